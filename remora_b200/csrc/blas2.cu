// Matrix-vector kernels of the cuda_tag device: GEMV, triangular solve with one vector
// (TRSV) and triangular products (TRMM, TRMV).
//
// Replace kernels::gemv / trsv / trmv / trmm for hip_tag (include/remora/kernels/hip/
// gemv.hpp:45-90, trsv.hpp:44-90, trmv.hpp:44-90, trmm.hpp:45-106, all forwarding to
// cuBLAS through hip/cublas_backend.hpp:170-213, :348-383). Here:
//  * GEMV is HBM-bound (every element of A is read once): y = A x (column-major A) sweeps
//    column slices with one thread per row (coalesced reads down each column) and sums the
//    slices' partial results in a second pass in slice order (deterministic); y = A^T x is
//    one warp per output, the lanes walking the column.
//  * TRSV is the blocked TRSM with one right-hand side (diagonal 128-blocks inverted in
//    FP64, then block-row products).
//  * TRMM / TRMV copy the triangle of op(A) (zero elsewhere, ones on a unit diagonal) and
//    the operand to workspace and multiply with the library's GEMM.
#include "assign.cuh"
#include "factor.cuh"
#include "gemm.cuh"

namespace rc {
namespace {

// part[s * m + i] = sum over the columns j of slice s of A(i, j) x[j * incx].
template <class T>
__global__ void __launch_bounds__(256) gemv_n_kernel(int64_t m, int64_t n, View<const T> A, const T* x,
                                                     int64_t incx, int64_t cols_per_slice, T* part) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t j0 = (int64_t)blockIdx.y * cols_per_slice;
    const int64_t j1 = (j0 + cols_per_slice) < n ? j0 + cols_per_slice : n;
    if (i >= m) return;
    T a0 = T(0), a1 = T(0);
    int64_t j = j0;
    for (; j + 1 < j1; j += 2) {
        a0 = fma(A(i, j), x[j * incx], a0);
        a1 = fma(A(i, j + 1), x[(j + 1) * incx], a1);
    }
    if (j < j1) a0 = fma(A(i, j), x[j * incx], a0);
    part[(int64_t)blockIdx.y * m + i] = a0 + a1;
}

// y[i] = alpha * sum_s part[s * m + i] + beta * y[i], slices summed in order.
template <class T>
__global__ void gemv_reduce_kernel(int64_t m, int slices, const T* part, T alpha, T beta, T* y, int64_t incy) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        T acc = T(0);
        for (int s = 0; s < slices; ++s) acc += part[s * m + i];
        T v = alpha * acc;
        if (beta != T(0)) v = fma(beta, y[i * incy], v);
        y[i * incy] = v;
    }
}

// y[c] = alpha * sum_j A(j, c) x[j] + beta * y[c]: one warp per output column c.
template <class T>
__global__ void __launch_bounds__(256) gemv_t_kernel(int64_t rows, int64_t cols, View<const T> A, const T* x,
                                                     int64_t incx, T alpha, T beta, T* y, int64_t incy) {
    const int64_t c = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (c >= cols) return;
    T acc = T(0);
    for (int64_t j = lane; j < rows; j += 32) acc = fma(A(j, c), x[j * incx], acc);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    if (lane == 0) {
        T v = alpha * acc;
        if (beta != T(0)) v = fma(beta, y[c * incy], v);
        y[c * incy] = v;
    }
}

// D = triangle of the k x k view S (lower, or upper), zero elsewhere, ones on a unit
// diagonal; D column-major with ld k.
template <class T>
__global__ void tri_copy_kernel(int64_t k, View<const T> S, bool upper, bool unit, T* D) {
    for (int64_t j = blockIdx.y; j < k; j += gridDim.y)
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < k; i += (int64_t)gridDim.x * blockDim.x) {
            T v = T(0);
            if (i == j) v = unit ? T(1) : S(i, j);
            else if (upper ? i < j : i > j) v = S(i, j);
            D[i + j * k] = v;
        }
}

// y = alpha x + beta y (beta == 0 does not read y).
template <class T>
__global__ void axpby_kernel(int64_t n, T alpha, const T* x, int64_t incx, T beta, T* y, int64_t incy) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        T v = alpha * x[i * incx];
        if (beta != T(0)) v = fma(beta, y[i * incy], v);
        y[i * incy] = v;
    }
}

dim3 sq_grid(int64_t rows, int64_t cols) {
    return dim3(ceil_div(rows, 256) < 256u ? ceil_div(rows, 256) : 256u, cols < 65535 ? (unsigned)cols : 65535u);
}

}  // namespace

// y <- alpha op(A) x + beta y for the m x n view A (op(A) = A, or A^T when trans).
template <class T>
int gemv(bool trans, int64_t m, int64_t n, T alpha, View<const T> A, const T* x, int64_t incx, T beta, T* y,
         int64_t incy, cudaStream_t s) {
    const int64_t rows_out = trans ? n : m, inner = trans ? m : n;
    if (rows_out <= 0) return RC_SUCCESS;
    if (inner <= 0 || alpha == T(0)) {
        RC_TRY(gemm<T>(rows_out, 1, 0, alpha, View<const T>{nullptr, 1, 1}, View<const T>{nullptr, 1, 1}, beta,
                       View<T>{y, incy, 1}, kFull, 0, s));
        return RC_SUCCESS;
    }
    // Reads run down the unit-stride direction of A: A x with column-major A, or A^T x
    // with row-major A, sweeps column slices; the other two cases are column dot products.
    const bool sweep = trans ? (A.cs == 1) : (A.rs == 1);
    if (sweep) {
        const View<const T> Ao = trans ? A.t() : A;  // rows_out x inner, unit stride down a column
        const int64_t row_blocks = ceil_div(rows_out, 256);
        int64_t slices = (2 * sm_count() + row_blocks - 1) / row_blocks;
        const int64_t max_slices = inner / 64 > 0 ? inner / 64 : 1;
        if (slices > max_slices) slices = max_slices;
        if (slices > 64) slices = 64;
        if (slices < 1) slices = 1;
        const int64_t per = (inner + slices - 1) / slices;
        slices = (inner + per - 1) / per;
        T* part = static_cast<T*>(workspace(s, (size_t)slices * rows_out * sizeof(T), 9));
        if (!part) return RC_ERR_ALLOC;
        gemv_n_kernel<T><<<dim3((unsigned)row_blocks, (unsigned)slices), 256, 0, s>>>(rows_out, inner, Ao, x, incx, per,
                                                                                       part);
        RC_TRY(check_launch());
        gemv_reduce_kernel<T><<<ceil_div(rows_out, 256) < 1024u ? ceil_div(rows_out, 256) : 1024u, 256, 0, s>>>(
            rows_out, (int)slices, part, alpha, beta, y, incy);
        return check_launch();
    }
    const View<const T> Ac = trans ? A : A.t();  // inner x rows_out: output c is column c
    gemv_t_kernel<T><<<ceil_div(rows_out, 8), 256, 0, s>>>(inner, rows_out, Ac, x, incx, alpha, beta, y, incy);
    return check_launch();
}

// B <- op(T) B (left) or B op(T) (right) for the triangle T of the k x k view A.
template <class T>
int trmm(bool left, bool upper, bool trans, bool unit, int64_t m, int64_t n, View<const T> A, View<T> B,
         cudaStream_t s) {
    if (m <= 0 || n <= 0) return RC_SUCCESS;
    const int64_t k = left ? m : n;
    T* w = static_cast<T*>(workspace(s, (size_t)(k * k + m * n) * sizeof(T), 10));
    if (!w) return RC_ERR_ALLOC;
    T* Tt = w;
    T* Bc = w + k * k;
    tri_copy_kernel<T><<<sq_grid(k, k), 256, 0, s>>>(k, A, upper, unit, Tt);
    RC_TRY(check_launch());
    RC_TRY(copy2d<T, T>(m, n, T(1), View<const T>{B.p, B.rs, B.cs}, colmajor(Bc, m), s));
    View<const T> Tv = colmajor(static_cast<const T*>(Tt), k);
    if (trans) Tv = Tv.t();
    const View<const T> Bv = colmajor(static_cast<const T*>(Bc), m);
    if (left) return gemm<T>(m, n, m, T(1), Tv, Bv, T(0), B, kFull, 0, s);
    return gemm<T>(m, n, n, T(1), Bv, Tv, T(0), B, kFull, 0, s);
}

}  // namespace rc

namespace {

template <class T>
int gemv_abi(int trans, size_t m, size_t n, T alpha, const T* A, size_t lda, const T* x, size_t incx, T beta, T* y,
             size_t incy, void* stream) {
    const size_t rows_out = trans ? n : m;
    if (rows_out == 0) return RC_SUCCESS;
    const size_t inner = trans ? m : n;
    if (!y || incy == 0 || lda < (m > 0 ? m : 1) || (inner > 0 && (!A || !x || incx == 0))) return RC_ERR_INVALID_ARGUMENT;
    return rc::gemv<T>(trans != 0, (int64_t)m, (int64_t)n, alpha, rc::colmajor(A, (int64_t)lda), x, (int64_t)incx,
                       beta, y, (int64_t)incy, static_cast<cudaStream_t>(stream));
}

template <class T>
int trsv_abi(int upper, int trans, int unit, size_t n, const T* A, size_t lda, T* x, size_t incx, void* stream) {
    if (n == 0) return RC_SUCCESS;
    if (!A || !x || lda < n || incx == 0) return RC_ERR_INVALID_ARGUMENT;
    rc::View<const T> Av = rc::colmajor(A, (int64_t)lda);
    bool up = upper != 0;
    if (trans) {
        Av = Av.t();
        up = !up;
    }
    return rc::trsm_left<T>(up, unit != 0, (int64_t)n, 1, T(1), Av, rc::View<T>{x, (int64_t)incx, (int64_t)n * (int64_t)incx},
                            nullptr, static_cast<cudaStream_t>(stream));
}

template <class T>
int trmm_abi(int left, int upper, int trans, int unit, size_t m, size_t n, const T* A, size_t lda, T* B, size_t ldb,
             void* stream) {
    if (m == 0 || n == 0) return RC_SUCCESS;
    const size_t k = left ? m : n;
    if (!A || !B || lda < k || ldb < m) return RC_ERR_INVALID_ARGUMENT;
    return rc::trmm<T>(left != 0, upper != 0, trans != 0, unit != 0, (int64_t)m, (int64_t)n,
                       rc::colmajor(A, (int64_t)lda), rc::colmajor(B, (int64_t)ldb), static_cast<cudaStream_t>(stream));
}

template <class T>
int axpby_abi(size_t n, T alpha, const T* x, size_t incx, T beta, T* y, size_t incy, void* stream) {
    if (n == 0) return RC_SUCCESS;
    if (!x || !y || incx == 0 || incy == 0) return RC_ERR_INVALID_ARGUMENT;
    const unsigned g = rc::ceil_div(n, 256) < 2048u ? rc::ceil_div(n, 256) : 2048u;
    rc::axpby_kernel<T><<<g, 256, 0, static_cast<cudaStream_t>(stream)>>>((int64_t)n, alpha, x, (int64_t)incx, beta, y,
                                                                          (int64_t)incy);
    return rc::check_launch();
}

template <class T>
int trmv_abi(int upper, int trans, int unit, size_t n, const T* A, size_t lda, T* x, size_t incx, void* stream) {
    if (n == 0) return RC_SUCCESS;
    if (!A || !x || lda < n || incx == 0) return RC_ERR_INVALID_ARGUMENT;
    return rc::trmm<T>(true, upper != 0, trans != 0, unit != 0, (int64_t)n, 1, rc::colmajor(A, (int64_t)lda),
                       rc::View<T>{x, (int64_t)incx, (int64_t)n * (int64_t)incx}, static_cast<cudaStream_t>(stream));
}

}  // namespace

extern "C" {

int rc_gemv_f64(int trans, size_t m, size_t n, double alpha, const double* A, size_t lda, const double* x,
                size_t incx, double beta, double* y, size_t incy, void* stream) {
    return gemv_abi<double>(trans, m, n, alpha, A, lda, x, incx, beta, y, incy, stream);
}
int rc_gemv_f32(int trans, size_t m, size_t n, float alpha, const float* A, size_t lda, const float* x, size_t incx,
                float beta, float* y, size_t incy, void* stream) {
    return gemv_abi<float>(trans, m, n, alpha, A, lda, x, incx, beta, y, incy, stream);
}
int rc_trsv_f64(int upper, int trans, int unit, size_t n, const double* A, size_t lda, double* x, size_t incx,
                void* stream) {
    return trsv_abi<double>(upper, trans, unit, n, A, lda, x, incx, stream);
}
int rc_trsv_f32(int upper, int trans, int unit, size_t n, const float* A, size_t lda, float* x, size_t incx,
                void* stream) {
    return trsv_abi<float>(upper, trans, unit, n, A, lda, x, incx, stream);
}
int rc_trmm_f64(int left, int upper, int trans, int unit, size_t m, size_t n, const double* A, size_t lda, double* B,
                size_t ldb, void* stream) {
    return trmm_abi<double>(left, upper, trans, unit, m, n, A, lda, B, ldb, stream);
}
int rc_trmm_f32(int left, int upper, int trans, int unit, size_t m, size_t n, const float* A, size_t lda, float* B,
                size_t ldb, void* stream) {
    return trmm_abi<float>(left, upper, trans, unit, m, n, A, lda, B, ldb, stream);
}
int rc_trmv_f64(int upper, int trans, int unit, size_t n, const double* A, size_t lda, double* x, size_t incx,
                void* stream) {
    return trmv_abi<double>(upper, trans, unit, n, A, lda, x, incx, stream);
}
int rc_trmv_f32(int upper, int trans, int unit, size_t n, const float* A, size_t lda, float* x, size_t incx,
                void* stream) {
    return trmv_abi<float>(upper, trans, unit, n, A, lda, x, incx, stream);
}
int rc_axpby_f64(size_t n, double alpha, const double* x, size_t incx, double beta, double* y, size_t incy,
                 void* stream) {
    return axpby_abi<double>(n, alpha, x, incx, beta, y, incy, stream);
}
int rc_axpby_f32(size_t n, float alpha, const float* x, size_t incx, float beta, float* y, size_t incy, void* stream) {
    return axpby_abi<float>(n, alpha, x, incx, beta, y, incy, stream);
}

}  // extern "C"
