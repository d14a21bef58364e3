// Copy / transpose / scale / fill of strided matrices: the assignment support that the
// reference's containers run as device kernels (include/remora/kernels/hip/
// matrix_assign.hpp:38-200, hip/dense.hpp:39-51 clear2d, hip/buffer.hpp:105-125 fill).
// A transposing copy goes through a 32x33 shared-memory tile so that both the read and
// the write are coalesced.
#include "assign.cuh"

namespace rc {
namespace {

template <class S, class D>
__global__ void __launch_bounds__(256) copy2d_kernel(int64_t m, int64_t n, D alpha, View<const S> A, View<D> B,
                                                     const int* abort) {
    __shared__ D tile[32][33];
    if (abort != nullptr && *(volatile const int*)abort != 0) return;
    const int64_t i0 = (int64_t)blockIdx.y * 32, j0 = (int64_t)blockIdx.x * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
    // Read with the thread index along A's unit stride when A is column-major.
    const bool a_col = A.rs == 1;
    for (int r = ty; r < 32; r += 8) {
        const int64_t i = i0 + (a_col ? tx : r), j = j0 + (a_col ? r : tx);
        if (i < m && j < n) tile[a_col ? r : tx][a_col ? tx : r] = alpha * (D)A(i, j);
    }
    __syncthreads();
    const bool b_col = B.rs == 1;
    for (int r = ty; r < 32; r += 8) {
        const int64_t i = i0 + (b_col ? tx : r), j = j0 + (b_col ? r : tx);
        if (i < m && j < n) B(i, j) = tile[b_col ? r : tx][b_col ? tx : r];
    }
}

template <class T>
__global__ void __launch_bounds__(256) fill_kernel(int64_t m, int64_t n, T value, View<T> A) {
    const bool col = A.rs == 1;
    const int64_t inner = col ? m : n, outer = col ? n : m;
    for (int64_t o = blockIdx.y; o < outer; o += gridDim.y)
        for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < inner;
             x += (int64_t)gridDim.x * blockDim.x) {
            if (col) A(x, o) = value; else A(o, x) = value;
        }
}

// B(i, j) = A(idx[i], j): a row gather with arbitrary element strides on both sides (the
// unit-stride index of B walks threadIdx.x). Rows whose index is outside [0, m) are not
// written.
template <class T>
__global__ void __launch_bounds__(256) gather_rows_kernel(int64_t m, int64_t n, const int* __restrict__ idx,
                                                          View<const T> A, View<T> B) {
    const bool col = B.rs == 1;
    const int64_t inner = col ? m : n, outer = col ? n : m;
    for (int64_t o = blockIdx.y; o < outer; o += gridDim.y)
        for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < inner;
             x += (int64_t)gridDim.x * blockDim.x) {
            const int64_t i = col ? x : o, j = col ? o : x;
            const int64_t r = idx[i];
            if (r >= 0 && r < m) B(i, j) = A(r, j);
        }
}

}  // namespace

template <class S, class D>
int copy2d(int64_t m, int64_t n, D alpha, View<const S> A, View<D> B, cudaStream_t s, const int* abort) {
    if (m <= 0 || n <= 0) return RC_SUCCESS;
    dim3 grid(ceil_div(n, 32), ceil_div(m, 32));
    if (grid.y > 65535) return RC_ERR_NOT_SUPPORTED;
    copy2d_kernel<S, D><<<grid, 256, 0, s>>>(m, n, alpha, A, B, abort);
    return check_launch();
}

template <class T>
int fill(int64_t m, int64_t n, T value, View<T> A, cudaStream_t s) {
    if (m <= 0 || n <= 0) return RC_SUCCESS;
    const bool col = A.rs == 1;
    const int64_t inner = col ? m : n, outer = col ? n : m;
    dim3 grid(ceil_div(inner, 256) < 1024u ? ceil_div(inner, 256) : 1024u, outer < 65535 ? (unsigned)outer : 65535u);
    fill_kernel<T><<<grid, 256, 0, s>>>(m, n, value, A);
    return check_launch();
}

template int copy2d<double, double>(int64_t, int64_t, double, View<const double>, View<double>, cudaStream_t,
                                           const int*);
template int copy2d<float, float>(int64_t, int64_t, float, View<const float>, View<float>, cudaStream_t,
                                           const int*);
template int copy2d<double, float>(int64_t, int64_t, float, View<const double>, View<float>, cudaStream_t,
                                           const int*);
template int copy2d<float, double>(int64_t, int64_t, double, View<const float>, View<double>, cudaStream_t,
                                           const int*);
template int fill<double>(int64_t, int64_t, double, View<double>, cudaStream_t);
template int fill<float>(int64_t, int64_t, float, View<float>, cudaStream_t);

}  // namespace rc

namespace {
template <class T>
int copy_abi(int trans, size_t m, size_t n, T alpha, const T* A, size_t lda, T* B, size_t ldb, void* stream) {
    if (m == 0 || n == 0) return RC_SUCCESS;
    if (!A || !B || ldb < m || lda < (trans ? n : m)) return RC_ERR_INVALID_ARGUMENT;
    rc::View<const T> a = rc::colmajor(A, (int64_t)lda);
    if (trans) a = a.t();
    return rc::copy2d<T, T>((int64_t)m, (int64_t)n, alpha, a, rc::colmajor(B, (int64_t)ldb),
                            static_cast<cudaStream_t>(stream));
}
template <class T>
int gather_abi(size_t m, size_t n, const int* idx, const T* A, ptrdiff_t ars, ptrdiff_t acs, T* B, ptrdiff_t brs,
               ptrdiff_t bcs, void* stream) {
    if (m == 0 || n == 0) return RC_SUCCESS;
    if (!idx || !A || !B || A == B) return RC_ERR_INVALID_ARGUMENT;
    const rc::View<T> b{B, (int64_t)brs, (int64_t)bcs};
    const bool col = brs == 1;
    const int64_t inner = col ? (int64_t)m : (int64_t)n, outer = col ? (int64_t)n : (int64_t)m;
    dim3 grid(rc::ceil_div(inner, 256) < 1024u ? rc::ceil_div(inner, 256) : 1024u,
              outer < 65535 ? (unsigned)outer : 65535u);
    rc::gather_rows_kernel<T><<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        (int64_t)m, (int64_t)n, idx, rc::View<const T>{A, (int64_t)ars, (int64_t)acs}, b);
    return rc::check_launch();
}
template <class T>
int fill_abi(size_t m, size_t n, T value, T* A, size_t lda, void* stream) {
    if (m == 0 || n == 0) return RC_SUCCESS;
    if (!A || lda < m) return RC_ERR_INVALID_ARGUMENT;
    return rc::fill<T>((int64_t)m, (int64_t)n, value, rc::colmajor(A, (int64_t)lda), static_cast<cudaStream_t>(stream));
}
}  // namespace

extern "C" {
int rc_copy2d_f64(int trans, size_t m, size_t n, double alpha, const double* A, size_t lda, double* B, size_t ldb,
                  void* stream) {
    return copy_abi<double>(trans, m, n, alpha, A, lda, B, ldb, stream);
}
int rc_copy2d_f32(int trans, size_t m, size_t n, float alpha, const float* A, size_t lda, float* B, size_t ldb,
                  void* stream) {
    return copy_abi<float>(trans, m, n, alpha, A, lda, B, ldb, stream);
}
int rc_gather_rows_f64(size_t m, size_t n, const int* idx, const double* A, ptrdiff_t a_rs, ptrdiff_t a_cs, double* B,
                       ptrdiff_t b_rs, ptrdiff_t b_cs, void* stream) {
    return gather_abi<double>(m, n, idx, A, a_rs, a_cs, B, b_rs, b_cs, stream);
}
int rc_gather_rows_f32(size_t m, size_t n, const int* idx, const float* A, ptrdiff_t a_rs, ptrdiff_t a_cs, float* B,
                       ptrdiff_t b_rs, ptrdiff_t b_cs, void* stream) {
    return gather_abi<float>(m, n, idx, A, a_rs, a_cs, B, b_rs, b_cs, stream);
}
int rc_fill_f64(size_t m, size_t n, double value, double* A, size_t lda, void* stream) {
    return fill_abi<double>(m, n, value, A, lda, stream);
}
int rc_fill_f32(size_t m, size_t n, float value, float* A, size_t lda, void* stream) {
    return fill_abi<float>(m, n, value, A, lda, stream);
}
}
