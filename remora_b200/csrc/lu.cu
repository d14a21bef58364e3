// LU with partial pivoting (getrf) and pivoted Cholesky (pstrf) on the GPU, in place on
// any strided view of the logical n x n matrix.
//
// getrf (kernels/getrf.hpp:50-59; CPU algorithm kernels/default/getrf.hpp:41-181):
// blocked right-looking LU with 64-column panels. One CTA factors a panel column by
// column -- pivot = the row of largest |A(i, j)| at or below the diagonal (the lowest
// row among equals, as the reference's strictly-larger scan), the swap of the two rows
// across the panel, the division of the column by the pivot (in double, as the
// reference), the rank-1 update of the panel -- then the panel's swaps are applied to
// the other columns in order, U12 = L11^-1 A12 (unit lower TRSM) and A22 -= L21 U12 (DMMA
// GEMM). piv[i] is the row swapped with row i at step i (LAPACK order, 0-based, as
// Remora's permutation_matrix). A zero pivot records its 1-based column in *info and
// stops every later kernel (the reference throws).
//
// pstrf (kernels/pstrf.hpp:62-70; CPU algorithm kernels/default/pstrf.hpp:40-147, the
// blocked pivoted Cholesky of LAWN 161): blocks of 32 columns. One CTA runs a block: the
// pivot values (the trailing diagonal, refreshed from the block's finished columns)
// choose the largest remaining pivot (the lowest index among equals, as std::max_element),
// rows and columns of the whole matrix are swapped, the factor stops with rank c when the
// pivot value is below n^2 eps max|A_ii| (the trailing square is cleared), else the
// column is finished by the dot products with the block's earlier columns and a division,
// and the row right of the diagonal is cleared. After the block the whole trailing square
// (both triangles, which later swaps read) is updated by a DMMA GEMM with the block's
// columns. piv as for getrf (identity where no swap happened); the rank goes to *rank.
#include <cfloat>
#include <cmath>

#include "factor.cuh"
#include "gemm.cuh"

namespace rc {
namespace {

constexpr int kLuNB = 64;       // getrf panel width
constexpr int kPsNB = 32;       // pstrf block width
constexpr int kLuThreads = 1024;

// Block-wide (value, index) reduction: larger value wins, the smaller index among equals.
__device__ __forceinline__ void argmax_pair(double& v, int64_t& i, double ov, int64_t oi) {
    if (ov > v || (ov == v && oi < i)) {
        v = ov;
        i = oi;
    }
}

__device__ void block_argmax(double& v, int64_t& i, double* sv, int64_t* si) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o; o >>= 1) argmax_pair(v, i, __shfl_xor_sync(0xffffffffu, v, o),
                                             __shfl_xor_sync(0xffffffffu, i, o));
    if (lane == 0) {
        sv[warp] = v;
        si[warp] = i;
    }
    __syncthreads();
    if (warp == 0) {
        v = lane < (int)(blockDim.x >> 5) ? sv[lane] : -DBL_MAX;
        i = lane < (int)(blockDim.x >> 5) ? si[lane] : INT64_MAX;
#pragma unroll
        for (int o = 16; o; o >>= 1) argmax_pair(v, i, __shfl_xor_sync(0xffffffffu, v, o),
                                                 __shfl_xor_sync(0xffffffffu, i, o));
        if (lane == 0) {
            sv[0] = v;
            si[0] = i;
        }
    }
    __syncthreads();
    v = sv[0];
    i = si[0];
    __syncthreads();
}

template <class T>
__global__ void __launch_bounds__(kLuThreads) getrf_panel_kernel(int64_t n, View<T> A, int64_t k0, int nb, int* piv,
                                                                 int* info) {
    __shared__ double sv[32];
    __shared__ int64_t si[32];
    if (*(volatile int*)info != 0) return;
    for (int j = 0; j < nb; ++j) {
        const int64_t c = k0 + j;
        double best = -1.0;
        int64_t bi = INT64_MAX;
        for (int64_t i = c + threadIdx.x; i < n; i += blockDim.x) {
            const double a = fabs((double)A(i, c));
            if (a > best) {
                best = a;
                bi = i;
            }
        }
        block_argmax(best, bi, sv, si);
        const int64_t p = bi;
        const double pv = (double)A(p, c);
        if (pv == 0.0) {  // also all-zero columns: the first row is the pivot, value 0
            if (threadIdx.x == 0) {
                piv[c] = (int)c;
                record_first(info, (int)(c + 1));
            }
            return;
        }
        if (threadIdx.x == 0) piv[c] = (int)p;
        if (p != c)
            for (int col = threadIdx.x; col < nb; col += blockDim.x) {
                const T t = A(c, k0 + col);
                A(c, k0 + col) = A(p, k0 + col);
                A(p, k0 + col) = t;
            }
        __syncthreads();
        for (int64_t i = c + 1 + threadIdx.x; i < n; i += blockDim.x) A(i, c) = (T)((double)A(i, c) / pv);
        __syncthreads();
        const int64_t rows = n - c - 1, cols = nb - j - 1;
        for (int64_t e = threadIdx.x; e < rows * cols; e += blockDim.x) {
            const int64_t i = c + 1 + e % rows, col = c + 1 + e / rows;
            A(i, col) -= A(i, c) * A(c, col);
        }
        __syncthreads();
    }
}

// The row swaps piv[k0 .. k0 + nb) in order, on the columns outside the panel.
template <class T>
__global__ void lu_swap_kernel(int64_t n, View<T> A, int64_t k0, int nb, const int* piv, const int* info) {
    if (*(volatile const int*)info != 0) return;
    for (int64_t col = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; col < n - nb;
         col += (int64_t)gridDim.x * blockDim.x) {
        const int64_t cc = col < k0 ? col : col + nb;
        for (int j = 0; j < nb; ++j) {
            const int64_t r = k0 + j, p = piv[r];
            if (p != r) {
                const T t = A(r, cc);
                A(r, cc) = A(p, cc);
                A(p, cc) = t;
            }
        }
    }
}

// eps = n^2 epsilon(T) max(A(0, 0), max_i |A(i, i)|); piv = identity; rank = n; stop = 0.
template <class T>
__global__ void pstrf_init_kernel(int64_t n, View<const T> A, double* eps, int* piv, int* rank, int* stop) {
    __shared__ double sv[32];
    __shared__ int64_t si[32];
    double mx = -DBL_MAX;
    int64_t dummy = 0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        mx = fmax(mx, i == 0 ? (double)A(0, 0) : fabs((double)A(i, i)));
        piv[i] = (int)i;
    }
    block_argmax(mx, dummy, sv, si);
    if (threadIdx.x == 0) {
        const double e = sizeof(T) == 8 ? DBL_EPSILON : (double)FLT_EPSILON;
        *eps = (double)(n * n) * e * mx;
        *rank = (int)n;
        *stop = 0;
    }
}

template <class T>
__global__ void __launch_bounds__(kLuThreads) pstrf_block_kernel(int64_t n, View<T> A, int64_t k, int cur, T* pv,
                                                                 const double* eps, int* piv, int* rank,
                                                                 int* stop) {
    __shared__ double sv[32];
    __shared__ int64_t si[32];
    if (*(volatile int*)stop != 0) return;
    const double epsv = *eps;
    for (int j = 0; j < cur; ++j) {
        const int64_t c = k + j;
        for (int64_t i = c + threadIdx.x; i < n; i += blockDim.x) {
            if (j == 0) pv[i] = A(i, i);
            else pv[i] -= A(i, c - 1) * A(i, c - 1);
        }
        __syncthreads();
        double best = -DBL_MAX;
        int64_t bi = INT64_MAX;
        for (int64_t i = c + threadIdx.x; i < n; i += blockDim.x)
            if ((double)pv[i] > best) {
                best = (double)pv[i];
                bi = i;
            }
        block_argmax(best, bi, sv, si);
        const int64_t p = bi;
        if (p != c) {
            if (threadIdx.x == 0) piv[c] = (int)p;
            for (int64_t t = threadIdx.x; t < n; t += blockDim.x) {
                const T x = A(c, t);
                A(c, t) = A(p, t);
                A(p, t) = x;
            }
            __syncthreads();
            for (int64_t t = threadIdx.x; t < n; t += blockDim.x) {
                const T x = A(t, c);
                A(t, c) = A(t, p);
                A(t, p) = x;
            }
            if (threadIdx.x == 0) {
                const T x = pv[c];
                pv[c] = pv[p];
                pv[p] = x;
            }
            __syncthreads();
        }
        const T v = pv[c];
        if ((double)v < epsv) {
            const int64_t m = n - c;
            for (int64_t e = threadIdx.x; e < m * m; e += blockDim.x) A(c + e % m, c + e / m) = T(0);
            if (threadIdx.x == 0) {
                *rank = (int)c;
                *stop = 1;
            }
            return;
        }
        const T d = sqrt(v);
        for (int64_t i = c + 1 + threadIdx.x; i < n; i += blockDim.x) {
            T s = A(i, c);
            for (int64_t t = k; t < c; ++t) s -= A(i, t) * A(c, t);
            A(i, c) = s / d;
        }
        __syncthreads();
        if (threadIdx.x == 0) A(c, c) = d;
        for (int64_t t = c + 1 + threadIdx.x; t < n; t += blockDim.x) A(c, t) = T(0);
        __syncthreads();
    }
}

template <class T>
View<T> view_of(int row_major, T* A, int64_t lda) {
    return row_major ? View<T>{A, lda, 1} : View<T>{A, 1, lda};
}

template <class T>
int getrf(int row_major, int64_t n, T* Ap, int64_t lda, int* piv, int* info, cudaStream_t s) {
    if (cudaMemsetAsync(info, 0, sizeof(int), s) != cudaSuccess) return RC_ERR_CUDA;
    const View<T> A = view_of(row_major, Ap, lda);
    for (int64_t k0 = 0; k0 < n; k0 += kLuNB) {
        const int nb = (int)(n - k0 < kLuNB ? n - k0 : kLuNB);
        getrf_panel_kernel<T><<<1, kLuThreads, 0, s>>>(n, A, k0, nb, piv, info);
        RC_TRY(check_launch());
        if (n > nb) {
            const int64_t cols = n - nb;
            lu_swap_kernel<T><<<ceil_div(cols, 256) < 1024u ? ceil_div(cols, 256) : 1024u, 256, 0, s>>>(n, A, k0, nb,
                                                                                                      piv, info);
            RC_TRY(check_launch());
        }
        const int64_t r = n - k0 - nb;
        if (r <= 0) continue;
        const View<const T> L11{A.sub(k0, k0).p, A.rs, A.cs};
        RC_TRY(trsm_left<T>(false, true, nb, r, T(1), L11, A.sub(k0, k0 + nb), nullptr, s, info));
        const View<const T> L21{A.sub(k0 + nb, k0).p, A.rs, A.cs}, U12{A.sub(k0, k0 + nb).p, A.rs, A.cs};
        RC_TRY(gemm<T>(r, r, nb, T(-1), L21, U12, T(1), A.sub(k0 + nb, k0 + nb), kFull, 0, s, info));
    }
    return RC_SUCCESS;
}

template <class T>
int pstrf(int row_major, int64_t n, T* Ap, int64_t lda, int* piv, int* rank, cudaStream_t s) {
    const size_t bytes = ((size_t)n * sizeof(T) + 255) / 256 * 256 + 256;
    char* ws = static_cast<char*>(workspace(s, bytes, 12));
    if (!ws) return RC_ERR_ALLOC;
    T* pv = reinterpret_cast<T*>(ws);
    double* eps = reinterpret_cast<double*>(ws + bytes - 256);
    int* stop = reinterpret_cast<int*>(ws + bytes - 128);
    const View<T> A = view_of(row_major, Ap, lda);
    pstrf_init_kernel<T><<<1, kLuThreads, 0, s>>>(n, View<const T>{A.p, A.rs, A.cs}, eps, piv, rank, stop);
    RC_TRY(check_launch());
    for (int64_t k = 0; k < n; k += kPsNB) {
        const int cur = (int)(n - k < kPsNB ? n - k : kPsNB);
        pstrf_block_kernel<T><<<1, kLuThreads, 0, s>>>(n, A, k, cur, pv, eps, piv, rank, stop);
        RC_TRY(check_launch());
        const int64_t r = n - k - cur;
        if (r <= 0) continue;
        const View<const T> L21{A.sub(k + cur, k).p, A.rs, A.cs};
        RC_TRY(gemm<T>(r, r, cur, T(-1), L21, L21.t(), T(1), A.sub(k + cur, k + cur), kFull, 0, s, stop));
    }
    return RC_SUCCESS;
}

}  // namespace
}  // namespace rc

extern "C" {

int rc_getrf_f64(int row_major, size_t n, double* A, size_t lda, int* piv, int* info, void* stream) {
    if (!info) return RC_ERR_INVALID_ARGUMENT;
    if (n == 0) return cudaMemsetAsync(info, 0, sizeof(int), static_cast<cudaStream_t>(stream)) == cudaSuccess
                           ? RC_SUCCESS
                           : RC_ERR_CUDA;
    if (!A || !piv || lda < n) return RC_ERR_INVALID_ARGUMENT;
    if (n > (size_t)INT32_MAX) return RC_ERR_NOT_SUPPORTED;
    return rc::getrf<double>(row_major, (int64_t)n, A, (int64_t)lda, piv, info, static_cast<cudaStream_t>(stream));
}

int rc_getrf_f32(int row_major, size_t n, float* A, size_t lda, int* piv, int* info, void* stream) {
    if (!info) return RC_ERR_INVALID_ARGUMENT;
    if (n == 0) return cudaMemsetAsync(info, 0, sizeof(int), static_cast<cudaStream_t>(stream)) == cudaSuccess
                           ? RC_SUCCESS
                           : RC_ERR_CUDA;
    if (!A || !piv || lda < n) return RC_ERR_INVALID_ARGUMENT;
    if (n > (size_t)INT32_MAX) return RC_ERR_NOT_SUPPORTED;
    return rc::getrf<float>(row_major, (int64_t)n, A, (int64_t)lda, piv, info, static_cast<cudaStream_t>(stream));
}

int rc_pstrf_f64(int row_major, size_t n, double* A, size_t lda, int* piv, int* rank, void* stream) {
    if (!rank) return RC_ERR_INVALID_ARGUMENT;
    if (n == 0) return cudaMemsetAsync(rank, 0, sizeof(int), static_cast<cudaStream_t>(stream)) == cudaSuccess
                           ? RC_SUCCESS
                           : RC_ERR_CUDA;
    if (!A || !piv || lda < n) return RC_ERR_INVALID_ARGUMENT;
    if (n > (size_t)INT32_MAX) return RC_ERR_NOT_SUPPORTED;
    return rc::pstrf<double>(row_major, (int64_t)n, A, (int64_t)lda, piv, rank, static_cast<cudaStream_t>(stream));
}

int rc_pstrf_f32(int row_major, size_t n, float* A, size_t lda, int* piv, int* rank, void* stream) {
    if (!rank) return RC_ERR_INVALID_ARGUMENT;
    if (n == 0) return cudaMemsetAsync(rank, 0, sizeof(int), static_cast<cudaStream_t>(stream)) == cudaSuccess
                           ? RC_SUCCESS
                           : RC_ERR_CUDA;
    if (!A || !piv || lda < n) return RC_ERR_INVALID_ARGUMENT;
    if (n > (size_t)INT32_MAX) return RC_ERR_NOT_SUPPORTED;
    return rc::pstrf<float>(row_major, (int64_t)n, A, (int64_t)lda, piv, rank, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
