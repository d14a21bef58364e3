// Blocked triangular solve (TRSM) and blocked right-looking Cholesky (POTRF).
//
// Replaces kernels::trsm / kernels::potrf for hip_tag (include/remora/kernels/hip/
// trsm.hpp:45-107 -> cublas trsm; include/remora/kernels/hip/potrf.hpp:41-141, a
// recursive split whose 16x16 leaves are factored by a single thread). Here:
//  * TRSM: every 128x128 diagonal block of the triangle is inverted at once (one CTA
//    per block, FP64 in shared memory); the solve then walks the block rows, each step
//    one GEMM with the inverted block and one GEMM update of the remaining rows, so
//    nearly all flops run in the tensor-core GEMM.
//  * POTRF: per 128-wide panel, one CTA factors the diagonal block in FP64 shared
//    memory (and inverts it), the panel below is solved by a GEMM with that inverse,
//    and the trailing matrix is updated by a lower-masked GEMM (the SYRK schedule).
//    A non-positive pivot writes its global index to the status word and every later
//    kernel of the factorization returns at once.
#include "factor.cuh"
#include "assign.cuh"
#include "gemm.cuh"
#include <type_traits>

namespace rc {
namespace {

constexpr int NB = kNB;
constexpr int SLD = NB + 1;  // shared-memory row stride (doubles)
constexpr size_t kBlockSmem = (size_t)NB * SLD * sizeof(double);

__device__ __forceinline__ bool aborted(const int* abort) { return abort != nullptr && *(volatile const int*)abort != 0; }

// In-place inversion of the unit/non-unit lower-triangular NB x NB matrix in S
// (row-major, stride SLD), one thread per column: row i of the inverse only needs row i
// of L and the rows < i of the inverse in the thread's own column.
__device__ void invert_lower_inplace(double* S, bool unit) {
    const int j = threadIdx.x;
    for (int i = 0; i < NB; ++i) {
        double x = 0.0;
        if (j <= i && j < NB) {
            const double dinv = unit ? 1.0 : 1.0 / S[i * SLD + i];
            if (j == i) {
                x = dinv;
            } else {
                double a0 = 0.0, a1 = 0.0;
                int k = j;
                for (; k + 1 < i; k += 2) {
                    a0 = fma(S[i * SLD + k], S[k * SLD + j], a0);
                    a1 = fma(S[i * SLD + k + 1], S[(k + 1) * SLD + j], a1);
                }
                if (k < i) a0 = fma(S[i * SLD + k], S[k * SLD + j], a0);
                x = -(a0 + a1) * dinv;
            }
        }
        __syncthreads();
        if (j <= i && j < NB) S[i * SLD + j] = x;
    }
    __syncthreads();
}

// Store the inverse (lower, zero above the diagonal) as an NB x NB block, column-major or
// (row_major) row-major.
template <class T>
__device__ void store_block(const double* S, T* W, bool row_major = false) {
    for (int e = threadIdx.x; e < NB * NB; e += blockDim.x) {
        const int i = row_major ? e / NB : e % NB, j = row_major ? e % NB : e / NB;
        W[e] = j <= i ? (T)S[i * SLD + j] : T(0);
    }
}

// One CTA per diagonal block: W_b = inverse of the lower-triangular block b of L.
template <class T>
__global__ void __launch_bounds__(NB) trtri_blocks(int64_t m, View<const T> L, bool unit, T* W, int* info,
                                                   const int* abort) {
    extern __shared__ double S[];
    if (aborted(abort)) return;
    const int64_t r0 = (int64_t)blockIdx.x * NB;
    const int sz = (int)(m - r0 < NB ? m - r0 : NB);
    for (int e = threadIdx.x; e < NB * NB; e += blockDim.x) {
        const int i = e % NB, j = e / NB;
        double v;
        if (i < sz && j < sz && j <= i) v = (i == j && unit) ? 1.0 : (double)L(r0 + i, r0 + j);
        else v = (i == j) ? 1.0 : 0.0;
        S[i * SLD + j] = v;
    }
    __syncthreads();
    if (!unit && info != nullptr && threadIdx.x < sz && S[threadIdx.x * SLD + threadIdx.x] == 0.0)
        record_first(info, (int)(r0 + threadIdx.x + 1));
    invert_lower_inplace(S, unit);
    store_block<T>(S, W + (size_t)blockIdx.x * NB * NB);
}

// In-CTA blocked factorisation of one NB x NB diagonal block (FP64 in shared memory S,
// row-major, odd stride SLD so that both row and column walks are bank-conflict free).
// Besides L (lower triangle of S) it keeps rd[i] = 1 / L(i, i) and builds inv(L) in the
// strict upper triangle: Inv(i, c), i > c, is stored at S[c * SLD + i].
constexpr int DB = 32;  // diagonal sub-block
constexpr size_t kDiagSmem = kBlockSmem + (NB + 64 * 65) * sizeof(double) + 16;  // S, rd, T, flag

// S[i][c] -= sum_{m in [C0, C0 + DB)} L(i, m) L(c, m) for C0 + DB <= c <= i < NB. Thread
// (ty, tx) of 16 x 16 owns rows ty + 16 r and columns tx + 16 q with r, q >= (C0 + DB) / 16.
template <int KB>
__device__ void trailing_update(double* S) {
    constexpr int C0 = DB * KB, R0 = (C0 + DB) / 16, G = NB / 16 - R0;
    const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
    double acc[G][G];
#pragma unroll
    for (int r = 0; r < G; ++r)
#pragma unroll
        for (int q = 0; q < G; ++q) acc[r][q] = 0.0;
#pragma unroll 4
    for (int m = C0; m < C0 + DB; ++m) {
        double lr[G], lc[G];
#pragma unroll
        for (int r = 0; r < G; ++r) lr[r] = S[(ty + 16 * (R0 + r)) * SLD + m];
#pragma unroll
        for (int q = 0; q < G; ++q) lc[q] = S[(tx + 16 * (R0 + q)) * SLD + m];
#pragma unroll
        for (int r = 0; r < G; ++r)
#pragma unroll
            for (int q = 0; q <= r; ++q) acc[r][q] = fma(lr[r], lc[q], acc[r][q]);
    }
#pragma unroll
    for (int r = 0; r < G; ++r)
#pragma unroll
        for (int q = 0; q <= r; ++q) {
            const int i = ty + 16 * (R0 + r), c = tx + 16 * (R0 + q);
            if (c <= i) S[i * SLD + c] -= acc[r][q];
        }
}

// One step of the recursive inverse, for blocks of H rows: with inv(A) (rows/columns
// [J0, J0 + H)) and inv(D) ([I0, I0 + H), I0 = J0 + H) in place, the off-diagonal block of
// inv([A 0; C D]) is X = -inv(D) (C inv(A)). Needs rd on the diagonal of S, so that
// Inv(i, c) = S[c * SLD + i] for i >= c. NT threads (index t); thread (ty, tx) of
// (NT / 16) x 16 computes rows ty + (NT / 16) r and columns tx + 16 q of the H x H
// products; T is an H x H scratch (pitch 65). Phase 0: T = C inv(A); phase 1: X.
template <int H, int NT>
__device__ void inverse_merge(double* S, double* T, int J0, int t, int phase) {
    constexpr int RY = NT / 16, NR = H / RY, NQ = H / 16;
    const int I0 = J0 + H, ty = t / 16, tx = t % 16;
    double acc[NR][NQ];
#pragma unroll
    for (int r = 0; r < NR; ++r)
#pragma unroll
        for (int q = 0; q < NQ; ++q) acc[r][q] = 0.0;
    // The triangular operand is walked in k-blocks matching this thread's row or column
    // blocks: blocks that are entirely zero are skipped, full blocks need no mask, and only
    // the diagonal block selects.
    if (phase == 0) {  // T(i, c) = sum_{k >= c} C(i, k) inv(A)(k, c); columns c = tx + 16 q
#pragma unroll
        for (int kb = 0; kb < NQ; ++kb) {
#pragma unroll 4
            for (int kk = 0; kk < 16; ++kk) {
                const int k = 16 * kb + kk;
                double lr[NR];
#pragma unroll
                for (int r = 0; r < NR; ++r) lr[r] = S[(I0 + ty + RY * r) * SLD + J0 + k];
#pragma unroll
                for (int q = 0; q <= kb; ++q) {
                    double v = S[(J0 + tx + 16 * q) * SLD + J0 + k];  // inv(A)(k, c)
                    if (q == kb) v = kk >= tx ? v : 0.0;
#pragma unroll
                    for (int r = 0; r < NR; ++r) acc[r][q] = fma(lr[r], v, acc[r][q]);
                }
            }
        }
    } else {           // X(i, c) = -sum_{k <= i} inv(D)(i, k) T(k, c); rows i = ty + RY r
#pragma unroll
        for (int kb = 0; kb < NR; ++kb) {
#pragma unroll 4
            for (int kk = 0; kk < RY; ++kk) {
                const int k = RY * kb + kk;
                double lc[NQ];
#pragma unroll
                for (int q = 0; q < NQ; ++q) lc[q] = T[k * 65 + tx + 16 * q];
#pragma unroll
                for (int r = kb; r < NR; ++r) {
                    double v = S[(I0 + k) * SLD + I0 + ty + RY * r];  // inv(D)(i, k)
                    if (r == kb) v = kk <= ty ? v : 0.0;
#pragma unroll
                    for (int q = 0; q < NQ; ++q) acc[r][q] = fma(v, lc[q], acc[r][q]);
                }
            }
        }
    }
#pragma unroll
    for (int r = 0; r < NR; ++r)
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            const int i = ty + RY * r, c = tx + 16 * q;
            if (phase == 0) T[i * 65 + c] = acc[r][q];
            else S[(J0 + c) * SLD + I0 + i] = -acc[r][q];  // X(i, c) stored transposed
        }
}

// Factor the sz x sz lower diagonal block (A already offset to it) in FP64 and store
// inv(L) into W (column-major, or row-major when w_row_major); g0 = global index of the
// block for the pivot status. Blocked in shared memory over 32-column sub-blocks k:
//   1. warp 0 factors the 32 x 32 diagonal sub-block right-looking with each lane's row
//      in registers (a column step: a shuffle of the pivot, one reciprocal square root,
//      the column broadcast through shared memory and independent FMAs, no CTA barrier);
//   2. warp 0 inverts that sub-block (each lane a column, in registers) while warps 1-3
//      solve the rows below it (each thread a row, in registers), both right-looking
//      substitutions reading L through shared-memory broadcasts;
//   3. all threads apply the rank-32 update to the trailing triangle (register tiles).
// inv(L) is then merged from the 32-block inverses: two 64-blocks at once, then the
// 128-block (X = -inv(D) C inv(A) at each merge).
template <class T>
__global__ void __launch_bounds__(256, 1) potrf_diag(View<T> A, int sz, int64_t g0, T* W, int* info,
                                                     bool w_row_major) {
    extern __shared__ double S[];
    double* rd = S + NB * SLD;
    double* Tm = rd + NB;
    int* fail = reinterpret_cast<int*>(Tm + 64 * 65);
    if (aborted(info)) return;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const bool rowmaj = A.cs == 1;
    // The block into shared memory, 16 loads per thread in flight at a time (the block was
    // just written by the previous update and comes from L2: one round trip per batch).
    constexpr int kPer = NB * NB / 256, kBatch = 16;
    static_assert(kPer % kBatch == 0, "load batches");
#pragma unroll 1
    for (int b0 = 0; b0 < kPer; b0 += kBatch) {
        double v[kBatch];
#pragma unroll
        for (int u = 0; u < kBatch; ++u) {
            const int e = tid + 256 * (b0 + u);
            const int i = rowmaj ? e / NB : e % NB, c = rowmaj ? e % NB : e / NB;
            v[u] = (i < sz && c < sz && c <= i) ? (double)A(i, c) : (i == c ? 1.0 : 0.0);
        }
#pragma unroll
        for (int u = 0; u < kBatch; ++u) {
            const int e = tid + 256 * (b0 + u);
            const int i = rowmaj ? e / NB : e % NB, c = rowmaj ? e % NB : e / NB;
            S[i * SLD + c] = v[u];
        }
    }
    if (tid == 0) *fail = 0;
    __syncthreads();
#pragma unroll 1
    for (int kb = 0; kb < NB / DB; ++kb) {
        const int c0 = DB * kb;
        if (warp == 0) {  // 1. right-looking factor of the diagonal sub-block, row `lane` in registers
            const int i = c0 + lane;
            double a[DB];
#pragma unroll
            for (int c = 0; c < DB; ++c) a[c] = c <= lane ? S[i * SLD + c0 + c] : 0.0;
            int bad = -1;  // first non-positive pivot (uniform across the warp); later steps run on 1
            double* colj = Tm;  // column j of L, broadcast through shared memory
#pragma unroll
            for (int j = 0; j < DB; ++j) {
                double d = __shfl_sync(0xffffffffu, a[j], j);
                if (!(d > 0.0)) {  // also catches NaN
                    if (bad < 0) bad = j;
                    d = 1.0;
                }
                const double r = rsqrt(d);
                const double l = lane == j ? d * r : a[j] * r;  // L(i, j); zero above the diagonal
                a[j] = l;
                if (lane == j) rd[c0 + j] = r;
                colj[lane] = l;
                __syncwarp();
#pragma unroll
                for (int c = 0; c < DB; ++c) {
                    if (c <= j) continue;
                    // a(i, c) -= L(i, j) L(c, j); lanes above the diagonal only touch their
                    // upper-triangle entries, which are neither read nor written back
                    a[c] = fma(-l, colj[c], a[c]);
                }
                __syncwarp();
            }
            if (bad >= 0) {
                if (lane == 0) {
                    record_first(info, (int)(g0 + c0 + bad + 1));
                    *fail = 1;
                }
            } else {
#pragma unroll
                for (int c = 0; c < DB; ++c)
                    if (c <= lane) S[i * SLD + c0 + c] = a[c];
            }
        }
        __syncthreads();
        if (*fail) return;
        if (warp == 0) {  // 2a. inverse of the sub-block, column `lane` in registers
            double x[DB];
#pragma unroll
            for (int q = 0; q < DB; ++q) x[q] = q == lane ? 1.0 : 0.0;
#pragma unroll
            for (int m = 0; m < DB; ++m) {
                x[m] *= rd[c0 + m];
#pragma unroll
                for (int q = m + 1; q < DB; ++q) x[q] = fma(-S[(c0 + q) * SLD + c0 + m], x[m], x[q]);
            }
#pragma unroll
            for (int q = 0; q < DB; ++q)
                if (q > lane) S[(c0 + lane) * SLD + c0 + q] = x[q];
        } else if (tid - 32 < NB - c0 - DB) {  // 2b. one row below the sub-block per thread
            const int i = c0 + DB + (tid - 32);
            double r[DB];
#pragma unroll
            for (int c = 0; c < DB; ++c) r[c] = S[i * SLD + c0 + c];
#pragma unroll
            for (int j = 0; j < DB; ++j) {
                r[j] *= rd[c0 + j];
#pragma unroll
                for (int c = j + 1; c < DB; ++c) r[c] = fma(-r[j], S[(c0 + c) * SLD + c0 + j], r[c]);
            }
#pragma unroll
            for (int c = 0; c < DB; ++c) S[i * SLD + c0 + c] = r[c];
        }
        __syncthreads();
        if (kb == 0) trailing_update<0>(S);  // 3.
        else if (kb == 1) trailing_update<1>(S);
        else if (kb == 2) trailing_update<2>(S);
        __syncthreads();
    }
    // L back to global memory (lower part).
    for (int e = tid; e < NB * NB; e += 256) {
        const int i = rowmaj ? e / NB : e % NB, c = rowmaj ? e % NB : e / NB;
        if (i < sz && c <= i) A(i, c) = (T)S[i * SLD + c];
    }
    __syncthreads();
    // inv(L): the inverse's diagonal replaces L's, then 32-blocks -> 64-blocks (two merges,
    // 128 threads each) -> the 128-block.
    if (tid < NB) S[tid * SLD + tid] = rd[tid];
    __syncthreads();
    double* Th = Tm + (tid >= 128 ? 32 * 65 : 0);
    inverse_merge<32, 128>(S, Th, tid >= 128 ? 64 : 0, tid & 127, 0);
    __syncthreads();
    inverse_merge<32, 128>(S, Th, tid >= 128 ? 64 : 0, tid & 127, 1);
    __syncthreads();
    inverse_merge<64, 256>(S, Tm, 0, tid, 0);
    __syncthreads();
    inverse_merge<64, 256>(S, Tm, 0, tid, 1);
    __syncthreads();
    for (int e = tid; e < NB * NB; e += 256) {
        const int i = w_row_major ? e / NB : e % NB, c = w_row_major ? e % NB : e / NB;
        const double v = S[c * SLD + i];
        W[e] = (T)(i >= c ? v : 0.0);
    }
}

template <class K>
int set_smem(K kernel, size_t bytes) {
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) == cudaSuccess
               ? RC_SUCCESS
               : RC_ERR_CUDA;
}

}  // namespace

template <class T>
int trsm_left(bool upper, bool unit, int64_t m, int64_t n, T alpha, View<const T> A, View<T> B, int* info,
              cudaStream_t s, const int* abort) {
    if (m <= 0 || n <= 0) return RC_SUCCESS;
    const int64_t nblk = (m + NB - 1) / NB;
    T* W = static_cast<T*>(workspace(s, (size_t)nblk * NB * NB * sizeof(T), 1));
    T* tmp = static_cast<T*>(workspace(s, (size_t)NB * n * sizeof(T), 2));
    if (!W || !tmp) return RC_ERR_ALLOC;
    const View<const T> L = upper ? A.t() : A;
    RC_TRY(set_smem(trtri_blocks<T>, kBlockSmem));
    trtri_blocks<T><<<(unsigned)nblk, NB, kBlockSmem, s>>>(m, L, unit, W, info, abort);
    RC_TRY(check_launch());
    if (alpha != T(1)) RC_TRY(copy2d<T, T>(m, n, alpha, View<const T>{B.p, B.rs, B.cs}, B, s, abort));
    const View<T> Tv = colmajor(tmp, (int64_t)NB);
    for (int64_t step = 0; step < nblk; ++step) {
        const int64_t b = upper ? nblk - 1 - step : step;
        const int64_t r0 = b * NB, sz = (m - r0 < NB) ? m - r0 : NB;
        const View<const T> X = {W + (size_t)b * NB * NB, 1, NB};
        View<T> Bb = B.sub(r0, 0);
        RC_TRY(gemm<T>(sz, n, sz, T(1), upper ? X.t() : X, View<const T>{Bb.p, Bb.rs, Bb.cs}, T(0), Tv, kFull, 0, s,
                       abort));
        RC_TRY(copy2d<T, T>(sz, n, T(1), View<const T>{Tv.p, Tv.rs, Tv.cs}, Bb, s, abort));
        const View<const T> Bc = {Bb.p, Bb.rs, Bb.cs};
        if (!upper && r0 + sz < m)
            RC_TRY(gemm<T>(m - r0 - sz, n, sz, T(-1), A.sub(r0 + sz, r0), Bc, T(1), B.sub(r0 + sz, 0), kFull, 0, s,
                           abort));
        if (upper && r0 > 0) RC_TRY(gemm<T>(r0, n, sz, T(-1), A.sub(0, r0), Bc, T(1), B, kFull, 0, s, abort));
    }
    return RC_SUCCESS;
}

template <class T>
int potrf_lower(int64_t n, View<T> A, int* info, cudaStream_t s) {
    if (!info) return RC_ERR_INVALID_ARGUMENT;
    if (cudaMemsetAsync(info, 0, sizeof(int), s) != cudaSuccess) return RC_ERR_CUDA;
    if (n <= 0) return RC_SUCCESS;
    T* W = static_cast<T*>(workspace(s, (size_t)NB * NB * sizeof(T), 1));
    if (!W) return RC_ERR_ALLOC;
    // FP64 panels run on the 128x128 DMMA tile, so one CTA owns every column of a panel
    // row block and the panel solve can write in place; other types go through a buffer.
    constexpr bool in_place = std::is_same<T, double>::value;
    T* tmp = nullptr;
    if (!in_place) {
        tmp = static_cast<T*>(workspace(s, (size_t)n * NB * sizeof(T), 2));
        if (!tmp) return RC_ERR_ALLOC;
    }
    RC_TRY(set_smem(potrf_diag<T>, kDiagSmem));
    const View<const T> Wt = {W, NB, 1};  // inv(L_jj)^T
    // Outer panels of kOuter columns: inner 128-column blocks update only the rest of
    // their panel, and the trailing matrix gets one update of depth kOuter per panel, so
    // the dominant GEMM streams its C tiles kOuter / 128 times less often.
    constexpr int64_t kOuter = 512;
    auto C_ = [](const View<T>& v) { return View<const T>{v.p, v.rs, v.cs}; };
    for (int64_t k0 = 0; k0 < n; k0 += kOuter) {
        const int64_t w = (n - k0) < kOuter ? n - k0 : kOuter;
        for (int64_t j0 = k0; j0 < k0 + w; j0 += NB) {
            const int jb = (int)((k0 + w - j0) < NB ? k0 + w - j0 : NB);
            potrf_diag<T><<<1, 256, kDiagSmem, s>>>(A.sub(j0, j0), jb, j0, W, info, false);
            RC_TRY(check_launch());
            const int64_t rows = n - j0 - jb;
            if (rows <= 0) continue;
            View<T> P = A.sub(j0 + jb, j0);
            if (in_place) {
                RC_TRY(gemm<T>(rows, jb, jb, T(1), C_(P), Wt, T(0), P, kFull, 0, s, info));
            } else {
                const View<T> Tv = colmajor(tmp, rows);
                RC_TRY(gemm<T>(rows, jb, jb, T(1), C_(P), Wt, T(0), Tv, kFull, 0, s, info));
                RC_TRY(copy2d<T, T>(rows, jb, T(1), C_(Tv), P, s, info));
            }
            const int64_t cw = k0 + w - (j0 + jb);
            if (cw > 0)
                RC_TRY(gemm<T>(rows, cw, jb, T(-1), C_(P), C_(P).t(), T(1), A.sub(j0 + jb, j0 + jb), kLower, 0, s,
                               info));
        }
        const int64_t rows = n - k0 - w;
        if (rows <= 0) continue;
        const View<T> Pk = A.sub(k0 + w, k0);
        RC_TRY(gemm<T>(rows, rows, w, T(-1), C_(Pk), C_(Pk).t(), T(1), A.sub(k0 + w, k0 + w), kLower, 0, s, info));
    }
    return RC_SUCCESS;
}

template <class T>
int potrf_diag_block(View<T> A, int sz, int64_t g0, T* W, bool w_row_major, int* info, cudaStream_t s) {
    RC_TRY(set_smem(potrf_diag<T>, kDiagSmem));
    potrf_diag<T><<<1, 256, kDiagSmem, s>>>(A, sz, g0, W, info, w_row_major);
    return check_launch();
}

template <class T>
int trsm_preinv(bool trans, int64_t m, int64_t n, View<const T> L, const T* Winv, View<T> B, T* tmp, cudaStream_t s) {
    if (m <= 0 || n <= 0) return RC_SUCCESS;
    const int64_t nblk = (m + NB - 1) / NB;
    const View<T> Tv = colmajor(tmp, (int64_t)NB);
    const View<const T> Tc = {tmp, 1, (int64_t)NB};
    for (int64_t step = 0; step < nblk; ++step) {
        const int64_t b = trans ? nblk - 1 - step : step;
        const int64_t r0 = b * NB, sz = (m - r0 < NB) ? m - r0 : NB;
        const View<const T> X = {Winv + (size_t)b * NB * NB, NB, 1};
        View<T> Bb = B.sub(r0, 0);
        const View<const T> Bc = {Bb.p, Bb.rs, Bb.cs};
        RC_TRY(gemm<T>(sz, n, sz, T(1), trans ? X.t() : X, Bc, T(0), Tv, kFull, 0, s));
        RC_TRY(copy2d<T, T>(sz, n, T(1), Tc, Bb, s));
        if (!trans && r0 + sz < m)
            RC_TRY(gemm<T>(m - r0 - sz, n, sz, T(-1), L.sub(r0 + sz, r0), Bc, T(1), B.sub(r0 + sz, 0), kFull, 0, s));
        if (trans && r0 > 0) RC_TRY(gemm<T>(r0, n, sz, T(-1), L.sub(r0, 0).t(), Bc, T(1), B, kFull, 0, s));
    }
    return RC_SUCCESS;
}

template <class T>
int trtri_blocks_launch(int64_t m, View<const T> L, bool unit, T* W, int* info, const int* abort, cudaStream_t s) {
    if (m <= 0) return RC_SUCCESS;
    RC_TRY(set_smem(trtri_blocks<T>, kBlockSmem));
    trtri_blocks<T><<<(unsigned)((m + NB - 1) / NB), NB, kBlockSmem, s>>>(m, L, unit, W, info, abort);
    return check_launch();
}

template int trtri_blocks_launch<double>(int64_t, View<const double>, bool, double*, int*, const int*, cudaStream_t);
template int potrf_diag_block<float>(View<float>, int, int64_t, float*, bool, int*, cudaStream_t);
template int potrf_diag_block<double>(View<double>, int, int64_t, double*, bool, int*, cudaStream_t);
template int trsm_preinv<float>(bool, int64_t, int64_t, View<const float>, const float*, View<float>, float*,
                                cudaStream_t);
template int trsm_preinv<double>(bool, int64_t, int64_t, View<const double>, const double*, View<double>, double*,
                                 cudaStream_t);
template int trsm_left<double>(bool, bool, int64_t, int64_t, double, View<const double>, View<double>, int*,
                               cudaStream_t, const int*);
template int trsm_left<float>(bool, bool, int64_t, int64_t, float, View<const float>, View<float>, int*,
                              cudaStream_t, const int*);
template int potrf_lower<double>(int64_t, View<double>, int*, cudaStream_t);
template int potrf_lower<float>(int64_t, View<float>, int*, cudaStream_t);

}  // namespace rc

namespace {

template <class T>
int trsm_abi(int left, int upper, int trans, int unit, size_t m, size_t n, T alpha, const T* A, size_t lda, T* B,
             size_t ldb, int* d_info, void* stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (d_info && cudaMemsetAsync(d_info, 0, sizeof(int), s) != cudaSuccess) return RC_ERR_CUDA;
    if (m == 0 || n == 0) return RC_SUCCESS;
    const size_t na = left ? m : n;
    if (!A || !B || lda < na || ldb < m) return RC_ERR_INVALID_ARGUMENT;
    rc::View<const T> a = rc::colmajor(A, (int64_t)lda);
    bool up = upper != 0;
    if (trans) { a = a.t(); up = !up; }
    rc::View<T> b = rc::colmajor(B, (int64_t)ldb);
    if (left) return rc::trsm_left<T>(up, unit != 0, (int64_t)m, (int64_t)n, alpha, a, b, d_info, s);
    // B op(A)^-1: solve op(A)^T X^T = alpha B^T on the left.
    return rc::trsm_left<T>(!up, unit != 0, (int64_t)n, (int64_t)m, alpha, a.t(), b.t(), d_info, s);
}

template <class T>
int potrf_abi(int upper, size_t n, T* A, size_t lda, int* d_info, void* stream) {
    if (!d_info) return RC_ERR_INVALID_ARGUMENT;
    if (n > 0 && (!A || lda < n)) return RC_ERR_INVALID_ARGUMENT;
    rc::View<T> a = rc::colmajor(A, (int64_t)lda);
    if (upper) a = a.t();
    return rc::potrf_lower<T>((int64_t)n, a, d_info, static_cast<cudaStream_t>(stream));
}

}  // namespace

extern "C" {

int rc_trsm_f64(int left, int upper, int trans, int unit, size_t m, size_t n, double alpha, const double* A,
                size_t lda, double* B, size_t ldb, int* d_info, void* stream) {
    return trsm_abi<double>(left, upper, trans, unit, m, n, alpha, A, lda, B, ldb, d_info, stream);
}
int rc_trsm_f32(int left, int upper, int trans, int unit, size_t m, size_t n, float alpha, const float* A,
                size_t lda, float* B, size_t ldb, int* d_info, void* stream) {
    return trsm_abi<float>(left, upper, trans, unit, m, n, alpha, A, lda, B, ldb, d_info, stream);
}
int rc_potrf_f64(int upper, size_t n, double* A, size_t lda, int* d_info, void* stream) {
    return potrf_abi<double>(upper, n, A, lda, d_info, stream);
}
int rc_potrf_f32(int upper, size_t n, float* A, size_t lda, int* d_info, void* stream) {
    return potrf_abi<float>(upper, n, A, lda, d_info, stream);
}

int rc_spd_solve_f64(size_t n, size_t nrhs, const double* A, size_t lda, double* B, size_t ldb, int* d_info,
                     void* stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (!d_info) return RC_ERR_INVALID_ARGUMENT;
    if (n == 0) return cudaMemsetAsync(d_info, 0, sizeof(int), s) == cudaSuccess ? RC_SUCCESS : RC_ERR_CUDA;
    if (!A || lda < n || (nrhs > 0 && (!B || ldb < n))) return RC_ERR_INVALID_ARGUMENT;
    // The reference copies A into the decomposition's own storage (decompositions.hpp:81-84).
    double* L = static_cast<double*>(rc::workspace(s, n * n * sizeof(double), 3));
    if (!L) return RC_ERR_ALLOC;
    const rc::View<double> Lv = rc::colmajor(L, (int64_t)n);
    RC_TRY(rc::copy2d<double, double>((int64_t)n, (int64_t)n, 1.0, rc::colmajor(A, (int64_t)lda), Lv, s));
    RC_TRY(rc::potrf_lower<double>((int64_t)n, Lv, d_info, s));
    if (nrhs == 0) return RC_SUCCESS;
    const rc::View<const double> Lc = {L, 1, (int64_t)n};
    const rc::View<double> Bv = rc::colmajor(B, (int64_t)ldb);
    RC_TRY(rc::trsm_left<double>(false, false, (int64_t)n, (int64_t)nrhs, 1.0, Lc, Bv, nullptr, s, d_info));
    return rc::trsm_left<double>(true, false, (int64_t)n, (int64_t)nrhs, 1.0, Lc.t(), Bv, nullptr, s, d_info);
}

}  // extern "C"
