// Mixed-precision refined SPD solve: an extension on top of the reference's
// cholesky_decomposition + solve (include/remora/decompositions.hpp:81-105), with no
// reference counterpart of its own.
//
//  1. Equilibrate and shift: W = fl32(S A S) + theta I with S = diag(A)^(-1/2), stored as
//     an FP32 row-major working copy (so every panel row is contiguous: the K-major layout
//     the tcgen05 GEMM reads through TMA). theta = shift_factor * u_f (u_f = 2^-11 for TF32,
//     2^-8 for BF16) keeps the low-precision factorisation from breaking down on
//     ill-conditioned A (Higham & Pranesh 2021, diagonal scaling + shift).
//  2. Factor W = L L^T, blocked right-looking: outer panels of `outer` columns, inner
//     128-column blocks whose diagonal block is factored (and inverted) in FP64 shared
//     memory; the panel below is solved with that inverse on the TF32 tensor cores; the
//     updates inside the panel and the trailing update run on the tcgen05 tensor cores in
//     TF32 or BF16 with FP32 accumulation (BF16 operands are packed per panel).
//  3. Refine in FP64: x0 = M^-1 b with M = S^-1 L L^T S^-1, then preconditioned conjugate
//     gradients on A (FP64 vectors, the FP32 factor as preconditioner), one independent
//     CG recurrence per right-hand side. The CG products A p and the starting residual
//     run on the int8 tensor cores on a digit split of A made in the same pass over A as
//     W (rows and columns scaled by 2^e_i >= sqrt(A_ii), which bounds every entry of an
//     SPD matrix; 56 bits below that bound, every digit product exact); every
//     residual that decides convergence is an FP64 DMMA product, and a failed check
//     moves the remaining products to the DMMA path too. Stopped per column when the
//     normwise backward error
//         ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf)
//     of the TRUE residual is at most tol (CG-based iterative refinement for SPD systems:
//     Higham & Pranesh 2021; GMRES-IR: Carson & Higham 2017/2018).
#include <cooperative_groups.h>

#include <cmath>
#include <cstdint>
#include <mutex>
#include <vector>

#include "assign.cuh"
#include "emu64.cuh"
#include "factor.cuh"
#include "gemm.cuh"
#include "mixed.cuh"
#include "ozaki.cuh"
#include "ozaki_digits.cuh"
#include "tc_gemm.cuh"

namespace cg = cooperative_groups;

namespace rc {
namespace {

// s_i = 1 / sqrt(A_ii) (1 where A_ii <= 0, which the factorisation then reports).
__global__ void diag_scale_kernel(int64_t n, View<const double> A, double* s) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double d = A(i, i);
        s[i] = d > 0.0 ? 1.0 / sqrt(d) : 1.0;
    }
}

// W[i * ldw + j] = fl32(s_i A(i, j) s_j) (+ theta on the diagonal) for the lower triangle
// (j <= i), through a 32 x 33 tile so reads of column-major A and writes of row-major W
// are both coalesced.
__global__ void __launch_bounds__(256) scale_to_f32_kernel(int64_t n, View<const double> A, const double* s,
                                                           double theta, float* W, int64_t ldw) {
    __shared__ float tile[32][33];
    const int64_t i0 = (int64_t)blockIdx.y * 32, j0 = (int64_t)blockIdx.x * 32;
    if (j0 > i0 + 31) return;  // tile strictly above the diagonal
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int r = ty; r < 32; r += 8) {  // read: consecutive threads walk i (A's unit stride)
        const int64_t i = i0 + tx, j = j0 + r;
        float v = 0.f;
        if (i < n && j < n && j <= i) v = (float)(s[i] * A(i, j) * s[j] + (i == j ? theta : 0.0));
        tile[r][tx] = v;
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {  // write: consecutive threads walk j (W's unit stride)
        const int64_t i = i0 + r, j = j0 + tx;
        if (i < n && j < n && j <= i) W[i * ldw + j] = tile[tx][r];
    }
}

// W64[i * ldw + j] = s_i A(i, j) s_j (+ theta on the diagonal) in FP64 for the lower
// triangle, through a 32 x 33 tile as scale_to_f32_kernel (the working copy of the
// factorisation whose trailing updates are digit products).
__global__ void __launch_bounds__(256) scale_to_f64_kernel(int64_t n, View<const double> A, const double* s,
                                                           double theta, double* W, int64_t ldw) {
    __shared__ double tile[32][33];
    const int64_t i0 = (int64_t)blockIdx.y * 32, j0 = (int64_t)blockIdx.x * 32;
    if (j0 > i0 + 31) return;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int r = ty; r < 32; r += 8) {
        const int64_t i = i0 + tx, j = j0 + r;
        double v = 0.0;
        if (i < n && j < n && j <= i) v = s[i] * A(i, j) * s[j] + (i == j ? theta : 0.0);
        tile[r][tx] = v;
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        const int64_t i = i0 + r, j = j0 + tx;
        if (i < n && j < n && j <= i) W[i * ldw + j] = tile[tx][r];
    }
}

// Z[:, j] = s .* R[:, j] for the c columns (column-major, leading dimensions ldr, ldz).
__global__ void col_scale_kernel(int64_t n, int64_t c, const double* s, const double* R, int64_t ldr, double* Z,
                                 int64_t ldz) {
    for (int64_t j = blockIdx.y; j < c; j += gridDim.y)
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
            Z[i + j * ldz] = s[i] * R[i + j * ldr];
}

// The first pass over A when the CG products run on its int8 digit split: one read of
// each 64-row x 128-column tile of column-major A (512 threads; a warp reads 64 rows of a
// column, 16 bytes per lane when A allows) writes
//  - W = fl32(S A S) + theta I on the tiles that meet the lower triangle (as
//    scale_to_f32_kernel: the same expression, zeros above the diagonal);
//  - the 8 digits of A_ij / 2^(e_i + e_j) (rexp from the diagonal) K-major, raising *flag
//    where an entry is not below its bound;
//  - per 128-column tile bx, the partial sums of |A_ij| of every row (rsum[bx * Mp + i]).
constexpr int kSplitRows = 64, kSplitThreads = 512;
__global__ void __launch_bounds__(kSplitThreads, 2) scale_split_kernel(int64_t n, const double* A, int64_t lda,
                                                                    const double* s, double theta, float* W,
                                                                    int64_t ldw, const int* rexp, int* flag,
                                                                    int8_t* Sa, int64_t Mp, int64_t ldk,
                                                                    double* rsum) {
    extern __shared__ double split_smem[];  // dynamic: above the 48 KB static limit
    double(*rs)[kSplitRows] = reinterpret_cast<double(*)[kSplitRows]>(split_smem);
    uint32_t(*sm)[kSplitRows][33] = reinterpret_cast<uint32_t(*)[kSplitRows][33]>(split_smem + 16 * kSplitRows);
    float(*wt)[129] = reinterpret_cast<float(*)[129]>(reinterpret_cast<uint32_t*>(sm) + kOzSlices * kSplitRows * 33);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t tiles_x = (n + 127) / 128;
    const int64_t bx = blockIdx.x % tiles_x, i0 = (int64_t)(blockIdx.x / tiles_x) * kSplitRows;
    const int64_t jb = bx * 128, j0 = jb + w * 8;
    const bool lower = W != nullptr && jb <= i0 + kSplitRows - 1;  // W null: digits and row sums only
    const bool vec = (lda % 2 == 0) && (reinterpret_cast<uintptr_t>(A) % 16 == 0);
    double x[2][8];  // rows i0 + 2 lane + h, columns j0 + c
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const int64_t j = j0 + c, ia = i0 + 2 * lane;
        if (vec && j < n && ia + 1 < n) {
            const double2 v = *reinterpret_cast<const double2*>(A + ia + j * lda);
            x[0][c] = v.x;
            x[1][c] = v.y;
        } else {
            x[0][c] = (j < n && ia < n) ? A[ia + j * lda] : 0.0;
            x[1][c] = (j < n && ia + 1 < n) ? A[ia + 1 + j * lda] : 0.0;
        }
    }
    int ej[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) ej[c] = j0 + c < n ? rexp[j0 + c] : 0;
    bool fine = true;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int row = 2 * lane + h;
        const int64_t i = i0 + row;
        const int e = rexp[i];
        double ra = 0.0;
#pragma unroll
        for (int c = 0; c < 8; ++c) ra += fabs(x[h][c]);
        rs[w][row] = ra;
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            uint32_t word[kOzSlices] = {};
#pragma unroll
            for (int c = 0; c < 4; ++c) fine &= digits(x[h][4 * q + c], e + ej[4 * q + c], word, c);
#pragma unroll
            for (int t = 0; t < kOzSlices; ++t) sm[t][row][w * 2 + q] = word[t];
        }
        if (lower) {
            const double si = i < n ? s[i] : 0.0;
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                const int64_t j = j0 + c;
                wt[row][w * 8 + c] =
                    (i < n && j < n && j <= i) ? (float)(si * x[h][c] * s[j] + (i == j ? theta : 0.0)) : 0.f;
            }
        }
    }
    if (!fine) atomicOr(flag, 1);
    __syncthreads();
    const int r = threadIdx.x >> 3, g = threadIdx.x & 7;
    const int64_t jw = jb + g * 16;
    if (jw < ldk) {
#pragma unroll
        for (int t = 0; t < kOzSlices; ++t) {
            const uint4 v = make_uint4(sm[t][r][4 * g], sm[t][r][4 * g + 1], sm[t][r][4 * g + 2], sm[t][r][4 * g + 3]);
            *reinterpret_cast<uint4*>(Sa + ((int64_t)t * Mp + i0 + r) * ldk + jw) = v;
        }
    }
    if (lower && i0 + r < n) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int64_t j = jw + 4 * q;
            if (j + 3 < ldw)
                *reinterpret_cast<float4*>(W + (i0 + r) * ldw + j) =
                    make_float4(wt[r][16 * g + 4 * q], wt[r][16 * g + 4 * q + 1], wt[r][16 * g + 4 * q + 2],
                                wt[r][16 * g + 4 * q + 3]);
        }
    }
    if (threadIdx.x < kSplitRows) {
        double t = 0.0;
#pragma unroll
        for (int q = 0; q < 16; ++q) t += rs[q][threadIdx.x];
        rsum[bx * Mp + i0 + threadIdx.x] = t;
    }
}
constexpr size_t kSplitSmem =
    16 * kSplitRows * sizeof(double) + kOzSlices * kSplitRows * 33 * 4 + kSplitRows * 129 * 4;

// out[i] = the row sums of |A|: rsum summed over the tile columns in a fixed order.
__global__ void row_sum_kernel(int64_t n, int64_t tiles_x, const double* rsum, int64_t Mp, double* out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double t = 0.0;
        for (int64_t b = 0; b < tiles_x; ++b) t += rsum[b * Mp + i];
        out[i] = t;
    }
}

// ||A||_inf of the symmetric A as the largest column sum of |A| (coalesced column walks).
__global__ void __launch_bounds__(256) col_abs_sum_kernel(int64_t n, View<const double> A, double* out) {
    __shared__ double red[256];
    for (int64_t j = blockIdx.x; j < n; j += gridDim.x) {
        double acc = 0.0;
        for (int64_t i = threadIdx.x; i < n; i += blockDim.x) acc += fabs(A(i, j));
        red[threadIdx.x] = acc;
        __syncthreads();
        for (int w = 128; w > 0; w >>= 1) {
            if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x == 0) out[j] = red[0];
        __syncthreads();
    }
}

// Per-column reductions of n x c column-major FP64 blocks: mode 0 max|u|, mode 1 u.v.
__global__ void __launch_bounds__(256) col_reduce_kernel(int64_t n, int64_t c, const double* U, int64_t ldu,
                                                         const double* V, int64_t ldv, int mode, double* out) {
    __shared__ double red[256];
    for (int64_t j = blockIdx.x; j < c; j += gridDim.x) {
        double acc = 0.0;
        for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
            const double u = U[i + j * ldu];
            acc = mode == 0 ? fmax(acc, fabs(u)) : fma(u, V[i + j * ldv], acc);
        }
        red[threadIdx.x] = acc;
        __syncthreads();
        for (int w = 128; w > 0; w >>= 1) {
            if (threadIdx.x < w)
                red[threadIdx.x] = mode == 0 ? fmax(red[threadIdx.x], red[threadIdx.x + w])
                                             : red[threadIdx.x] + red[threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x == 0) out[j] = red[0];
        __syncthreads();
    }
}

// Y[:, j] += a[j] * X[:, j] (sign folded into a).
__global__ void col_axpy_kernel(int64_t n, int64_t c, const double* a, const double* X, int64_t ldx, double* Y,
                                int64_t ldy) {
    for (int64_t j = blockIdx.y; j < c; j += gridDim.y) {
        const double aj = a[j];
        if (aj == 0.0) continue;
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
            Y[i + j * ldy] = fma(aj, X[i + j * ldx], Y[i + j * ldy]);
    }
}

// P[:, j] = Z[:, j] + b[j] * P[:, j] for active columns (b[j] >= 0); inactive: untouched.
__global__ void col_xpby_kernel(int64_t n, int64_t c, const double* b, const double* Z, int64_t ldz, double* P,
                                int64_t ldp) {
    for (int64_t j = blockIdx.y; j < c; j += gridDim.y) {
        const double bj = b[j];
        if (bj < 0.0) continue;
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
            P[i + j * ldp] = fma(bj, P[i + j * ldp], Z[i + j * ldz]);
    }
}

// ---------------------------------------------------------------------------------------
// Few-right-hand-side triangular solves with the FP32 factor (the CG preconditioner).
// After the factorisation the strict lower triangle of W is truncated to TF32 in place and
// the strict upper triangle receives the transpose (W(i, j) = L'(j, i) for j > i), so that
// both solve directions read contiguous ROW segments of W, K-major for the tensor cores:
//   forward  step b: R[r0+sz:]  -= L'[r0+sz:, r0:r0+sz] X_b   (rows of the lower part)
//   backward step b: R[:r0]     -= L'[r0:r0+sz, :r0]^T  X_b   (rows of the upper part)
// The preconditioner is therefore the fixed operator (L' L'^T)^-1 with L' = the factor's
// diagonal BS x BS blocks (exact FP32, applied through their inverses Y) and its
// off-diagonal blocks rounded down to TF32 -- symmetric and positive definite like
// (L L^T)^-1 and as close to A^-1 as the TF32 factor itself. The vectors stay FP32: each
// diagonal step writes X_b also as its exact TF32 split [X_hi; X_lo] (128 columns), and the
// update runs on the tcgen05 tensor cores as one TF32 GEMM against that 128-row operand
// whose two column halves are summed in the epilogue, i.e. L' times X to FP32 accuracy.
// Y holds the row-major inverses of the BS x BS diagonal blocks (BS = 1024, built once
// per solve from the 128-block inverses of the factorisation); block b occupies rows
// [b BS, (b + 1) BS) of the n x BS array Y. Right-hand sides, solutions and the split
// are column-major with leading dimension ldx (a multiple of 32), 64 columns per chunk
// (padding columns zero).
constexpr int RHS = 64;
constexpr int BS = 1024;  // diagonal block of the preconditioner solves
constexpr int UK = 32;    // K slice staged in shared memory

__device__ __forceinline__ float tf32_hi(float v) { return __uint_as_float(__float_as_uint(v) & 0xFFFFE000u); }

// T[:, j] = fl32(s .* R[:, j]) for j < c, zero for the padding columns up to gridDim.y;
// and back: Z = s .* T.
__global__ void to_f32_scaled_kernel(int64_t n, int64_t c, const double* s, const double* R, int64_t ldr, float* T,
                                     int64_t ldx) {
    const int64_t j = blockIdx.y;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        T[j * ldx + i] = j < c ? (float)(s[i] * R[i + j * ldr]) : 0.f;
}
__global__ void from_f32_scaled_kernel(int64_t n, int64_t c, const double* s, const float* T, int64_t ldx, double* Z,
                                       int64_t ldz) {
    const int64_t j = blockIdx.y;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        Z[i + j * ldz] = s[i] * (double)T[j * ldx + i];
}

// Strict lower triangle of W rounded down to TF32 in place and mirrored into the strict
// upper triangle. 32 x 32 tiles: the CTA of upper tile (bi, bj), bj >= bi, reads lower tile
// (bj, bi) into shared memory, then writes it back truncated and writes its transpose.
__global__ void mirror_lower_kernel(int64_t n, float* W, int64_t ldw) {
    __shared__ float tile[32][33];
    const int64_t bi = blockIdx.y, bj = blockIdx.x;
    if (bj < bi) return;
    for (int r = threadIdx.y; r < 32; r += 8) {  // lower tile rows bj*32 + r, columns bi*32 + tx
        const int64_t i = bj * 32 + r, j = bi * 32 + threadIdx.x;
        if (i < n && j <= i) tile[r][threadIdx.x] = W[i * ldw + j];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += 8) {
        const int64_t i = bj * 32 + r, j = bi * 32 + threadIdx.x;
        if (i < n && j < i) W[i * ldw + j] = tf32_hi(tile[r][threadIdx.x]);
    }
    for (int r = threadIdx.y; r < 32; r += 8) {  // upper tile rows bi*32 + r, columns bj*32 + tx
        const int64_t i = bi * 32 + r, j = bj * 32 + threadIdx.x;
        if (j < n && j > i) W[i * ldw + j] = tf32_hi(tile[threadIdx.x][r]);
    }
}

// Diagonal step X_b = M_b R_b for rows [0, sz) of one block: M_b(i, k) = Yb[i BS + k]
// (TRANS = false, forward) or Yb[k BS + i] (backward), R_b the block's rows of the
// right-hand sides. Writes X_b to Xp and its TF32 split to Xs (columns j and 64 + j).
// 64 threads, 16-row tiles: 8 column groups (columns 4 tx + {0..3} and 32 + 4 tx + {0..3})
// x 8 row pairs. K is split over the gridDim.y CTAs of a thread-block cluster (1, parts,
// 1), each taking a contiguous run of UK-slices staged in shared memory through registers
// (the next slice is fetched while the current one is multiplied); the partial tiles are
// summed through distributed shared memory in rank order (deterministic), each CTA
// finishing 16 / parts rows.
template <bool TRANS>
__global__ void __launch_bounds__(64) pre_diag_kernel(int sz, const float* Yb, const float* Rb, int64_t ldx, float* Xp,
                                                      float* Xs) {
    constexpr int NT = 64, TM = 2, UM = 16, UAP = UM + 4, XP = RHS + 4;
    constexpr int NA = UM * UK / 4 / NT;   // float4 of M per thread and slice (2)
    constexpr int NX = UK * RHS / 4 / NT;  // float4 of R per thread and slice (8)
    __shared__ __align__(16) float sm[UK * UAP + UK * XP];
    float* As = sm;             // As[k * UAP + i]
    float* Rs = sm + UK * UAP;  // Rs[k * XP + j]
    const int tid = threadIdx.x;
    const int i0 = blockIdx.x * UM;
    const int ty = tid / 8, tx = tid % 8;
    const int parts = gridDim.y, part = blockIdx.y;
    const int kper = ((sz + UK - 1) / UK + parts - 1) / parts * UK;  // whole slices per rank
    const int kb = part * kper < sz ? part * kper : sz;
    const int ke = kb + kper < sz ? kb + kper : sz;
    float4 a_reg[NA], x_reg[NX];
    auto fetch = [&](int k0) {
#pragma unroll
        for (int q = 0; q < NA; ++q) {
            const int e = tid + NT * q;
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (!TRANS) {  // row ii, k = 4 kq .. 4 kq + 3
                const int ii = e % UM, kq = e / UM;
                const int gi = i0 + ii, k = k0 + 4 * kq;
                if (gi < sz) {
                    const float* src = Yb + (int64_t)gi * BS + k;
                    if (k + 3 < ke) {
                        v = *reinterpret_cast<const float4*>(src);
                    } else {
                        if (k < ke) v.x = src[0];
                        if (k + 1 < ke) v.y = src[1];
                        if (k + 2 < ke) v.z = src[2];
                    }
                }
            } else {       // row k, rows of the tile 4 g4 .. 4 g4 + 3
                const int g4 = e % (UM / 4), k = k0 + e / (UM / 4);
                const int gi = i0 + 4 * g4;
                if (k < ke) {
                    const float* src = Yb + (int64_t)k * BS + gi;
                    if (gi + 3 < sz) {
                        v = *reinterpret_cast<const float4*>(src);
                    } else {
                        if (gi < sz) v.x = src[0];
                        if (gi + 1 < sz) v.y = src[1];
                        if (gi + 2 < sz) v.z = src[2];
                    }
                }
            }
            a_reg[q] = v;
        }
#pragma unroll
        for (int q = 0; q < NX; ++q) {  // column j, rows k .. k + 3 (column-major R)
            const int e = tid + NT * q;
            const int k = k0 + 4 * (e % (UK / 4)), j = e / (UK / 4);
            const float* src = Rb + (int64_t)j * ldx + k;
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (k + 3 < ke) {
                v = *reinterpret_cast<const float4*>(src);
            } else {
                if (k < ke) v.x = src[0];
                if (k + 1 < ke) v.y = src[1];
                if (k + 2 < ke) v.z = src[2];
            }
            x_reg[q] = v;
        }
    };
    auto stage = [&]() {
#pragma unroll
        for (int q = 0; q < NA; ++q) {
            const int e = tid + NT * q;
            if (!TRANS) {
                const int ii = e % UM, kq = e / UM;
                As[(4 * kq + 0) * UAP + ii] = a_reg[q].x;
                As[(4 * kq + 1) * UAP + ii] = a_reg[q].y;
                As[(4 * kq + 2) * UAP + ii] = a_reg[q].z;
                As[(4 * kq + 3) * UAP + ii] = a_reg[q].w;
            } else {
                const int g4 = e % (UM / 4), k = e / (UM / 4);
                *reinterpret_cast<float4*>(&As[k * UAP + 4 * g4]) = a_reg[q];
            }
        }
#pragma unroll
        for (int q = 0; q < NX; ++q) {
            const int e = tid + NT * q;
            const int k = 4 * (e % (UK / 4)), j = e / (UK / 4);
            Rs[(k + 0) * XP + j] = x_reg[q].x;
            Rs[(k + 1) * XP + j] = x_reg[q].y;
            Rs[(k + 2) * XP + j] = x_reg[q].z;
            Rs[(k + 3) * XP + j] = x_reg[q].w;
        }
    };
    float acc[TM][8];
#pragma unroll
    for (int u = 0; u < TM; ++u)
#pragma unroll
        for (int v = 0; v < 8; ++v) acc[u][v] = 0.f;
    if (kb < ke) fetch(kb);
    for (int k0 = kb; k0 < ke; k0 += UK) {
        stage();
        __syncthreads();
        if (k0 + UK < ke) fetch(k0 + UK);
#pragma unroll 4
        for (int k = 0; k < UK; ++k) {  // slices past ke are zero-filled
            const float a0 = As[k * UAP + TM * ty], a1 = As[k * UAP + TM * ty + 1];
            const float4 x0 = *reinterpret_cast<const float4*>(&Rs[k * XP + 4 * tx]);
            const float4 x1 = *reinterpret_cast<const float4*>(&Rs[k * XP + 32 + 4 * tx]);
            const float xv[8] = {x0.x, x0.y, x0.z, x0.w, x1.x, x1.y, x1.z, x1.w};
#pragma unroll
            for (int v = 0; v < 8; ++v) {
                acc[0][v] = fmaf(a0, xv[v], acc[0][v]);
                acc[1][v] = fmaf(a1, xv[v], acc[1][v]);
            }
        }
        __syncthreads();
    }
    auto emit = [&](int gi, int j, float v) {  // X_b(gi, j) and its split
        const float h = tf32_hi(v);
        Xp[(int64_t)j * ldx + gi] = v;
        Xs[(int64_t)j * ldx + gi] = h;
        Xs[(int64_t)(j + RHS) * ldx + gi] = v - h;
    };
    if (parts == 1) {
#pragma unroll
        for (int u = 0; u < TM; ++u) {
            const int gi = i0 + TM * ty + u;
            if (gi >= sz) continue;
#pragma unroll
            for (int v = 0; v < 8; ++v) emit(gi, (v < 4 ? 4 * tx : 32 + 4 * tx) + (v & 3), acc[u][v]);
        }
        return;
    }
    // Cluster reduction: partial tile (16 x 64, row-major) in this CTA's shared memory,
    // then rank p sums rows [p 16 / parts, (p + 1) 16 / parts) over ranks 0..parts-1.
#pragma unroll
    for (int u = 0; u < TM; ++u) {
        float* r = sm + (TM * ty + u) * RHS;
        *reinterpret_cast<float4*>(r + 4 * tx) = make_float4(acc[u][0], acc[u][1], acc[u][2], acc[u][3]);
        *reinterpret_cast<float4*>(r + 32 + 4 * tx) = make_float4(acc[u][4], acc[u][5], acc[u][6], acc[u][7]);
    }
    cg::cluster_group cluster = cg::this_cluster();
    cluster.sync();
    const int rows_per = UM / parts;
    for (int e = tid; e < rows_per * RHS; e += NT) {
        const int row = part * rows_per + e / RHS, col = e % RHS;
        float sum = 0.f;
        for (int q = 0; q < parts; ++q) sum += cluster.map_shared_rank(sm, q)[row * RHS + col];
        if (i0 + row < sz) emit(i0 + row, col, sum);
    }
    cluster.sync();  // the other ranks may still read this CTA's partial tile
}

// Split K over a cluster of up to 8 CTAs so that the launch fills about one wave of
// resident CTAs with at least two UK-slices per CTA.
template <bool TRANS>
int launch_pre_diag(int sz, const float* Yb, const float* Rb, int64_t ldx, float* Xp, float* Xs, cudaStream_t st) {
    static int slots = 0;
    if (slots == 0) {
        int per_sm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pre_diag_kernel<TRANS>, 64, 0) != cudaSuccess)
            return RC_ERR_CUDA;
        slots = (per_sm > 0 ? per_sm : 1) * sm_count();
    }
    const int tiles = (sz + 15) / 16;
    int parts = 1;
    while (parts < 8 && tiles * parts * 2 <= slots && sz >= parts * 2 * 2 * UK) parts *= 2;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)tiles, (unsigned)parts, 1);
    cfg.blockDim = dim3(64, 1, 1);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 1;
    attr[0].val.clusterDim.y = parts;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (cudaLaunchKernelEx(&cfg, pre_diag_kernel<TRANS>, sz, Yb, Rb, ldx, Xp, Xs) != cudaSuccess) return RC_ERR_CUDA;
    return check_launch();
}

// Solve L' X = R (bwd = false) or L'^T X = R (bwd = true) for one 64-column chunk
// (column-major, ld ldx): R is consumed (updated in place), X receives the solution, S
// (128 columns) holds each step's TF32 split of X_b.
int trsm_few(bool bwd, int64_t n, const float* W, int64_t ldw, const float* Y, float* R, float* X, float* S,
             int64_t ldx, cudaStream_t st) {
    if (ldw % 4 != 0 || ldx % 4 != 0 || reinterpret_cast<uintptr_t>(W) % 16 != 0 ||
        reinterpret_cast<uintptr_t>(Y) % 16 != 0 || reinterpret_cast<uintptr_t>(R) % 16 != 0 ||
        reinterpret_cast<uintptr_t>(X) % 16 != 0 || reinterpret_cast<uintptr_t>(S) % 16 != 0)
        return RC_ERR_INVALID_ARGUMENT;
    const int64_t nblk = (n + BS - 1) / BS;
    for (int64_t step = 0; step < nblk; ++step) {
        const int64_t b = bwd ? nblk - 1 - step : step;
        const int64_t r0 = b * BS;
        const int sz = (int)((n - r0) < BS ? n - r0 : BS);
        const float* Yb = Y + r0 * BS;
        if (bwd) RC_TRY(launch_pre_diag<true>(sz, Yb, R + r0, ldx, X + r0, S + r0, st));
        else RC_TRY(launch_pre_diag<false>(sz, Yb, R + r0, ldx, X + r0, S + r0, st));
        // rows [rb, re) of R -= W[rows, r0 : r0 + sz] (X_hi + X_lo)
        const int64_t rb = bwd ? 0 : r0 + sz, re = bwd ? r0 : n;
        if (re > rb)
            RC_TRY(gemm_tc_fold_kmajor(re - rb, sz, -1.f, W + rb * ldw + r0, ldw, S + r0, ldx, 1.f,
                                       View<float>{R + rb, 1, ldx}, st));
    }
    return RC_SUCCESS;
}

// Batched C_z (=, alpha) A_z B_z for the block-inverse merges, one z per grid.z, 64 x 64
// tiles of 256 threads (4 x 4 each). Operand z is at p + (z zr + i) ld + (z zc mod cm) + j:
// the merges of one level sit at every 2h-aligned position of the n x n factor, and the
// inverses of a BS block at its rows of the n x BS array Y.
struct BatchView {
    float* p;
    int64_t ld, zr, zc, cm;
    __device__ float* at(int64_t z, int64_t i, int64_t j) const { return p + (z * zr + i) * ld + (z * zc) % cm + j; }
};
// Merge level h: for each z with g = 2 h z, g + h < n, d = min(h, n - g - h):
//   step 0: T_z = C_z Ainv_z   (d x h, k = h)
//   step 1: X_z = -Dinv_z T_z  (d x h, k = d)
__global__ void __launch_bounds__(256) merge_gemm_kernel(int64_t n, int64_t h, int step, BatchView A, BatchView B,
                                                          BatchView C) {
    constexpr int BM = 64, BN = 64, BK = 16;
    __shared__ float sA[BK][BM + 1];
    __shared__ float sB[BK][BN + 1];
    const int64_t z = blockIdx.z, g = 2 * h * z;
    if (g + h >= n) return;
    const int64_t d = (n - g - h) < h ? n - g - h : h;
    const int64_t m = d, nn = h, k = step == 0 ? h : d;
    const int64_t m0 = (int64_t)blockIdx.y * BM, n0 = (int64_t)blockIdx.x * BN;
    if (m0 >= m) return;
    const int tid = threadIdx.x, tm = tid / 16, tn = tid % 16;
    float acc[4][4] = {};
    for (int64_t k0 = 0; k0 < k; k0 += BK) {
        for (int e = tid; e < BM * BK; e += 256) {
            const int kk = e % BK, mm = e / BK;  // A rows are K-contiguous
            sA[kk][mm] = (m0 + mm < m && k0 + kk < k) ? *A.at(z, m0 + mm, k0 + kk) : 0.f;
            const int nb = e % BN, kb = e / BN;  // B rows are N-contiguous
            sB[kb][nb] = (n0 + nb < nn && k0 + kb < k) ? *B.at(z, k0 + kb, n0 + nb) : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            float a[4], b[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) a[r] = sA[kk][tm + 16 * r];
#pragma unroll
            for (int c = 0; c < 4; ++c) b[c] = sB[kk][tn + 16 * c];
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int c = 0; c < 4; ++c) acc[r][c] = fmaf(a[r], b[c], acc[r][c]);
        }
        __syncthreads();
    }
    const float alpha = step == 0 ? 1.f : -1.f;
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int64_t i = m0 + tm + 16 * r, j = n0 + tn + 16 * c;
            if (i < m && j < nn) *C.at(z, i, j) = alpha * acc[r][c];
        }
}

// Y rows [q kNB, q kNB + kNB), columns (q kNB mod BS) + [0, kNB) <- the 128-block inverse q.
__global__ void place_inverses_kernel(int64_t n, const float* Winv, float* Y) {
    const int64_t q = blockIdx.y;
    const int64_t r0 = q * kNB, c0 = r0 % BS;
    const int64_t qs = (n - r0) < kNB ? n - r0 : kNB;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < qs * qs; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e / qs, j = e % qs;
        Y[(r0 + i) * BS + c0 + j] = Winv[q * kNB * kNB + i * kNB + j];
    }
}

// Inverses of the BS x BS diagonal blocks of L (row-major rows of the n x BS array Y, zero
// above the diagonal) from the 128-block inverses Winv: inv([A 0; C D]) = [inv(A) 0;
// -inv(D) C inv(A)  inv(D)], applied level by level (h = 128, 256, ..., BS / 2) to every
// block at once. T is an n x BS / 2 scratch array.
int build_block_inverses(int64_t n, const float* W, int64_t ldw, const float* Winv, float* Y, float* T,
                         cudaStream_t st) {
    const int64_t nblk = (n + BS - 1) / BS;
    if (cudaMemsetAsync(Y, 0, (size_t)nblk * BS * BS * sizeof(float), st) != cudaSuccess) return RC_ERR_CUDA;
    const int64_t nq = (n + kNB - 1) / kNB;
    place_inverses_kernel<<<dim3(16, (unsigned)nq), 256, 0, st>>>(n, Winv, Y);
    RC_TRY(check_launch());
    const int64_t big = INT64_MAX / 4;
    for (int64_t h = kNB; h < BS; h *= 2) {
        const int64_t nz = (n + 2 * h - 1) / (2 * h);
        const dim3 grid((unsigned)ceil_div(h, 64), (unsigned)ceil_div(h, 64), (unsigned)nz);
        // T_z (d x h, ld h) = C_z Ainv_z: C_z = L(g + h.., g..), Ainv_z = Y rows g.., cols g mod BS
        const BatchView C = {const_cast<float*>(W) + h * ldw, ldw, 2 * h, 2 * h, big};
        const BatchView Ainv = {Y, BS, 2 * h, 2 * h, BS};
        const BatchView Tv = {T, h, h, 0, big};
        merge_gemm_kernel<<<grid, 256, 0, st>>>(n, h, 0, C, Ainv, Tv);
        RC_TRY(check_launch());
        // X_z = -Dinv_z T_z: Dinv_z = Y rows g + h.., cols (g + h) mod BS; X_z = Y rows g + h.., cols g mod BS
        const BatchView Dinv = {Y + h * BS + h, BS, 2 * h, 2 * h, BS};
        const BatchView Xz = {Y + h * BS, BS, 2 * h, 2 * h, BS};
        merge_gemm_kernel<<<grid, 256, 0, st>>>(n, h, 1, Dinv, Tv, Xz);
        RC_TRY(check_launch());
    }
    return RC_SUCCESS;
}

dim3 vec_grid(int64_t n, int64_t c) {
    return dim3(ceil_div(n, 256) < 256u ? ceil_div(n, 256) : 256u, c < 65535 ? (unsigned)c : 65535u);
}

struct Buf {
    char* base;
    size_t used = 0;
    template <class T>
    T* take(size_t count) {
        T* p = reinterpret_cast<T*>(base + used);
        used += (count * sizeof(T) + 255) & ~size_t(255);
        return p;
    }
};

}  // namespace

// CG products on the int8 digit split of A: up to 64 right-hand sides, n large enough
// for the split (one pass over A) to pay off.
static bool sliced_products(int64_t n, int64_t nrhs) { return nrhs <= 64 && n >= 512 && n <= (1 << 21) - 128; }

int mixed_workspace_bytes(int64_t n, int64_t nrhs, int prec, int outer, size_t* bytes) {
    const int64_t ldw = (n + 31) / 32 * 32;
    const int64_t nblk = (n + kNB - 1) / kNB;
    // the panel width the solve uses (as normalised by spd_solve_mixed)
    int64_t ow = (outer > 0 && outer % kNB == 0) ? outer : 1024;
    if (prec == RC_PREC_EMU64 && ow > 4096) ow = 1024;
    size_t b = 0;
    auto add = [&](size_t x) { b += (x + 255) & ~size_t(255); };
    if (prec == RC_PREC_EMU64) {
        add((size_t)n * ldw * sizeof(double));           // W (FP64)
        add((size_t)nblk * kNB * kNB * sizeof(double));  // diagonal-block inverses (FP64)
        add(emu_panel_bytes(n, ow));                     // digit splits of two outer panels
        add(emu_panel_bytes(n, ow));
        add((size_t)kNB * nrhs * sizeof(double));        // TRSM tile buffer
    } else {
        add((size_t)n * ldw * sizeof(float));           // W
        add((size_t)nblk * kNB * kNB * sizeof(float));  // diagonal-block inverses
        if (prec == RC_PREC_BF16) {
            add((size_t)n * ((ow + 63) / 64 * 64) * 2);  // BF16 outer panels (two)
            add((size_t)n * ((ow + 63) / 64 * 64) * 2);
            add((size_t)n * kNB * 2);                    // BF16 128-column block
        }
        const size_t chunked = (size_t)ldw * ((nrhs + RHS - 1) / RHS) * RHS;  // 64-column chunks, ld ldw
        add(chunked * sizeof(float));                    // FP32 right-hand side of the preconditioner
        add(chunked * sizeof(float));                    // FP32 intermediate of the preconditioner
        add((size_t)ldw * 2 * RHS * sizeof(float));      // TF32 split of one solution block
        add((size_t)kNB * nrhs * sizeof(float));         // TRSM tile buffer
        add((size_t)((n + BS - 1) / BS) * BS * BS * sizeof(float));      // BS-block inverses
        add((size_t)((n + BS - 1) / BS) * BS * BS / 2 * sizeof(float));  // their scratch
    }
    add((size_t)n * sizeof(double));                    // s
    add((size_t)n * sizeof(double));                    // column sums
    for (int i = 0; i < 4; ++i) add((size_t)n * nrhs * sizeof(double));  // R, Z, P, Q
    add((size_t)8 * nrhs * sizeof(double));             // per-column scalars
    if (sliced_products(n, nrhs)) {
        add(ozaki_a_bytes(n, n));        // digit split of A
        add(ozaki_p_bytes(n, n, nrhs));  // digits of one product's right-hand side, partials
        add((size_t)((n + 127) / 128) * ((n + 127) / 128 * 128) * sizeof(double));  // row-sum partials
    }
    *bytes = b;
    return RC_SUCCESS;
}

namespace {

// One high-priority non-blocking stream per device for the factorisation's look-ahead
// (kept for the life of the process).
cudaStream_t lookahead_stream() {
    static cudaStream_t streams[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    if (!streams[dev]) {
        int lo = 0, hi = 0;
        if (cudaDeviceGetStreamPriorityRange(&lo, &hi) != cudaSuccess) return nullptr;
        cudaStream_t st = nullptr;
        if (cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, hi) != cudaSuccess) return nullptr;
        streams[dev] = st;
    }
    return streams[dev];
}

struct Mixed {
    int64_t n, nrhs, ldw, nblk;
    int prec;
    cudaStream_t s;
    const double* A;
    int64_t lda;
    float* W;
    float* Winv;
    void* Pb[2];  // BF16 outer panels, alternating
    void* Pi;     // BF16 128-column block of the panel steps
    int64_t ldpb;
    double* sc;
    double* colsum;
    double *R, *Z, *P, *Q;
    float* T32;   // FP32 right-hand sides / solutions of the preconditioner (ld ldv)
    float* T32b;  // its intermediate
    float* T32s;  // TF32 split of one block of the solution (128 columns)
    int64_t ldv;
    float* Y;  // BS-block inverses
    float* Tinv;
    float* tmp;
    double* dev_scalars;  // 8 x nrhs
    OzakiA oz;            // digit split of A (valid when use_oz)
    void* oz_p = nullptr; // one sliced product's buffers
    bool use_oz = false;
    int* errw = nullptr;  // the library's device error word (a timed-out wait sets it)
    // RC_PREC_EMU64: the FP64 working copy, its FP64 diagonal-block inverses (row-major),
    // the digit splits of two outer panels and the TRSM tile buffer of the preconditioner.
    double* W64 = nullptr;
    double* Winv64 = nullptr;
    void* Pe[2] = {nullptr, nullptr};
    EmuPanel pe[2];
    double* tmp64 = nullptr;
    View<const double> Av() const { return {A, 1, lda}; }
    View<float> Wv() const { return {W, ldw, 1}; }
    View<double> W64v() const { return {W64, ldw, 1}; }

    // The 128-column steps of one outer panel [k0, k0 + w) of the FP64 working copy, on
    // stream st: factor (and invert, row-major) the diagonal block, solve the rows below it
    // in place with that inverse on the 128 x 128 FP64 DMMA tile (one CTA owns every column
    // of a row block), update the rest of the panel's columns in FP64.
    int panel_chain64(int64_t k0, int64_t w, int* info, cudaStream_t st) {
        const View<double> Wm = W64v();
        for (int64_t j0 = k0; j0 < k0 + w; j0 += kNB) {
            const int jb = (int)((k0 + w - j0) < kNB ? k0 + w - j0 : kNB);
            double* Wb = Winv64 + (size_t)(j0 / kNB) * kNB * kNB;
            RC_TRY(potrf_diag_block<double>(Wm.sub(j0, j0), jb, j0, Wb, true, info, st));
            const int64_t rows = n - j0 - jb;
            if (rows <= 0) continue;
            const View<double> Pj = Wm.sub(j0 + jb, j0);
            const View<const double> Pc = {Pj.p, Pj.rs, Pj.cs};
            RC_TRY(gemm<double>(rows, jb, jb, 1.0, Pc, View<const double>{Wb, 1, kNB}, 0.0, Pj, kFull, 0, st, info));
            const int64_t cw = k0 + w - (j0 + jb);
            if (cw <= 0) continue;
            RC_TRY(gemm<double>(rows, cw, jb, -1.0, Pc, Pc.t(), 1.0, Wm.sub(j0 + jb, j0 + jb), kLower, 0, st, info));
        }
        return RC_SUCCESS;
    }

    // The look-ahead schedule of factor() with an FP64 working copy: each factored outer
    // panel is split into its int8 digits on the look-ahead stream, and T1 / T2 are digit-
    // product updates (emu_update) instead of TF32/BF16 GEMMs. Panel p's split lives in
    // Pe[p & 1]; the look-ahead stream has waited for T2(p - 2), its last reader, before it
    // splits panel p (it waits for T2(p - 1) before T1(p), and T2(p - 2) ran before that).
    int factor_emu(int outer, int* info) {
        cudaStream_t la = lookahead_stream();
        if (!la) return RC_ERR_CUDA;
        cudaEvent_t ev_fork, ev_packed, ev_t2, ev_join;
        if (cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&ev_packed, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&ev_t2, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming) != cudaSuccess)
            return RC_ERR_CUDA;
        struct Events {
            cudaEvent_t e[4];
            ~Events() { for (cudaEvent_t x : e) cudaEventDestroy(x); }
        } guard{{ev_fork, ev_packed, ev_t2, ev_join}};
        auto ok = [](cudaError_t e) { return e == cudaSuccess ? RC_SUCCESS : RC_ERR_CUDA; };
        RC_TRY(ok(cudaEventRecord(ev_fork, s)));
        RC_TRY(ok(cudaStreamWaitEvent(la, ev_fork, 0)));
        RC_TRY(panel_chain64(0, n < outer ? n : outer, info, la));
        bool t2_pending = false;
        for (int64_t p = 0, k0 = 0; k0 < n; ++p, k0 += outer) {
            const int64_t w = (n - k0 < outer) ? n - k0 : outer;
            const int64_t k1 = k0 + w, rows = n - k1;
            if (rows <= 0) break;
            EmuPanel& pn = pe[p & 1];
            RC_TRY(emu_panel_layout(rows, w, Pe[p & 1], &pn));
            RC_TRY(emu_slice_panel(pn, W64 + k1 * ldw + k0, ldw, la));
            RC_TRY(ok(cudaEventRecord(ev_packed, la)));
            if (t2_pending) RC_TRY(ok(cudaStreamWaitEvent(la, ev_t2, 0)));
            const int64_t w1 = rows < outer ? rows : outer;  // width of panel p + 1
            // T1: rows [k1, n) x columns [k1, k1 + w1) on the look-ahead stream
            RC_TRY(emu_update(pn, 0, 0, rows, w1, -1.0, 1.0, W64 + k1 * ldw + k1, ldw, true, la, info));
            // T2: rows and columns [k1 + w1, n) on the main stream
            const int64_t r2 = rows - w1;
            if (r2 > 0) {
                RC_TRY(ok(cudaStreamWaitEvent(s, ev_packed, 0)));
                RC_TRY(emu_update(pn, w1, w1, r2, r2, -1.0, 1.0, W64 + (k1 + w1) * ldw + (k1 + w1), ldw, true, s,
                                  info));
                RC_TRY(ok(cudaEventRecord(ev_t2, s)));
                t2_pending = true;
            } else {
                t2_pending = false;
            }
            RC_TRY(panel_chain64(k1, w1, info, la));
        }
        RC_TRY(ok(cudaEventRecord(ev_join, la)));
        return ok(cudaStreamWaitEvent(s, ev_join, 0));
    }

    // Zout = M^-1 Rin = S L^-T L^-1 S Rin, all in FP64, on st: block forward and backward
    // substitution with the FP64 diagonal-block inverses (trsm_preinv) on the FP64 factor.
    int precond_on64(const double* Rin, int64_t ldr, double* Zout, int64_t ldz, cudaStream_t st) {
        const dim3 g = vec_grid(n, nrhs);
        col_scale_kernel<<<g, 256, 0, st>>>(n, nrhs, sc, Rin, ldr, Zout, ldz);
        RC_TRY(check_launch());
        const View<const double> L = {W64, ldw, 1};
        RC_TRY(trsm_preinv<double>(false, n, nrhs, L, Winv64, colmajor(Zout, ldz), tmp64, st));
        RC_TRY(trsm_preinv<double>(true, n, nrhs, L, Winv64, colmajor(Zout, ldz), tmp64, st));
        col_scale_kernel<<<g, 256, 0, st>>>(n, nrhs, sc, Zout, ldz, Zout, ldz);
        return check_launch();
    }

    // The 128-column steps of one outer panel [k0, k0 + w), on stream st: factor (and
    // invert) the diagonal block in FP64, solve the rows below it with that inverse on the
    // TF32 tensor cores, update the rest of the panel's columns.
    int panel_chain(int64_t k0, int64_t w, int* info, cudaStream_t st) {
        const View<float> Wm = Wv();
        for (int64_t j0 = k0; j0 < k0 + w; j0 += kNB) {
            const int jb = (int)((k0 + w - j0) < kNB ? k0 + w - j0 : kNB);
            float* Wb = Winv + (size_t)(j0 / kNB) * kNB * kNB;
            RC_TRY(potrf_diag_block<float>(Wm.sub(j0, j0), jb, j0, Wb, true, info, st));
            const int64_t rows = n - j0 - jb;
            if (rows <= 0) continue;
            View<float> Pj = Wm.sub(j0 + jb, j0);
            // Panel solve in place: P <- P inv(L_jj)^T (TF32 tensor cores, one column tile).
            RC_TRY(gemm_tc_kmajor(false, rows, jb, jb, 1.f, Pj.p, ldw, Wb, kNB, 0.f, Pj, kFull, 0, st, info, 128));
            const int64_t cw = k0 + w - (j0 + jb);
            if (cw <= 0) continue;
            const void* op = Pj.p;
            int64_t ldo = ldw;
            if (prec == RC_PREC_BF16) {
                RC_TRY(pack_kmajor(rows, jb, View<const float>{Pj.p, Pj.rs, Pj.cs}, Pi, kNB, true, st));
                op = Pi;
                ldo = kNB;
            }
            RC_TRY(gemm_tc_kmajor(prec == RC_PREC_BF16, rows, cw, jb, -1.f, op, ldo, op, ldo, 1.f,
                                  Wm.sub(j0 + jb, j0 + jb), kLower, 0, st, info));
        }
        return RC_SUCCESS;
    }

    // Blocked right-looking factorisation with a look-ahead of one outer panel. With panel
    // p factored, the look-ahead stream (high priority) updates the columns of panel p + 1
    // (T1) and factors that panel while the main stream applies panel p to everything to
    // its right (T2, the bulk of the flops), so the latency-bound 128-column steps run in
    // the shadow of the trailing update:
    //   look-ahead: pack(p) -> rec(packed) -> wait(T2(p-1)) -> T1(p) -> chain(p + 1)
    //   main:       wait(packed) -> T2(p) -> rec(T2(p))      (T2 on CTA pairs, 256 x 256 tiles)
    // T1(p) and T2(p) write disjoint columns; T1(p) waits for T2(p - 1), whose columns
    // include panel p + 1's. BF16 panels are packed into two alternating buffers.
    int factor(int outer, int* info) {
        const View<float> Wm = Wv();
        cudaStream_t la = lookahead_stream();
        if (!la) return RC_ERR_CUDA;
        cudaEvent_t ev_fork, ev_packed, ev_t2, ev_join;
        if (cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&ev_packed, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&ev_t2, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming) != cudaSuccess)
            return RC_ERR_CUDA;
        struct Events {
            cudaEvent_t e[4];
            ~Events() { for (cudaEvent_t x : e) cudaEventDestroy(x); }
        } guard{{ev_fork, ev_packed, ev_t2, ev_join}};
        auto ok = [](cudaError_t e) { return e == cudaSuccess ? RC_SUCCESS : RC_ERR_CUDA; };
        RC_TRY(ok(cudaEventRecord(ev_fork, s)));
        RC_TRY(ok(cudaStreamWaitEvent(la, ev_fork, 0)));
        RC_TRY(panel_chain(0, n < outer ? n : outer, info, la));
        bool t2_pending = false;
        for (int64_t p = 0, k0 = 0; k0 < n; ++p, k0 += outer) {
            const int64_t w = (n - k0 < outer) ? n - k0 : outer;
            const int64_t k1 = k0 + w, rows = n - k1;
            if (rows <= 0) break;
            View<float> Pk = Wm.sub(k1, k0);
            const void* op = Pk.p;
            int64_t ldo = ldw;
            const bool bf16 = prec == RC_PREC_BF16;
            if (bf16) {
                op = Pb[p & 1];
                ldo = ldpb;
                RC_TRY(pack_kmajor(rows, w, View<const float>{Pk.p, Pk.rs, Pk.cs}, Pb[p & 1], ldpb, true, la));
            }
            RC_TRY(ok(cudaEventRecord(ev_packed, la)));
            if (t2_pending) RC_TRY(ok(cudaStreamWaitEvent(la, ev_t2, 0)));
            const int64_t w1 = rows < outer ? rows : outer;  // width of panel p + 1
            // T1: rows [k1, n) x columns [k1, k1 + w1) on the look-ahead stream
            RC_TRY(gemm_tc_kmajor(bf16, rows, w1, w, -1.f, op, ldo, op, ldo, 1.f, Wm.sub(k1, k1), kLower, 0, la, info));
            // T2: rows and columns [k1 + w1, n) on the main stream
            const int64_t r2 = rows - w1;
            if (r2 > 0) {
                const size_t esz = bf16 ? 2 : 4;
                const void* op2 = static_cast<const char*>(op) + (size_t)w1 * ldo * esz;
                RC_TRY(ok(cudaStreamWaitEvent(s, ev_packed, 0)));
                // Two SMs stay free of pair CTAs for the look-ahead's diagonal blocks.
                RC_TRY(gemm_tc_pair_kmajor(bf16, r2, r2, w, -1.f, op2, ldo, op2, ldo, 1.f, Wm.sub(k1 + w1, k1 + w1),
                                           kLower, 0, s, info, 2, true));
                RC_TRY(ok(cudaEventRecord(ev_t2, s)));
                t2_pending = true;
            } else {
                t2_pending = false;
            }
            RC_TRY(panel_chain(k1, w1, info, la));
        }
        RC_TRY(ok(cudaEventRecord(ev_join, la)));
        return ok(cudaStreamWaitEvent(s, ev_join, 0));
    }

    // Zout = M^-1 Rin = S L^-T L^-1 S Rin (FP64 in/out, FP32 triangular solves), on st.
    int precond_on(const double* Rin, int64_t ldr, double* Zout, int64_t ldz, cudaStream_t st) {
        if (W64) return precond_on64(Rin, ldr, Zout, ldz, st);
        const int64_t nch = (nrhs + RHS - 1) / RHS;  // 64-column chunks
        const dim3 g(ceil_div(n, 256) < 128u ? ceil_div(n, 256) : 128u, (unsigned)(nch * RHS));
        to_f32_scaled_kernel<<<g, 256, 0, st>>>(n, nrhs, sc, Rin, ldr, T32, ldv);
        RC_TRY(check_launch());
        for (int64_t q = 0; q < nch; ++q) {
            float* R1 = T32 + q * RHS * ldv;
            float* R2 = T32b + q * RHS * ldv;
            RC_TRY(trsm_few(false, n, W, ldw, Y, R1, R2, T32s, ldv, st));  // R2 = L'^-1 R1
            RC_TRY(trsm_few(true, n, W, ldw, Y, R2, R1, T32s, ldv, st));   // R1 = L'^-T R2
        }
        from_f32_scaled_kernel<<<dim3(g.x, (unsigned)nrhs), 256, 0, st>>>(n, nrhs, sc, T32, ldv, Zout, ldz);
        return check_launch();
    }

    // The CG preconditioner R -> Z is replayed as one CUDA graph: its ~6 n/128 small
    // launches per application would otherwise be bound by launch latency. Every buffer it
    // touches lies in the solve's workspace, so the instantiated graph is kept for later
    // solves with the same workspace, sizes and precision (g_graphs).
    const void* ws_base = nullptr;
    size_t ws_bytes = 0;
    int outer = 0;
    cudaGraphExec_t graph_exec = nullptr;
    size_t graph_kernels = 0;
    int precond_RZ();

    // Rout = B - A X: FP64 DMMA, or (sliced) on the int8 digit split of A.
    int residual(const double* B, int64_t ldb, const double* X, int64_t ldx, double* Rout, bool sliced = false) {
        RC_TRY(copy2d<double, double>(n, nrhs, 1.0, View<const double>{B, 1, ldb}, colmajor(Rout, n), s));
        if (sliced) return ozaki_gemm(oz, nrhs, -1.0, X, ldx, 1.0, Rout, n, oz_p, s);
        return gemm<double>(n, nrhs, n, -1.0, Av(), View<const double>{X, 1, ldx}, 1.0, colmajor(Rout, n), kFull, 0,
                            s);
    }

    int col_reduce(const double* U, int64_t ldu, const double* V, int64_t ldv, int mode, std::vector<double>& out,
                   double* dst) {
        col_reduce_kernel<<<(unsigned)(nrhs < 1024 ? nrhs : 1024), 256, 0, s>>>(n, nrhs, U, ldu, V, ldv, mode, dst);
        RC_TRY(check_launch());
        out.resize(nrhs);
        int e = 0;  // every host synchronisation of the refinement also reads the error word
        if (cudaMemcpyAsync(out.data(), dst, nrhs * sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaMemcpyAsync(&e, errw, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            return RC_ERR_CUDA;
        return e != 0 ? RC_ERR_TIMEOUT : RC_SUCCESS;
    }

    int upload(const std::vector<double>& v, double* dst) {
        return cudaMemcpyAsync(dst, v.data(), nrhs * sizeof(double), cudaMemcpyHostToDevice, s) == cudaSuccess
                   ? RC_SUCCESS
                   : RC_ERR_CUDA;
    }
};

// Instantiated preconditioner graphs, one per (device, workspace address), valid for the
// key it was built from: the workspace size (all buffers are carved from it in a fixed
// layout), the sizes, the precision, the panel width and the wait limit of the tensor-core
// kernels. A workspace belongs to one stream, whose calls are ordered, so a graph that a
// new key replaces ran last on the calling stream.
struct PrecondGraph {
    int dev;
    const void* base;
    size_t bytes;
    int64_t n, nrhs;
    int prec, outer;
    uint64_t limit_ns;
    cudaGraphExec_t exec;
    size_t kernels;
};
std::mutex g_graph_mutex;
std::vector<PrecondGraph> g_graphs;

int Mixed::precond_RZ() {
    if (!graph_exec) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess) return RC_ERR_CUDA;
        const uint64_t lim = wait_limit_ns();
        std::lock_guard<std::mutex> lock(g_graph_mutex);
        PrecondGraph* slot = nullptr;
        for (PrecondGraph& g : g_graphs)
            if (g.dev == dev && g.base == ws_base) slot = &g;
        if (slot && slot->bytes == ws_bytes && slot->n == n && slot->nrhs == nrhs && slot->prec == prec &&
            slot->outer == outer && slot->limit_ns == lim) {
            graph_exec = slot->exec;
            graph_kernels = slot->kernels;
        } else {
            cudaStream_t cs;
            if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) return RC_ERR_CUDA;
            const unsigned long long before = rc_launch_count();
            cudaGraph_t gr = nullptr;
            cudaGraphExec_t exec = nullptr;
            int st = RC_SUCCESS;
            if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed) != cudaSuccess) st = RC_ERR_CUDA;
            if (st == RC_SUCCESS) st = precond_on(R, n, Z, n, cs);
            if (cudaStreamEndCapture(cs, &gr) != cudaSuccess && st == RC_SUCCESS) st = RC_ERR_CUDA;
            cudaStreamDestroy(cs);
            const size_t kernels = (size_t)(rc_launch_count() - before);
            if (st == RC_SUCCESS && cudaGraphInstantiate(&exec, gr, 0) != cudaSuccess) st = RC_ERR_CUDA;
            if (gr) cudaGraphDestroy(gr);
            if (st != RC_SUCCESS) {
                cudaGetLastError();
                return st;
            }
            if (slot) {
                if (cudaStreamSynchronize(s) != cudaSuccess) return RC_ERR_CUDA;
                cudaGraphExecDestroy(slot->exec);
                *slot = {dev, ws_base, ws_bytes, n, nrhs, prec, outer, lim, exec, kernels};
            } else {
                g_graphs.push_back({dev, ws_base, ws_bytes, n, nrhs, prec, outer, lim, exec, kernels});
            }
            graph_exec = exec;
            graph_kernels = kernels;
        }
    }
    if (cudaGraphLaunch(graph_exec, s) != cudaSuccess) return RC_ERR_CUDA;
    for (size_t i = 0; i < graph_kernels; ++i) count_launch();
    return RC_SUCCESS;
}

}  // namespace

int spd_solve_mixed(int prec, int64_t n, int64_t nrhs, const double* A, int64_t lda, const double* B, int64_t ldb,
                    double* X, int64_t ldx, const rc_mixed_options* opt, int* d_info, rc_refine_info* out,
                    cudaStream_t s) {
    rc_mixed_options o = {};
    o.tol = 1e-15;
    o.max_iter = 100;
    o.outer = 1024;
    o.shift_factor = -1.0;
    if (opt) o = *opt;  // shift_factor < 0 selects the adaptive shift
    if (o.outer <= 0 || o.outer % kNB) o.outer = 1024;
    if (o.tol <= 0) o.tol = 1e-15;
    if (o.max_iter < 0) o.max_iter = 100;
    const bool emu = prec == RC_PREC_EMU64;
    if (emu && o.outer > 4096) o.outer = 1024;  // int32 digit sums: K * 7 * 127^2 < 2^31
    // u_f: the unit of the factor's trailing updates (about 2^-40 of the row maxima for
    // the 7-digit products).
    const double uf = prec == RC_PREC_BF16 ? std::ldexp(1.0, -8)
                      : emu               ? std::ldexp(1.0, -40)
                                          : std::ldexp(1.0, -11);
    // shift_factor < 0: adaptive -- theta = u_f / 4 first, then 2 and 16 u_f after a
    // breakdown of the low-precision factorisation. Measured CG steps at n = 16384 (TF32)
    // for theta = 0, u_f / 16, u_f / 4, u_f: kappa 1e2: 5, 5, 5, 6; kappa 1e4: 14, 14, 14,
    // 16; kappa 1e6: 191, 100, 83, 100 -- no shift starves the ill-conditioned case, a
    // full u_f over-damps the well-conditioned one.
    const bool adaptive = o.shift_factor < 0.0;
    double theta = adaptive ? 0.25 * uf : o.shift_factor * uf;

    // The error word is sticky: a timeout left by an earlier call (not yet read by
    // rc_device_status) would make every tensor-core kernel of this solve return at once.
    int* errw = error_word();
    if (!errw) return RC_ERR_ALLOC;
    {
        const int e = pending_error(s);
        if (e != RC_SUCCESS) return e;
    }
    size_t bytes = 0;
    mixed_workspace_bytes(n, nrhs, prec, o.outer, &bytes);
    char* base = static_cast<char*>(workspace(s, bytes, 6));
    if (!base) return RC_ERR_ALLOC;
    Buf buf{base};
    Mixed M;
    M.ws_base = base;
    M.ws_bytes = bytes;
    M.outer = o.outer;
    M.n = n; M.nrhs = nrhs; M.prec = prec; M.s = s; M.A = A; M.lda = lda; M.errw = errw;
    M.ldw = (n + 31) / 32 * 32;
    M.nblk = (n + kNB - 1) / kNB;
    M.ldv = (n + 31) / 32 * 32;
    M.ldpb = (o.outer + 63) / 64 * 64;
    M.W = nullptr;
    M.Winv = M.T32 = M.T32b = M.T32s = M.tmp = M.Y = M.Tinv = nullptr;
    M.Pb[0] = M.Pb[1] = M.Pi = nullptr;
    if (emu) {
        M.W64 = buf.take<double>((size_t)n * M.ldw);
        M.Winv64 = buf.take<double>((size_t)M.nblk * kNB * kNB);
        for (int q = 0; q < 2; ++q) M.Pe[q] = buf.take<char>(emu_panel_bytes(n, o.outer));
        M.tmp64 = buf.take<double>((size_t)kNB * nrhs);
    } else {
        M.W = buf.take<float>((size_t)n * M.ldw);
        M.Winv = buf.take<float>((size_t)M.nblk * kNB * kNB);
        for (int q = 0; q < 2; ++q)
            M.Pb[q] = prec == RC_PREC_BF16 ? static_cast<void*>(buf.take<uint16_t>((size_t)n * M.ldpb)) : nullptr;
        M.Pi = prec == RC_PREC_BF16 ? static_cast<void*>(buf.take<uint16_t>((size_t)n * kNB)) : nullptr;
        M.T32 = buf.take<float>((size_t)M.ldv * ((nrhs + RHS - 1) / RHS) * RHS);
        M.T32b = buf.take<float>((size_t)M.ldv * ((nrhs + RHS - 1) / RHS) * RHS);
        M.T32s = buf.take<float>((size_t)M.ldv * 2 * RHS);
        M.tmp = buf.take<float>((size_t)kNB * nrhs);
        M.Y = buf.take<float>((size_t)((n + BS - 1) / BS) * BS * BS);
        M.Tinv = buf.take<float>((size_t)((n + BS - 1) / BS) * BS * BS / 2);
    }
    M.sc = buf.take<double>(n);
    M.colsum = buf.take<double>(n);
    M.R = buf.take<double>((size_t)n * nrhs);
    M.Z = buf.take<double>((size_t)n * nrhs);
    M.P = buf.take<double>((size_t)n * nrhs);
    M.Q = buf.take<double>((size_t)n * nrhs);
    M.dev_scalars = buf.take<double>((size_t)8 * nrhs);
    void* oz_a = nullptr;
    double* rsum = nullptr;
    if (sliced_products(n, nrhs)) {
        oz_a = buf.take<char>(ozaki_a_bytes(n, n));
        M.oz_p = buf.take<char>(ozaki_p_bytes(n, n, nrhs));
        rsum = buf.take<double>((size_t)((n + 127) / 128) * ((n + 127) / 128 * 128));
    }

    struct Timers {  // destroyed on every return path
        cudaEvent_t e[3] = {nullptr, nullptr, nullptr};
        ~Timers() {
            for (cudaEvent_t x : e)
                if (x) cudaEventDestroy(x);
        }
    } tm;
    for (cudaEvent_t& x : tm.e)
        if (cudaEventCreate(&x) != cudaSuccess) return RC_ERR_CUDA;
    cudaEvent_t e0 = tm.e[0], e1 = tm.e[1], e2 = tm.e[2];
    if (cudaEventRecord(e0, s) != cudaSuccess) return RC_ERR_CUDA;
    const View<const double> Av = M.Av();
    diag_scale_kernel<<<ceil_div(n, 256) < 1024u ? ceil_div(n, 256) : 1024u, 256, 0, s>>>(n, Av, M.sc);
    RC_TRY(check_launch());
    int h_info = 0;
    for (int attempt = 0;; ++attempt) {
        if (cudaMemsetAsync(d_info, 0, sizeof(int), s) != cudaSuccess) return RC_ERR_CUDA;
        // The first attempt reads A once for W, the digit split and the row sums of |A|. (A
        // split run on another stream beside the factorisation slows its latency-bound
        // diagonal chain by more than the split costs.)
        if (attempt == 0 && oz_a && ozaki_layout_a(n, n, oz_a, true, &M.oz) == RC_SUCCESS) {
            RC_TRY(ozaki_diag_exponents(M.oz, A, lda, s));
            if (cudaFuncSetAttribute(scale_split_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)kSplitSmem) != cudaSuccess)
                return RC_ERR_CUDA;
            const int64_t tiles = ((n + 127) / 128) * (M.oz.Mp / kSplitRows);
            scale_split_kernel<<<(unsigned)tiles, kSplitThreads, kSplitSmem, s>>>(n, A, lda, M.sc, theta, M.W, M.ldw, M.oz.rexp,
                                                                        M.oz.flag, M.oz.slices, M.oz.Mp, M.oz.ldk,
                                                                        rsum);
            RC_TRY(check_launch());
            row_sum_kernel<<<ceil_div(n, 256) < 1024u ? ceil_div(n, 256) : 1024u, 256, 0, s>>>(
                n, (n + 127) / 128, rsum, M.oz.Mp, M.colsum);
            RC_TRY(check_launch());
            M.use_oz = true;
            if (emu) {
                scale_to_f64_kernel<<<dim3(ceil_div(n, 32), ceil_div(n, 32)), 256, 0, s>>>(n, Av, M.sc, theta, M.W64,
                                                                                          M.ldw);
                RC_TRY(check_launch());
            }
        } else if (emu) {
            scale_to_f64_kernel<<<dim3(ceil_div(n, 32), ceil_div(n, 32)), 256, 0, s>>>(n, Av, M.sc, theta, M.W64,
                                                                                      M.ldw);
            RC_TRY(check_launch());
        } else {
            scale_to_f32_kernel<<<dim3(ceil_div(n, 32), ceil_div(n, 32)), 256, 0, s>>>(n, Av, M.sc, theta, M.W,
                                                                                      M.ldw);
            RC_TRY(check_launch());
        }
        RC_TRY(emu ? M.factor_emu(o.outer, d_info) : M.factor(o.outer, d_info));
        int h_err = 0;
        if (cudaMemcpyAsync(&h_info, d_info, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaMemcpyAsync(&h_err, errw, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            return RC_ERR_CUDA;
        if (h_err != 0) return RC_ERR_TIMEOUT;  // a wait of the factorisation ran out
        if (h_info == 0 || !adaptive || attempt == 2) break;
        theta = (attempt == 0 ? 2.0 : 16.0) * uf;
    }
    if (cudaEventRecord(e1, s) != cudaSuccess) return RC_ERR_CUDA;
    rc_refine_info info = {};
    info.shift = theta;
    if (h_info != 0) {
        if (out) *out = info;
        return RC_SUCCESS;  // d_info reports the failing pivot of the low-precision factor
    }

    // ||A||_inf (the row sums of |A| from the first pass when the split ran, else the
    // column sums of the symmetric A), ||b||_inf per column.
    if (!M.use_oz) {
        col_abs_sum_kernel<<<(unsigned)(n < 4096 ? n : 4096), 256, 0, s>>>(n, Av, M.colsum);
        RC_TRY(check_launch());
    }
    std::vector<double> tmpv;
    {
        // max over the n column sums: reuse the column reduction with c = 1 on an n x 1 block
        col_reduce_kernel<<<1, 256, 0, s>>>(n, 1, M.colsum, n, nullptr, 0, 0, M.dev_scalars);
        RC_TRY(check_launch());
    }
    double normA = 0.0;
    int split_flag = 0;
    int h_err = 0;
    if (cudaMemcpyAsync(&normA, M.dev_scalars, sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        (M.use_oz && cudaMemcpyAsync(&split_flag, M.oz.flag, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess) ||
        cudaMemcpyAsync(&h_err, errw, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return RC_ERR_CUDA;
    if (h_err != 0) return RC_ERR_TIMEOUT;
    if (split_flag) M.use_oz = false;  // the diagonal did not bound A: FP64 DMMA products
    std::vector<double> normB, normX, normR, rz, pq, alpha(nrhs), beta(nrhs);
    RC_TRY(M.col_reduce(B, ldb, nullptr, 0, 0, normB, M.dev_scalars));

    // x0 = M^-1 b, after L^T is mirrored into W's upper triangle and the BS-block
    // inverses are built
    if (!emu) {
        const unsigned nt = ceil_div(n, 32);
        mirror_lower_kernel<<<dim3(nt, nt), dim3(32, 8), 0, s>>>(n, M.W, M.ldw);
        RC_TRY(check_launch());
        RC_TRY(build_block_inverses(n, M.W, M.ldw, M.Winv, M.Y, M.Tinv, s));
    }
    // x0 = M^-1 B through the same CUDA graph as the CG steps (R = B, Z = M^-1 R, X = Z):
    // the FP64 preconditioner of RC_PREC_EMU64 is ~6 n / 128 launches.
    RC_TRY(copy2d<double, double>(n, nrhs, 1.0, View<const double>{B, 1, ldb}, colmajor(M.R, n), s));
    RC_TRY(M.precond_RZ());
    RC_TRY(copy2d<double, double>(n, nrhs, 1.0, View<const double>{M.Z, 1, n}, View<double>{X, 1, ldx}, s));
    bool sliced = M.use_oz;  // CG products on the digit split until a convergence check fails
    std::vector<char> done(nrhs, 0);
    int iters = 0, residuals = 0;
    double worst = 0.0;
    bool restart = true;
    double* const Rm = M.R;
    const int64_t ldm = n;
    while (true) {
        if (restart) {
            // The starting residual may come from the digit split; a residual that ends
            // the solve (or checks a converged recurrence) is always an FP64 DMMA product.
            bool all = true;
            for (int pass = 0; pass < 2; ++pass) {
                const bool from_split = sliced && iters == 0 && pass == 0;
                RC_TRY(M.residual(B, ldb, X, ldx, Rm, from_split));
                ++residuals;
                RC_TRY(M.col_reduce(Rm, ldm, nullptr, 0, 0, normR, M.dev_scalars));
                RC_TRY(M.col_reduce(X, ldx, nullptr, 0, 0, normX, M.dev_scalars + nrhs));
                worst = 0.0;
                for (int64_t j = 0; j < nrhs; ++j) {
                    const double eta = normR[j] / (normA * normX[j] + normB[j]);
                    done[j] = !(eta > o.tol);
                    if (std::isfinite(eta)) worst = std::max(worst, eta);
                    else worst = INFINITY;
                }
                all = true;
                for (char d : done) all = all && d;
                if (!from_split || !(all || iters >= o.max_iter)) break;
            }
            if (iters > 0 && !all) sliced = false;
            if (all || iters >= o.max_iter) break;
            // (re)start CG from the true residual: Z = M^-1 R, P = Z, rz = R.Z
            RC_TRY(M.precond_RZ());
            RC_TRY(copy2d<double, double>(n, nrhs, 1.0, View<const double>{M.Z, 1, ldm}, colmajor(M.P, ldm), s));
            RC_TRY(M.col_reduce(Rm, ldm, M.Z, ldm, 1, rz, M.dev_scalars));
            restart = false;
        }
        // Q = A P; alpha = rz / (P.Q) on the active columns.
        if (sliced) RC_TRY(ozaki_gemm(M.oz, nrhs, 1.0, M.P, ldm, 0.0, M.Q, ldm, M.oz_p, s));
        else
            RC_TRY(gemm<double>(n, nrhs, n, 1.0, Av, View<const double>{M.P, 1, ldm}, 0.0, colmajor(M.Q, ldm),
                                kFull, 0, s));
        RC_TRY(M.col_reduce(M.P, ldm, M.Q, ldm, 1, pq, M.dev_scalars));
        for (int64_t j = 0; j < nrhs; ++j) alpha[j] = (done[j] || pq[j] <= 0.0) ? 0.0 : rz[j] / pq[j];
        RC_TRY(M.upload(alpha, M.dev_scalars + 2 * nrhs));
        const dim3 g = vec_grid(n, nrhs);
        col_axpy_kernel<<<g, 256, 0, s>>>(n, nrhs, M.dev_scalars + 2 * nrhs, M.P, ldm, X, ldx);
        for (int64_t j = 0; j < nrhs; ++j) alpha[j] = -alpha[j];
        RC_TRY(M.upload(alpha, M.dev_scalars + 3 * nrhs));
        col_axpy_kernel<<<g, 256, 0, s>>>(n, nrhs, M.dev_scalars + 3 * nrhs, M.Q, ldm, Rm, ldm);
        RC_TRY(check_launch());
        ++iters;
        // Convergence estimate from the recurrence residual; confirm with a true residual.
        RC_TRY(M.col_reduce(Rm, ldm, nullptr, 0, 0, normR, M.dev_scalars));
        RC_TRY(M.col_reduce(X, ldx, nullptr, 0, 0, normX, M.dev_scalars + nrhs));
        bool all = true;
        for (int64_t j = 0; j < nrhs; ++j) {
            if (done[j]) continue;
            const double eta = normR[j] / (normA * normX[j] + normB[j]);
            if (!(eta > 0.5 * o.tol)) done[j] = 1;
            all = all && done[j];
        }
        if (all || iters >= o.max_iter) {
            restart = true;  // verify with the true residual (and restart CG where it fails)
            continue;
        }
        // Z = M^-1 R; beta = rz_new / rz; P = Z + beta P
        RC_TRY(M.precond_RZ());
        std::vector<double> rz_new;
        RC_TRY(M.col_reduce(Rm, ldm, M.Z, ldm, 1, rz_new, M.dev_scalars));
        for (int64_t j = 0; j < nrhs; ++j) {
            beta[j] = done[j] ? -1.0 : (rz[j] != 0.0 ? rz_new[j] / rz[j] : 0.0);
            rz[j] = rz_new[j];
        }
        RC_TRY(M.upload(beta, M.dev_scalars + 4 * nrhs));
        col_xpby_kernel<<<g, 256, 0, s>>>(n, nrhs, M.dev_scalars + 4 * nrhs, M.Z, ldm, M.P, ldm);
        RC_TRY(check_launch());
    }
    if (cudaEventRecord(e2, s) != cudaSuccess || cudaEventSynchronize(e2) != cudaSuccess) return RC_ERR_CUDA;
    {
        const int e = pending_error(s);  // the last products ran after the last check
        if (e != RC_SUCCESS) return e;
    }
    float t_f = 0.f, t_r = 0.f;
    cudaEventElapsedTime(&t_f, e0, e1);
    cudaEventElapsedTime(&t_r, e1, e2);
    info.iterations = iters;
    info.residuals = residuals;
    info.backward_error = worst;
    info.converged = worst <= o.tol ? 1 : 0;
    info.factor_ms = t_f;
    info.refine_ms = t_r;
    info.shift = theta;
    if (out) *out = info;
    return info.converged ? RC_SUCCESS : RC_ERR_NOT_CONVERGED;
}

}  // namespace rc

extern "C" {

int rc_spd_solve_mixed(int precision, size_t n, size_t nrhs, const double* A, size_t lda, const double* B, size_t ldb,
                       double* X, size_t ldx, const rc_mixed_options* options, int* d_info, rc_refine_info* info,
                       void* stream) {
    if (precision != RC_PREC_TF32 && precision != RC_PREC_BF16 && precision != RC_PREC_EMU64)
        return RC_ERR_INVALID_ARGUMENT;
    if (!d_info) return RC_ERR_INVALID_ARGUMENT;
    if (n == 0 || nrhs == 0) return RC_SUCCESS;
    if (!A || !B || !X || lda < n || ldb < n || ldx < n) return RC_ERR_INVALID_ARGUMENT;
    if (n > (size_t)INT32_MAX) return RC_ERR_NOT_SUPPORTED;
    return rc::spd_solve_mixed(precision, (int64_t)n, (int64_t)nrhs, A, (int64_t)lda, B, (int64_t)ldb, X, (int64_t)ldx,
                               options, d_info, info, static_cast<cudaStream_t>(stream));
}

int rc_spd_solve_mixed_workspace(int precision, size_t n, size_t nrhs, const rc_mixed_options* options,
                                 size_t* bytes) {
    if (!bytes) return RC_ERR_INVALID_ARGUMENT;
    return rc::mixed_workspace_bytes((int64_t)n, (int64_t)nrhs, precision, options ? options->outer : 0, bytes);
}

}  // extern "C"
