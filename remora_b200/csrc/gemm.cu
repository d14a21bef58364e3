// Dense GEMM / SYRK for Remora's cuda_tag.
//
// Replaces the reference's cuBLAS calls behind kernels::gemm and kernels::syrk
// (include/remora/hip/cublas_backend.hpp:121-166, :389-431, called from
// include/remora/kernels/hip/gemm.hpp:46-112 and kernels/hip/syrk.hpp:44-85).
//
// Two kernels:
//  * gemm_dmma_f64: the FP64 tensor-core path (DMMA, mma.sync m16n8k4 f64). 128x128x16
//    CTA tiles, 8 warps of 64x32, a 3-stage cp.async pipeline. Operand tiles are staged
//    in shared memory in one canonical layout ([k][m] and [k][n], rows padded by 4
//    doubles so every fragment load of a half-warp hits 16 distinct 8-byte bank pairs);
//    the transposition that a K-major operand needs happens in the 8-byte cp.async
//    scatter, so all four transpose combinations share one inner loop.
//  * gemm_simt: a generic strided FP32/FP64 kernel (64x64x16 tiles, 4x4 outer products
//    per thread) for operands with no unit stride and for FP32.
// Both honour a triangle mask (SYRK writes one triangle; whole tiles outside it exit at
// once) and an abort word (a failed Cholesky pivot stops the trailing updates).
#include "gemm.cuh"
#include "tc_gemm.cuh"
#include <type_traits>

namespace rc {
namespace {

__device__ __forceinline__ bool aborted(const int* abort) { return abort != nullptr && *(volatile const int*)abort != 0; }

__device__ __forceinline__ bool tile_outside(Mask mask, int64_t off, int64_t m0, int64_t n0, int bm, int bn) {
    if (mask == kLower) return (m0 + bm - 1) - n0 - off < 0;
    if (mask == kUpper) return m0 - (n0 + bn - 1) - off > 0;
    return false;
}

__device__ __forceinline__ bool in_mask(Mask mask, int64_t off, int64_t i, int64_t j) {
    if (mask == kLower) return i - j >= off;
    if (mask == kUpper) return i - j <= off;
    return true;
}

// ------------------------------------------------------------------------------------
// Generic SIMT kernel.
template <class T>
__global__ void __launch_bounds__(256) gemm_simt(int64_t m, int64_t n, int64_t k, T alpha, View<const T> A,
                                                 View<const T> B, T beta, View<T> C, Mask mask, int64_t off,
                                                 const int* abort) {
    constexpr int BM = 64, BN = 64, BK = 16;
    __shared__ T sA[BK][BM + 1];
    __shared__ T sB[BK][BN + 1];
    const int64_t m0 = (int64_t)blockIdx.y * BM, n0 = (int64_t)blockIdx.x * BN;
    if (aborted(abort) || tile_outside(mask, off, m0, n0, BM, BN)) return;
    const int tid = threadIdx.x;
    const int tm = tid / 16, tn = tid % 16;  // 16 x 16 threads, 4 x 4 each
    T acc[4][4] = {};
    for (int64_t k0 = 0; k0 < k; k0 += BK) {
        for (int e = tid; e < BM * BK; e += 256) {
            // A tile: consecutive threads walk the unit-stride direction when there is one.
            int mm, kk;
            if (A.rs == 1) { mm = e % BM; kk = e / BM; } else { kk = e % BK; mm = e / BK; }
            const int64_t gi = m0 + mm, gk = k0 + kk;
            sA[kk][mm] = (gi < m && gk < k) ? A(gi, gk) : T(0);
            int nn, kb;
            if (B.cs == 1) { nn = e % BN; kb = e / BN; } else { kb = e % BK; nn = e / BK; }
            const int64_t gj = n0 + nn, gk2 = k0 + kb;
            sB[kb][nn] = (gj < n && gk2 < k) ? B(gk2, gj) : T(0);
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            T a[4], b[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) a[r] = sA[kk][tm + 16 * r];
#pragma unroll
            for (int c = 0; c < 4; ++c) b[c] = sB[kk][tn + 16 * c];
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int c = 0; c < 4; ++c) acc[r][c] = fma(a[r], b[c], acc[r][c]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const int64_t i = m0 + tm + 16 * r;
        if (i >= m) continue;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int64_t j = n0 + tn + 16 * c;
            if (j >= n || !in_mask(mask, off, i, j)) continue;
            T v = alpha * acc[r][c];
            if (beta != T(0)) v = fma(beta, C(i, j), v);
            C(i, j) = v;
        }
    }
}

// ------------------------------------------------------------------------------------
// FP64 DMMA kernel: 128 x BN tiles (BN = 128 or 64 for skinny right-hand sides), k-step 16
// staged through a 4-deep cp.async ring,
// 8 warps. gridDim.z > 1 splits K: slice z covers [z * kchunk, (z + 1) * kchunk) and
// writes its partial product (alpha = 1, beta = 0) to Cz + z * zstride; a second kernel
// then reduces the slices into C.
constexpr int DM = 128, DK = 16, DSTAGES = 4, DPAD = 4;
constexpr int DLDA = DM + DPAD;

template <int BN>
struct DmmaCfg {
    static constexpr int LDB = BN + DPAD;
    static constexpr int WARPS_N = BN == 128 ? 4 : 2;  // warps along N
    static constexpr int WARPS_M = 8 / WARPS_N;
    static constexpr int WM = DM / WARPS_M, WN = BN / WARPS_N;  // warp tile
    static constexpr int MI = WM / 16, NI = WN / 8;
    static constexpr size_t SMEM = (size_t)DSTAGES * DK * (DLDA + LDB) * sizeof(double);
};

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool pred) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const int bytes = pred ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ void dmma_16x8x4(double (&d)[4], double a0, double a1, double b0) {
    asm volatile(
        "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
        : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
        : "d"(a0), "d"(a1), "d"(b0));
}

// Shared-memory tiles are k-rows of DLDA / LDB doubles; the row offset of element (k, c) is
// c ^ dswz(k): when the global layout is K-major, consecutive lanes store consecutive k
// rows, and the XOR spreads their 8-byte stores over all banks (without it the row strides
// 132 and 68 put four lanes on each bank pair). The fragment loads of one 4-deep k step
// share one XOR value, which only permutes columns inside groups of four.
__device__ __forceinline__ int dswz(int k) { return (k >> 2) & 3; }

// A_KMAJOR: A(i, k) is contiguous along k (A.cs == 1), else along i (A.rs == 1).
// B_KMAJOR: B(k, j) is contiguous along k (B.rs == 1), else along j (B.cs == 1).
template <bool A_KMAJOR, bool B_KMAJOR, int BN>
__device__ __forceinline__ void dmma_load_tile(double* sA, double* sB, const View<const double>& A,
                                               const View<const double>& B, int64_t m, int64_t n, int64_t k,
                                               int64_t m0, int64_t n0, int64_t k0, int tid) {
    constexpr int LDB = DmmaCfg<BN>::LDB;
#pragma unroll
    for (int r = 0; r < DM * DK / 256; ++r) {
        int mm, kk;
        if (A_KMAJOR) { kk = tid % DK; mm = tid / DK + (256 / DK) * r; } else { mm = tid % DM; kk = tid / DM + (256 / DM) * r; }
        const int64_t gi = m0 + mm, gk = k0 + kk;
        const bool ok = gi < m && gk < k;
        cp_async8(sA + kk * DLDA + (mm ^ dswz(kk)), ok ? &A(gi, gk) : A.p, ok);
    }
#pragma unroll
    for (int r = 0; r < BN * DK / 256; ++r) {
        int nn, kk;
        if (B_KMAJOR) { kk = tid % DK; nn = tid / DK + (256 / DK) * r; } else { nn = tid % BN; kk = tid / BN + (256 / BN) * r; }
        const int64_t gj = n0 + nn, gk = k0 + kk;
        const bool ok = gj < n && gk < k;
        cp_async8(sB + kk * LDB + (nn ^ dswz(kk)), ok ? &B(gk, gj) : B.p, ok);
    }
}

template <bool A_KMAJOR, bool B_KMAJOR, int BN>
__global__ void __launch_bounds__(256, 1) gemm_dmma_f64(int64_t m, int64_t n, int64_t k, double alpha,
                                                         View<const double> A, View<const double> B, double beta,
                                                         View<double> C, Mask mask, int64_t off,
                                                         const int* abort, int64_t kchunk, int64_t zstride) {
    using Cfg = DmmaCfg<BN>;
    constexpr int LDB = Cfg::LDB, MI = Cfg::MI, NI = Cfg::NI;
    extern __shared__ __align__(16) double dsmem[];
    double* sA = dsmem;
    double* sB = dsmem + DSTAGES * DK * DLDA;
    // Grouped tile order: consecutive CTAs take kGroupM row tiles of one column tile before
    // the next column tile, so that a wave holds a few A row blocks and B column blocks in L2
    // instead of streaming all of B once per row of tiles.
    constexpr int64_t kGroupM = 8;
    const int64_t lin = (int64_t)blockIdx.y * gridDim.x + blockIdx.x, per = kGroupM * gridDim.x;
    const int64_t first = lin / per * kGroupM, rest = (int64_t)gridDim.y - first;
    const int64_t gsz = rest < kGroupM ? rest : kGroupM, r = lin % per;
    const int64_t m0 = (first + r % gsz) * DM, n0 = r / gsz * BN;
    if (aborted(abort) || tile_outside(mask, off, m0, n0, DM, BN)) return;
    if (gridDim.z > 1) {  // K slice of a split-K product
        const int64_t kz = (int64_t)blockIdx.z * kchunk;
        A = A.sub(0, kz);
        B = B.sub(kz, 0);
        k = (k - kz) < kchunk ? k - kz : kchunk;
        C.p += (int64_t)blockIdx.z * zstride;
    }
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int wm = (warp / Cfg::WARPS_N) * Cfg::WM, wn = (warp % Cfg::WARPS_N) * Cfg::WN;
    double acc[MI][NI][4];
#pragma unroll
    for (int a = 0; a < MI; ++a)
#pragma unroll
        for (int b = 0; b < NI; ++b)
#pragma unroll
            for (int c = 0; c < 4; ++c) acc[a][b][c] = 0.0;

    const int KT = (int)((k + DK - 1) / DK);
#pragma unroll
    for (int s = 0; s < DSTAGES - 1; ++s) {
        if (s < KT)
            dmma_load_tile<A_KMAJOR, B_KMAJOR, BN>(sA + s * DK * DLDA, sB + s * DK * LDB, A, B, m, n, k, m0, n0,
                                                   (int64_t)s * DK, tid);
        cp_async_commit();
    }
    for (int kt = 0; kt < KT; ++kt) {
        cp_async_wait<DSTAGES - 2>();
        __syncthreads();
        const int pf = kt + DSTAGES - 1;
        if (pf < KT) {
            const int st = pf % DSTAGES;
            dmma_load_tile<A_KMAJOR, B_KMAJOR, BN>(sA + st * DK * DLDA, sB + st * DK * LDB, A, B, m, n, k, m0, n0,
                                                   (int64_t)pf * DK, tid);
        }
        cp_async_commit();
        const double* a_s = sA + (kt % DSTAGES) * DK * DLDA;
        const double* b_s = sB + (kt % DSTAGES) * DK * LDB;
#pragma unroll
        for (int ks = 0; ks < DK; ks += 4) {
            double af[MI][2], bf[NI];
            const int sx = dswz(ks);  // == dswz(ks + t) for t < 4
#pragma unroll
            for (int mi = 0; mi < MI; ++mi) {
                af[mi][0] = a_s[(ks + t) * DLDA + ((wm + mi * 16 + g) ^ sx)];
                af[mi][1] = a_s[(ks + t) * DLDA + ((wm + mi * 16 + g + 8) ^ sx)];
            }
#pragma unroll
            for (int ni = 0; ni < NI; ++ni) bf[ni] = b_s[(ks + t) * LDB + ((wn + ni * 8 + g) ^ sx)];
#pragma unroll
            for (int mi = 0; mi < MI; ++mi)
#pragma unroll
                for (int ni = 0; ni < NI; ++ni) dmma_16x8x4(acc[mi][ni], af[mi][0], af[mi][1], bf[ni]);
        }
    }
    cp_async_wait<0>();
    // Epilogue: element (g, 2t + c) and (g + 8, 2t + c) of each 16x8 accumulator tile.
#pragma unroll
    for (int mi = 0; mi < MI; ++mi)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int64_t i = m0 + wm + mi * 16 + g + 8 * h;
            if (i >= m) continue;
#pragma unroll
            for (int ni = 0; ni < NI; ++ni)
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    const int64_t j = n0 + wn + ni * 8 + 2 * t + c;
                    if (j >= n || !in_mask(mask, off, i, j)) continue;
                    double v = alpha * acc[mi][ni][2 * h + c];
                    if (beta != 0.0) v = fma(beta, C(i, j), v);
                    C(i, j) = v;
                }
        }
}

// C = alpha * sum_z P_z + beta * C over the split-K slices (column-major m x n, ld m each).
__global__ void splitk_reduce(int64_t m, int64_t n, int nz, const double* P, int64_t zstride, double alpha,
                              double beta, View<double> C) {
    for (int64_t j = blockIdx.y; j < n; j += gridDim.y)
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
            double acc = 0.0;
            for (int z = 0; z < nz; ++z) acc += P[z * zstride + i + j * m];
            double v = alpha * acc;
            if (beta != 0.0) v = fma(beta, C(i, j), v);
            C(i, j) = v;
        }
}

template <bool AK, bool BK, int BN>
int launch_dmma(int64_t m, int64_t n, int64_t k, double alpha, View<const double> A, View<const double> B,
                double beta, View<double> C, Mask mask, int64_t off, cudaStream_t s, const int* abort) {
    const size_t smem = DmmaCfg<BN>::SMEM;
    if (cudaFuncSetAttribute(gemm_dmma_f64<AK, BK, BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
        return RC_ERR_CUDA;
    dim3 grid(ceil_div(n, BN), ceil_div(m, DM));
    // Long K: split it into nz slices when that packs the CTAs into the GPU's resident
    // slots with less wave quantisation -- nz minimises ceil(tiles nz / slots) / nz (the
    // time in units of one full-K tile) plus a small charge per slice for the reduction.
    static int per_sm = 0;
    if (per_sm == 0 &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gemm_dmma_f64<AK, BK, BN>, 256, smem) != cudaSuccess)
        return RC_ERR_CUDA;
    const int64_t tiles = (int64_t)grid.x * grid.y, slots = (int64_t)(per_sm > 0 ? per_sm : 1) * sm_count();
    int nz = 1;
    if (mask == kFull && k >= 2048 && tiles < 4 * slots) {  // few waves: quantisation matters
        double best = 1e30;
        for (int z = 1; z <= 8 && (int64_t)z * 1024 <= k; ++z) {
            const double cost = (double)((tiles * z + slots - 1) / slots) / z + 0.01 * (z - 1);
            if (cost < best - 1e-9) {
                best = cost;
                nz = z;
            }
        }
    }
    if (nz > 1) {
        const int64_t kchunk = ((k + nz - 1) / nz + DK - 1) / DK * DK;
        nz = (int)((k + kchunk - 1) / kchunk);
        const int64_t zstride = m * n;
        double* P = static_cast<double*>(workspace(s, (size_t)nz * zstride * sizeof(double), 7));
        if (!P) return RC_ERR_ALLOC;
        grid.z = nz;
        gemm_dmma_f64<AK, BK, BN><<<grid, 256, smem, s>>>(m, n, k, 1.0, A, B, 0.0, colmajor(P, m), kFull, 0, abort,
                                                          kchunk, zstride);
        RC_TRY(check_launch());
        dim3 rg(ceil_div(m, 256) < 1024u ? ceil_div(m, 256) : 1024u, n < 65535 ? (unsigned)n : 65535u);
        splitk_reduce<<<rg, 256, 0, s>>>(m, n, nz, P, zstride, alpha, beta, C);
        return check_launch();
    }
    gemm_dmma_f64<AK, BK, BN><<<grid, 256, smem, s>>>(m, n, k, alpha, A, B, beta, C, mask, off, abort, k, 0);
    return check_launch();
}

template <bool AK, bool BK>
int launch_dmma_bn(int64_t m, int64_t n, int64_t k, double alpha, View<const double> A, View<const double> B,
                   double beta, View<double> C, Mask mask, int64_t off, cudaStream_t s, const int* abort) {
    if (n <= 64) return launch_dmma<AK, BK, 64>(m, n, k, alpha, A, B, beta, C, mask, off, s, abort);
    return launch_dmma<AK, BK, 128>(m, n, k, alpha, A, B, beta, C, mask, off, s, abort);
}

// Scale (beta != 1) the masked part of C when k == 0 or alpha == 0.
template <class T>
__global__ void scale_masked(int64_t m, int64_t n, T beta, View<T> C, Mask mask, int64_t off, const int* abort) {
    if (aborted(abort)) return;
    for (int64_t j = blockIdx.y; j < n; j += gridDim.y)
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x)
            if (in_mask(mask, off, i, j)) C(i, j) = beta == T(0) ? T(0) : beta * C(i, j);
}

}  // namespace

template <class T>
int gemm(int64_t m, int64_t n, int64_t k, T alpha, View<const T> A, View<const T> B, T beta, View<T> C, Mask mask,
         int64_t off, cudaStream_t s, const int* abort) {
    if (m <= 0 || n <= 0) return RC_SUCCESS;
    if (k <= 0 || alpha == T(0)) {
        if (beta == T(1)) return RC_SUCCESS;
        dim3 grid(ceil_div(m, 256) < 1024u ? ceil_div(m, 256) : 1024u, n < 65535 ? (unsigned)n : 65535u);
        scale_masked<T><<<grid, 256, 0, s>>>(m, n, beta, C, mask, off, abort);
        return check_launch();
    }
    if constexpr (std::is_same<T, double>::value) {
        const bool a_k = A.cs == 1, a_m = A.rs == 1, b_k = B.rs == 1, b_n = B.cs == 1;
        if ((a_k || a_m) && (b_k || b_n)) {
            if (a_k && b_k) return launch_dmma_bn<true, true>(m, n, k, alpha, A, B, beta, C, mask, off, s, abort);
            if (a_k) return launch_dmma_bn<true, false>(m, n, k, alpha, A, B, beta, C, mask, off, s, abort);
            if (b_k) return launch_dmma_bn<false, true>(m, n, k, alpha, A, B, beta, C, mask, off, s, abort);
            return launch_dmma_bn<false, false>(m, n, k, alpha, A, B, beta, C, mask, off, s, abort);
        }
    }
    dim3 grid(ceil_div(n, 64), ceil_div(m, 64));
    gemm_simt<T><<<grid, 256, 0, s>>>(m, n, k, alpha, A, B, beta, C, mask, off, abort);
    return check_launch();
}

template int gemm<double>(int64_t, int64_t, int64_t, double, View<const double>, View<const double>, double,
                          View<double>, Mask, int64_t, cudaStream_t, const int*);
template int gemm<float>(int64_t, int64_t, int64_t, float, View<const float>, View<const float>, float,
                         View<float>, Mask, int64_t, cudaStream_t, const int*);

}  // namespace rc

namespace {

template <class T>
int gemm_abi(int transA, int transB, size_t m, size_t n, size_t k, T alpha, const T* A, size_t lda, const T* B,
             size_t ldb, T beta, T* C, size_t ldc, void* stream) {
    if (m == 0 || n == 0) return RC_SUCCESS;
    if (!C || ldc < m) return RC_ERR_INVALID_ARGUMENT;
    if (k > 0) {
        if (!A || !B) return RC_ERR_INVALID_ARGUMENT;
        if (lda < (transA ? k : m) || ldb < (transB ? n : k)) return RC_ERR_INVALID_ARGUMENT;
    }
    rc::View<const T> a = rc::colmajor(A, (int64_t)lda);
    rc::View<const T> b = rc::colmajor(B, (int64_t)ldb);
    if (transA) a = a.t();
    if (transB) b = b.t();
    return rc::gemm<T>((int64_t)m, (int64_t)n, (int64_t)k, alpha, a, b, beta, rc::colmajor(C, (int64_t)ldc),
                       rc::kFull, 0, static_cast<cudaStream_t>(stream));
}

template <class T>
int syrk_abi(int upper, int trans, size_t n, size_t k, T alpha, const T* A, size_t lda, T beta, T* C, size_t ldc,
             void* stream) {
    if (n == 0) return RC_SUCCESS;
    if (!C || ldc < n) return RC_ERR_INVALID_ARGUMENT;
    if (k > 0 && (!A || lda < (trans ? k : n))) return RC_ERR_INVALID_ARGUMENT;
    rc::View<const T> a = rc::colmajor(A, (int64_t)lda);
    if (trans) a = a.t();  // op(A) = A^T, n x k
    return rc::gemm<T>((int64_t)n, (int64_t)n, (int64_t)k, alpha, a, a.t(), beta, rc::colmajor(C, (int64_t)ldc),
                       upper ? rc::kUpper : rc::kLower, 0, static_cast<cudaStream_t>(stream));
}

}  // namespace

extern "C" {

int rc_gemm_f64(int transA, int transB, size_t m, size_t n, size_t k, double alpha, const double* A, size_t lda,
                const double* B, size_t ldb, double beta, double* C, size_t ldc, void* stream) {
    return gemm_abi<double>(transA, transB, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, stream);
}
int rc_gemm_f32(int transA, int transB, size_t m, size_t n, size_t k, float alpha, const float* A, size_t lda,
                const float* B, size_t ldb, float beta, float* C, size_t ldc, void* stream) {
    return gemm_abi<float>(transA, transB, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, stream);
}
int rc_syrk_f64(int upper, int trans, size_t n, size_t k, double alpha, const double* A, size_t lda, double beta,
                double* C, size_t ldc, void* stream) {
    return syrk_abi<double>(upper, trans, n, k, alpha, A, lda, beta, C, ldc, stream);
}
int rc_syrk_f32(int upper, int trans, size_t n, size_t k, float alpha, const float* A, size_t lda, float beta,
                float* C, size_t ldc, void* stream) {
    return syrk_abi<float>(upper, trans, n, k, alpha, A, lda, beta, C, ldc, stream);
}

}  // extern "C"
