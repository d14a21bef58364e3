// Trailing updates of an FP64 Cholesky factorisation as exact int8 digit products: the
// near-FP64 factor of the mixed-precision solve for ill-conditioned systems.
//
// An outer panel P (rows of the trailing matrix x K panel columns, FP64) is split once,
// row by row, into kEmuSlices signed 7-bit digits below the row's largest entry
// (Ozaki, Ogita, Oishi and Rump, Numer. Algorithms 2012, in the integer form of Ootomo,
// Ozaki and Yokota, IJHPCA 2024):
//
//   P(i, k) = 2^e_i sum_{t=1..7} a_t(i, k) 2^-7t + r,   |r| < 2^(e_i - 49).
//
// Then (P P^T)(i, j) = 2^(e_i + e_j) sum_{d=2..8} 2^-7d sum_{t+u=d} (a_t a_u^T)(i, j) up to
// the truncations, and every a_t a_u^T is an exact int8 GEMM with int32 accumulation
// (7 * 127^2 * K < 2^31 for K <= 16384). One tcgen05.mma of slice t against the stacked
// slices [a_1 .. a_(8-t)] of the 64 B rows lands in the accumulators d = t+1 .. 8 side by
// side in TMEM (7 x 64 columns), as in the right-hand-side products of ozaki.cu; the
// epilogue combines the seven int32 accumulators (two exact int64 partial sums, one FP64
// rounding) and adds
// alpha 2^(e_i + e_j - 14) times the result into C. Each product term then misses the pairs
// of weight 2^-63 and below and the truncated remainders: at most 2^-46 2^(e_i + e_j), so
// an update of depth K is within K 2^-46 2^(e_i + e_j) <= K 2^-44 m_i m_j (m_i the row's
// largest |entry|) of the exact one -- against 2^-11 and 2^-8 relative for TF32 and BF16,
// within reach of FP64 refinement for condition numbers up to ~1e12.
//
// Per CTA: a 128-row x 64-column tile of C. Warp 0 streams, per 128-wide K block, the
// seven 128-row slices of the A rows through a 7-deep ring and the seven 64-row slices of
// the B rows (one 3-D TMA box) through a 2-deep ring; warp 1 issues the MMAs; warps 2..5
// finish the tile: during the main loop they load their rows of the C tile into registers
// (a row per load across the lanes), then combine the accumulators into a staging tile in the
// (by then idle) A ring and update C a row at a time across the lanes, so that every C
// access is coalesced and none waits after the MMAs. Every mbarrier wait
// is bounded, as in the other tensor-core kernels.
#include <climits>
#include <cudaTypedefs.h>

#include "emu64.cuh"
#include "ozaki_digits.cuh"
#include "tc_common.cuh"
#include "tc_gemm.cuh"

namespace rc {
namespace {

using namespace tc;
constexpr int S = kEmuSlices;
constexpr int EMU_THREADS = 192;
constexpr int A_STAGES = 7;
constexpr int A_TILE = 128 * 128;     // one slice of 128 rows x 128 bytes
constexpr int B_TILE = 64 * 128 * S;  // all slices of 64 rows x 128 bytes
constexpr size_t EMU_SMEM = 1024 + (size_t)A_STAGES * A_TILE + 2 * (size_t)B_TILE + 256;
static_assert(EMU_SMEM <= 232448, "shared memory of the digit-product update");
// The epilogue's staging tile (128 rows x 64 FP64 values, rows padded to 65) reuses the A ring.
constexpr int kStageLd = 65;
static_assert(128 * kStageLd * 8 <= A_STAGES * A_TILE, "staging tile");

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
int64_t round_up(int64_t x, int64_t q) { return (x + q - 1) / q * q; }

// One warp per row r < Mp: the row's exponent from its largest |P(r, k)|, then its digits,
// four columns per lane and step so that both the reads (32 bytes per lane) and the writes
// (a 4-byte word per slice and lane) are contiguous across the warp. Rows r >= rows and
// columns k >= width get zero digits.
__global__ void __launch_bounds__(256) emu_slice_kernel(int64_t rows, int64_t width, const double* __restrict__ P,
                                                        int64_t ldp, int64_t Mp, int64_t ldk, int8_t* __restrict__ D,
                                                        int* __restrict__ rexp) {
    const int lane = threadIdx.x & 31;
    const int64_t r = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
    if (r >= Mp) return;
    const bool live = r < rows;
    const double* row = P + r * ldp;
    unsigned long long mx = 0;
    if (live)
        for (int64_t k = lane; k < width; k += 32) {
            const unsigned long long b = (unsigned long long)__double_as_longlong(row[k]) & 0x7FFFFFFFFFFFFFFFull;
            mx = b > mx ? b : mx;
        }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        const unsigned long long y = __shfl_xor_sync(0xffffffffu, mx, o);
        mx = y > mx ? y : mx;
    }
    const int e = live ? scale_exp(mx) : 0;
    if (lane == 0) rexp[r] = e;
    const bool ok = live && e != kOzBadExp;
    for (int64_t k0 = 4 * (int64_t)lane; k0 < ldk; k0 += 128) {
        uint32_t word[kOzSlices] = {};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int64_t k = k0 + q;
            digits((ok && k < width) ? row[k] : 0.0, e, word, q);
        }
#pragma unroll
        for (int t = 0; t < S; ++t) *reinterpret_cast<uint32_t*>(D + ((int64_t)t * Mp + r) * ldk + k0) = word[t];
    }
}

__device__ __forceinline__ uint32_t i8_idesc(int n) {
    // D = S32 (bits 4-5), A and B signed 8-bit (bits 7-9, 10-12), K-major, N >> 3, M = 128.
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* tm, uint64_t* bar, int x, int y, int z) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];" ::
            "r"(smem_u32(dst)),
        "l"(tm), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
        : "memory");
}

// 8 int32 accumulator columns of this warp's TMEM lanes, without waiting (tmem_wait_ld).
__device__ __forceinline__ void tmem_ld8_async(uint32_t taddr, uint32_t (&r)[8]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Shared-space accesses of the staging tile (explicitly .shared, so that the compiler and the
// memory pipeline never order them behind the epilogue's global loads and stores).
__device__ __forceinline__ void sts_f64(uint32_t addr, double v) {
    asm volatile("st.shared.f64 [%0], %1;" ::"r"(addr), "d"(v) : "memory");
}
__device__ __forceinline__ double lds_f64(uint32_t addr) {
    double v;
    asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(addr) : "memory");
    return v;
}

// 2^e as a double for e in [-1022, 1023] (the exponent field alone).
__device__ __forceinline__ double pow2(int e) { return __longlong_as_double((long long)(e + 1023) << 52); }

// h * 2^e, correctly rounded (as ldexp(h, e)), for |h| in {0} u [2^-42, 2^35) (a
// combination of the seven accumulators), without a branch: e is clamped to [-2044, 2044]
// (beyond it the result is 0 or Inf either way) and split into halves e1 + e2, both within
// the normal exponents; h 2^e1 is then exact (normal, |e1| <= 1022 keeps it far from
// overflow, and it is subnormal only when the final result rounds to zero), so the second
// product is the one rounding.
__device__ __forceinline__ double scale_pow2(double h, int e) {
    e = max(-2044, min(e, 2044));
    const int e1 = e >> 1;
    return (h * pow2(e1)) * pow2(e - e1);
}

// The seven int32 accumulators v[0] (weight 1) .. v[6] (weight 2^-42) as one FP64 value:
// v0 2^21 + v1 2^14 + v2 2^7 + v3 and v4 2^14 + v5 2^7 + v6 are exact in int64 (|v| < 2^31),
// and exact in FP64 (below 2^53 and 2^46), so h has one rounding.
template <int W>
__device__ __forceinline__ double combine7(const uint32_t (&v)[S][W], int x) {
    const long long hi = ((((long long)(int)v[0][x] * 128 + (int)v[1][x]) * 128 + (int)v[2][x]) * 128) + (int)v[3][x];
    const long long lo = ((long long)(int)v[4][x] * 128 + (int)v[5][x]) * 128 + (int)v[6][x];
    return fma((double)hi, 0x1p-21, (double)lo * 0x1p-42);
}

// C(i, j) <- alpha * (P_A P_B^T)(i, j) + beta * C(i, j) on one 128 x 64 tile (see the file
// comment); beta == 0 does not read C.
__global__ void __launch_bounds__(EMU_THREADS, 1)
    emu_update_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, int64_t Mp,
                      int64_t a0, int64_t b0, int64_t M, int64_t N, int64_t K, double alpha, double beta, double* C,
                      int64_t ldc,
                      const int* __restrict__ rexp, int lower, const int* abort, int* err, uint64_t limit_ns) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* sA = smem;
    uint8_t* sB = smem + A_STAGES * A_TILE;
    uint64_t* afull = reinterpret_cast<uint64_t*>(sB + 2 * B_TILE);
    uint64_t* aempty = afull + A_STAGES;
    uint64_t* bfull = aempty + A_STAGES;
    uint64_t* bempty = bfull + 2;
    uint64_t* done = bempty + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
    volatile int* stop = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int64_t i0 = (int64_t)blockIdx.y * 128, j0 = (int64_t)blockIdx.x * 64;
    if (lower && j0 > i0 + 127) return;  // the tile lies above the diagonal
    if (aborted(abort) || aborted(err)) return;
    const int KB = (int)((K + 127) / 128);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int q = 0; q < A_STAGES; ++q) {
            mbar_init(&afull[q], 1);
            mbar_init(&aempty[q], 1);
        }
        for (int q = 0; q < 2; ++q) {
            mbar_init(&bfull[q], 1);
            mbar_init(&bempty[q], 1);
        }
        mbar_init(done, 1);
        *stop = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(&tmA) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(&tmB) : "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(512u));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            int a_issued = 0, b_issued = 0;
            for (int kb = 0; kb < KB && !*stop; ++kb) {
                const int bs = kb & 1;
                const int w = mbar_wait_bounded(&bempty[bs], ((kb >> 1) & 1) ^ 1, stop, err, abort, limit_ns);
                if (w != kWaitOk) {
                    raise_stop(stop, err, w, kSiteEmu * 100 + kRoleProducer * 10);
                    break;
                }
                mbar_expect_tx(&bfull[bs], (uint32_t)B_TILE);
                tma_load_3d(sB + bs * B_TILE, &tmB, &bfull[bs], kb * 128, (int)(b0 + j0), 0);
                ++b_issued;
                for (int t = 0; t < S; ++t) {
                    const int as = a_issued % A_STAGES;
                    const int wa =
                        mbar_wait_bounded(&aempty[as], ((a_issued / A_STAGES) & 1) ^ 1, stop, err, abort, limit_ns);
                    if (wa != kWaitOk) {
                        raise_stop(stop, err, wa, kSiteEmu * 100 + kRoleProducer * 10);
                        break;
                    }
                    mbar_expect_tx(&afull[as], (uint32_t)A_TILE);
                    tma_load_2d(sA + as * A_TILE, &tmA, &afull[as], kb * 128, (int)(t * Mp + a0 + i0));
                    ++a_issued;
                }
            }
            if (*stop) {
                // Let the copies this thread started land before the CTA's shared memory goes away.
                volatile int never = 0;
                bool drained = true;
                for (int q = (a_issued > A_STAGES ? a_issued - A_STAGES : 0); q < a_issued; ++q)
                    drained &= mbar_wait_bounded(&afull[q % A_STAGES], (q / A_STAGES) & 1, &never, nullptr, nullptr,
                                                 limit_ns) == kWaitOk;
                for (int q = (b_issued > 2 ? b_issued - 2 : 0); q < b_issued; ++q)
                    drained &= mbar_wait_bounded(&bfull[q & 1], (q >> 1) & 1, &never, nullptr, nullptr, limit_ns) ==
                               kWaitOk;
                if (!drained) settle(kSettleNs);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // The tensor pipe idles through every instruction this thread runs between two
            // MMAs (its queue is shallow: a pause after a slice's MMAs shows up one for one in
            // the main loop), so the slices are unrolled with their descriptors, shapes and
            // accumulator columns fixed at compile time: A stage t always holds slice t and is
            // filled once per K block (phase parity kb & 1).
            static_assert(A_STAGES == S, "one A stage per slice");
            uint64_t adesc[S];
#pragma unroll
            for (int t = 0; t < S; ++t) adesc[t] = sw128_kmajor_desc(sA + t * A_TILE);
            const uint64_t b0d0 = sw128_kmajor_desc(sB), b0d1 = sw128_kmajor_desc(sB + 256 * 128);
            const uint64_t b1d0 = sw128_kmajor_desc(sB + B_TILE), b1d1 = sw128_kmajor_desc(sB + B_TILE + 256 * 128);
            bool ok = true;
            for (int kb = 0; kb < KB && ok; ++kb) {
                const int bs = kb & 1;
                const uint32_t par = (uint32_t)kb & 1u;
                int w = mbar_wait_bounded(&bfull[bs], (kb >> 1) & 1, stop, err, abort, limit_ns);
                if (w != kWaitOk) {
                    raise_stop(stop, err, w, kSiteEmu * 100 + kRoleMma * 10);
                    break;
                }
                tc_fence_after();
                const uint64_t bd0 = bs ? b1d0 : b0d0, bd1 = bs ? b1d1 : b0d1;
#pragma unroll
                for (int t = 0; t < S; ++t) {
                    w = mbar_wait_bounded(&afull[t], par, stop, err, abort, limit_ns);
                    if (w != kWaitOk) {
                        raise_stop(stop, err, w, kSiteEmu * 100 + kRoleMma * 10);
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    // a_t x [b_1 .. b_(S-t)] -> accumulators d = t .. S-1 (columns 64 t ..)
                    constexpr int kCols = 64;
                    const int n_all = kCols * (S - t);
                    const int n1 = n_all < 256 ? n_all : 256;
#pragma unroll
                    for (int kk = 0; kk < 4; ++kk) {
                        const uint32_t acc = (kb | t | kk) != 0 ? 1u : 0u;
                        umma_i8(tmem + (uint32_t)(kCols * t), adesc[t] + 2 * kk, bd0 + 2 * kk, i8_idesc(n1), acc);
                        if (n_all > 256)
                            umma_i8(tmem + (uint32_t)(kCols * t + 256), adesc[t] + 2 * kk, bd1 + 2 * kk,
                                    i8_idesc(n_all - 256), acc);
                    }
                    umma_commit(&aempty[t]);
                }
                if (ok) umma_commit(&bempty[bs]);
            }
            umma_commit(done);
            if (*stop) {
                // The epilogue leaves at once on a stop: the MMAs issued so far finish before
                // the accumulator columns and the operand ring are released.
                volatile int never = 0;
                if (mbar_wait_bounded(done, 0, &never, nullptr, nullptr, limit_ns) != kWaitOk) settle(kSettleNs);
            }
        }
    } else {
        // Epilogue warps: warp w owns TMEM lanes 32 (w % 4) .. and the same 32 rows of the tile.
        const int q = warp & 3;
        const int r0 = 32 * q;
        const int64_t i = i0 + r0 + lane;  // the row whose accumulators this thread reads
        const int ei = i < M ? rexp[a0 + i] : 0;
        // Tile-local indices: row rl = r0 + rr, column cl = lane + 32 u; C(rl, cl) is written
        // when rl < mrem, cl < nrem and, for the lower triangle, cl - rl <= dlim.
        const int mrem = (int)(M - i0 < 128 ? M - i0 : 128), nrem = (int)(N - j0 < 64 ? N - j0 : 64);
        const int dlim = lower ? (int)(i0 - j0 < 256 ? i0 - j0 : 256) : 256;
        const bool rd = beta != 0.0;
        double* cw = C + (i0 + r0) * ldc + j0 + lane;  // this lane's column of the warp's first row
        // While the main loop runs: the warp's 32 rows of the C tile (columns lane and
        // lane + 32) into registers, a row per load across the lanes.
        double cv[32][2];
#pragma unroll
        for (int rr = 0; rr < 32; ++rr)
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const int rl = r0 + rr, cl = lane + 32 * u;
                cv[rr][u] = (rd && rl < mrem && cl < nrem && cl - rl <= dlim) ? cw[(int64_t)rr * ldc + 32 * u] : 0.0;
            }
        int ej[2];
#pragma unroll
        for (int u = 0; u < 2; ++u) ej[u] = lane + 32 * u < nrem ? rexp[b0 + j0 + lane + 32 * u] : 0;
        const int w = mbar_wait_bounded(done, 0, stop, err, abort, limit_ns);
        const bool ok = w == kWaitOk;
        if (!ok) raise_stop(stop, err, w, kSiteEmu * 100 + kRoleEpilogue * 10);
        tc_fence_after();
        if (__all_sync(0xffffffffu, ok && !*stop)) {
            // 1. The seven accumulators of this thread's row, combined, into this warp's 32 rows
            //    of a staging tile in the operand ring (idle now: every load has been consumed
            //    and every MMA has completed).
            const uint32_t stage = smem_u32(sA) + (uint32_t)(r0 * kStageLd * 8);
            const uint32_t srow = stage + (uint32_t)(lane * kStageLd * 8);
#pragma unroll 1
            for (int cc = 0; cc < 64; cc += 8) {
                uint32_t v[S][8];
#pragma unroll
                for (int d = 0; d < S; ++d) tmem_ld8_async(tmem + ((uint32_t)r0 << 16) + (uint32_t)(64 * d + cc), v[d]);
                tmem_wait_ld();
#pragma unroll
                for (int x = 0; x < 8; ++x) sts_f64(srow + (uint32_t)((cc + x) * 8), combine7(v, x));
            }
            __syncwarp();
            // 2. The warp's 32 rows of C, a row at a time across the lanes.
#pragma unroll
            for (int rr = 0; rr < 32; ++rr) {
                const int rl = r0 + rr;
                const int er = __shfl_sync(0xffffffffu, ei, rr);
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const int cl = lane + 32 * u;
                    const double h = lds_f64(stage + (uint32_t)((rr * kStageLd + cl) * 8));
                    const bool bad = er == kOzBadExp || ej[u] == kOzBadExp;
                    double val = scale_pow2(h, bad ? 0 : er + ej[u] - 14);
                    val = bad ? __longlong_as_double(0x7FF8000000000000ll) : val;
                    const double out = rd ? fma(alpha, val, beta * cv[rr][u]) : alpha * val;
                    if (rl < mrem && cl < nrem && cl - rl <= dlim) cw[(int64_t)rr * ldc + 32 * u] = out;
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512u));
    }
}

// C(i, j) <- beta C(i, j) on the lower triangle of the row-major n x n C (k = 0 updates).
__global__ void lower_scale_kernel(int64_t n, double beta, double* C, int64_t ldc) {
    for (int64_t i = blockIdx.y; i < n; i += gridDim.y)
        for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j <= i; j += (int64_t)gridDim.x * blockDim.x)
            C[i * ldc + j] = beta == 0.0 ? 0.0 : beta * C[i * ldc + j];
}

bool make_u8_map(CUtensorMap* tm, const void* base, int rank, const cuuint64_t* dims, const cuuint64_t* strides,
                 const cuuint32_t* box) {
    auto enc = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(tensor_map_encoder());
    if (!enc) return false;
    cuuint32_t estr[3] = {1, 1, 1};
    return enc(tm, CU_TENSOR_MAP_DATA_TYPE_UINT8, (cuuint32_t)rank, const_cast<void*>(base), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

size_t emu_panel_bytes(int64_t rows, int64_t width) {
    const int64_t Mp = round_up(rows > 0 ? rows : 1, 128), ldk = round_up(width > 0 ? width : 1, 128);
    return align256((size_t)S * Mp * ldk) + align256((size_t)Mp * sizeof(int));
}

int emu_panel_layout(int64_t rows, int64_t width, void* ws, EmuPanel* out) {
    if (rows <= 0 || width <= 0 || width > 16384 || !ws || !out) return RC_ERR_INVALID_ARGUMENT;
    EmuPanel pn;
    pn.rows = rows;
    pn.width = width;
    pn.Mp = round_up(rows, 128);
    pn.ldk = round_up(width, 128);
    if ((int64_t)S * pn.Mp > INT32_MAX) return RC_ERR_NOT_SUPPORTED;
    char* p = static_cast<char*>(ws);
    pn.digits = reinterpret_cast<int8_t*>(p);
    pn.rexp = reinterpret_cast<int*>(p + align256((size_t)S * pn.Mp * pn.ldk));
    const cuuint64_t da[2] = {(cuuint64_t)pn.ldk, (cuuint64_t)(S * pn.Mp)};
    const cuuint64_t sa[1] = {(cuuint64_t)pn.ldk};
    const cuuint32_t ba[2] = {128u, 128u};
    const cuuint64_t db[3] = {(cuuint64_t)pn.ldk, (cuuint64_t)pn.Mp, (cuuint64_t)S};
    const cuuint64_t sb[2] = {(cuuint64_t)pn.ldk, (cuuint64_t)(pn.Mp * pn.ldk)};
    const cuuint32_t bb[3] = {128u, 64u, (cuuint32_t)S};
    if (!make_u8_map(&pn.tmA, pn.digits, 2, da, sa, ba) || !make_u8_map(&pn.tmB, pn.digits, 3, db, sb, bb))
        return RC_ERR_NOT_SUPPORTED;
    *out = pn;
    return RC_SUCCESS;
}

int emu_slice_panel(const EmuPanel& pn, const double* P, int64_t ldp, cudaStream_t s) {
    emu_slice_kernel<<<(unsigned)(pn.Mp / 8), 256, 0, s>>>(pn.rows, pn.width, P, ldp, pn.Mp, pn.ldk, pn.digits,
                                                          pn.rexp);
    return check_launch();
}

int emu_update(const EmuPanel& pn, int64_t a0, int64_t b0, int64_t M, int64_t N, double alpha, double beta,
               double* C, int64_t ldc, bool lower, cudaStream_t s, const int* abort) {
    if (M <= 0 || N <= 0) return RC_SUCCESS;
    if (a0 < 0 || b0 < 0 || a0 + M > pn.rows || b0 + N > pn.rows || !C || ldc < N) return RC_ERR_INVALID_ARGUMENT;
    if (cudaFuncSetAttribute(emu_update_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)EMU_SMEM) !=
        cudaSuccess)
        return RC_ERR_CUDA;
    const dim3 grid((unsigned)((N + 63) / 64), (unsigned)((M + 127) / 128));
    if (grid.y > 65535) return RC_ERR_NOT_SUPPORTED;
    emu_update_kernel<<<grid, EMU_THREADS, EMU_SMEM, s>>>(pn.tmA, pn.tmB, pn.Mp, a0, b0, M, N, pn.width, alpha, beta,
                                                          C, ldc, pn.rexp, lower ? 1 : 0, abort, error_word(),
                                                          wait_limit_ns());
    return check_launch();
}

}  // namespace rc

extern "C" {

int rc_syrk_emu64(size_t n, size_t k, double alpha, const double* P, size_t ldp, double beta, double* C, size_t ldc,
                  void* stream) {
    if (n == 0) return RC_SUCCESS;
    if (!C || ldc < n || (k > 0 && (!P || ldp < k))) return RC_ERR_INVALID_ARGUMENT;
    if (k > 16384 || n > (size_t)INT32_MAX / rc::kEmuSlices - 128) return RC_ERR_NOT_SUPPORTED;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (k == 0 || alpha == 0.0) {
        if (beta == 1.0) return RC_SUCCESS;
        const dim3 g(n < 256 ? 1u : (unsigned)((n + 255) / 256 < 64 ? (n + 255) / 256 : 64),
                     n < 65535 ? (unsigned)n : 65535u);
        rc::lower_scale_kernel<<<g, 256, 0, s>>>((int64_t)n, beta, C, (int64_t)ldc);
        return rc::check_launch();
    }
    void* ws = rc::workspace(s, rc::emu_panel_bytes((int64_t)n, (int64_t)k), 13);
    if (!ws) return RC_ERR_ALLOC;
    rc::EmuPanel pn;
    RC_TRY(rc::emu_panel_layout((int64_t)n, (int64_t)k, ws, &pn));
    RC_TRY(rc::emu_slice_panel(pn, P, (int64_t)ldp, s));
    return rc::emu_update(pn, 0, 0, (int64_t)n, (int64_t)n, alpha, beta, C, (int64_t)ldc, true, s, nullptr);
}

}  // extern "C"
