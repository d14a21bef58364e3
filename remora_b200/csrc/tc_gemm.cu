// Tensor-core GEMM on the 5th-generation tensor cores (tcgen05) for FP32 data:
// TF32 or BF16 operands, FP32 accumulation in tensor memory (TMEM).
//
//   D(m, n) = alpha * sum_k A(m, k) * B(n, k) + beta * C(m, n)
//
// A (M x K) and B (N x K) are K-major (k contiguous) in global memory; C is any strided
// FP32 view. One CTA computes a 128 x BN tile (BN = 128 or 256):
//   warp 0      one elected thread issues TMA loads of 128-byte-wide K slices of A and B
//               into a STAGES-deep ring of 128B-swizzled shared-memory buffers;
//   warp 1      allocates BN TMEM columns and one elected thread issues tcgen05.mma
//               (M = 128, N = BN, K = 32 bytes per instruction), committing each stage
//               back to the producer through an mbarrier;
//   warps 2..5  wait for the final commit, read the accumulator with tcgen05.ld (each warp
//               its 32-lane quadrant of TMEM) and apply alpha/beta and the triangle mask.
// Every mbarrier wait is bounded (tc_common.cuh); a wait that runs out records
// RC_ERR_TIMEOUT in the library's device error word, stops the other roles, lets the
// copies it issued land, frees TMEM and returns. A kernel that starts while the error word
// or its abort word (a failed pivot) is set returns at once, and waits in flight give up
// when either is raised, so one failure ends the whole factorisation within microseconds.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <cstring>

#include "assign.cuh"
#include "gemm.cuh"
#include "tc_gemm.cuh"
#include "tc_common.cuh"

namespace rc {
namespace {

using namespace tc;
constexpr int KB_BYTES = 128;  // K extent of one pipeline stage, in bytes (one swizzle row)
constexpr int TC_THREADS = 192;

template <int BN, bool FOLD = false>
struct TcCfg {
    // Every configuration runs two CTAs per SM (~96 KB of rings each): a second CTA's main
    // loop overlaps one CTA's pipeline fill and epilogue, and the factorisation's
    // look-ahead kernels fit beside a trailing-update CTA.
    static constexpr int STAGES = FOLD ? 3 : (BN == 256 ? 2 : 3);
    static constexpr int A_BYTES = 128 * KB_BYTES;
    static constexpr int B_BYTES = BN * KB_BYTES;
    static constexpr size_t SMEM = (size_t)STAGES * (A_BYTES + B_BYTES) + 1024 + 256;
};

// FOLD (BN = 128): the product's columns j and j + 64 are summed into column j of C (an
// m x 64 result from a 128-row B = [B_hi; B_lo], the two halves of an exact TF32 split).
template <int BN, bool BF16, bool FOLD = false>
__global__ void __launch_bounds__(TC_THREADS, 2)
    tc_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, int64_t M,
                   int64_t N, int64_t K, float alpha, float beta, View<float> C, Mask mask, int64_t off,
                   const int* abort, int* err, uint64_t limit_ns) {
    using Cfg = TcCfg<BN, FOLD>;
    constexpr int STAGES = Cfg::STAGES;
    constexpr int KB_ELEMS = KB_BYTES / (BF16 ? 2 : 4);
    constexpr int MMAS_PER_STAGE = KB_BYTES / 32;  // each MMA consumes 32 bytes of K
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* sA = smem;
    uint8_t* sB = smem + STAGES * Cfg::A_BYTES;
    uint64_t* full = reinterpret_cast<uint64_t*>(sB + STAGES * Cfg::B_BYTES);
    uint64_t* empty = full + STAGES;
    uint64_t* done = empty + STAGES;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
    volatile int* stop = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int64_t m0 = (int64_t)blockIdx.y * 128, n0 = (int64_t)blockIdx.x * BN;
    if (aborted(abort) || aborted(err) || outside(mask, off, m0, n0, 128, BN)) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(done, 1);
        *stop = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(&tmA) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(&tmB) : "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"((uint32_t)BN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const int KB = (int)((K + KB_ELEMS - 1) / KB_ELEMS);

    if (warp == 0) {
        if (lane == 0) {
            int issued = 0;
            for (int kb = 0; kb < KB; ++kb) {
                const int s = kb % STAGES;
                const uint32_t ph = (kb / STAGES) & 1;
                const int w = mbar_wait_bounded(&empty[s], ph ^ 1, stop, err, abort, limit_ns);
                if (w != kWaitOk) {
                    raise_stop(stop, err, w, kSiteTcGemm * 100 + kRoleProducer * 10);
                    break;
                }
                mbar_expect_tx(&full[s], Cfg::A_BYTES + Cfg::B_BYTES);
                tma_load_2d(sA + s * Cfg::A_BYTES, &tmA, &full[s], kb * KB_ELEMS, (int)m0);
                tma_load_2d(sB + s * Cfg::B_BYTES, &tmB, &full[s], kb * KB_ELEMS, (int)n0);
                ++issued;
            }
            if (*stop) {
                // Let the copies this thread started land before the CTA's shared memory goes
                // away (every copy completes on its own barrier; no other thread waits now).
                volatile int never = 0;
                bool drained = true;
                for (int kb = (issued > STAGES ? issued - STAGES : 0); kb < issued; ++kb)
                    drained &= mbar_wait_bounded(&full[kb % STAGES], (kb / STAGES) & 1, &never, nullptr, nullptr,
                                                 limit_ns) == kWaitOk;
                if (!drained) settle(kSettleNs);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t fmt = BF16 ? 1u : 2u;
            const uint32_t idesc = (1u << 4) | (fmt << 7) | (fmt << 10) | ((uint32_t)(BN >> 3) << 17) |
                                   ((uint32_t)(128 >> 4) << 24);
            // The tensor pipe idles through every instruction this thread runs between two
            // MMAs: the ring position is carried incrementally and the descriptors advance by
            // a fixed stride.
            const uint64_t ad0 = sw128_kmajor_desc(sA), bd0 = sw128_kmajor_desc(sB);
            constexpr uint64_t kAStep = Cfg::A_BYTES >> 4, kBStep = Cfg::B_BYTES >> 4;
            int s = 0;
            uint32_t ph = 0;
            for (int kb = 0; kb < KB; ++kb) {
                const int w = mbar_wait_bounded(&full[s], ph, stop, err, abort, limit_ns);
                if (w != kWaitOk) {
                    raise_stop(stop, err, w, kSiteTcGemm * 100 + kRoleMma * 10);
                    break;
                }
                tc_fence_after();
                const uint64_t ad = ad0 + (uint64_t)s * kAStep, bd = bd0 + (uint64_t)s * kBStep;
#pragma unroll
                for (int kk = 0; kk < MMAS_PER_STAGE; ++kk)
                    umma<BF16>(tmem, ad + 2 * kk, bd + 2 * kk, idesc, (kb | kk) != 0 ? 1u : 0u);
                umma_commit(&empty[s]);
                if (++s == STAGES) {
                    s = 0;
                    ph ^= 1u;
                }
            }
            umma_commit(done);
        }
    } else {
        const int q = warp & 3;  // TMEM lane quadrant this warp may access
        // FOLD: the rows of C this thread finishes are read while the main loop runs.
        float cpre[FOLD ? BN / 2 : 1];
        if constexpr (FOLD) {
            const int64_t i = m0 + 32 * q + lane;
#pragma unroll
            for (int j = 0; j < BN / 2; ++j) cpre[j] = (beta != 0.f && i < M && j < N) ? C(i, j) : 0.f;
        }
        const int w = mbar_wait_bounded(done, 0, stop, err, abort, limit_ns);
        const bool ok = w == kWaitOk;
        if (!ok) raise_stop(stop, err, w, kSiteTcGemm * 100 + kRoleEpilogue * 10);
        tc_fence_after();
        // tcgen05.ld is warp-collective: the whole warp takes one decision.
        if (__all_sync(0xffffffffu, ok && !*stop)) {
            const int64_t i = m0 + 32 * q + lane;
            const bool row_ok = i < M;
            const bool vec = C.cs == 1 && (C.rs % 4 == 0) && (reinterpret_cast<uintptr_t>(C.p) % 16 == 0);
            if constexpr (FOLD) {
#pragma unroll
                for (int c0 = 0; c0 < BN / 2; c0 += 16) {
                    float v[16], w[16];
                    tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)c0, v);
                    tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(c0 + BN / 2), w);
                    if (!row_ok) continue;
#pragma unroll
                    for (int u = 0; u < 16; ++u) {
                        const int j = c0 + u;
                        if (j < N) C(i, j) = fmaf(beta, cpre[j], alpha * (v[u] + w[u]));
                    }
                }
            }
#pragma unroll 1
            for (int c0 = 0; c0 < (FOLD ? 0 : BN); c0 += 16) {
                float v[16];
                tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)c0, v);
                if (!row_ok) continue;
                const int64_t j0 = n0 + c0;
                if (vec && j0 + 15 < N && keep(mask, off, i, j0 + 15) && keep(mask, off, i, j0)) {
                    float4* dst = reinterpret_cast<float4*>(C.p + i * C.rs + j0);
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        float4 r = make_float4(alpha * v[4 * u], alpha * v[4 * u + 1], alpha * v[4 * u + 2],
                                               alpha * v[4 * u + 3]);
                        if (beta != 0.f) {
                            const float4 c = dst[u];
                            r.x = fmaf(beta, c.x, r.x); r.y = fmaf(beta, c.y, r.y);
                            r.z = fmaf(beta, c.z, r.z); r.w = fmaf(beta, c.w, r.w);
                        }
                        dst[u] = r;
                    }
                } else {
#pragma unroll
                    for (int u = 0; u < 16; ++u) {
                        const int64_t j = j0 + u;
                        if (j >= N || !keep(mask, off, i, j)) continue;
                        float r = alpha * v[u];
                        if (beta != 0.f) r = fmaf(beta, C(i, j), r);
                        C(i, j) = r;
                    }
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)BN));
    }
}

// Pair kernel: persistent clusters of two CTAs, each computing 256 x 256 tiles with
// tcgen05.mma.cta_group::2. CTA rank r (0 = the leader) stages rows [128 r, 128 r + 128)
// of the tile's A rows and of its B rows (K-major) in its own shared memory at the same
// offsets, and holds the accumulator of its 128 rows (x 256 columns) in its own TMEM.
// Both CTAs issue their TMA loads against the leader's full barrier (peer bit cleared),
// whose expected byte count covers both; one thread of the leader issues the MMAs and
// commits every stage to the empty barriers of both CTAs and every finished tile to both
// tfull barriers. Per SM and k-slice this moves 32 KB for a 128 x 256 x 32 product instead
// of 48 KB, half the B traffic of a single-CTA 128 x 256 tile.
//
// Persistence. Cluster c takes tiles c, c + C, c + 2C, ... of a fixed enumeration (all
// tiles, or the tiles on and below the diagonal of a square C). The loads of the next tile
// stream into the ring while the epilogue still drains the accumulator; the leader's MMAs
// of the next tile wait on its tempty barrier, which both CTAs' epilogue groups arrive on
// once their TMEM reads are done.
//
// Epilogue. Four warps, one per TMEM lane quadrant (warp w may read lanes 32 (w mod 4) ..),
// each finishing the 256 columns of its 32 rows. Fast path (beta = 1, C row-major and
// 16-byte aligned with a multiple of 32 columns, tile off the diagonal): TMEM -> registers
// (x alpha) -> a staging box in shared memory (32 rows x EPI_BLK blocks of 32 columns,
// 128-byte swizzled) -> one TMA reduce-add of the box into C through a 3-D tensor map
// (column-in-block, row, column block), EPI_BUFS boxes per warp in flight; C is never read
// by the SM. The boxes are large because the TMA unit serialises its operations: with 2 KB
// boxes the reduce-adds of one tile (64 per CTA) took as long as a third of its MMAs.
// Otherwise the rows are finished element by element (the triangle mask, general beta).
//
// One CTA per SM. The shared-memory footprint is at least half an SM's, so no SM holds two
// pair CTAs and no TPC holds two pairs. (Two pairs on one TPC can allocate TMEM in crossed
// order -- each pair holding on one SM the columns the other pair waits for on the other
// SM -- and then both wait forever.) A single-CTA tcgen05 kernel (at most 256 columns, it
// waits on no other CTA) may run beside a pair CTA; the pair's collective allocation then
// waits at most until that CTA finishes. Two configurations:
//   PairCo    (3 stages, one 32-column box per warp, 113 KB, one 256-column accumulator):
//             leaves room beside it for one single-CTA tcgen05 kernel (~97 KB, at most 256
//             TMEM columns) -- the factorisation's look-ahead chain runs there;
//   PairAlone (5 stages, two 64-column boxes per warp, 225 KB, two 256-column accumulators:
//             the MMAs of the next tile run while the epilogue drains the last one): a
//             launch that has the SMs to itself (rc_syrk_tc, rc_gemm_tf32).
//
// Failure handling. Every mbarrier wait is bounded and gives up as soon as the device
// error word or the abort word is raised; the epilogue warps take each decision together
// (a barrier-reduction over their threads). The two CTAs may still take different
// decisions, so neither returns early: each reaches the closing cluster barrier, having
// written its stop flag into both CTAs' `any_stop`; when either stopped, both stay
// resident for a settle period so that copies still in flight land first.
constexpr int PAIR_A_BYTES = 128 * KB_BYTES, PAIR_B_BYTES = 128 * KB_BYTES;
constexpr int PAIR_THREADS = 192;
template <int STAGES_, int EPI_BLK_, int EPI_BUFS_, int TMEM_BUFS_>
struct PairCfg {
    static constexpr int STAGES = STAGES_;
    static constexpr int TMEM_BUFS = TMEM_BUFS_;               // 256-column accumulators per CTA
    static constexpr int EPI_BLK = EPI_BLK_;                   // 32-column blocks per staged box
    static constexpr int EPI_COLS = 32 * EPI_BLK;              // columns per box
    static constexpr int EPI_BOX_BYTES = 32 * EPI_COLS * 4;    // 32 rows
    static constexpr int EPI_BUFS = EPI_BUFS_;                 // boxes in flight per warp
    static constexpr int STAGING = 4 * EPI_BUFS * EPI_BOX_BYTES;
    static constexpr size_t SMEM = 1024 + (size_t)STAGES * (PAIR_A_BYTES + PAIR_B_BYTES) + STAGING + 256;
};
// 115,968 bytes: with the 1 KB the hardware reserves per CTA, a 99,584-byte single-CTA
// kernel still fits beside it in an SM's 233,472.
using PairCo = PairCfg<3, 1, 1, 1>;
using PairAlone = PairCfg<5, 2, 2, 2>;
static_assert(PairCo::SMEM + 1024 + 99584 + 1024 <= 233472, "a look-ahead CTA must fit beside a pair CTA");

// The tile enumeration of one pair launch: mode 0 all tm_count x tn_count tiles, mode 1
// the tiles (tm, tn) with tn <= tm of a square grid, mode 2 those with tn >= tm. Tiles are
// grouped into blocks of kGroup x kGroup (kGroup tile rows, taken block by block along them,
// row by row inside a block; triangular blocks on the diagonal), so that the clusters,
// which take consecutive tiles, share a few A and B row blocks in L2 at any time instead
// of sweeping the whole panel once per tile row.
constexpr int64_t kGroup = 8;
struct PairTiles {
    int mode;
    int64_t tm_count, tn_count, total;
};

__device__ __forceinline__ int64_t tri_row(int64_t t) {  // r with r(r+1)/2 <= t < (r+1)(r+2)/2
    int64_t r = (int64_t)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
    while ((r + 1) * (r + 2) / 2 <= t) ++r;
    while (r * (r + 1) / 2 > t) --r;
    return r;
}

__device__ __forceinline__ void pair_tile(const PairTiles& pt, int64_t t, int64_t& tm, int64_t& tn) {
    for (int64_t sr = 0;; ++sr) {  // super row sr: tile rows [kGroup sr, kGroup sr + r)
        const int64_t r0 = kGroup * sr;
        const int64_t r = pt.tm_count - r0 < kGroup ? pt.tm_count - r0 : kGroup;
        const int64_t full_blocks = pt.mode == 0 ? pt.tn_count / kGroup : sr;  // r x kGroup blocks
        const int64_t tail = pt.mode == 0 ? pt.tn_count - full_blocks * kGroup : 0;  // a last narrower block
        const int64_t diag = pt.mode == 0 ? 0 : r * (r + 1) / 2;
        const int64_t count = full_blocks * r * kGroup + tail * r + diag;
        if (t >= count) {
            t -= count;
            continue;
        }
        if (t < full_blocks * r * kGroup) {
            const int64_t blk = t / (r * kGroup), in = t % (r * kGroup);
            tm = r0 + in / kGroup;
            tn = blk * kGroup + in % kGroup;
        } else if (pt.mode == 0) {
            const int64_t in = t - full_blocks * r * kGroup;
            tm = r0 + in / tail;
            tn = full_blocks * kGroup + in % tail;
        } else {
            const int64_t in = t - full_blocks * r * kGroup;
            const int64_t a = tri_row(in);
            tm = r0 + a;
            tn = r0 + (in - a * (a + 1) / 2);
        }
        if (pt.mode == 2) {
            const int64_t x = tm;
            tm = tn;
            tn = x;
        }
        return;
    }
}

template <bool BF16, class Cfg>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(PAIR_THREADS, 1)
    tc_gemm_pair_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                        const __grid_constant__ CUtensorMap tmC, int64_t M, int64_t N, int64_t K, float alpha,
                        float beta, View<float> C, Mask mask, PairTiles pt, int fast, const int* abort, int* err,
                        uint64_t limit_ns) {
    constexpr int KB_ELEMS = KB_BYTES / (BF16 ? 2 : 4);
    constexpr int MMAS_PER_STAGE = KB_BYTES / 32;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* sA = smem;
    constexpr int PAIR_STAGES = Cfg::STAGES, EPI_COLS = Cfg::EPI_COLS, EPI_BOX_BYTES = Cfg::EPI_BOX_BYTES;
    constexpr int EPI_BUFS = Cfg::EPI_BUFS, TBUFS = Cfg::TMEM_BUFS;
    constexpr uint32_t TMEM_COLS = 256u * TBUFS;
    uint8_t* sB = sA + PAIR_STAGES * PAIR_A_BYTES;
    uint8_t* stage_c = sB + PAIR_STAGES * PAIR_B_BYTES;  // 4 warps x EPI_BUFS boxes
    uint64_t* full = reinterpret_cast<uint64_t*>(stage_c + Cfg::STAGING);
    uint64_t* empty = full + PAIR_STAGES;
    uint64_t* tfull = empty + PAIR_STAGES;  // per accumulator buffer
    uint64_t* tempty = tfull + TBUFS;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tempty + TBUFS);
    volatile int* stop = reinterpret_cast<volatile int*>(tmem_slot + 1);
    volatile int* any_stop = stop + 1;

    const uint32_t rank = cluster_rank();
    const int64_t cluster = blockIdx.x >> 1, nclusters = gridDim.x >> 1;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int s = 0; s < PAIR_STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < TBUFS; ++b) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], 2);  // one arrival per CTA's epilogue group (used in the leader)
        }
        // A word already raised stops this CTA's roles before they start (no early return:
        // the peer may have read the word as zero and waits at the cluster barriers).
        *stop = (aborted(abort) || aborted(err)) ? 1 : 0;
        *any_stop = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(&tmA) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(&tmB) : "memory");
        if (fast) asm volatile("prefetch.tensormap [%0];" ::"l"(&tmC) : "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
    }
    tc_fence_before();
    cluster_sync_all();  // barriers of both CTAs initialised, TMEM allocated in both
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const int KB = (int)((K + KB_ELEMS - 1) / KB_ELEMS);
    const int site = kSiteTcPair * 100 + (int)rank;

    if (warp == 0) {
        if (lane == 0) {
            int64_t g = 0;  // k-blocks issued so far, over all tiles of this cluster
            for (int64_t t = cluster; t < pt.total && !*stop; t += nclusters) {
                int64_t tm, tn;
                pair_tile(pt, t, tm, tn);
                const int am = (int)(tm * 256 + 128 * rank), bn = (int)(tn * 256 + 128 * rank);
                for (int kb = 0; kb < KB; ++kb, ++g) {
                    const int s = (int)(g % PAIR_STAGES);
                    const uint32_t ph = (uint32_t)((g / PAIR_STAGES) & 1);
                    const int w = mbar_wait_bounded(&empty[s], ph ^ 1, stop, err, abort, limit_ns);
                    if (w != kWaitOk) {
                        raise_stop(stop, err, w, site + kRoleProducer * 10);
                        break;
                    }
                    if (rank == 0) mbar_expect_tx(&full[s], 2 * (PAIR_A_BYTES + PAIR_B_BYTES));
                    tma_load_2d_pair(sA + s * PAIR_A_BYTES, &tmA, &full[s], kb * KB_ELEMS, am);
                    tma_load_2d_pair(sB + s * PAIR_B_BYTES, &tmB, &full[s], kb * KB_ELEMS, bn);
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0 && rank == 0) {
            const uint32_t fmt = BF16 ? 1u : 2u;
            const uint32_t idesc = (1u << 4) | (fmt << 7) | (fmt << 10) | ((uint32_t)(256 >> 3) << 17) |
                                   ((uint32_t)(256 >> 4) << 24);
            // The tensor pipe idles through every instruction this thread runs between two
            // MMAs, so the ring position is carried incrementally (no division) and the stage
            // descriptors advance by a fixed stride.
            const uint64_t ad0 = sw128_kmajor_desc(sA), bd0 = sw128_kmajor_desc(sB);
            constexpr uint64_t kAStep = PAIR_A_BYTES >> 4, kBStep = PAIR_B_BYTES >> 4;
            int s = 0;
            uint32_t ph = 0;
            int it = 0;
            for (int64_t t = cluster; t < pt.total && !*stop; t += nclusters, ++it) {
                // Both epilogue groups have read the accumulator this tile reuses (tile
                // it - TBUFS); a fresh barrier passes parity 1 at once.
                const int ab = it % TBUFS;
                const uint32_t acc_col = 256u * (uint32_t)ab;
                {
                    const int w = mbar_wait_bounded(&tempty[ab], (uint32_t)(((it / TBUFS) & 1) ^ 1), stop, err,
                                                    abort, limit_ns);
                    if (w != kWaitOk) {
                        raise_stop(stop, err, w, site + kRoleMma * 10);
                        break;
                    }
                    tc_fence_after();
                }
                for (int kb = 0; kb < KB; ++kb) {
                    const int w = mbar_wait_bounded(&full[s], ph, stop, err, abort, limit_ns);
                    if (w != kWaitOk) {
                        raise_stop(stop, err, w, site + kRoleMma * 10);
                        break;
                    }
                    tc_fence_after();
                    const uint64_t ad = ad0 + (uint64_t)s * kAStep, bd = bd0 + (uint64_t)s * kBStep;
#pragma unroll
                    for (int kk = 0; kk < MMAS_PER_STAGE; ++kk)
                        umma_pair<BF16>(tmem + acc_col, ad + 2 * kk, bd + 2 * kk, idesc, (kb | kk) != 0 ? 1u : 0u);
                    umma_commit_pair(&empty[s]);
                    if (++s == PAIR_STAGES) {
                        s = 0;
                        ph ^= 1u;
                    }
                }
                // The tile's accumulator is complete once the MMAs issued so far finish (on a
                // stop: whatever was issued; the epilogue then skips the tile).
                umma_commit_pair(&tfull[ab]);
            }
        }
    } else {
        const int q = warp & 3;  // TMEM lane quadrant this warp may access
        constexpr int EPI_THREADS = 128;
        uint8_t* my_stage = stage_c + q * EPI_BUFS * EPI_BOX_BYTES;
        const bool vec = C.cs == 1 && (C.rs % 4 == 0) && (reinterpret_cast<uintptr_t>(C.p) % 16 == 0);
        int it = 0, issued = 0;
        for (int64_t t = cluster; t < pt.total; t += nclusters, ++it) {
            const int ab = it % TBUFS;
            const uint32_t tacc = tmem + 256u * (uint32_t)ab;
            const int w = mbar_wait_bounded(&tfull[ab], (uint32_t)((it / TBUFS) & 1), stop, err, abort, limit_ns);
            // One decision for all epilogue warps (their barrier below counts them all).
            if (epilogue_any(w != kWaitOk || *stop, EPI_THREADS)) {
                if (w != kWaitOk) raise_stop(stop, err, w, site + kRoleEpilogue * 10);
                else *stop = 1;
                break;
            }
            tc_fence_after();
            int64_t tm, tn;
            pair_tile(pt, t, tm, tn);
            const int64_t m0 = tm * 256, n0 = tn * 256;
            const int64_t r0 = m0 + 128 * rank + 32 * q;  // this warp's first row
            const int64_t i = r0 + lane;
            const bool diag = mask != kFull && tm == tn;
            if (fast && !diag) {
#pragma unroll 1
                for (int c0 = 0; c0 < 256; c0 += EPI_COLS) {
                    float v[16];
                    tmem_ld16(tacc + ((uint32_t)(32 * q) << 16) + (uint32_t)c0, v);
                    uint8_t* box = my_stage + (issued % EPI_BUFS) * EPI_BOX_BYTES;
                    if (issued >= EPI_BUFS) {  // the box written EPI_BUFS steps ago has been read
                        if (lane == 0) bulk_wait_read<EPI_BUFS - 1>();
                        __syncwarp();
                    }
                    // block b of the box: 32 rows x 128 bytes, 16-byte chunks swizzled by row mod 8
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int chunk = u ^ (lane & 7);
                        *reinterpret_cast<float4*>(box + lane * 128 + chunk * 16) =
                            make_float4(alpha * v[4 * u], alpha * v[4 * u + 1], alpha * v[4 * u + 2],
                                        alpha * v[4 * u + 3]);
                    }
#pragma unroll
                    for (int sub = 16; sub < EPI_COLS; sub += 16) {
                        tmem_ld16(tacc + ((uint32_t)(32 * q) << 16) + (uint32_t)(c0 + sub), v);
                        uint8_t* blk = box + (sub / 32) * 4096;
#pragma unroll
                        for (int u = 0; u < 4; ++u) {
                            const int chunk = (((sub % 32) / 4) + u) ^ (lane & 7);
                            *reinterpret_cast<float4*>(blk + lane * 128 + chunk * 16) =
                                make_float4(alpha * v[4 * u], alpha * v[4 * u + 1], alpha * v[4 * u + 2],
                                            alpha * v[4 * u + 3]);
                        }
                    }
                    fence_proxy_async_smem();
                    __syncwarp();
                    if (lane == 0) {
                        tma_reduce_add_3d(&tmC, box, 0, (int)r0, (int)((n0 + c0) / 32));
                        bulk_commit();
                    }
                    ++issued;
                }
            } else {
                const bool row_ok = i < M;
#pragma unroll 1
                for (int c0 = 0; c0 < 256; c0 += 16) {
                    float v[16];
                    tmem_ld16(tacc + ((uint32_t)(32 * q) << 16) + (uint32_t)c0, v);
                    if (!row_ok) continue;
                    const int64_t j0 = n0 + c0;
                    if (vec && j0 + 15 < N && keep(mask, 0, i, j0 + 15) && keep(mask, 0, i, j0)) {
                        float4* dst = reinterpret_cast<float4*>(C.p + i * C.rs + j0);
#pragma unroll
                        for (int u = 0; u < 4; ++u) {
                            float4 r = make_float4(alpha * v[4 * u], alpha * v[4 * u + 1], alpha * v[4 * u + 2],
                                                   alpha * v[4 * u + 3]);
                            if (beta != 0.f) {
                                const float4 c = dst[u];
                                r.x = fmaf(beta, c.x, r.x); r.y = fmaf(beta, c.y, r.y);
                                r.z = fmaf(beta, c.z, r.z); r.w = fmaf(beta, c.w, r.w);
                            }
                            dst[u] = r;
                        }
                    } else {
#pragma unroll
                        for (int u = 0; u < 16; ++u) {
                            const int64_t j = j0 + u;
                            if (j >= N || !keep(mask, 0, i, j)) continue;
                            float r = alpha * v[u];
                            if (beta != 0.f) r = fmaf(beta, C(i, j), r);
                            C(i, j) = r;
                        }
                    }
                }
            }
            // This CTA's reads of the accumulator are done: release it to the leader's MMAs.
            tc_fence_before();
            asm volatile("bar.sync 1, %0;" ::"r"(EPI_THREADS) : "memory");
            if (warp == 2 && lane == 0) mbar_arrive_cluster(&tempty[ab], 0);
        }
        if (lane == 0) bulk_wait_all();  // every reduce-add of this warp has landed
    }
    tc_fence_before();
    __syncthreads();  // this CTA's roles are over: *stop is final
    if (threadIdx.x == 0 && *stop) {
        st_cluster_u32((const void*)any_stop, 0, 1u);
        st_cluster_u32((const void*)any_stop, 1, 1u);
    }
    __syncwarp();
    cluster_sync_all();  // the leader's MMAs read this CTA's shared memory until its last tfull
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
    }
    if (threadIdx.x == 0 && *any_stop) settle(kSettleNs);
}

// x rounded to the nearest TF32 value (10 explicit mantissa bits, the low 13 bits zero;
// ties away from zero): exactly what the tensor cores read from a kind::tf32 operand.
__device__ __forceinline__ float tf32_rn(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// Split x into hi = tf32_rn(x) and lo = tf32_rn(x - hi) (x - hi is exact in FP32 and below
// half an ulp of hi, so |x - hi - lo| <= 2^-22 |x|), writing K-major copies: dst row r =
// [part(p0) | part(p1) | part(p2)], each segment of width K (0 = hi, 1 = lo). Both parts
// are TF32 values, so the tensor cores drop none of their bits.
__global__ void split3_kernel(int64_t rows, int64_t K, View<const float> X, float* dst, int64_t ldd, int p0, int p1,
                              int p2) {
    for (int64_t r = blockIdx.y; r < rows; r += gridDim.y)
        for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < K; k += (int64_t)gridDim.x * blockDim.x) {
            const float x = X(r, k);
            const float hi = tf32_rn(x);
            const float lo = tf32_rn(x - hi);
            float* row = dst + r * ldd;
            row[k] = p0 ? lo : hi;
            row[K + k] = p1 ? lo : hi;
            row[2 * K + k] = p2 ? lo : hi;
        }
}

template <class Src>
__global__ void pack_kmajor_kernel(int64_t rows, int64_t K, View<const Src> X, void* dst, int64_t ldd, bool bf16) {
    for (int64_t r = blockIdx.y; r < rows; r += gridDim.y)
        for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < K; k += (int64_t)gridDim.x * blockDim.x) {
            const float x = (float)X(r, k);
            if (bf16) static_cast<__nv_bfloat16*>(dst)[r * ldd + k] = __float2bfloat16_rn(x);
            else static_cast<float*>(dst)[r * ldd + k] = x;
        }
}

PFN_cuTensorMapEncodeTiled_v12000 encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

bool make_tmap(CUtensorMap* tm, const void* base, bool bf16, int64_t rows, int64_t kdim, int64_t ld, int box_rows) {
    auto enc = encoder();
    if (!enc) return false;
    const int es = bf16 ? 2 : 4;
    cuuint64_t dims[2] = {(cuuint64_t)kdim, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)ld * es};
    cuuint32_t box[2] = {(cuuint32_t)(KB_BYTES / es), (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    return enc(tm, bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
               const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Tensor map of a row-major FP32 C (rows x cols, row stride ld, cols a multiple of 32) for
// the pair epilogue's reduce-adds, as (column within a 32-column block, row, block): boxes
// of 32 rows x blk blocks, 128-byte swizzle (the staging layout).
bool make_c_tmap(CUtensorMap* tm, const float* base, int64_t rows, int64_t cols, int64_t ld, int blk) {
    auto enc = encoder();
    if (!enc || cols % 32) return false;
    cuuint64_t dims[3] = {32u, (cuuint64_t)rows, (cuuint64_t)(cols / 32)};
    cuuint64_t strides[2] = {(cuuint64_t)ld * 4, 128u};
    cuuint32_t box[3] = {32u, 32u, (cuuint32_t)blk};
    cuuint32_t estr[3] = {1, 1, 1};
    return enc(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_NONE,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Dynamic shared memory of a pair CTA: the configuration's ring, staging boxes and barriers,
// and at least half of an SM's shared memory so that no SM ever holds two pair CTAs.
size_t pair_smem_bytes(size_t base) {
    static int per_sm[64] = {}, reserved[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
    if (!per_sm[dev]) {
        if (cudaDeviceGetAttribute(&per_sm[dev], cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&reserved[dev], cudaDevAttrReservedSharedMemoryPerBlock, dev) != cudaSuccess)
            return 0;
    }
    const size_t half = (size_t)per_sm[dev] / 2 + 16 - (size_t)reserved[dev];  // two such CTAs do not fit
    return base > half ? base : (half + 127) / 128 * 128;
}

template <bool BF16, class Cfg>
int launch_tc_pair(const CUtensorMap& ta, const CUtensorMap& tb, int64_t m, int64_t n, int64_t k, float alpha,
                   float beta, View<float> C, Mask mask, int64_t off, cudaStream_t s, const int* abort,
                   int reserve_sms) {
    PairTiles pt;
    pt.tm_count = (m + 255) / 256;
    pt.tn_count = (n + 255) / 256;
    if (mask == kFull) {
        pt.mode = 0;
        pt.total = pt.tm_count * pt.tn_count;
    } else if (off == 0 && m == n) {
        pt.mode = mask == kLower ? 1 : 2;
        pt.total = pt.tm_count * (pt.tm_count + 1) / 2;
    } else {
        return RC_ERR_NOT_SUPPORTED;
    }
    CUtensorMap tc;
    std::memset(&tc, 0, sizeof(tc));
    const bool fast = beta == 1.f && C.cs == 1 && C.rs % 4 == 0 && reinterpret_cast<uintptr_t>(C.p) % 16 == 0 &&
                      make_c_tmap(&tc, C.p, m, n, C.rs, Cfg::EPI_BLK);
    const size_t smem = pair_smem_bytes(Cfg::SMEM);
    if (smem == 0 || smem > 232448) return RC_ERR_NOT_SUPPORTED;
    if (cudaFuncSetAttribute(tc_gemm_pair_kernel<BF16, Cfg>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) != cudaSuccess)
        return RC_ERR_CUDA;
    const int64_t avail = (int64_t)(sm_count() - (reserve_sms > 0 ? reserve_sms : 0)) / 2;
    const int64_t clusters = pt.total < (avail > 0 ? avail : 1) ? pt.total : (avail > 0 ? avail : 1);
    tc_gemm_pair_kernel<BF16, Cfg><<<(unsigned)(2 * clusters), PAIR_THREADS, smem, s>>>(
        ta, tb, tc, m, n, k, alpha, beta, C, mask, pt, fast ? 1 : 0, abort, error_word(), wait_limit_ns());
    return check_launch();
}

template <int BN, bool BF16, bool FOLD = false>
int launch_tc(const CUtensorMap& ta, const CUtensorMap& tb, int64_t m, int64_t n, int64_t k, float alpha, float beta,
              View<float> C, Mask mask, int64_t off, cudaStream_t s, const int* abort) {
    const size_t smem = TcCfg<BN, FOLD>::SMEM;
    if (cudaFuncSetAttribute(tc_gemm_kernel<BN, BF16, FOLD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) != cudaSuccess)
        return RC_ERR_CUDA;
    dim3 grid(FOLD ? 1u : ceil_div(n, BN), ceil_div(m, 128));
    if (grid.y > 65535) return RC_ERR_NOT_SUPPORTED;
    tc_gemm_kernel<BN, BF16, FOLD><<<grid, TC_THREADS, smem, s>>>(ta, tb, m, n, k, alpha, beta, C, mask, off, abort,
                                                                  error_word(), wait_limit_ns());
    return check_launch();
}

}  // namespace

void* tensor_map_encoder() { return reinterpret_cast<void*>(encoder()); }

int gemm_tc_kmajor(bool bf16, int64_t m, int64_t n, int64_t k, float alpha, const void* A, int64_t lda, const void* B,
                   int64_t ldb, float beta, View<float> C, Mask mask, int64_t off, cudaStream_t s, const int* abort,
                   int bn) {
    if (m <= 0 || n <= 0) return RC_SUCCESS;
    if (k <= 0) return gemm<float>(m, n, 0, alpha, View<const float>{nullptr, 1, 1}, View<const float>{nullptr, 1, 1},
                                   beta, C, mask, off, s, abort);
    const int es = bf16 ? 2 : 4;
    if ((reinterpret_cast<uintptr_t>(A) % 16) || (reinterpret_cast<uintptr_t>(B) % 16) || ((lda * es) % 16) ||
        ((ldb * es) % 16) || m > (int64_t)INT32_MAX || n > (int64_t)INT32_MAX || k > (int64_t)INT32_MAX)
        return RC_ERR_NOT_SUPPORTED;
    if (bn != 128 && bn != 256) bn = n > 128 ? 256 : 128;
    CUtensorMap ta, tb;
    if (!make_tmap(&ta, A, bf16, m, k, lda, 128) || !make_tmap(&tb, B, bf16, n, k, ldb, bn)) return RC_ERR_NOT_SUPPORTED;
    if (bf16) {
        return bn == 256 ? launch_tc<256, true>(ta, tb, m, n, k, alpha, beta, C, mask, off, s, abort)
                         : launch_tc<128, true>(ta, tb, m, n, k, alpha, beta, C, mask, off, s, abort);
    }
    return bn == 256 ? launch_tc<256, false>(ta, tb, m, n, k, alpha, beta, C, mask, off, s, abort)
                     : launch_tc<128, false>(ta, tb, m, n, k, alpha, beta, C, mask, off, s, abort);
}

int gemm_tc_pair_kmajor(bool bf16, int64_t m, int64_t n, int64_t k, float alpha, const void* A, int64_t lda,
                        const void* B, int64_t ldb, float beta, View<float> C, Mask mask, int64_t off, cudaStream_t s,
                        const int* abort, int reserve_sms, bool beside) {
    if (m <= 0 || n <= 0) return RC_SUCCESS;
    const int es = bf16 ? 2 : 4;
    if (k <= 0 || (reinterpret_cast<uintptr_t>(A) % 16) || (reinterpret_cast<uintptr_t>(B) % 16) || ((lda * es) % 16) ||
        ((ldb * es) % 16) || m > (int64_t)INT32_MAX || n > (int64_t)INT32_MAX || k > (int64_t)INT32_MAX)
        return RC_ERR_NOT_SUPPORTED;
    CUtensorMap ta, tb;
    if (!make_tmap(&ta, A, bf16, m, k, lda, 128) || !make_tmap(&tb, B, bf16, n, k, ldb, 128)) return RC_ERR_NOT_SUPPORTED;
    if (beside)
        return bf16 ? launch_tc_pair<true, PairCo>(ta, tb, m, n, k, alpha, beta, C, mask, off, s, abort, reserve_sms)
                    : launch_tc_pair<false, PairCo>(ta, tb, m, n, k, alpha, beta, C, mask, off, s, abort, reserve_sms);
    return bf16 ? launch_tc_pair<true, PairAlone>(ta, tb, m, n, k, alpha, beta, C, mask, off, s, abort, reserve_sms)
                : launch_tc_pair<false, PairAlone>(ta, tb, m, n, k, alpha, beta, C, mask, off, s, abort, reserve_sms);
}

int gemm_tc_fold_kmajor(int64_t m, int64_t k, float alpha, const float* A, int64_t lda, const float* B, int64_t ldb,
                        float beta, View<float> C, cudaStream_t s, const int* abort) {
    if (m <= 0) return RC_SUCCESS;
    if (k <= 0 || (reinterpret_cast<uintptr_t>(A) % 16) || (reinterpret_cast<uintptr_t>(B) % 16) ||
        ((lda * 4) % 16) || ((ldb * 4) % 16) || m > (int64_t)INT32_MAX || k > (int64_t)INT32_MAX)
        return RC_ERR_NOT_SUPPORTED;
    CUtensorMap ta, tb;
    if (!make_tmap(&ta, A, false, m, k, lda, 128) || !make_tmap(&tb, B, false, 128, k, ldb, 128))
        return RC_ERR_NOT_SUPPORTED;
    return launch_tc<128, false, true>(ta, tb, m, 64, k, alpha, beta, C, kFull, 0, s, abort);
}

// One warp waits, bounded, on an mbarrier phase that nothing completes: exercises the
// timeout path of every tcgen05 kernel's waits without touching any other state.
__global__ void wait_selftest_kernel(int* err, uint64_t limit_ns) {
    __shared__ uint64_t bar;
    __shared__ int stop;
    if (threadIdx.x == 0) {
        stop = 0;
        mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    if (threadIdx.x == 0) {
        const int w = mbar_wait_bounded(&bar, 0, &stop, err, nullptr, limit_ns);
        if (w != kWaitOk) raise_stop(&stop, err, w, kSiteSelftest * 100);
    }
}

int pack_kmajor(int64_t rows, int64_t K, View<const float> X, void* dst, int64_t ldd, bool bf16, cudaStream_t s) {
    if (rows <= 0 || K <= 0) return RC_SUCCESS;
    dim3 grid(ceil_div(K, 256) < 64u ? ceil_div(K, 256) : 64u, rows < 65535 ? (unsigned)rows : 65535u);
    pack_kmajor_kernel<float><<<grid, 256, 0, s>>>(rows, K, X, dst, ldd, bf16);
    return check_launch();
}

int gemm_tf32(int64_t m, int64_t n, int64_t k, float alpha, View<const float> A, View<const float> B, float beta,
              View<float> C, Mask mask, int64_t off, bool split, cudaStream_t s, const int* abort) {
    if (m <= 0 || n <= 0) return RC_SUCCESS;
    if (k <= 0) return gemm<float>(m, n, k, alpha, A, B, beta, C, mask, off, s, abort);
    // Operands as K-major buffers: A (m x k) rows, B^T (n x k) rows; ld rounded to 32 floats.
    const int64_t kk = split ? 3 * k : k;
    const int64_t ld = (kk + 31) / 32 * 32;
    float* a = static_cast<float*>(workspace(s, (size_t)m * ld * sizeof(float), 4));
    float* b = static_cast<float*>(workspace(s, (size_t)n * ld * sizeof(float), 5));
    if (!a || !b) return RC_ERR_ALLOC;
    const View<const float> Bt = B.t();  // n x k
    dim3 ga(ceil_div(k, 256) < 64u ? ceil_div(k, 256) : 64u, m < 65535 ? (unsigned)m : 65535u);
    dim3 gb(ceil_div(k, 256) < 64u ? ceil_div(k, 256) : 64u, n < 65535 ? (unsigned)n : 65535u);
    if (split) {
        split3_kernel<<<ga, 256, 0, s>>>(m, k, A, a, ld, 0, 0, 1);
        split3_kernel<<<gb, 256, 0, s>>>(n, k, Bt, b, ld, 0, 1, 0);
    } else {
        pack_kmajor_kernel<float><<<ga, 256, 0, s>>>(m, k, A, a, ld, false);
        pack_kmajor_kernel<float><<<gb, 256, 0, s>>>(n, k, Bt, b, ld, false);
    }
    RC_TRY(check_launch());
    // CTA pairs on 256 x 256 tiles where the pair kernel takes the mask; else 128-row tiles.
    if (m >= 256 && n >= 256 && (mask == kFull || (off == 0 && m == n)))
        return gemm_tc_pair_kmajor(false, m, n, kk, alpha, a, ld, b, ld, beta, C, mask, off, s, abort, 0, false);
    return gemm_tc_kmajor(false, m, n, kk, alpha, a, ld, b, ld, beta, C, mask, off, s, abort, 0);
}

}  // namespace rc

extern "C" {

int rc_gemm_tf32(int transA, int transB, size_t m, size_t n, size_t k, float alpha, const float* A, size_t lda,
                 const float* B, size_t ldb, float beta, float* C, size_t ldc, void* stream) {
    if (m == 0 || n == 0) return RC_SUCCESS;
    if (!C || ldc < m) return RC_ERR_INVALID_ARGUMENT;
    if (k > 0 && (!A || !B || lda < (transA ? k : m) || ldb < (transB ? n : k))) return RC_ERR_INVALID_ARGUMENT;
    rc::View<const float> a = rc::colmajor(A, (int64_t)lda), b = rc::colmajor(B, (int64_t)ldb);
    if (transA) a = a.t();
    if (transB) b = b.t();
    return rc::gemm_tf32((int64_t)m, (int64_t)n, (int64_t)k, alpha, a, b, beta, rc::colmajor(C, (int64_t)ldc),
                         rc::kFull, 0, false, static_cast<cudaStream_t>(stream));
}

int rc_gemm_bf16(int transA, int transB, size_t m, size_t n, size_t k, float alpha, const float* A, size_t lda,
                 const float* B, size_t ldb, float beta, float* C, size_t ldc, void* stream) {
    if (m == 0 || n == 0) return RC_SUCCESS;
    if (!C || ldc < m) return RC_ERR_INVALID_ARGUMENT;
    if (k > 0 && (!A || !B || lda < (transA ? k : m) || ldb < (transB ? n : k))) return RC_ERR_INVALID_ARGUMENT;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    rc::View<const float> a = rc::colmajor(A, (int64_t)lda), b = rc::colmajor(B, (int64_t)ldb);
    if (transA) a = a.t();
    if (transB) b = b.t();
    if (k == 0)
        return rc::gemm<float>((int64_t)m, (int64_t)n, 0, alpha, a, b, beta, rc::colmajor(C, (int64_t)ldc), rc::kFull,
                               0, s);
    const int64_t ld = ((int64_t)k + 63) / 64 * 64;
    void* pa = rc::workspace(s, m * ld * 2, 4);
    void* pb = rc::workspace(s, n * ld * 2, 5);
    if (!pa || !pb) return RC_ERR_ALLOC;
    RC_TRY(rc::pack_kmajor((int64_t)m, (int64_t)k, a, pa, ld, true, s));
    RC_TRY(rc::pack_kmajor((int64_t)n, (int64_t)k, b.t(), pb, ld, true, s));
    return rc::gemm_tc_kmajor(true, (int64_t)m, (int64_t)n, (int64_t)k, alpha, pa, ld, pb, ld, beta,
                              rc::colmajor(C, (int64_t)ldc), rc::kFull, 0, s);
}

int rc_syrk_tc_ex(int precision, size_t n, size_t k, float alpha, const void* P, size_t ldp, float beta, float* C,
                  size_t ldc, int flags, void* stream) {
    if (precision != RC_PREC_TF32 && precision != RC_PREC_BF16) return RC_ERR_INVALID_ARGUMENT;
    if (flags & ~RC_SYRK_BESIDE) return RC_ERR_INVALID_ARGUMENT;
    if (n == 0) return RC_SUCCESS;
    if (!C || ldc < n || (k > 0 && (!P || ldp < k))) return RC_ERR_INVALID_ARGUMENT;
    const bool bf16 = precision == RC_PREC_BF16;
    const rc::View<float> Cv{C, (int64_t)ldc, 1};
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (k > 0 && n >= 256)  // CTA pairs on 256 x 256 tiles
        return rc::gemm_tc_pair_kmajor(bf16, (int64_t)n, (int64_t)n, (int64_t)k, alpha, P, (int64_t)ldp, P,
                                       (int64_t)ldp, beta, Cv, rc::kLower, 0, s, nullptr, 0,
                                       (flags & RC_SYRK_BESIDE) != 0);
    return rc::gemm_tc_kmajor(bf16, (int64_t)n, (int64_t)n, (int64_t)k, alpha, P, (int64_t)ldp, P, (int64_t)ldp, beta,
                              Cv, rc::kLower, 0, s);
}

int rc_syrk_tc(int precision, size_t n, size_t k, float alpha, const void* P, size_t ldp, float beta, float* C,
               size_t ldc, void* stream) {
    return rc_syrk_tc_ex(precision, n, k, alpha, P, ldp, beta, C, ldc, 0, stream);
}

int rc_selftest_wait_timeout(uint64_t limit_ns, void* stream) {
    int* err = rc::error_word();
    if (!err) return RC_ERR_ALLOC;
    rc::wait_selftest_kernel<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(err, limit_ns);
    return rc::check_launch();
}

int rc_device_error_site(void* stream, int* site) {
    if (cudaStreamSynchronize(static_cast<cudaStream_t>(stream)) != cudaSuccess) return RC_ERR_CUDA;
    int* w = rc::error_word();
    if (!w) return RC_ERR_ALLOC;
    int v[2] = {0, 0};
    if (cudaMemcpy(v, w, sizeof(v), cudaMemcpyDeviceToHost) != cudaSuccess) return RC_ERR_CUDA;
    if ((v[0] != 0 || v[1] != 0) && cudaMemset(w, 0, sizeof(v)) != cudaSuccess) return RC_ERR_CUDA;
    if (site) *site = v[1];
    return v[0];
}

int rc_device_status(void* stream) { return rc_device_error_site(stream, nullptr); }

}  // extern "C"
