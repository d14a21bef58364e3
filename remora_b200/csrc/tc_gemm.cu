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
            for (int kb = 0; kb < KB; ++kb) {
                const int s = kb % STAGES;
                const uint32_t ph = (kb / STAGES) & 1;
                const int w = mbar_wait_bounded(&full[s], ph, stop, err, abort, limit_ns);
                if (w != kWaitOk) {
                    raise_stop(stop, err, w, kSiteTcGemm * 100 + kRoleMma * 10);
                    break;
                }
                tc_fence_after();
                const uint64_t ad = sw128_kmajor_desc(sA + s * Cfg::A_BYTES);
                const uint64_t bd = sw128_kmajor_desc(sB + s * Cfg::B_BYTES);
#pragma unroll
                for (int kk = 0; kk < MMAS_PER_STAGE; ++kk)
                    umma<BF16>(tmem, ad + 2 * kk, bd + 2 * kk, idesc, (kb | kk) != 0 ? 1u : 0u);
                umma_commit(&empty[s]);
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

// Pair kernel: a cluster of two CTAs computes one 256 x 256 tile with
// tcgen05.mma.cta_group::2. CTA rank r (0 = the leader) stages rows [128 r, 128 r + 128)
// of the tile's A rows and of its B rows (K-major) in its own shared memory at the same
// offsets, and holds the accumulator of its 128 rows (x 256 columns) in its own TMEM.
// Both CTAs issue their TMA loads against the leader's full barrier (peer bit cleared),
// whose expected byte count covers both; one thread of the leader issues the MMAs and
// commits every stage to the empty barriers of both CTAs and the final product to both
// done barriers. Per SM and k-slice this moves 32 KB for a 128 x 256 x 32 product instead
// of 48 KB, halving the B traffic of the single-CTA 128 x 256 tile. Two CTAs per SM
// (3 stages each, 256 TMEM columns each).
//
// Failure handling. Every mbarrier wait is bounded and gives up as soon as the device error
// word or the abort word is raised. The two CTAs may take different decisions (one sees a
// word the other read as zero), so neither returns early after the first cluster barrier:
// a stopped CTA still reaches the closing barrier, and before it each CTA writes its stop
// flag into both CTAs' `any_stop`. When either stopped, both stay resident for a settle
// period after the closing barrier, so that copies issued by either CTA (whose completion
// counts on the leader's barrier, which nobody waits for any more) land first. Neither
// cluster barrier can wait forever: every thread of both CTAs reaches each one after a
// bounded number of bounded waits. TMEM allocation cannot wait forever either: at most two
// tcgen05 CTAs (of any of this library's kernels) fit on an SM by shared memory, each
// holding at most 256 of the 512 columns, and a CTA holding columns never waits on a CTA
// that does not.
constexpr int PAIR_STAGES = 3;
constexpr int PAIR_A_BYTES = 128 * KB_BYTES, PAIR_B_BYTES = 128 * KB_BYTES;
constexpr size_t PAIR_SMEM = (size_t)PAIR_STAGES * (PAIR_A_BYTES + PAIR_B_BYTES) + 1024 + 256;

template <bool BF16>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(TC_THREADS, 2)
    tc_gemm_pair_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, int64_t M,
                        int64_t N, int64_t K, float alpha, float beta, View<float> C, Mask mask, int64_t off,
                        const int* abort, int* err, uint64_t limit_ns) {
    constexpr int KB_ELEMS = KB_BYTES / (BF16 ? 2 : 4);
    constexpr int MMAS_PER_STAGE = KB_BYTES / 32;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* sA = smem;
    uint8_t* sB = smem + PAIR_STAGES * PAIR_A_BYTES;
    uint64_t* full = reinterpret_cast<uint64_t*>(sB + PAIR_STAGES * PAIR_B_BYTES);
    uint64_t* empty = full + PAIR_STAGES;
    uint64_t* done = empty + PAIR_STAGES;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
    volatile int* stop = reinterpret_cast<volatile int*>(tmem_slot + 1);
    volatile int* any_stop = stop + 1;

    const uint32_t rank = cluster_rank();
    const int64_t m0 = (int64_t)blockIdx.y * 256, n0 = (int64_t)(blockIdx.x >> 1) * 256;
    if (outside(mask, off, m0, n0, 256, 256)) return;  // the same decision in both CTAs
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int s = 0; s < PAIR_STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(done, 1);
        // A word already raised stops this CTA's roles before they start (no early return:
        // the peer may have read the word as zero and waits at the cluster barriers).
        *stop = (aborted(abort) || aborted(err)) ? 1 : 0;
        *any_stop = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(&tmA) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(&tmB) : "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(256u));
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
            for (int kb = 0; kb < KB && !*stop; ++kb) {
                const int s = kb % PAIR_STAGES;
                const uint32_t ph = (kb / PAIR_STAGES) & 1;
                const int w = mbar_wait_bounded(&empty[s], ph ^ 1, stop, err, abort, limit_ns);
                if (w != kWaitOk) {
                    raise_stop(stop, err, w, site + kRoleProducer * 10);
                    break;
                }
                if (rank == 0) mbar_expect_tx(&full[s], 2 * (PAIR_A_BYTES + PAIR_B_BYTES));
                tma_load_2d_pair(sA + s * PAIR_A_BYTES, &tmA, &full[s], kb * KB_ELEMS, (int)(m0 + 128 * rank));
                tma_load_2d_pair(sB + s * PAIR_B_BYTES, &tmB, &full[s], kb * KB_ELEMS, (int)(n0 + 128 * rank));
            }
        }
    } else if (warp == 1) {
        if (lane == 0 && rank == 0) {
            const uint32_t fmt = BF16 ? 1u : 2u;
            const uint32_t idesc = (1u << 4) | (fmt << 7) | (fmt << 10) | ((uint32_t)(256 >> 3) << 17) |
                                   ((uint32_t)(256 >> 4) << 24);
            for (int kb = 0; kb < KB && !*stop; ++kb) {
                const int s = kb % PAIR_STAGES;
                const uint32_t ph = (kb / PAIR_STAGES) & 1;
                const int w = mbar_wait_bounded(&full[s], ph, stop, err, abort, limit_ns);
                if (w != kWaitOk) {
                    raise_stop(stop, err, w, site + kRoleMma * 10);
                    break;
                }
                tc_fence_after();
                const uint64_t ad = sw128_kmajor_desc(sA + s * PAIR_A_BYTES);
                const uint64_t bd = sw128_kmajor_desc(sB + s * PAIR_B_BYTES);
#pragma unroll
                for (int kk = 0; kk < MMAS_PER_STAGE; ++kk)
                    umma_pair<BF16>(tmem, ad + 2 * kk, bd + 2 * kk, idesc, (kb | kk) != 0 ? 1u : 0u);
                umma_commit_pair(&empty[s]);
            }
            // Always committed: the done barriers of both CTAs complete once the MMAs issued
            // so far (possibly none) are finished.
            umma_commit_pair(done);
        }
    } else {
        const int q = warp & 3;  // TMEM lane quadrant this warp may access
        const int w = mbar_wait_bounded(done, 0, stop, err, abort, limit_ns);
        const bool ok = w == kWaitOk;
        if (!ok) raise_stop(stop, err, w, site + kRoleEpilogue * 10);
        tc_fence_after();
        if (__all_sync(0xffffffffu, ok && !*stop)) {
            const int64_t i = m0 + 128 * rank + 32 * q + lane;
            const bool row_ok = i < M;
            const bool vec = C.cs == 1 && (C.rs % 4 == 0) && (reinterpret_cast<uintptr_t>(C.p) % 16 == 0);
#pragma unroll 1
            for (int c0 = 0; c0 < 256; c0 += 16) {
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
    __syncthreads();  // this CTA's roles are over: *stop is final
    if (threadIdx.x == 0 && *stop) {
        st_cluster_u32((const void*)any_stop, 0, 1u);
        st_cluster_u32((const void*)any_stop, 1, 1u);
    }
    cluster_sync_all();  // the leader's MMAs read this CTA's shared memory until `done`
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256u));
    }
    if (threadIdx.x == 0 && *any_stop) settle(kSettleNs);
}

template <bool BF16>
int launch_tc_pair(const CUtensorMap& ta, const CUtensorMap& tb, int64_t m, int64_t n, int64_t k, float alpha,
                   float beta, View<float> C, Mask mask, int64_t off, cudaStream_t s, const int* abort) {
    if (cudaFuncSetAttribute(tc_gemm_pair_kernel<BF16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)PAIR_SMEM) != cudaSuccess)
        return RC_ERR_CUDA;
    dim3 grid(2 * ceil_div(n, 256), ceil_div(m, 256));
    if (grid.y > 65535) return RC_ERR_NOT_SUPPORTED;
    tc_gemm_pair_kernel<BF16><<<grid, TC_THREADS, PAIR_SMEM, s>>>(ta, tb, m, n, k, alpha, beta, C, mask, off, abort,
                                                                  error_word(), wait_limit_ns());
    return check_launch();
}

// Split x into TF32 high part (low 13 mantissa bits cleared) and the FP32 remainder,
// writing K-major copies: dst row r = [hi(.., k) | hi or lo | ...] per `pattern`.
// Operand layout in dst (rows x 3K, ld = ldd): segments s = 0, 1, 2 of width K hold
// part[pattern[s]] (0 = hi, 1 = lo).
__global__ void split3_kernel(int64_t rows, int64_t K, View<const float> X, float* dst, int64_t ldd, int p0, int p1,
                              int p2) {
    for (int64_t r = blockIdx.y; r < rows; r += gridDim.y)
        for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < K; k += (int64_t)gridDim.x * blockDim.x) {
            const float x = X(r, k);
            const float hi = __uint_as_float(__float_as_uint(x) & 0xFFFFE000u);
            const float lo = x - hi;
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
                        const int* abort) {
    if (m <= 0 || n <= 0) return RC_SUCCESS;
    const int es = bf16 ? 2 : 4;
    if (k <= 0 || (reinterpret_cast<uintptr_t>(A) % 16) || (reinterpret_cast<uintptr_t>(B) % 16) || ((lda * es) % 16) ||
        ((ldb * es) % 16) || m > (int64_t)INT32_MAX || n > (int64_t)INT32_MAX || k > (int64_t)INT32_MAX)
        return RC_ERR_NOT_SUPPORTED;
    CUtensorMap ta, tb;
    if (!make_tmap(&ta, A, bf16, m, k, lda, 128) || !make_tmap(&tb, B, bf16, n, k, ldb, 128)) return RC_ERR_NOT_SUPPORTED;
    return bf16 ? launch_tc_pair<true>(ta, tb, m, n, k, alpha, beta, C, mask, off, s, abort)
                : launch_tc_pair<false>(ta, tb, m, n, k, alpha, beta, C, mask, off, s, abort);
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

int rc_syrk_tc(int precision, size_t n, size_t k, float alpha, const void* P, size_t ldp, float beta, float* C,
               size_t ldc, void* stream) {
    if (precision != RC_PREC_TF32 && precision != RC_PREC_BF16) return RC_ERR_INVALID_ARGUMENT;
    if (n == 0) return RC_SUCCESS;
    if (!C || ldc < n || (k > 0 && (!P || ldp < k))) return RC_ERR_INVALID_ARGUMENT;
    const bool bf16 = precision == RC_PREC_BF16;
    const rc::View<float> Cv{C, (int64_t)ldc, 1};
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (k > 0 && n >= 256)  // CTA pairs on 256 x 256 tiles
        return rc::gemm_tc_pair_kmajor(bf16, (int64_t)n, (int64_t)n, (int64_t)k, alpha, P, (int64_t)ldp, P,
                                       (int64_t)ldp, beta, Cv, rc::kLower, 0, s);
    return rc::gemm_tc_kmajor(bf16, (int64_t)n, (int64_t)n, (int64_t)k, alpha, P, (int64_t)ldp, P, (int64_t)ldp, beta,
                              Cv, rc::kLower, 0, s);
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
