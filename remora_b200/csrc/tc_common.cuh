// Device helpers for the tcgen05 / TMA / mbarrier kernels (sm_100a inline PTX).
#pragma once
#include <cuda.h>
#include "common.cuh"
#include "gemm.cuh"

namespace rc {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Bounded waits. Every spin of the tensor-core pipelines is limited by the SM's own cycle
// counter (clock64: per SM, monotonic, unaffected by changes of the GPU's global timer),
// 2 cycles per nanosecond of the library's wait limit, i.e. at least that wall time at any
// SM clock up to 2 GHz.
__device__ __forceinline__ long long wait_cycles(uint64_t limit_ns) { return (long long)(limit_ns * 2u); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ bool aborted(const int* abort) { return abort != nullptr && *(volatile const int*)abort != 0; }

// Outcome of a bounded wait.
enum WaitResult { kWaitOk = 0, kWaitAborted = 1, kWaitTimeout = 2 };

// Bounded wait on an mbarrier phase. kWaitAborted: this CTA's *stop was raised, or one of
// the device-wide words err (the library's error word: a wait somewhere timed out) and
// abort (a failed pivot of the factorisation) became non-zero -- every CTA of every
// tensor-core kernel gives up within microseconds of the first failure instead of waiting
// out its own limit. kWaitTimeout: the limit ran out.
__device__ __forceinline__ int mbar_wait_bounded(uint64_t* bar, uint32_t parity, volatile int* stop, const int* err,
                                                 const int* abort, uint64_t limit_ns) {
    if (mbar_try(bar, parity)) return kWaitOk;
    const long long t0 = clock64(), lim = wait_cycles(limit_ns);
    for (uint32_t it = 1;; ++it) {
        if (mbar_try(bar, parity)) return kWaitOk;
        if (*stop) return kWaitAborted;
        if ((it & 15u) == 0 && (aborted(err) || aborted(abort))) return kWaitAborted;
        if (clock64() - t0 > lim) return kWaitTimeout;
    }
}

// Where a wait ran out (the second int of the error word): kernel * 100 + role * 10 + the
// CTA's rank in its cluster.
enum WaitKernel { kSiteTcGemm = 1, kSiteTcPair = 2, kSiteOzaki = 3, kSiteEmu = 4, kSiteSelftest = 9 };
enum WaitRole { kRoleProducer = 0, kRoleMma = 1, kRoleEpilogue = 2, kRoleDrain = 3 };

// Stop this CTA's roles; on a timeout also record RC_ERR_TIMEOUT (and, for the first one on
// the device, its site) in the error word, which stops every other CTA's waits.
__device__ __forceinline__ void raise_stop(volatile int* stop, int* err, int result, int site) {
    *stop = 1;
    if (result == kWaitTimeout && err != nullptr) {
        if (atomicCAS(err, 0, RC_ERR_TIMEOUT) == 0) atomicExch(err + 1, site);
        __threadfence();
    }
}

// After a stop, keep the CTA (and its shared memory) alive for about `ns` so that bulk copies
// it or its pair peer issued, and that nothing waits for any more, land before the memory is
// handed to another CTA.
__device__ __forceinline__ void settle(uint64_t ns) {
    const long long t0 = clock64(), lim = wait_cycles(ns);
    while (clock64() - t0 < lim) __nanosleep(1000);
}
constexpr uint64_t kSettleNs = 2000000;  // 2 ms: a bulk copy of a few KB takes microseconds

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* tm, uint64_t* bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::
            "r"(smem_u32(dst)),
        "l"(tm), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 128B-swizzled K-major operand tile: rows of 128 bytes, 8-row groups 1024 bytes apart
// (stride byte offset), descriptor version 1, layout type 2 (SWIZZLE_128B).
__device__ __forceinline__ uint64_t sw128_kmajor_desc(const void* p) {
    const uint64_t addr = (smem_u32(p) >> 4) & 0x3FFF;
    return addr | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}

template <bool BF16>
__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
    if constexpr (BF16) {
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
            "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc));
    } else {
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
            "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc));
    }
}

// Signed 8-bit operands, exact 32-bit integer accumulation (K = 32 bytes per instruction).
__device__ __forceinline__ void umma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// ---- CTA pairs (a cluster of two CTAs sharing one tcgen05.mma.cta_group::2) ----------
// Bit 24 of a shared::cluster address selects the CTA of the pair; cleared, the address
// names the same offset in the pair's first CTA (whose barriers gate the pair's MMAs).
constexpr uint32_t kPairLeaderMask = 0xFEFFFFFFu;

__device__ __forceinline__ uint32_t cluster_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// Store v to the same shared-memory offset in CTA `rank` of the cluster (distributed shared
// memory); ordered before the next cluster barrier's release.
__device__ __forceinline__ void st_cluster_u32(const void* local, uint32_t rank, uint32_t v) {
    uint32_t remote;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(remote) : "r"(smem_u32(local)), "r"(rank));
    asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(remote), "r"(v) : "memory");
}
// TMA load into this CTA's shared memory whose completion counts on the pair leader's
// barrier (the same barrier offset with the peer bit cleared). No multicast.
__device__ __forceinline__ void tma_load_2d_pair(void* dst, const CUtensorMap* tm, uint64_t* bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, "
        "%4}], [%2];" ::"r"(smem_u32(dst)),
        "l"(tm), "r"(smem_u32(bar) & kPairLeaderMask), "r"(x), "r"(y)
        : "memory");
}
template <bool BF16>
__device__ __forceinline__ void umma_pair(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t acc) {
    const uint32_t z = 0;
    if constexpr (BF16) {
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5, %5, %5, %5, %5}, p;\n}\n" ::"r"(
                tmem_d),
            "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc), "r"(z));
    } else {
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::2.kind::tf32 [%0], %1, %2, %3, {%5, %5, %5, %5, %5, %5, %5, %5}, p;\n}\n" ::"r"(
                tmem_d),
            "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc), "r"(z));
    }
}
// Arrive on the barrier at this offset in both CTAs of the pair when the issuing thread's
// previous pair MMAs complete.
__device__ __forceinline__ void umma_commit_pair(uint64_t* bar) {
    const uint16_t both = 0x3;
    asm volatile(
        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
            smem_u32(bar)),
        "h"(both)
        : "memory");
}

// Arrive once on the mbarrier at this shared-memory offset in CTA `rank` of the cluster.
__device__ __forceinline__ void mbar_arrive_cluster(const void* local_bar, uint32_t rank) {
    uint32_t remote;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(remote) : "r"(smem_u32(local_bar)), "r"(rank));
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(remote) : "memory");
}

// Barrier 1 over the `count` threads of the epilogue warps, returning whether any of them
// passed a true `flag` (one decision for all of them).
__device__ __forceinline__ bool epilogue_any(bool flag, int count) {
    uint32_t r;
    asm volatile(
        "{\n .reg .pred p, q;\n setp.ne.u32 q, %1, 0;\n bar.red.or.pred p, 1, %2, q;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(r)
        : "r"((uint32_t)flag), "r"(count)
        : "memory");
    return r != 0;
}

// TMA reduction of a shared-memory box into global memory: C[y .. y + box) += box, FP32
// adds performed in the memory system (elements outside the tensor map are not touched).
__device__ __forceinline__ void tma_reduce_add_2d(const CUtensorMap* tm, const void* src, int x, int y) {
    asm volatile(
        "cp.reduce.async.bulk.tensor.2d.global.shared::cta.add.tile.bulk_group [%0, {%1, %2}], [%3];" ::"l"(tm),
        "r"(x), "r"(y), "r"(smem_u32(src))
        : "memory");
}
__device__ __forceinline__ void tma_reduce_add_3d(const CUtensorMap* tm, const void* src, int x, int y, int z) {
    asm volatile(
        "cp.reduce.async.bulk.tensor.3d.global.shared::cta.add.tile.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(tm),
        "r"(x), "r"(y), "r"(z), "r"(smem_u32(src))
        : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// Wait until at most N of this thread's bulk groups still read their shared-memory sources.
template <int N>
__device__ __forceinline__ void bulk_wait_read() {
    asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}
// Wait until every bulk group of this thread has completed.
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
// Order this thread's shared-memory writes before later bulk copies that read them.
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_ld16i(uint32_t taddr, int (&v)[16]) {
    float f[16];
    tmem_ld16(taddr, f);
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __float_as_int(f[i]);
}

__device__ __forceinline__ bool outside(Mask mask, int64_t off, int64_t m0, int64_t n0, int bm, int bn) {
    if (mask == kLower) return (m0 + bm - 1) - n0 - off < 0;
    if (mask == kUpper) return m0 - (n0 + bn - 1) - off > 0;
    return false;
}

__device__ __forceinline__ bool keep(Mask mask, int64_t off, int64_t i, int64_t j) {
    if (mask == kLower) return i - j >= off;
    if (mask == kUpper) return i - j <= off;
    return true;
}

}  // namespace tc
}  // namespace rc
