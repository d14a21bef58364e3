// Internal triangular-solve and Cholesky entry points.
#pragma once
#include "common.cuh"

namespace rc {

// Block size of the blocked TRSM / POTRF: one diagonal block per CTA, and the width of
// the panel GEMMs (equal to the FP64 DMMA tile so in-place panel updates are race free).
constexpr int kNB = 128;

// Writes v into *info if *info is 0 or larger than v (first failing index wins).
__device__ __forceinline__ void record_first(int* info, int v) {
    int old = *(volatile int*)info;
    while (old == 0 || old > v) {
        const int prev = atomicCAS(info, old, v);
        if (prev == old) break;
        old = prev;
    }
}

// Solves op(A) X = alpha * B in place for B (m x n), op(A) the m x m view A restricted to
// its lower (upper = false) or upper triangle. info (device, may be null): receives the
// 1-based index of the first exactly-zero diagonal when !unit. abort (may be null): the
// whole solve is skipped when *abort != 0 at launch time.
template <class T>
int trsm_left(bool upper, bool unit, int64_t m, int64_t n, T alpha, View<const T> A, View<T> B, int* info,
              cudaStream_t s, const int* abort = nullptr);

// In-place Cholesky A = L L^T of the lower triangle of the n x n view A (the strictly
// upper part is never written). info (device, required) is set to 0 first and then to the
// global 1-based index of the first non-positive pivot.
template <class T>
int potrf_lower(int64_t n, View<T> A, int* info, cudaStream_t s);

// Factor one sz x sz (sz <= kNB) lower diagonal block of A (view offset to the block)
// in FP64 shared memory, write L back and store inv(L) as a kNB x kNB block into W
// (row-major when w_row_major). g0 is the block's global index for the pivot status.
template <class T>
int potrf_diag_block(View<T> A, int sz, int64_t g0, T* W, bool w_row_major, int* info, cudaStream_t s);

// Blocked triangular solve with precomputed inverses of the kNB diagonal blocks of the
// lower-triangular L (row-major blocks, as potrf_diag_block stores them):
// trans = false: B <- L^-1 B; trans = true: B <- L^-T B. tmp holds kNB x n elements.
template <class T>
int trsm_preinv(bool trans, int64_t m, int64_t n, View<const T> L, const T* Winv, View<T> B, T* tmp, cudaStream_t s);

// Invert every kNB x kNB diagonal block of the lower-triangular m x m view L into W
// (column-major kNB x kNB blocks, block b at W + b * kNB * kNB); skipped when *abort != 0.
template <class T>
int trtri_blocks_launch(int64_t m, View<const T> L, bool unit, T* W, int* info, const int* abort, cudaStream_t s);

}  // namespace rc
