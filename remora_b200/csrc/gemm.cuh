// Internal GEMM entry points shared by gemm/syrk/trsm/potrf.
#pragma once
#include "common.cuh"

namespace rc {

// Which part of C a (masked) GEMM may write: kFull writes every element; kLower writes
// C(i, j) only when i - j >= off; kUpper only when i - j <= off. Tiles that lie entirely
// outside the mask are skipped, which turns a masked GEMM into SYRK's triangle schedule.
enum Mask { kFull = 0, kLower = 1, kUpper = 2 };

// C <- alpha * A * B + beta * C (A m x k, B k x n, C m x n, arbitrary strided views).
// beta == 0 does not read C. abort (device int, may be null): when *abort != 0 at launch
// time the kernel returns without touching C (used after a failed Cholesky pivot).
template <class T>
int gemm(int64_t m, int64_t n, int64_t k, T alpha, View<const T> A, View<const T> B, T beta, View<T> C,
         Mask mask, int64_t off, cudaStream_t s, const int* abort = nullptr);

// FP32 GEMM on the tensor cores with TF32 products (reduced precision) or, with
// split = true, with the 3-term hi/lo TF32 split that keeps FP32 accuracy. Returns
// RC_ERR_NOT_SUPPORTED when the views do not meet the TMA layout rules; callers then use
// gemm<float>.
int gemm_tf32(int64_t m, int64_t n, int64_t k, float alpha, View<const float> A, View<const float> B,
              float beta, View<float> C, Mask mask, int64_t off, bool split, cudaStream_t s,
              const int* abort = nullptr);

}  // namespace rc
