// Internal entry points of the tcgen05 GEMM.
#pragma once
#include "gemm.cuh"

namespace rc {

// D = alpha * A * B^T + beta * C with A (m x k) and B (n x k) K-major buffers (row r at
// ptr + r * ld) of FP32 (TF32 products) or BF16; 16-byte aligned pointers and rows.
// bn: tile width (128 or 256; 0 picks one). Returns RC_ERR_NOT_SUPPORTED on layouts the
// TMA cannot describe.
int gemm_tc_kmajor(bool bf16, int64_t m, int64_t n, int64_t k, float alpha, const void* A, int64_t lda,
                   const void* B, int64_t ldb, float beta, View<float> C, Mask mask, int64_t off, cudaStream_t s,
                   const int* abort = nullptr, int bn = 0);

// The same product on persistent CTA pairs (tcgen05.mma.cta_group::2, 256 x 256 tiles,
// K-major A and B as for gemm_tc_kmajor, one pair CTA per SM): half the operand traffic per
// SM of the 128 x 256 tiles; with beta = 1 and a row-major 16-byte-aligned C the epilogue
// adds into C with TMA reduce-adds. Masks: kFull, or kLower / kUpper with off = 0 and
// m = n (else RC_ERR_NOT_SUPPORTED). reserve_sms SMs are left to kernels that need a whole
// SM's shared memory (the factorisation's diagonal blocks). beside: the configuration that
// leaves room on every SM for one single-CTA tcgen05 kernel (for a launch that runs beside
// other tensor-core work); otherwise the deeper-ring configuration. abort (device int, may
// be null): when non-zero the pairs stop (C is then left partly updated).
int gemm_tc_pair_kmajor(bool bf16, int64_t m, int64_t n, int64_t k, float alpha, const void* A, int64_t lda,
                        const void* B, int64_t ldb, float beta, View<float> C, Mask mask, int64_t off, cudaStream_t s,
                        const int* abort = nullptr, int reserve_sms = 0, bool beside = false);

// C (m x 64) = alpha * (A B^T folded) + beta * C for a 128-row K-major B = [B_hi; B_lo]:
// column j of the product is A B_hi(j)^T + A B_lo(j)^T, i.e. A times B_hi + B_lo with
// B's TF32 split exact. TF32 products, FP32 accumulation.
int gemm_tc_fold_kmajor(int64_t m, int64_t k, float alpha, const float* A, int64_t lda, const float* B, int64_t ldb,
                        float beta, View<float> C, cudaStream_t s, const int* abort = nullptr);

// The driver's cuTensorMapEncodeTiled (a PFN_cuTensorMapEncodeTiled_v12000), or null.
void* tensor_map_encoder();

// Copy rows x K of X into a K-major buffer (row stride ldd), as FP32 or rounded to BF16.
int pack_kmajor(int64_t rows, int64_t K, View<const float> X, void* dst, int64_t ldd, bool bf16, cudaStream_t s);

}  // namespace rc
