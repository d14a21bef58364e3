// FP64 matrix products on the int8 tensor cores (error-free digit splitting).
#pragma once
#include <cuda.h>

#include "common.cuh"

namespace rc {

// Digits per operand: |x| / 2^e = sum_{t=1..8} d_t 2^-7t + r, 0 <= r < 2^-56.
constexpr int kOzSlices = 8;

// The m x k left operand, split once and reused by every product with it.
struct OzakiA {
    int64_t m = 0, k = 0, Mp = 0, ldk = 0;
    int8_t* slices = nullptr;  // kOzSlices x Mp rows of ldk bytes, K-major
    int* rexp = nullptr;       // per row: e with max_j |A(i, j)| < 2^e (INT_MIN: non-finite row)
    unsigned long long* rowbits = nullptr;
    int* flag = nullptr;    // device int: nonzero when the diagonal scaling did not bound A
    bool diagonal = false;  // rows AND columns scaled by 2^e_i (symmetric positive definite A)
    CUtensorMap tmap;
};

// Device bytes of the split left operand and of one product's right-hand buffers.
size_t ozaki_a_bytes(int64_t m, int64_t k);
size_t ozaki_p_bytes(int64_t m, int64_t k, int64_t nrhs);

// Split column-major A (m x k, lda) into `ws` (ozaki_a_bytes(m, k) bytes, 256-byte aligned).
int ozaki_prepare_a(int64_t m, int64_t k, const double* A, int64_t lda, void* ws, OzakiA* out, cudaStream_t s);

// For callers that write the digits with kernels of their own: the buffer layout and
// tensor map (no launch), and -- diagonal scaling of a square SPD A, 2^e_i >= sqrt(A_ii),
// which bounds every |A_ij| by 2^(e_i + e_j) without a pass over A -- the exponents (rexp)
// with *flag cleared first. The digits of A_ij / 2^(e_i + e_j) must then be written at
// slices + (t * Mp + i) * ldk + j, and *flag raised where an entry is not below its bound;
// a raised flag means the split must not be used.
int ozaki_layout_a(int64_t m, int64_t k, void* ws, bool diagonal, OzakiA* out);
int ozaki_diag_exponents(const OzakiA& a, const double* A, int64_t lda, cudaStream_t s);

// C (m x nrhs, column-major, ldc) = alpha * A P + beta * C for column-major P (k x nrhs,
// ldp), nrhs <= 64, through `ws` (ozaki_p_bytes bytes). Every digit product is exact; the
// result differs from the exact product by at most the truncations of A and P to 56
// bits below their row / column maxima, the dropped digit pairs of weight <= 2^-70 and
// the final FP64 roundings.
int ozaki_gemm(const OzakiA& a, int64_t nrhs, double alpha, const double* P, int64_t ldp, double beta, double* C,
               int64_t ldc, void* ws, cudaStream_t s);

}  // namespace rc
