// Trailing updates of an FP64 Cholesky factorisation as exact int8 digit products.
#pragma once
#include <cuda.h>

#include "common.cuh"

namespace rc {

// Digits kept per panel entry: |x| / 2^e_i = sum_{t=1..kEmuSlices} d_t 2^-7t + r with
// 0 <= r < 2^-7 kEmuSlices (e_i from the row's largest entry). With 7 digits the update
// keeps 49 bits below each row maximum (the dropped digit pairs weigh at most 2^-56).
constexpr int kEmuSlices = 7;

// The digit split of one outer panel: rows [0, rows) of the panel (rows of the trailing
// matrix, K = the panel's width), slice t of row r at digits + (t * Mp + r) * ldk.
struct EmuPanel {
    int64_t rows = 0, width = 0, Mp = 0, ldk = 0;
    int8_t* digits = nullptr;
    int* rexp = nullptr;  // per row: e with max_k |P(r, k)| < 2^e (INT_MIN: a non-finite entry)
    CUtensorMap tmA;      // 128 x 128-byte boxes of the stacked slices (A operand)
    CUtensorMap tmB;      // 64 rows x 128 bytes x kEmuSlices slices per box (B operand)
};

// Bytes of the digit split of a panel of up to `rows` rows and `width` columns.
size_t emu_panel_bytes(int64_t rows, int64_t width);

// Lay out the split in `ws` (emu_panel_bytes bytes, 256-byte aligned) and encode its maps.
int emu_panel_layout(int64_t rows, int64_t width, void* ws, EmuPanel* out);

// Split the row-major FP64 panel P (rows x width, row stride ldp): per row its exponent,
// then its digits (rows and columns of the split beyond the panel are zero).
int emu_slice_panel(const EmuPanel& pn, const double* P, int64_t ldp, cudaStream_t s);

// C <- alpha * P_A P_B^T + beta * C on the M x N block C (row-major, row stride ldc; with
// lower, only its lower triangle i >= j), where P_A = panel rows [a0, a0 + M) and P_B =
// panel rows [b0, b0 + N), every digit product exact (int32 accumulation) and the seven
// weights combined in FP64; beta == 0 does not read C. Tiles of 128 rows x 64 columns, one
// CTA per SM; abort (device int, may be null) and the library's error word stop it as for
// the other tensor-core kernels.
int emu_update(const EmuPanel& pn, int64_t a0, int64_t b0, int64_t M, int64_t N, double alpha, double beta,
               double* C, int64_t ldc, bool lower, cudaStream_t s, const int* abort);

}  // namespace rc
