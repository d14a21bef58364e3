// Internal entry of the mixed-precision refined SPD solver.
#pragma once
#include "common.cuh"

namespace rc {
int mixed_workspace_bytes(int64_t n, int64_t nrhs, int prec, int outer, size_t* bytes);
int spd_solve_mixed(int prec, int64_t n, int64_t nrhs, const double* A, int64_t lda, const double* B, int64_t ldb,
                    double* X, int64_t ldx, const rc_mixed_options* opt, int* d_info, rc_refine_info* out,
                    cudaStream_t s);
}  // namespace rc
