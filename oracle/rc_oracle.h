/* Test infrastructure: the CPU oracle. A restatement, in plain loops, of the reference's
 * algorithms for the hot path (Remora's CPU kernels and its device RNG stream). Only the
 * tests, the smoke check and the CPU-baseline leg of bench.py load it, and only as the
 * checker; the product library never links it.
 *
 * Matrices are strided views: element (i, j) lives at p[i * rs + j * cs]. A row-major
 * matrix with leading dimension ld is (rs, cs) = (ld, 1); a column-major one is (1, ld).
 */
#ifndef RC_ORACLE_H
#define RC_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Threefry-4x32, 12 rounds, with the reference's key-injection schedule. */
void orc_threefry(const uint32_t ctr[4], const uint32_t key[4], uint32_t out[4]);
/* Counter of the 4-element group that holds element (i, 4*j4): (i & 0xffff, i >> 32,
 * j & 0xffff, j >> 32) with j = 4*j4. */
void orc_counter(uint64_t i, uint64_t j, uint32_t ctr[4]);

/* Fills of a rows x cols strided matrix. kind: 0 = raw Threefry words (as uint32),
 * 1 = uniform(a, b), 2 = normal(mean a, stddev b), 3 = discrete [ia, ib] as float,
 * 4 = discrete [ia, ib] as int32. fused: 1 = the fused multiply-adds that nvcc emits for
 * the reference's float transforms (the default target), 0 = unfused. */
void orc_rng_fill(int kind, const uint32_t key[4], size_t rows, size_t cols, void* A,
                  ptrdiff_t rs, ptrdiff_t cs, float a, float b, int ia, int ib, int fused);
/* The same fill for the sub-block of rows [row0, row0 + rows) and columns
 * [col0, col0 + cols) of a larger matrix (col0 a multiple of 4). */
void orc_rng_fill_block(int kind, const uint32_t key[4], uint64_t row0, uint64_t col0, size_t rows,
                        size_t cols, void* A, ptrdiff_t rs, ptrdiff_t cs, float a, float b, int ia,
                        int ib, int fused);

/* std::mt19937 generator handle and the reference CPU input generator on it. */
void* orc_rng_create(uint32_t seed);
void orc_rng_destroy(void* rng);
void orc_rng_key(void* rng, uint32_t key[4]);
void orc_generate_normal_f64(void* rng, size_t rows, size_t cols, double* A, ptrdiff_t rs, ptrdiff_t cs,
                             double mean, double variance);
void orc_generate_uniform_f64(void* rng, size_t rows, size_t cols, double* A, ptrdiff_t rs, ptrdiff_t cs,
                              double low, double high);
void orc_generate_normal_f32(void* rng, size_t rows, size_t cols, float* A, ptrdiff_t rs, ptrdiff_t cs,
                             float mean, float variance);
void orc_generate_uniform_f32(void* rng, size_t rows, size_t cols, float* A, ptrdiff_t rs, ptrdiff_t cs,
                              float low, float high);

/* C += alpha * A * B (m x k times k x n). */
void orc_gemm_f64(size_t m, size_t n, size_t k, double alpha, const double* A, ptrdiff_t ars, ptrdiff_t acs,
                  const double* B, ptrdiff_t brs, ptrdiff_t bcs, double* C, ptrdiff_t crs, ptrdiff_t ccs);
void orc_gemm_f32(size_t m, size_t n, size_t k, float alpha, const float* A, ptrdiff_t ars, ptrdiff_t acs,
                  const float* B, ptrdiff_t brs, ptrdiff_t bcs, float* C, ptrdiff_t crs, ptrdiff_t ccs);
/* C_tri += alpha * A * A^T on the upper (upper = 1) or lower triangle only; A is n x k. */
void orc_syrk_f64(int upper, size_t n, size_t k, double alpha, const double* A, ptrdiff_t ars, ptrdiff_t acs,
                  double* C, ptrdiff_t crs, ptrdiff_t ccs);
void orc_syrk_f32(int upper, size_t n, size_t k, float alpha, const float* A, ptrdiff_t ars, ptrdiff_t acs,
                  float* C, ptrdiff_t crs, ptrdiff_t ccs);
/* B <- op(A)^-1 B (left) or B op(A)^-1 (right); A is the triangle named by upper; unit
 * skips the diagonal. B is m x n. Returns 1 on an exact zero on the diagonal, else 0. */
int orc_trsm_f64(int left, int upper, int unit, size_t m, size_t n, const double* A, ptrdiff_t ars, ptrdiff_t acs,
                 double* B, ptrdiff_t brs, ptrdiff_t bcs);
int orc_trsm_f32(int left, int upper, int unit, size_t m, size_t n, const float* A, ptrdiff_t ars, ptrdiff_t acs,
                 float* B, ptrdiff_t brs, ptrdiff_t bcs);
/* y += alpha * A x (A m x n; x, y with strides incx, incy). */
void orc_gemv_f64(size_t m, size_t n, double alpha, const double* A, ptrdiff_t ars, ptrdiff_t acs, const double* x,
                  ptrdiff_t incx, double* y, ptrdiff_t incy);
void orc_gemv_f32(size_t m, size_t n, float alpha, const float* A, ptrdiff_t ars, ptrdiff_t acs, const float* x,
                  ptrdiff_t incx, float* y, ptrdiff_t incy);
/* x <- op(A)^-1 x (left) or solves x A = b in place (right); A the named triangle. */
int orc_trsv_f64(int left, int upper, int unit, size_t n, const double* A, ptrdiff_t ars, ptrdiff_t acs, double* x,
                 ptrdiff_t incx);
int orc_trsv_f32(int left, int upper, int unit, size_t n, const float* A, ptrdiff_t ars, ptrdiff_t acs, float* x,
                 ptrdiff_t incx);
/* B <- T B for the named triangle T of A (m x m); B is m x n (n = 1: trmv). */
void orc_trmm_f64(int upper, int unit, size_t m, size_t n, const double* A, ptrdiff_t ars, ptrdiff_t acs, double* B,
                  ptrdiff_t brs, ptrdiff_t bcs);
void orc_trmm_f32(int upper, int unit, size_t m, size_t n, const float* A, ptrdiff_t ars, ptrdiff_t acs, float* B,
                  ptrdiff_t brs, ptrdiff_t bcs);
/* In-place Cholesky of the lower (upper = 0) or upper triangle; the other triangle is
 * left untouched. Returns 0, or the 1-based GLOBAL index of the first non-positive pivot. */
size_t orc_potrf_f64(int upper, size_t n, double* A, ptrdiff_t rs, ptrdiff_t cs);
size_t orc_potrf_f32(int upper, size_t n, float* A, ptrdiff_t rs, ptrdiff_t cs);
/* LU with partial pivoting in place (unit lower L below the diagonal, U on and above):
 * piv[i] = the row swapped with row i, in order i = 0, 1, ... (kernels/getrf.hpp:50-59).
 * Returns 0, or the 1-based column of the first zero pivot (the reference throws). */
size_t orc_getrf_f64(size_t n, double* A, ptrdiff_t rs, ptrdiff_t cs, int* piv);
size_t orc_getrf_f32(size_t n, float* A, ptrdiff_t rs, ptrdiff_t cs, int* piv);
/* Pivoted Cholesky P^T A P = L L^T of a symmetric positive semidefinite A, L in the lower
 * triangle (zeros above), piv as for getrf (kernels/pstrf.hpp:62-70); returns the rank,
 * the columns from the rank on are zero. */
size_t orc_pstrf_f64(size_t n, double* A, ptrdiff_t rs, ptrdiff_t cs, int* piv);
size_t orc_pstrf_f32(size_t n, float* A, ptrdiff_t rs, ptrdiff_t cs, int* piv);
/* cholesky_decomposition(A).solve(B, left): A n x n SPD (lower triangle read), B n x nrhs.
 * Returns the potrf status. A is not modified. */
size_t orc_cholesky_solve_f64(size_t n, size_t nrhs, const double* A, ptrdiff_t ars, ptrdiff_t acs,
                              double* B, ptrdiff_t brs, ptrdiff_t bcs);

#ifdef __cplusplus
}
#endif
#endif
