/* remora_cuda.h -- the C-ABI of libremora_cuda.so, the sm_100a (B200) kernels behind
 * Remora's `cuda_tag` device.
 *
 * Conventions (the cuBLAS-style column-major convention that the reference's HIP
 * backend maps every orientation onto, include/remora/kernels/hip/gemm.hpp:46-88):
 *  - matrices are column-major with a leading dimension; `trans*` flags select op(X) = X
 *    or X^T. A row-major matrix is passed as its transpose (swap the dimensions, flip
 *    the flag), exactly as the reference's row-major overloads do;
 *  - all pointers are device pointers unless stated; every call is asynchronous on the
 *    caller's `stream` (a cudaStream_t; NULL = the legacy default stream);
 *  - the return value is a status (RC_SUCCESS = 0); numerical outcomes that are only
 *    known on the device (a failing pivot, a zero diagonal) are written to a
 *    caller-provided device int `d_info` (may be NULL where stated);
 *  - the library allocates only internal workspaces, cached per device and stream
 *    (released by rc_release_workspaces).
 */
#ifndef REMORA_CUDA_H
#define REMORA_CUDA_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    RC_SUCCESS = 0,
    RC_ERR_INVALID_ARGUMENT = 1, /* a size, leading dimension or flag is out of range */
    RC_ERR_CUDA = 2,             /* a CUDA runtime call or kernel launch failed */
    RC_ERR_ALLOC = 3,            /* a workspace allocation failed */
    RC_ERR_NOT_SUPPORTED = 4,    /* a combination the library does not implement */
    RC_ERR_TIMEOUT = 5,          /* a bounded device-side wait gave up */
    RC_ERR_NOT_CONVERGED = 6,    /* iterative refinement did not reach its tolerance */
    RC_ERR_SIZE_LIMIT = 7        /* the problem exceeds an entry point's fixed scratch */
};

/* Library version (major * 10000 + minor * 100 + patch). */
int rc_version(void);
/* Static description of a status code. */
const char* rc_error_string(int status);
/* Number of kernels the library has launched so far in this process (all devices). */
unsigned long long rc_launch_count(void);
/* Number of device allocations the library has made for its own use so far in this
 * process (workspaces, the error word, batched plans; not rc_malloc on a caller's behalf).
 * No reference counterpart: it lets a host check that a call allocated nothing. */
unsigned long long rc_allocation_count(void);
/* Free every cached workspace of the current device (synchronises the device). */
int rc_release_workspaces(void);
/* Failure detection. Every device-side wait (the mbarrier phases of the tensor-core
 * pipelines, the grid barriers of the cooperative getrf panel) is bounded: by the SM's cycle counter, 2 cycles per nanosecond of the limit
 * set here (default 2 s), i.e. at least that long at SM clocks up to 2 GHz. A wait that
 * runs out records RC_ERR_TIMEOUT and where it happened (kernel * 100 + role * 10 + CTA
 * rank in its cluster; kernels 1 = tcgen05 GEMM, 2 = CTA-pair GEMM, 3 = int8 product,
 * 4 = int8 digit-product trailing update, 5 = getrf panel grid barrier (site 500),
 * 9 = self-test; roles 0 = loads, 1 = MMAs, 2 = epilogue) in a per-device error word and
 * its kernel returns, leaving the context usable. The word is sticky: while it is set,
 * every tensor-core kernel returns at once and waits in flight give up, and
 * rc_spd_solve_mixed returns RC_ERR_TIMEOUT. rc_device_status synchronises the stream
 * and returns (then clears) the status; rc_device_error_site also writes the site.
 * rc_selftest_wait_timeout launches one bounded wait on a barrier that nothing
 * completes, to exercise that path. These have no reference counterpart (the reference
 * checks no launch, hip/exception.hpp:41-63). */
int rc_set_wait_limit_ns(uint64_t ns);
int rc_device_status(void* stream);
int rc_device_error_site(void* stream, int* site);
int rc_selftest_wait_timeout(uint64_t limit_ns, void* stream);

/* ---------------------------------------------------------------------------------
 * Device runtime for hosts compiled without the CUDA toolkit (the cuda_tag headers).
 * Replace the HIP runtime plumbing of include/remora/hip/device.hpp:41-180 (device,
 * stream per thread), include/remora/hip/buffer.hpp:41-102 (owning allocation) and the
 * transport of include/remora/hip/copy.hpp:131-410 (here: pitched asynchronous copies
 * through page-locked staging chunks, rc_host_alloc; a copy from pageable host memory is
 * synchronous with respect to the host). */
enum { RC_COPY_H2D = 1, RC_COPY_D2H = 2, RC_COPY_D2D = 3 };
int rc_device_count(int* count);
int rc_set_device(int device);
int rc_get_device(int* device);
int rc_malloc(void** ptr, size_t bytes);
int rc_free(void* ptr);
/* Copy `rows` rows of width_bytes bytes; row r of src starts at src + r * spitch. */
int rc_memcpy2d(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width_bytes,
                size_t rows, int kind, void* stream);
/* Page-locked host memory (the staging chunks of the transport: DMA at the link's rate,
 * asynchronous with respect to the host) and events to order reuse of such chunks. */
int rc_host_alloc(void** ptr, size_t bytes);
int rc_host_free(void* ptr);
int rc_event_create(void** event);
int rc_event_record(void* event, void* stream);
int rc_event_synchronize(void* event);
int rc_event_destroy(void* event);
int rc_stream_create(void** stream);
int rc_stream_destroy(void* stream);
int rc_stream_synchronize(void* stream);

/* ---------------------------------------------------------------------------------
 * Counter-based RNG fills of a rows x cols float/int matrix (Threefry-4x32, 12 rounds).
 * Replaces bindings::generate_normal/uniform/discrete for hip_tag,
 * include/remora/kernels/hip/random.hpp:218-323 (kernels :163-210, generator :40-161).
 * key: the 4 words the reference draws from the host generator (:225-227).
 * Element (i, j) is component j % 4 of Threefry(ctr(i, 4*floor(j/4)), key) with
 * ctr(i, j) = (i & 0xffff, i >> 32, j & 0xffff, j >> 32) (:167), independent of storage
 * order; row_major selects the layout of A (leading dimension ld). Elements outside
 * rows x cols are never written (the reference writes past the end, :172, :186). */
int rc_rng_bits_u32(const uint32_t key[4], size_t rows, size_t cols, uint32_t* A, size_t ld,
                    int row_major, void* stream);
int rc_rng_uniform_f32(const uint32_t key[4], size_t rows, size_t cols, float* A, size_t ld,
                       int row_major, float low, float high, void* stream);
int rc_rng_normal_f32(const uint32_t key[4], size_t rows, size_t cols, float* A, size_t ld,
                      int row_major, float mean, float stddev, void* stream);
/* Discrete values low + (x % (high - low + 1)); requires low <= high and a range below 2^32. */
int rc_rng_discrete_f32(const uint32_t key[4], size_t rows, size_t cols, float* A, size_t ld,
                        int row_major, int low, int high, void* stream);
int rc_rng_discrete_i32(const uint32_t key[4], size_t rows, size_t cols, int32_t* A, size_t ld,
                        int row_major, int low, int high, void* stream);

/* ---------------------------------------------------------------------------------
 * C <- alpha * op(A) * op(B) + beta * C, C m x n, op(A) m x k, op(B) k x n.
 * Replaces kernels::gemm for hip_tag (include/remora/kernels/hip/gemm.hpp:46-112 ->
 * include/remora/hip/cublas_backend.hpp:121-166). beta == 0 does not read C.
 * rc_gemm_f64: FP64 on the DMMA tensor path; rc_gemm_f32: FP32 FMA (IEEE FP32 accuracy). */
int rc_gemm_f64(int transA, int transB, size_t m, size_t n, size_t k, double alpha,
                const double* A, size_t lda, const double* B, size_t ldb, double beta,
                double* C, size_t ldc, void* stream);
int rc_gemm_f32(int transA, int transB, size_t m, size_t n, size_t k, float alpha,
                const float* A, size_t lda, const float* B, size_t ldb, float beta,
                float* C, size_t ldc, void* stream);
/* FP64 C <- alpha * A * B + beta * C (column-major, no transposes, n <= 64) on the int8
 * tensor cores: A and B are split into 8 signed 7-bit digits below their row (A) and column
 * (B) maxima and the 36 digit-pair products of weight above 2^-70 run as exact int8 GEMMs
 * (Ozaki-Ootomo-Yokota error-free splitting). |error(i, j)| <= ~(2k + 9k) 2^-56
 * 2^(e_i + f_j) with 2^e_i > max|A(i, :)|, 2^f_j > max|B(:, j)|, plus FP64 rounding of the
 * sum: FP64-level normwise accuracy. Rows of A / columns of B holding Inf or NaN give NaN.
 * No reference counterpart (an alternative FP64 product for the skinny products of
 * iterative refinement). RC_ERR_NOT_SUPPORTED for n > 64. */
int rc_gemm_f64_sliced(size_t m, size_t n, size_t k, double alpha, const double* A, size_t lda,
                       const double* B, size_t ldb, double beta, double* C, size_t ldc,
                       void* stream);
/* Reduced-precision FP32 GEMMs on the tcgen05 tensor cores with FP32 accumulation:
 * rc_gemm_tf32 truncates the operands to TF32 (10 mantissa bits), rc_gemm_bf16 rounds
 * them to BF16. No reference counterpart (the reference's FP32 gemm is cuBLAS SGEMM);
 * they are the precisions of the mixed-precision solve's trailing updates. */
int rc_gemm_tf32(int transA, int transB, size_t m, size_t n, size_t k, float alpha,
                 const float* A, size_t lda, const float* B, size_t ldb, float beta,
                 float* C, size_t ldc, void* stream);
int rc_gemm_bf16(int transA, int transB, size_t m, size_t n, size_t k, float alpha,
                 const float* A, size_t lda, const float* B, size_t ldb, float beta,
                 float* C, size_t ldc, void* stream);

/* C_tri <- alpha * op(A) * op(A)^T + beta * C_tri on the upper or lower triangle of the
 * n x n matrix C; op(A) is n x k (trans = 0: A is n x k; trans = 1: A is k x n). The
 * other triangle is not touched. Replaces kernels::syrk for hip_tag
 * (include/remora/kernels/hip/syrk.hpp:44-85 -> hip/cublas_backend.hpp:389-431). */
int rc_syrk_f64(int upper, int trans, size_t n, size_t k, double alpha, const double* A,
                size_t lda, double beta, double* C, size_t ldc, void* stream);
int rc_syrk_f32(int upper, int trans, size_t n, size_t k, float alpha, const float* A,
                size_t lda, float beta, float* C, size_t ldc, void* stream);

/* Triangular solve with m x n B: left: B <- alpha * op(A)^-1 B (A m x m);
 * right: B <- alpha * B op(A)^-1 (A n x n). upper names the stored triangle of A,
 * unit assumes a unit diagonal. d_info (may be NULL): set to 0, or to the 1-based index
 * of the first exactly-zero diagonal element of A when !unit (the reference CPU kernel
 * throws there, include/remora/kernels/default/trsm.hpp:86-87).
 * Replaces kernels::trsm for hip_tag (include/remora/kernels/hip/trsm.hpp:45-107 ->
 * hip/cublas_backend.hpp:303-344). */
int rc_trsm_f64(int left, int upper, int trans, int unit, size_t m, size_t n, double alpha,
                const double* A, size_t lda, double* B, size_t ldb, int* d_info, void* stream);
int rc_trsm_f32(int left, int upper, int trans, int unit, size_t m, size_t n, float alpha,
                const float* A, size_t lda, float* B, size_t ldb, int* d_info, void* stream);

/* y <- alpha * op(A) x + beta * y with A column-major m x n (lda >= m); op(A) = A (trans = 0:
 * x has n entries, y has m) or A^T (trans = 1: x has m, y has n); incx, incy >= 1 are the
 * vector strides. Replaces kernels::gemv for hip_tag (include/remora/kernels/hip/
 * gemv.hpp:45-90, cuBLAS gemv through hip/cublas_backend.hpp:170-213). */
int rc_gemv_f64(int trans, size_t m, size_t n, double alpha, const double* A, size_t lda, const double* x,
                size_t incx, double beta, double* y, size_t incy, void* stream);
int rc_gemv_f32(int trans, size_t m, size_t n, float alpha, const float* A, size_t lda, const float* x,
                size_t incx, float beta, float* y, size_t incy, void* stream);

/* x <- op(T)^-1 x for the lower (upper = 0) or upper triangle T of the column-major n x n A
 * (unit: ones assumed on the diagonal), op(T) = T or T^T (trans); x has stride incx.
 * Replaces kernels::trsv for hip_tag (include/remora/kernels/hip/trsv.hpp:44-90). */
int rc_trsv_f64(int upper, int trans, int unit, size_t n, const double* A, size_t lda, double* x, size_t incx,
                void* stream);
int rc_trsv_f32(int upper, int trans, int unit, size_t n, const float* A, size_t lda, float* x, size_t incx,
                void* stream);

/* B <- op(T) B (left) or B op(T) (right) for the lower/upper triangle T of the column-major A
 * (k x k, k = m on the left, n on the right; unit: ones on the diagonal); B column-major
 * m x n. Replaces kernels::trmm for hip_tag (include/remora/kernels/hip/trmm.hpp:45-106). */
int rc_trmm_f64(int left, int upper, int trans, int unit, size_t m, size_t n, const double* A, size_t lda,
                double* B, size_t ldb, void* stream);
int rc_trmm_f32(int left, int upper, int trans, int unit, size_t m, size_t n, const float* A, size_t lda,
                float* B, size_t ldb, void* stream);

/* x <- op(T) x for the triangle T of the column-major n x n A; x has stride incx. Replaces
 * kernels::trmv for hip_tag (include/remora/kernels/hip/trmv.hpp:44-90). */
int rc_trmv_f64(int upper, int trans, int unit, size_t n, const double* A, size_t lda, double* x, size_t incx,
                void* stream);
int rc_trmv_f32(int upper, int trans, int unit, size_t n, const float* A, size_t lda, float* x, size_t incx,
                void* stream);

/* In-place Cholesky of the lower (A = L L^T) or upper (A = U^T U) triangle of the n x n
 * column-major A; the opposite triangle is never written. d_info (required): set to 0 on
 * success, else to the GLOBAL 1-based index of the first pivot that is not positive
 * (the reference CPU kernel returns an index relative to its recursive sub-block,
 * include/remora/kernels/default/potrf.hpp:125-133; the HIP kernel always returns 0,
 * kernels/hip/potrf.hpp:139). Replaces kernels::potrf for hip_tag
 * (include/remora/kernels/hip/potrf.hpp:41-141). */
int rc_potrf_f64(int upper, size_t n, double* A, size_t lda, int* d_info, void* stream);
int rc_potrf_f32(int upper, size_t n, float* A, size_t lda, int* d_info, void* stream);

/* LU with partial pivoting in place on the n x n matrix A (column-major; row-major when
 * row_major = 1): A = P L U, L unit lower below the diagonal, U on and above it.
 * d_piv (device, n ints): the row swapped with row i at step i, 0-based, applied in the
 * order i = 0, 1, ... (Remora's permutation_matrix). d_info (device): 0, or the 1-based
 * column of the first zero pivot, where the factorisation stops (the reference throws).
 * Replaces kernels::getrf (include/remora/kernels/getrf.hpp:50-59; CPU algorithm
 * kernels/default/getrf.hpp:41-181). */
int rc_getrf_f64(int row_major, size_t n, double* A, size_t lda, int* d_piv, int* d_info, void* stream);
int rc_getrf_f32(int row_major, size_t n, float* A, size_t lda, int* d_piv, int* d_info, void* stream);

/* Pivoted Cholesky P^T A P = L L^T of the symmetric positive semidefinite n x n A in place:
 * L in the lower triangle, zeros above it and in the columns from the rank on. d_piv as
 * for rc_getrf (identity where no swap happened); *d_rank (device) = the rank: the
 * factorisation stops once the largest remaining pivot is below n^2 eps max|A_ii|.
 * Replaces kernels::pstrf<lower> (include/remora/kernels/pstrf.hpp:62-70; CPU algorithm
 * kernels/default/pstrf.hpp:40-147). */
int rc_pstrf_f64(int row_major, size_t n, double* A, size_t lda, int* d_piv, int* d_rank, void* stream);
int rc_pstrf_f32(int row_major, size_t n, float* A, size_t lda, int* d_piv, int* d_rank, void* stream);

/* X = A^-1 B for SPD A via Cholesky: cholesky_decomposition(A).solve(B, left())
 * (include/remora/decompositions.hpp:81-84, :101-105; solve.hpp:165-170). A (n x n,
 * lower triangle read) is not modified; B (n x nrhs) is overwritten with X. d_info as
 * in rc_potrf_*; on failure B is left unchanged. */
int rc_spd_solve_f64(size_t n, size_t nrhs, const double* A, size_t lda, double* B, size_t ldb,
                     int* d_info, void* stream);

/* The same solve without any device allocation, for callers that cannot let a library
 * allocate while they run: services whose device memory is reserved up front by their
 * own pool allocator, and latency-bound loops where cudaMalloc/cudaFree (which can
 * synchronise the device) are not allowed. No counterpart in the reference. Scratch is
 * one 9.19 MiB __device__ array inside the library, held by every GPU that loads it until
 * the process exits: n <= 1024 and nrhs <= 64, else RC_ERR_SIZE_LIMIT. The first call on
 * a device looks up the array's device address (cudaGetSymbolAddress); make that first
 * call before any stream capture. All calls share the array: calls whose work overlaps
 * on the GPU (other streams, other host threads) race on it. d_info, A and B as in
 * rc_spd_solve_f64. */
int rc_spd_solve_f64_noalloc(size_t n, size_t nrhs, const double* A, size_t lda, double* B,
                             size_t ldb, int* d_info, void* stream);

/* ---------------------------------------------------------------------------------
 * Batched uneven SPD solves (extension; the reference solves one system per
 * cholesky_decomposition, decompositions.hpp:81-115). System i: the n_i x n_i SPD matrix
 * at d_A[i] (column-major, ld = n_i, lower triangle read, overwritten by its Cholesky
 * factor) and the right-hand side at d_b[i] (overwritten by the solution);
 * 1 <= n_i <= 512. d_A and d_b are DEVICE arrays of device pointers, h_n a HOST array of
 * sizes, d_info a device array receiving 0 or each system's failing pivot (1-based).
 * One persistent launch replayed as a CUDA graph; the graph and the tile configuration
 * (autotune = 1: timed on this batch the first time, cached per precision and size
 * bucket) are kept per (device, d_A, d_b, d_info, count) until rc_batched_release_plans. */
int rc_potrf_trsm_batched_f64(size_t count, const int* h_n, double* const* d_A, double* const* d_b,
                              int* d_info, int autotune, void* stream);
int rc_potrf_trsm_batched_f32(size_t count, const int* h_n, float* const* d_A, float* const* d_b,
                              int* d_info, int autotune, void* stream);
int rc_batched_release_plans(void);

/* ---------------------------------------------------------------------------------
 * Mixed-precision refined SPD solve (extension; no reference counterpart -- the reference
 * solves SPD systems only in the working precision, decompositions.hpp:81-105).
 * X = A^-1 B for a symmetric positive definite A given in FULL (both triangles), FP64:
 *  - factor S A S + theta I (S = diag(A)^-1/2, theta a multiple of u_f) in FP32 storage
 *    with FP64 diagonal blocks and TF32 or BF16 tensor-core trailing updates (FP32
 *    accumulation);
 *  - refine in FP64 by preconditioned conjugate gradients with that factor, per
 *    right-hand side, until the normwise backward error
 *    ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf) <= tol on every column. With at
 *    most 64 right-hand sides and n >= 512, the CG products A p run on the int8 tensor
 *    cores on an exact digit split of A (as rc_gemm_f64_sliced, rows and columns scaled
 *    from the diagonal), which adds 8 n^2 bytes to the workspace; every residual that
 *    decides convergence is an FP64 DMMA product.
 * RC_PREC_EMU64 (for condition numbers up to about 1e12, where a TF32/BF16 factor is too
 * coarse for CG to converge): the factor is kept in FP64 storage and its trailing updates
 * are exact int8 digit products on the tensor cores (7 signed 7-bit digits per entry below
 * its row's largest, 28 digit-pair GEMMs with int32 accumulation, combined in FP64), within
 * k 2^-44 of the row maxima per update of depth k; the diagonal blocks and panel solves are FP64 DMMA,
 * and the preconditioner is applied in FP64. The outer panel width is at most 4096 (wider
 * requests use 1024).
 * The call synchronises the stream (convergence is decided on the host). Returns
 * RC_ERR_NOT_CONVERGED when max_iter is reached first; d_info receives the failing pivot
 * when the low-precision factorisation breaks down (then X is not written). */
enum { RC_PREC_TF32 = 0, RC_PREC_BF16 = 1, RC_PREC_EMU64 = 2 };
typedef struct {
    double tol;          /* backward-error target (<= 0: 1e-15) */
    int max_iter;        /* CG iterations allowed in total (< 0: 100) */
    int outer;           /* outer panel width, a multiple of 128 (<= 0: 1024) */
    double shift_factor; /* theta = shift_factor * u_f; < 0: adaptive (u_f / 4, then 2 and 16 u_f
                            after a breakdown of the low-precision factorisation) */
} rc_mixed_options;
typedef struct {
    int iterations;        /* preconditioned CG iterations */
    int residuals;         /* true FP64 residual evaluations */
    int converged;         /* 1 when every column met tol */
    double backward_error; /* max over columns, from the last true residual */
    double factor_ms;      /* device time of the low-precision factorisation */
    double refine_ms;      /* device + host time of the refinement */
    double shift;          /* theta actually used */
} rc_refine_info;
int rc_spd_solve_mixed(int precision, size_t n, size_t nrhs, const double* A, size_t lda,
                       const double* B, size_t ldb, double* X, size_t ldx,
                       const rc_mixed_options* options, int* d_info, rc_refine_info* info,
                       void* stream);
/* The trailing update of the mixed-precision factorisation as a standalone call: the
 * lower triangle of the row-major n x n FP32 matrix C (element (i, j), j <= i, at
 * C[i * ldc + j]) <- alpha * P P^T + beta * C on the tcgen05 tensor cores, with P a
 * row-major n x k matrix of FP32 (RC_PREC_TF32) or BF16 (RC_PREC_BF16) elements, rows
 * 16-byte aligned. The strictly upper triangle is not touched. (A lower-triangle SYRK,
 * kernels::syrk<false> of include/remora/kernels/syrk.hpp:55-67, in reduced precision.) */
int rc_syrk_tc(int precision, size_t n, size_t k, float alpha, const void* P, size_t ldp,
               float beta, float* C, size_t ldc, void* stream);
/* rc_syrk_tc with options. RC_SYRK_BESIDE: the configuration that leaves room on every SM
 * for one more tensor-core CTA (a shallower operand ring), for a call that runs beside
 * other tensor-core work on another stream -- the configuration the mixed factorisation
 * uses for its trailing updates, whose look-ahead runs beside them. Without it (and in
 * rc_syrk_tc) the call takes the deeper ring and a whole SM per CTA. */
enum { RC_SYRK_BESIDE = 1 };
int rc_syrk_tc_ex(int precision, size_t n, size_t k, float alpha, const void* P, size_t ldp,
                  float beta, float* C, size_t ldc, int flags, void* stream);
/* The trailing update of the RC_PREC_EMU64 factorisation as a standalone call: the lower
 * triangle of the row-major n x n FP64 C <- alpha * P P^T + beta * C with P a row-major
 * n x k FP64 matrix (k <= 16384), P split per row into 7 signed 7-bit digits below the
 * row's largest |entry| and the 28 digit-pair products run as exact int8 GEMMs on the
 * tcgen05 tensor cores (int32 accumulation), combined in FP64: every entry of P P^T is
 * within k 2^-44 max_k |P(i, k)| max_k |P(j, k)| of the exact product (the digits truncate
 * toward zero and the pairs of weight below 2^-56 are dropped). beta == 0 does not read C;
 * the strictly upper triangle is not touched. Inf/NaN in a row of P gives NaN in its row
 * and column of the product. (kernels::syrk<false>, include/remora/kernels/syrk.hpp:55-67,
 * with emulated FP64 products.) */
int rc_syrk_emu64(size_t n, size_t k, double alpha, const double* P, size_t ldp, double beta,
                  double* C, size_t ldc, void* stream);
/* Device workspace the solve caches for these sizes, in bytes. */
int rc_spd_solve_mixed_workspace(int precision, size_t n, size_t nrhs,
                                 const rc_mixed_options* options, size_t* bytes);

/* ---------------------------------------------------------------------------------
 * Reverse-mode adjoints (extension; the reference has no derivatives of its
 * decompositions). Column-major FP64, device pointers.
 * rc_potrf_backward_f64: for A = L L^T (L lower, e.g. from rc_potrf_f64; only its lower
 *   triangle is read) and the adjoint Lbar of L (lower triangle read), writes the full
 *   symmetric adjoint Abar = 1/2 L^-T (P + P^T) L^-1, P = Phi(L^T Lbar) (Murray 2016),
 *   computed from L alone with blocked GEMM/TRSM kernels.
 * rc_trsm_backward_f64: reverse mode of X = L^-1 B (trans = 0) or X = L^-T B (trans = 1)
 *   with n x nrhs X: Xbar is overwritten by Bbar, and the lower triangle of Lbar
 *   accumulates -tril(Bbar X^T) (trans = 0) or -tril(X Bbar^T) (trans = 1). */
int rc_potrf_backward_f64(size_t n, const double* L, size_t ldl, const double* Lbar, size_t ldlb,
                          double* Abar, size_t ldab, void* stream);
int rc_trsm_backward_f64(int trans, size_t n, size_t nrhs, const double* L, size_t ldl,
                         const double* X, size_t ldx, double* Xbar, size_t ldxb, double* Lbar,
                         size_t ldlb, void* stream);
/* Gaussian-process RBF kernel around the differentiated Cholesky: X is n x d row-major
 * (d <= 16), ls the d lengthscales. rc_rbf_kernel_f64 writes
 * K_ij = exp(-1/2 sum_q ((x_iq - x_jq) / ls_q)^2) + noise [i == j]; the gradient call
 * writes grad_q = sum_ij Kbar_ij k_ij (x_iq - x_jq)^2 / ls_q^3 (the chain rule from the
 * adjoint Kbar of K to the lengthscales). */
int rc_rbf_kernel_f64(size_t n, int d, const double* X, const double* ls, double noise, double* K,
                      size_t ldk, void* stream);
int rc_rbf_lengthscale_grad_f64(size_t n, int d, const double* X, const double* ls,
                                const double* Kbar, size_t ldk, double* grad, void* stream);

/* ---------------------------------------------------------------------------------
 * Assignment support for the containers (include/remora/kernels/hip/matrix_assign.hpp:
 * 38-200, include/remora/hip/dense.hpp:39-51, hip/buffer.hpp:105-125).
 * rc_copy2d_*: B <- alpha * op(A) (A m x n if !trans, n x m if trans; B m x n).
 * rc_fill_*: every element of the m x n matrix set to value. */
int rc_copy2d_f64(int trans, size_t m, size_t n, double alpha, const double* A, size_t lda,
                  double* B, size_t ldb, void* stream);
int rc_copy2d_f32(int trans, size_t m, size_t n, float alpha, const float* A, size_t lda,
                  float* B, size_t ldb, void* stream);
int rc_fill_f64(size_t m, size_t n, double value, double* A, size_t lda, void* stream);
/* rc_axpby_*: y <- alpha * x + beta * y for vectors of n entries with strides incx, incy (the
 * dense vector assignments of include/remora/kernels/hip/vector_assign.hpp:55-130; beta = 0
 * does not read y). */
int rc_axpby_f64(size_t n, double alpha, const double* x, size_t incx, double beta, double* y, size_t incy,
                 void* stream);
int rc_axpby_f32(size_t n, float alpha, const float* x, size_t incx, float beta, float* y, size_t incy, void* stream);
int rc_fill_f32(size_t m, size_t n, float value, float* A, size_t lda, void* stream);
/* Row gather B(i, j) = A(idx[i], j) for the m x n matrices A and B given by element strides
 * (element (i, j) at p + i * rs + j * cs; a vector is m x 1, columns are rows of the
 * transposed strides); idx (device, m ints) must index rows of A, other rows of B are not
 * written; B must not be A. The device-side row and column swaps of Remora's permutations
 * (include/remora/permutation.hpp:51-131: swap_rows, swap_rows_inverted,
 * swap_columns_inverted) for the cuda_tag, applied as one gather. */
int rc_gather_rows_f64(size_t m, size_t n, const int* idx, const double* A, ptrdiff_t a_rs,
                       ptrdiff_t a_cs, double* B, ptrdiff_t b_rs, ptrdiff_t b_cs, void* stream);
int rc_gather_rows_f32(size_t m, size_t n, const int* idx, const float* A, ptrdiff_t a_rs,
                       ptrdiff_t a_cs, float* B, ptrdiff_t b_rs, ptrdiff_t b_cs, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* REMORA_CUDA_H */
