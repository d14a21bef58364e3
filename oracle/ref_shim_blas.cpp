// Test infrastructure, not product code: a C-ABI shim over the reference's own CPU
// kernels (Remora, header-only C++), compiled from the reference headers where they
// lie by oracle/Makefile into oracle/_ref/libremora_ref.so. It is used to pin the
// oracle restatement (oracle/rc_oracle.cpp), to make the golden fixtures under
// tests/golden/, and as the timed CPU baseline ("kind": "reference") in bench.py.
// Nothing in the product links or loads this file.
//
// Every entry point forwards to the reference's public kernel API:
//   kernels::potrf<Tri>(A)            include/remora/kernels/potrf.hpp:56-62
//   kernels::trsm<Tri,Side>(A,B)      include/remora/kernels/trsm.hpp:55-65
//   kernels::syrk<Upper>(A,C,alpha)   include/remora/kernels/syrk.hpp:55-67
//   kernels::gemm(A,B,C,alpha)        include/remora/kernels/gemm.hpp:85-106
//   kernels::gemv(A,x,y,alpha)        include/remora/kernels/gemv.hpp:56-69
//   kernels::trsv<Tri,Side>(A,b)      include/remora/kernels/trsv.hpp:56-65
//   kernels::trmv<Upper,Unit>(A,b)    include/remora/kernels/trmv.hpp:54-65
//   kernels::trmm<Upper,Unit>(A,B)    include/remora/kernels/trmm.hpp:53-64
//   cholesky_decomposition + solve    include/remora/decompositions.hpp:70-115
//   kernels::getrf(A,P)               include/remora/kernels/getrf.hpp:50-59
//   kernels::pstrf<lower>(A,P)        include/remora/kernels/pstrf.hpp:62-70
//   kernels::generate_normal/uniform/discrete (CPU input generator)
//                                     include/remora/kernels/default/random.hpp:37-122
#include <remora/remora.hpp>
#include <random>
#include <cstdint>
#include <cstddef>

using namespace remora;

namespace {
template<class T, class O> using view = dense_matrix_adaptor<T, O, continuous_dense_tag, cpu_tag>;

// kernels::potrf takes a matrix_container, so the strided input is copied into a
// matrix<T,O> of the same orientation and back.
template<class T, class O, class Tri>
std::size_t potrf_impl(std::size_t n, T* A, std::size_t ld) {
	view<T, O> a(A, n, n, ld);
	matrix<T, O> m = a;
	std::size_t r = kernels::potrf<Tri>(m);
	noalias(a) = m;
	return r;
}

template<class T, class OA, class OB, class Tri, class Side>
void trsm_impl(std::size_t m, std::size_t n, T const* A, std::size_t lda, T* B, std::size_t ldb) {
	std::size_t na = Side::is_left ? m : n;
	view<T const, OA> a(A, na, na, lda);
	view<T, OB> b(B, m, n, ldb);
	kernels::trsm<Tri, Side>(a, b);
}

template<class T, class OA, class OB>
void trsm_dispatch(int left, int upper, int unit, std::size_t m, std::size_t n,
                   T const* A, std::size_t lda, T* B, std::size_t ldb) {
	if (left) {
		if (upper) {
			if (unit) trsm_impl<T, OA, OB, unit_upper, remora::left>(m, n, A, lda, B, ldb);
			else trsm_impl<T, OA, OB, remora::upper, remora::left>(m, n, A, lda, B, ldb);
		} else {
			if (unit) trsm_impl<T, OA, OB, unit_lower, remora::left>(m, n, A, lda, B, ldb);
			else trsm_impl<T, OA, OB, remora::lower, remora::left>(m, n, A, lda, B, ldb);
		}
	} else {
		if (upper) {
			if (unit) trsm_impl<T, OA, OB, unit_upper, remora::right>(m, n, A, lda, B, ldb);
			else trsm_impl<T, OA, OB, remora::upper, remora::right>(m, n, A, lda, B, ldb);
		} else {
			if (unit) trsm_impl<T, OA, OB, unit_lower, remora::right>(m, n, A, lda, B, ldb);
			else trsm_impl<T, OA, OB, remora::lower, remora::right>(m, n, A, lda, B, ldb);
		}
	}
}

template<class T>
int trsm_all(int left, int upper, int unit, int a_rm, int b_rm, std::size_t m, std::size_t n,
             T const* A, std::size_t lda, T* B, std::size_t ldb) {
	try {
		if (a_rm && b_rm) trsm_dispatch<T, row_major, row_major>(left, upper, unit, m, n, A, lda, B, ldb);
		else if (a_rm) trsm_dispatch<T, row_major, column_major>(left, upper, unit, m, n, A, lda, B, ldb);
		else if (b_rm) trsm_dispatch<T, column_major, row_major>(left, upper, unit, m, n, A, lda, B, ldb);
		else trsm_dispatch<T, column_major, column_major>(left, upper, unit, m, n, A, lda, B, ldb);
	} catch (std::invalid_argument const&) {
		return 1;  // zero diagonal: kernels/default/trsm.hpp:86-87 throws
	}
	return 0;
}

template<class T, class OA, class OC>
void syrk_impl(int upper, std::size_t n, std::size_t k, T alpha, T const* A, std::size_t lda, T* C, std::size_t ldc) {
	view<T const, OA> a(A, n, k, lda);
	view<T, OC> c(C, n, n, ldc);
	if (upper) kernels::syrk<true>(a, c, alpha);
	else kernels::syrk<false>(a, c, alpha);
}

template<class T>
void syrk_all(int upper, int a_rm, int c_rm, std::size_t n, std::size_t k, T alpha,
              T const* A, std::size_t lda, T* C, std::size_t ldc) {
	if (a_rm && c_rm) syrk_impl<T, row_major, row_major>(upper, n, k, alpha, A, lda, C, ldc);
	else if (a_rm) syrk_impl<T, row_major, column_major>(upper, n, k, alpha, A, lda, C, ldc);
	else if (c_rm) syrk_impl<T, column_major, row_major>(upper, n, k, alpha, A, lda, C, ldc);
	else syrk_impl<T, column_major, column_major>(upper, n, k, alpha, A, lda, C, ldc);
}

template<class T, class OA, class OB, class OC>
void gemm_impl(std::size_t m, std::size_t n, std::size_t k, T alpha, T const* A, std::size_t lda,
               T const* B, std::size_t ldb, T* C, std::size_t ldc) {
	view<T const, OA> a(A, m, k, lda);
	view<T const, OB> b(B, k, n, ldb);
	view<T, OC> c(C, m, n, ldc);
	kernels::gemm(a, b, c, alpha);
}

template<class T, class OA, class OB>
void gemm_c(int c_rm, std::size_t m, std::size_t n, std::size_t k, T alpha, T const* A, std::size_t lda,
            T const* B, std::size_t ldb, T* C, std::size_t ldc) {
	if (c_rm) gemm_impl<T, OA, OB, row_major>(m, n, k, alpha, A, lda, B, ldb, C, ldc);
	else gemm_impl<T, OA, OB, column_major>(m, n, k, alpha, A, lda, B, ldb, C, ldc);
}

template<class T>
void gemm_all(int a_rm, int b_rm, int c_rm, std::size_t m, std::size_t n, std::size_t k, T alpha,
              T const* A, std::size_t lda, T const* B, std::size_t ldb, T* C, std::size_t ldc) {
	if (a_rm && b_rm) gemm_c<T, row_major, row_major>(c_rm, m, n, k, alpha, A, lda, B, ldb, C, ldc);
	else if (a_rm) gemm_c<T, row_major, column_major>(c_rm, m, n, k, alpha, A, lda, B, ldb, C, ldc);
	else if (b_rm) gemm_c<T, column_major, row_major>(c_rm, m, n, k, alpha, A, lda, B, ldb, C, ldc);
	else gemm_c<T, column_major, column_major>(c_rm, m, n, k, alpha, A, lda, B, ldb, C, ldc);
}

template<class O, class OB>
int chol_solve_impl(std::size_t n, std::size_t nrhs, double const* A, std::size_t lda, double* B, std::size_t ldb) {
	view<double const, O> a(A, n, n, lda);
	view<double, OB> b(B, n, nrhs, ldb);
	cholesky_decomposition<matrix<double, O> > chol(a);
	chol.solve(b, left());
	return 0;
}

template<class T, class O>
void gen_normal(std::mt19937& rng, std::size_t rows, std::size_t cols, T* A, std::size_t ld, T mean, T variance) {
	view<T, O> a(A, rows, cols, ld);
	kernels::generate_normal(a, rng, mean, variance);
}
template<class T, class O>
void gen_uniform(std::mt19937& rng, std::size_t rows, std::size_t cols, T* A, std::size_t ld, T low, T high) {
	view<T, O> a(A, rows, cols, ld);
	kernels::generate_uniform(a, rng, low, high);
}
template<class T, class O>
void gemv_impl(std::size_t m, std::size_t n, T alpha, T const* A, std::size_t lda, T const* x, T* y) {
	view<T const, O> a(A, m, n, lda);
	vector<T> xv(n), yv(m);
	for (std::size_t j = 0; j != n; ++j) xv(j) = x[j];
	for (std::size_t i = 0; i != m; ++i) yv(i) = y[i];
	kernels::gemv(a, xv, yv, alpha);
	for (std::size_t i = 0; i != m; ++i) y[i] = yv(i);
}

template<class T, class O, class Tri, class Side>
void trsv_impl(std::size_t n, T const* A, std::size_t lda, T* x) {
	view<T const, O> a(A, n, n, lda);
	vector<T> xv(n);
	for (std::size_t j = 0; j != n; ++j) xv(j) = x[j];
	kernels::trsv<Tri, Side>(a, xv);
	for (std::size_t j = 0; j != n; ++j) x[j] = xv(j);
}

template<class T, class O, class Tri>
void trsv_side(int left, std::size_t n, T const* A, std::size_t lda, T* x) {
	if (left) trsv_impl<T, O, Tri, remora::left>(n, A, lda, x);
	else trsv_impl<T, O, Tri, remora::right>(n, A, lda, x);
}

template<class T, class O>
void trsv_tri(int upper, int unit, int left, std::size_t n, T const* A, std::size_t lda, T* x) {
	if (upper) {
		if (unit) trsv_side<T, O, unit_upper>(left, n, A, lda, x);
		else trsv_side<T, O, remora::upper>(left, n, A, lda, x);
	} else {
		if (unit) trsv_side<T, O, unit_lower>(left, n, A, lda, x);
		else trsv_side<T, O, remora::lower>(left, n, A, lda, x);
	}
}

template<class T, class O, bool Upper, bool Unit>
void trmv_impl(std::size_t n, T const* A, std::size_t lda, T* x) {
	view<T const, O> a(A, n, n, lda);
	vector<T> xv(n);
	for (std::size_t j = 0; j != n; ++j) xv(j) = x[j];
	kernels::trmv<Upper, Unit>(a, xv);
	for (std::size_t j = 0; j != n; ++j) x[j] = xv(j);
}

template<class T, class O>
void trmv_tri(int upper, int unit, std::size_t n, T const* A, std::size_t lda, T* x) {
	if (upper) {
		if (unit) trmv_impl<T, O, true, true>(n, A, lda, x);
		else trmv_impl<T, O, true, false>(n, A, lda, x);
	} else {
		if (unit) trmv_impl<T, O, false, true>(n, A, lda, x);
		else trmv_impl<T, O, false, false>(n, A, lda, x);
	}
}

template<class T, class OA, class OB, bool Upper, bool Unit>
void trmm_impl(std::size_t m, std::size_t n, T const* A, std::size_t lda, T* B, std::size_t ldb) {
	view<T const, OA> a(A, m, m, lda);
	view<T, OB> b(B, m, n, ldb);
	kernels::trmm<Upper, Unit>(a, b);
}

template<class T, class OA, class OB>
void trmm_tri(int upper, int unit, std::size_t m, std::size_t n, T const* A, std::size_t lda, T* B, std::size_t ldb) {
	if (upper) {
		if (unit) trmm_impl<T, OA, OB, true, true>(m, n, A, lda, B, ldb);
		else trmm_impl<T, OA, OB, true, false>(m, n, A, lda, B, ldb);
	} else {
		if (unit) trmm_impl<T, OA, OB, false, true>(m, n, A, lda, B, ldb);
		else trmm_impl<T, OA, OB, false, false>(m, n, A, lda, B, ldb);
	}
}

template<class T>
void trmm_all(int upper, int unit, int a_rm, int b_rm, std::size_t m, std::size_t n, T const* A, std::size_t lda,
              T* B, std::size_t ldb) {
	if (a_rm && b_rm) trmm_tri<T, row_major, row_major>(upper, unit, m, n, A, lda, B, ldb);
	else if (a_rm) trmm_tri<T, row_major, column_major>(upper, unit, m, n, A, lda, B, ldb);
	else if (b_rm) trmm_tri<T, column_major, row_major>(upper, unit, m, n, A, lda, B, ldb);
	else trmm_tri<T, column_major, column_major>(upper, unit, m, n, A, lda, B, ldb);
}
// kernels::getrf / kernels::pstrf take matrix containers too: copy in and out. P starts as
// the identity (permutation_matrix); getrf's "rank deficient" exception becomes -1.
template<class T, class O>
long getrf_impl(std::size_t n, T* A, std::size_t ld, int* P) {
	view<T, O> a(A, n, n, ld);
	matrix<T, O> m = a;
	permutation_matrix p(n);
	try {
		kernels::getrf(m, p);
	} catch (std::invalid_argument const&) {
		return -1;
	}
	noalias(a) = m;
	for (std::size_t i = 0; i != n; ++i) P[i] = p(i);
	return 0;
}

template<class T, class O>
std::size_t pstrf_impl(std::size_t n, T* A, std::size_t ld, int* P) {
	view<T, O> a(A, n, n, ld);
	matrix<T, O> m = a;
	permutation_matrix p(n);
	std::size_t rank = kernels::pstrf<remora::lower>(m, p);
	noalias(a) = m;
	for (std::size_t i = 0; i != n; ++i) P[i] = p(i);
	return rank;
}

}  // namespace

extern "C" {

std::size_t ref_potrf_f64(int upper, int row_major_, std::size_t n, double* A, std::size_t ld) {
	if (row_major_) return upper ? potrf_impl<double, row_major, remora::upper>(n, A, ld)
	                             : potrf_impl<double, row_major, remora::lower>(n, A, ld);
	return upper ? potrf_impl<double, column_major, remora::upper>(n, A, ld)
	             : potrf_impl<double, column_major, remora::lower>(n, A, ld);
}

// FP32 potrf compiles in the reference only for row-major lower and column-major upper:
// the other two bind a float element to `double&` (kernels/default/potrf.hpp:74).
// Returns (size_t)-1 for the two layouts it cannot build.
std::size_t ref_potrf_f32(int upper, int row_major_, std::size_t n, float* A, std::size_t ld) {
	if (row_major_ && !upper) return potrf_impl<float, row_major, remora::lower>(n, A, ld);
	if (!row_major_ && upper) return potrf_impl<float, column_major, remora::upper>(n, A, ld);
	return (std::size_t)-1;
}

long ref_getrf_f64(int row_major_, std::size_t n, double* A, std::size_t ld, int* P) {
	return row_major_ ? getrf_impl<double, row_major>(n, A, ld, P) : getrf_impl<double, column_major>(n, A, ld, P);
}
long ref_getrf_f32(int row_major_, std::size_t n, float* A, std::size_t ld, int* P) {
	return row_major_ ? getrf_impl<float, row_major>(n, A, ld, P) : getrf_impl<float, column_major>(n, A, ld, P);
}
std::size_t ref_pstrf_f64(int row_major_, std::size_t n, double* A, std::size_t ld, int* P) {
	return row_major_ ? pstrf_impl<double, row_major>(n, A, ld, P) : pstrf_impl<double, column_major>(n, A, ld, P);
}
// FP32 pstrf does not compile in the reference (kernels/default/pstrf.hpp:78 calls
// std::max(double&, float)): (size_t)-1.
std::size_t ref_pstrf_f32(int, std::size_t, float*, std::size_t, int*) { return (std::size_t)-1; }

int ref_trsm_f64(int left, int upper, int unit, int a_rm, int b_rm, std::size_t m, std::size_t n,
                 double const* A, std::size_t lda, double* B, std::size_t ldb) {
	return trsm_all<double>(left, upper, unit, a_rm, b_rm, m, n, A, lda, B, ldb);
}
int ref_trsm_f32(int left, int upper, int unit, int a_rm, int b_rm, std::size_t m, std::size_t n,
                 float const* A, std::size_t lda, float* B, std::size_t ldb) {
	return trsm_all<float>(left, upper, unit, a_rm, b_rm, m, n, A, lda, B, ldb);
}

void ref_syrk_f64(int upper, int a_rm, int c_rm, std::size_t n, std::size_t k, double alpha,
                  double const* A, std::size_t lda, double* C, std::size_t ldc) {
	syrk_all<double>(upper, a_rm, c_rm, n, k, alpha, A, lda, C, ldc);
}
void ref_syrk_f32(int upper, int a_rm, int c_rm, std::size_t n, std::size_t k, float alpha,
                  float const* A, std::size_t lda, float* C, std::size_t ldc) {
	syrk_all<float>(upper, a_rm, c_rm, n, k, alpha, A, lda, C, ldc);
}

void ref_gemm_f64(int a_rm, int b_rm, int c_rm, std::size_t m, std::size_t n, std::size_t k, double alpha,
                  double const* A, std::size_t lda, double const* B, std::size_t ldb, double* C, std::size_t ldc) {
	gemm_all<double>(a_rm, b_rm, c_rm, m, n, k, alpha, A, lda, B, ldb, C, ldc);
}
void ref_gemm_f32(int a_rm, int b_rm, int c_rm, std::size_t m, std::size_t n, std::size_t k, float alpha,
                  float const* A, std::size_t lda, float const* B, std::size_t ldb, float* C, std::size_t ldc) {
	gemm_all<float>(a_rm, b_rm, c_rm, m, n, k, alpha, A, lda, B, ldb, C, ldc);
}

// cholesky_decomposition<matrix<double,O>>(A).solve(B, left()): decompositions.hpp:81-84, :101-105
int ref_cholesky_solve_f64(int a_rm, int b_rm, std::size_t n, std::size_t nrhs,
                           double const* A, std::size_t lda, double* B, std::size_t ldb) {
	if (a_rm && b_rm) return chol_solve_impl<row_major, row_major>(n, nrhs, A, lda, B, ldb);
	if (a_rm) return chol_solve_impl<row_major, column_major>(n, nrhs, A, lda, B, ldb);
	if (b_rm) return chol_solve_impl<column_major, row_major>(n, nrhs, A, lda, B, ldb);
	return chol_solve_impl<column_major, column_major>(n, nrhs, A, lda, B, ldb);
}

// Matrix-vector kernels; x and y are contiguous.
void ref_gemv_f64(int a_rm, std::size_t m, std::size_t n, double alpha, double const* A, std::size_t lda,
                  double const* x, double* y) {
	if (a_rm) gemv_impl<double, row_major>(m, n, alpha, A, lda, x, y);
	else gemv_impl<double, column_major>(m, n, alpha, A, lda, x, y);
}
void ref_gemv_f32(int a_rm, std::size_t m, std::size_t n, float alpha, float const* A, std::size_t lda,
                  float const* x, float* y) {
	if (a_rm) gemv_impl<float, row_major>(m, n, alpha, A, lda, x, y);
	else gemv_impl<float, column_major>(m, n, alpha, A, lda, x, y);
}
void ref_trsv_f64(int upper, int unit, int left, int a_rm, std::size_t n, double const* A, std::size_t lda,
                  double* x) {
	if (a_rm) trsv_tri<double, row_major>(upper, unit, left, n, A, lda, x);
	else trsv_tri<double, column_major>(upper, unit, left, n, A, lda, x);
}
void ref_trsv_f32(int upper, int unit, int left, int a_rm, std::size_t n, float const* A, std::size_t lda,
                  float* x) {
	if (a_rm) trsv_tri<float, row_major>(upper, unit, left, n, A, lda, x);
	else trsv_tri<float, column_major>(upper, unit, left, n, A, lda, x);
}
void ref_trmv_f64(int upper, int unit, int a_rm, std::size_t n, double const* A, std::size_t lda, double* x) {
	if (a_rm) trmv_tri<double, row_major>(upper, unit, n, A, lda, x);
	else trmv_tri<double, column_major>(upper, unit, n, A, lda, x);
}
void ref_trmv_f32(int upper, int unit, int a_rm, std::size_t n, float const* A, std::size_t lda, float* x) {
	if (a_rm) trmv_tri<float, row_major>(upper, unit, n, A, lda, x);
	else trmv_tri<float, column_major>(upper, unit, n, A, lda, x);
}
void ref_trmm_f64(int upper, int unit, int a_rm, int b_rm, std::size_t m, std::size_t n, double const* A,
                  std::size_t lda, double* B, std::size_t ldb) {
	trmm_all<double>(upper, unit, a_rm, b_rm, m, n, A, lda, B, ldb);
}
void ref_trmm_f32(int upper, int unit, int a_rm, int b_rm, std::size_t m, std::size_t n, float const* A,
                  std::size_t lda, float* B, std::size_t ldb) {
	trmm_all<float>(upper, unit, a_rm, b_rm, m, n, A, lda, B, ldb);
}

// Seeded host generator (std::mt19937), as the reference's CPU tests and benchmarks use.
void* ref_rng_create(std::uint32_t seed) { return new std::mt19937(seed); }
void ref_rng_destroy(void* rng) { delete static_cast<std::mt19937*>(rng); }

// The device generators draw their key this way: kernels/hip/random.hpp:225-227.
void ref_rng_key(void* rng, std::uint32_t key[4]) {
	std::uniform_int_distribution<std::uint32_t> dist(0, 0xffffffff);
	auto& g = *static_cast<std::mt19937*>(rng);
	for (int i = 0; i != 4; ++i) key[i] = dist(g);
}

void ref_generate_normal_f64(void* rng, int row_major_, std::size_t rows, std::size_t cols,
                             double* A, std::size_t ld, double mean, double variance) {
	auto& g = *static_cast<std::mt19937*>(rng);
	if (row_major_) gen_normal<double, row_major>(g, rows, cols, A, ld, mean, variance);
	else gen_normal<double, column_major>(g, rows, cols, A, ld, mean, variance);
}
void ref_generate_normal_f32(void* rng, int row_major_, std::size_t rows, std::size_t cols,
                             float* A, std::size_t ld, float mean, float variance) {
	auto& g = *static_cast<std::mt19937*>(rng);
	if (row_major_) gen_normal<float, row_major>(g, rows, cols, A, ld, mean, variance);
	else gen_normal<float, column_major>(g, rows, cols, A, ld, mean, variance);
}
void ref_generate_uniform_f64(void* rng, int row_major_, std::size_t rows, std::size_t cols,
                              double* A, std::size_t ld, double low, double high) {
	auto& g = *static_cast<std::mt19937*>(rng);
	if (row_major_) gen_uniform<double, row_major>(g, rows, cols, A, ld, low, high);
	else gen_uniform<double, column_major>(g, rows, cols, A, ld, low, high);
}
void ref_generate_uniform_f32(void* rng, int row_major_, std::size_t rows, std::size_t cols,
                              float* A, std::size_t ld, float low, float high) {
	auto& g = *static_cast<std::mt19937*>(rng);
	if (row_major_) gen_uniform<float, row_major>(g, rows, cols, A, ld, low, high);
	else gen_uniform<float, column_major>(g, rows, cols, A, ld, low, high);
}

}  // extern "C"
