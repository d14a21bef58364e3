// Test infrastructure: the CPU oracle (see rc_oracle.h). Each function restates the
// reference algorithm it names, in plain loops over strided views. Nothing in the product
// path links this file; tests, the smoke check and bench.py's CPU-baseline leg load it as
// the checker only.
#include "rc_oracle.h"
#include <cmath>
#include <cstring>
#include <random>
#include <limits>
#include <vector>

namespace {

template<class T>
struct View {
	T* p;
	ptrdiff_t rs, cs;
	T& operator()(size_t i, size_t j) const { return p[(ptrdiff_t)i * rs + (ptrdiff_t)j * cs]; }
	View sub(size_t i0, size_t j0) const { return {p + (ptrdiff_t)i0 * rs + (ptrdiff_t)j0 * cs, rs, cs}; }
	View t() const { return {p, cs, rs}; }
};

// ---------------------------------------------------------------------------------------
// Threefry-4x32 with 12 rounds: include/remora/kernels/hip/random.hpp:40-108.
// Rotation constants per round (r, mix of the first pair, mix of the second pair); even
// rounds mix (x,y),(z,w), odd rounds mix (x,w),(z,y) (random.hpp:45-54, :66-101).
const unsigned kRot[8][2] = {{10, 26}, {11, 21}, {13, 27}, {23, 5}, {6, 20}, {17, 11}, {25, 10}, {18, 20}};

inline uint32_t rotl(uint32_t v, unsigned r) { return (v << (r & 31)) | (v >> ((32 - r) & 31)); }

inline void four_rounds(uint32_t X[4], int first) {
	for (int r = 0; r < 4; ++r) {
		const unsigned* R = kRot[first + r];
		if ((r & 1) == 0) {
			X[0] += X[1]; X[1] = rotl(X[1], R[0]); X[1] ^= X[0];
			X[2] += X[3]; X[3] = rotl(X[3], R[1]); X[3] ^= X[2];
		} else {
			X[0] += X[3]; X[3] = rotl(X[3], R[0]); X[3] ^= X[0];
			X[2] += X[1]; X[1] = rotl(X[1], R[1]); X[1] ^= X[2];
		}
	}
}

// float(x) / 2^32: the divisor 0xffffffff of random.hpp:111 converts to the float 2^32.
inline float unit_float(uint32_t x) { return (float)x / 4294967296.0f; }

inline float affine(float z, float scale, float offset, int fused) {
	if (fused) return std::fmaf(z, scale, offset);
	float prod = z * scale;
	return offset + prod;
}

// uniform4_32_device: random.hpp:110-118
inline void uniform4(float low, float high, const uint32_t x[4], float out[4], int fused) {
	for (int c = 0; c < 4; ++c) out[c] = std::nextafterf(affine(unit_float(x[c]), high - low, low, fused), low);
}

// normal4_32_device: random.hpp:119-132 (Box-Muller on the four uniforms)
inline void normal4(float mean, float stddev, const uint32_t x[4], float out[4], int fused) {
	float u[4];
	uniform4(0.0f, 1.0f, x, u, fused);
	float r0 = std::sqrt(-2.0f * logf(u[0]));
	float r1 = std::sqrt(-2.0f * logf(u[1]));
	const float two_pi = 2.0f * (float)M_PI;
	float s0, c0, s1, c1;
	sincosf(two_pi * u[2], &s0, &c0);
	sincosf(two_pi * u[3], &s1, &c1);
	out[0] = affine(stddev * r0, s0, mean, fused);
	out[1] = affine(stddev * r0, c0, mean, fused);
	out[2] = affine(stddev * r1, s1, mean, fused);
	out[3] = affine(stddev * r1, c1, mean, fused);
}

// ---------------------------------------------------------------------------------------
// BLAS-3 restatements.
template<class T>
void gemm(size_t m, size_t n, size_t k, T alpha, View<const T> A, View<const T> B, View<T> C) {
	for (size_t i = 0; i < m; ++i)
		for (size_t j = 0; j < n; ++j) {
			T s = 0;
			for (size_t l = 0; l < k; ++l) s += A(i, l) * B(l, j);
			C(i, j) += alpha * s;
		}
}

template<class T>
void syrk(bool upper, size_t n, size_t k, T alpha, View<const T> A, View<T> C) {
	for (size_t i = 0; i < n; ++i)
		for (size_t j = 0; j < n; ++j) {
			if (upper ? (j < i) : (j > i)) continue;
			T s = 0;
			for (size_t l = 0; l < k; ++l) s += A(i, l) * A(j, l);
			C(i, j) += alpha * s;
		}
}

// trsm_block: kernels/default/trsm.hpp:44-225 (substitution per right-hand side column).
template<class T>
int trsm_block(bool upper, bool unit, size_t size, size_t nrhs, View<const T> A, View<T> B) {
	for (size_t c = 0; c < nrhs; ++c) {
		for (size_t step = 0; step < size; ++step) {
			size_t i = upper ? size - 1 - step : step;
			T v = B(i, c);
			if (upper) {
				for (size_t j = i + 1; j < size; ++j) v -= A(i, j) * B(j, c);
			} else {
				for (size_t j = 0; j < i; ++j) v -= A(i, j) * B(j, c);
			}
			if (!unit) {
				if (A(i, i) == T(0)) return 1;  // trsm.hpp:86-87 throws "Matrix is singular"
				v /= A(i, i);
			}
			B(i, c) = v;
		}
	}
	return 0;
}

// trsm_recursive (left): kernels/default/trsm.hpp:227-261 -- halve at a multiple of 32,
// solve one half, update the other with a gemm, solve the other half.
template<class T>
int trsm_left(bool upper, bool unit, size_t size, size_t nrhs, View<const T> A, View<T> B) {
	const size_t block = 32;
	if (size <= block) return trsm_block(upper, unit, size, nrhs, A, B);
	size_t split = (size + block - 1) / block / 2 * block;
	View<const T> A11 = A, A22 = A.sub(split, split);
	View<T> Bf = B, Bb = B.sub(split, 0);
	int r;
	if (upper) {
		if ((r = trsm_left(upper, unit, size - split, nrhs, A22, Bb))) return r;
		gemm<T>(split, nrhs, size - split, T(-1), A.sub(0, split), View<const T>{Bb.p, Bb.rs, Bb.cs}, Bf);
		return trsm_left(upper, unit, split, nrhs, A11, Bf);
	}
	if ((r = trsm_left(upper, unit, split, nrhs, A11, Bf))) return r;
	gemm<T>(size - split, nrhs, split, T(-1), A.sub(split, 0), View<const T>{Bf.p, Bf.rs, Bf.cs}, Bb);
	return trsm_left(upper, unit, size - split, nrhs, A22, Bb);
}

// Right side: trsm.hpp:263-275 -- transpose A and B and solve on the left with the
// transposed triangle.
template<class T>
int trsm(bool left, bool upper, bool unit, size_t m, size_t n, View<const T> A, View<T> B) {
	if (left) return trsm_left(upper, unit, m, n, A, B);
	return trsm_left(!upper, unit, n, m, A.t(), B.t());
}

// gemv: kernels/default/gemv.hpp:41-92 -- y += alpha * A x (one dot product per row).
template<class T>
void gemv(size_t m, size_t n, T alpha, View<const T> A, const T* x, ptrdiff_t incx, T* y, ptrdiff_t incy) {
	for (size_t i = 0; i < m; ++i) {
		T s = 0;
		for (size_t j = 0; j < n; ++j) s += A(i, j) * x[(ptrdiff_t)j * incx];
		y[(ptrdiff_t)i * incy] += alpha * s;
	}
}

// trmm / trmv: kernels/default/trmm.hpp:40-120, trmv.hpp:40-96 -- B <- T B for the named
// triangle T of A (ones on the diagonal when unit), evaluated into a copy.
template<class T>
void trmm(bool upper, bool unit, size_t m, size_t n, View<const T> A, View<T> B) {
	std::vector<T> out(m * n);
	for (size_t c = 0; c < n; ++c)
		for (size_t i = 0; i < m; ++i) {
			T s = unit ? B(i, c) : A(i, i) * B(i, c);
			if (upper) {
				for (size_t j = i + 1; j < m; ++j) s += A(i, j) * B(j, c);
			} else {
				for (size_t j = 0; j < i; ++j) s += A(i, j) * B(j, c);
			}
			out[c * m + i] = s;
		}
	for (size_t c = 0; c < n; ++c)
		for (size_t i = 0; i < m; ++i) B(i, c) = out[c * m + i];
}

// potrf_block (lower, left-looking, double accumulator): kernels/default/potrf.hpp:42-64.
// Returns the 1-based index inside the block of the first pivot s <= 0.
template<class T>
size_t potrf_block(size_t m, View<T> A) {
	for (size_t j = 0; j < m; ++j) {
		for (size_t i = j; i < m; ++i) {
			double s = A(i, j);
			for (size_t k = 0; k < j; ++k) s -= (double)(T)(A(i, k) * A(j, k));
			if (i == j) {
				if (!(s > 0)) return i + 1;
				A(i, j) = (T)std::sqrt(s);
			} else {
				A(i, j) = (T)(s / A(j, j));
			}
		}
	}
	return 0;
}

// potrf_recursive (lower): kernels/default/potrf.hpp:106-134 -- block 32, split at a
// multiple of 32, then trsm<upper,right>(trans(A11), A21) and syrk<lower>(A21, A22, -1).
// Unlike the reference (:125-133, which returns an index relative to the sub-block), the
// failing pivot is reported as a global 1-based index.
template<class T>
size_t potrf_rec(size_t size, View<T> A, size_t offset) {
	const size_t block = 32;
	if (size <= block) {
		size_t r = potrf_block<T>(size, A);
		return r ? r + offset : 0;
	}
	size_t split = (size + block - 1) / block / 2 * block;
	size_t r = potrf_rec<T>(split, A, offset);
	if (r) return r;
	View<T> A21 = A.sub(split, 0), A22 = A.sub(split, split);
	View<const T> L11t{A.p, A.cs, A.rs};
	trsm<T>(false, true, false, size - split, split, L11t, A21);
	syrk<T>(false, size - split, split, T(-1), View<const T>{A21.p, A21.rs, A21.cs}, A22);
	return potrf_rec<T>(size - split, A22, offset + split);
}

template<class T>
size_t potrf(int upper, size_t n, View<T> A) {
	// upper: kernels/default/potrf.hpp:136-145 -- the lower algorithm on the transpose.
	return potrf_rec<T>(n, upper ? A.t() : A, 0);
}

// ---------------------------------------------------------------------------------------
// LU with partial pivoting and pivoted Cholesky.

// Row swaps r <-> piv[r] (r = 0, 1, ...) on rows x cols of A; piv relative to A's first row.
template<class T>
void swap_rows_seq(size_t count, const int* piv, size_t cols, View<T> A) {
	for (size_t r = 0; r < count; ++r) {
		const size_t q = (size_t)piv[r];
		if (q == r) continue;
		for (size_t c = 0; c < cols; ++c) std::swap(A(r, c), A(q, c));
	}
}

// getrf_block (column-major order): kernels/default/getrf.hpp:41-79 -- per column j the
// pivot is the first row of largest |A(i, j)| (a later row replaces it only when strictly
// larger), rows j and pivot are swapped across the panel's columns, the column below the
// diagonal is divided by the pivot (in double) and the rank-1 update is applied to the
// panel's remaining columns. Returns j + 1 for a zero pivot (the reference throws).
template<class T>
size_t getrf_panel(size_t rows, size_t cols, View<T> A, int* piv) {
	for (size_t j = 0; j < cols; ++j) {
		double pv = A(j, j);
		piv[j] = (int)j;
		for (size_t i = j + 1; i < rows; ++i)
			if (std::abs((double)A(i, j)) > std::abs(pv)) {
				piv[j] = (int)i;
				pv = A(i, j);
			}
		if (pv == 0) return j + 1;
		if ((size_t)piv[j] != j)
			for (size_t c = 0; c < cols; ++c) std::swap(A(j, c), A((size_t)piv[j], c));
		for (size_t i = j + 1; i < rows; ++i) A(i, j) = (T)(A(i, j) / pv);
		for (size_t k = j + 1; k < cols; ++k)
			for (size_t i = j + 1; i < rows; ++i) A(i, k) -= A(i, j) * A(j, k);
	}
	return 0;
}

// getrf_recursive: kernels/default/getrf.hpp:117-166 -- columns [start, end) of the n x n A,
// split at a multiple of 4 columns: left half recursively, its row swaps applied to the
// right half's columns, A12 <- L11^-1 A12 (unit lower), A22 -= A21 A12, right half
// recursively, its row swaps applied to A21 and its pivots made relative to `start`.
template<class T>
size_t getrf_rec(size_t n, View<T> A, int* piv, size_t start, size_t end) {
	const size_t block = 4, size = end - start, rows = n - start;
	if (size <= block) {
		const size_t r = getrf_panel<T>(rows, size, A.sub(start, start), piv + start);
		return r ? r + start : 0;
	}
	const size_t split = start + (size + block - 1) / block / 2 * block;
	size_t r = getrf_rec<T>(n, A, piv, start, split);
	if (r) return r;
	swap_rows_seq<T>(split - start, piv + start, end - split, A.sub(start, split));
	View<const T> L11{A.sub(start, start).p, A.rs, A.cs};
	trsm<T>(true, false, true, split - start, end - split, L11, A.sub(start, split));
	View<const T> A21{A.sub(split, start).p, A.rs, A.cs}, A12{A.sub(start, split).p, A.rs, A.cs};
	gemm<T>(n - split, end - split, split - start, T(-1), A21, A12, A.sub(split, split));
	if ((r = getrf_rec<T>(n, A, piv, split, end))) return r;
	swap_rows_seq<T>(end - split, piv + split, split - start, A.sub(split, start));
	for (size_t i = split; i < end; ++i) piv[i] += (int)(split - start);
	return 0;
}

// pstrf (lower): kernels/default/pstrf.hpp:40-147, the blocked pivoted Cholesky of LAWN 161
// with blocks of 20 columns. Inside a block the pivot values (the diagonal of the updated
// trailing matrix) are refreshed from the block's finished columns; the largest remaining
// one (first of equals) is swapped into place, rows and columns of the whole matrix; the
// factor stops with rank k + j once a pivot value falls below n^2 eps max|A_ii| (the
// trailing square is cleared); each column is finished by a gemv against the block's
// earlier columns and a division; the row right of the diagonal is cleared; after the
// block, the trailing square is updated with the block's columns. piv[i] is set only where
// a swap happens (callers start from the identity). Returns the rank.
template<class T>
size_t pstrf_lower(size_t m, View<T> A, int* piv) {
	const size_t block = 20;
	double max_diag = A(0, 0);
	for (size_t i = 1; i < m; ++i) max_diag = std::max(max_diag, (double)std::abs(A(i, i)));
	const double eps = (double)(m * m) * std::numeric_limits<T>::epsilon() * max_diag;
	std::vector<T> pv(m);
	for (size_t k = 0; k < m; k += block) {
		const size_t cur = std::min(m - k, block), rest = m - k;
		View<T> Ak = A.sub(k, k);
		for (size_t j = 0; j < cur; ++j) {
			if (j == 0) {
				for (size_t i = 0; i < rest; ++i) pv[i] = Ak(i, i);
			} else {
				for (size_t i = j; i < rest; ++i) pv[i] -= Ak(i, j - 1) * Ak(i, j - 1);
			}
			size_t p = j;
			for (size_t i = j + 1; i < rest; ++i)
				if (pv[i] > pv[p]) p = i;
			if (p != j) {
				piv[k + j] = (int)(k + p);
				for (size_t c = 0; c < m; ++c) std::swap(A(k + j, c), A(k + p, c));
				for (size_t r = 0; r < m; ++r) std::swap(A(r, k + j), A(r, k + p));
				std::swap(pv[j], pv[p]);
			}
			const T v = pv[j];
			if (v < eps) {
				for (size_t i = j; i < rest; ++i)
					for (size_t c = j; c < rest; ++c) Ak(i, c) = T(0);
				return k + j;
			}
			Ak(j, j) = std::sqrt(v);
			if (j > 0) {
				std::vector<T> row(j);
				for (size_t c = 0; c < j; ++c) row[c] = Ak(j, c);
				View<const T> LL{Ak.sub(j + 1, 0).p, Ak.rs, Ak.cs};
				gemv<T>(rest - j - 1, j, T(-1), LL, row.data(), 1, &Ak(j + 1, j), Ak.rs);
			}
			for (size_t i = j + 1; i < rest; ++i) Ak(i, j) /= Ak(j, j);
			for (size_t c = j + 1; c < rest; ++c) Ak(j, c) = T(0);
		}
		if (k + cur < m) {
			View<const T> LL{Ak.sub(block, 0).p, Ak.rs, Ak.cs};
			gemm<T>(rest - block, rest - block, block, T(-1), LL, LL.t(), Ak.sub(block, block));
		}
	}
	return m;
}

}  // namespace

extern "C" {

void orc_counter(uint64_t i, uint64_t j, uint32_t ctr[4]) {
	// random.hpp:167: make_uint4(id_x & 0x0000ffff, id_x >> 32, id_y & 0x0000ffff, id_y >> 32)
	ctr[0] = (uint32_t)(i & 0xffffu);
	ctr[1] = (uint32_t)(i >> 32);
	ctr[2] = (uint32_t)(j & 0xffffu);
	ctr[3] = (uint32_t)(j >> 32);
}

void orc_threefry(const uint32_t ctr[4], const uint32_t key[4], uint32_t out[4]) {
	const uint32_t k4 = 0x1BD11BDAu ^ key[0] ^ key[1] ^ key[2] ^ key[3];
	uint32_t X[4];
	for (int c = 0; c < 4; ++c) X[c] = ctr[c] + key[c];
	four_rounds(X, 0);
	X[0] += key[1]; X[1] += key[2]; X[2] += key[3]; X[3] += k4 + 1u;   // random.hpp:74-78
	four_rounds(X, 4);
	X[0] += key[2]; X[1] += key[3]; X[2] += k4; X[3] += key[0] + 2u;   // random.hpp:88-92
	four_rounds(X, 0);
	// random.hpp:102-106: the third injection leaves .z alone and adds key[0] AND key[1]
	// to .w (textbook Threefry adds key[0] to .z and key[1] to .w).
	X[0] += key[3]; X[1] += k4; X[3] += key[0] + key[1] + 3u;
	for (int c = 0; c < 4; ++c) out[c] = X[c];
}

void orc_rng_fill_block(int kind, const uint32_t key[4], uint64_t row0, uint64_t col0, size_t rows,
                        size_t cols, void* A, ptrdiff_t rs, ptrdiff_t cs, float a, float b, int ia,
                        int ib, int fused) {
	// generate_*32_kernel: random.hpp:163-210 -- one Threefry call per (row i, 4-column
	// group); component c of the result goes to column 4*j4 + c if it is in range.
	const uint32_t N = (uint32_t)(ib - ia) + 1u;
	for (size_t i = 0; i < rows; ++i) {
		for (size_t j4 = 0; j4 < cols; j4 += 4) {
			uint32_t ctr[4], x[4];
			orc_counter(row0 + i, col0 + j4, ctr);
			orc_threefry(ctr, key, x);
			float f[4];
			if (kind == 1) uniform4(a, b, x, f, fused);
			if (kind == 2) normal4(a, b, x, f, fused);
			for (size_t c = 0; c < 4 && j4 + c < cols; ++c) {
				ptrdiff_t off = (ptrdiff_t)i * rs + (ptrdiff_t)(j4 + c) * cs;
				switch (kind) {
				case 0: ((uint32_t*)A)[off] = x[c]; break;
				case 1: case 2: ((float*)A)[off] = f[c]; break;
				case 3: ((float*)A)[off] = (float)ia + (float)(x[c] % N); break;  // :202 low + float(z)
				case 4: ((int32_t*)A)[off] = ia + (int32_t)(x[c] % N); break;
				}
			}
		}
	}
}

void orc_rng_fill(int kind, const uint32_t key[4], size_t rows, size_t cols, void* A,
                  ptrdiff_t rs, ptrdiff_t cs, float a, float b, int ia, int ib, int fused) {
	orc_rng_fill_block(kind, key, 0, 0, rows, cols, A, rs, cs, a, b, ia, ib, fused);
}

void orc_gemm_f64(size_t m, size_t n, size_t k, double alpha, const double* A, ptrdiff_t ars, ptrdiff_t acs,
                  const double* B, ptrdiff_t brs, ptrdiff_t bcs, double* C, ptrdiff_t crs, ptrdiff_t ccs) {
	gemm<double>(m, n, k, alpha, {A, ars, acs}, {B, brs, bcs}, {C, crs, ccs});
}
void orc_gemm_f32(size_t m, size_t n, size_t k, float alpha, const float* A, ptrdiff_t ars, ptrdiff_t acs,
                  const float* B, ptrdiff_t brs, ptrdiff_t bcs, float* C, ptrdiff_t crs, ptrdiff_t ccs) {
	gemm<float>(m, n, k, alpha, {A, ars, acs}, {B, brs, bcs}, {C, crs, ccs});
}
void orc_syrk_f64(int upper, size_t n, size_t k, double alpha, const double* A, ptrdiff_t ars, ptrdiff_t acs,
                  double* C, ptrdiff_t crs, ptrdiff_t ccs) {
	syrk<double>(upper != 0, n, k, alpha, {A, ars, acs}, {C, crs, ccs});
}
void orc_syrk_f32(int upper, size_t n, size_t k, float alpha, const float* A, ptrdiff_t ars, ptrdiff_t acs,
                  float* C, ptrdiff_t crs, ptrdiff_t ccs) {
	syrk<float>(upper != 0, n, k, alpha, {A, ars, acs}, {C, crs, ccs});
}
int orc_trsm_f64(int left, int upper, int unit, size_t m, size_t n, const double* A, ptrdiff_t ars, ptrdiff_t acs,
                 double* B, ptrdiff_t brs, ptrdiff_t bcs) {
	return trsm<double>(left != 0, upper != 0, unit != 0, m, n, {A, ars, acs}, {B, brs, bcs});
}
int orc_trsm_f32(int left, int upper, int unit, size_t m, size_t n, const float* A, ptrdiff_t ars, ptrdiff_t acs,
                 float* B, ptrdiff_t brs, ptrdiff_t bcs) {
	return trsm<float>(left != 0, upper != 0, unit != 0, m, n, {A, ars, acs}, {B, brs, bcs});
}
void orc_gemv_f64(size_t m, size_t n, double alpha, const double* A, ptrdiff_t ars, ptrdiff_t acs, const double* x,
                  ptrdiff_t incx, double* y, ptrdiff_t incy) {
	gemv<double>(m, n, alpha, {A, ars, acs}, x, incx, y, incy);
}
void orc_gemv_f32(size_t m, size_t n, float alpha, const float* A, ptrdiff_t ars, ptrdiff_t acs, const float* x,
                  ptrdiff_t incx, float* y, ptrdiff_t incy) {
	gemv<float>(m, n, alpha, {A, ars, acs}, x, incx, y, incy);
}
// trsv: kernels/default/trsv.hpp -- the one-column case of trsm (left), or x A = b as
// A^T x^T = b^T (right).
int orc_trsv_f64(int left, int upper, int unit, size_t n, const double* A, ptrdiff_t ars, ptrdiff_t acs, double* x,
                 ptrdiff_t incx) {
	if (left) return trsm<double>(true, upper != 0, unit != 0, n, 1, {A, ars, acs}, {x, incx, 0});
	return trsm<double>(true, upper == 0, unit != 0, n, 1, View<const double>{A, ars, acs}.t(), {x, incx, 0});
}
int orc_trsv_f32(int left, int upper, int unit, size_t n, const float* A, ptrdiff_t ars, ptrdiff_t acs, float* x,
                 ptrdiff_t incx) {
	if (left) return trsm<float>(true, upper != 0, unit != 0, n, 1, {A, ars, acs}, {x, incx, 0});
	return trsm<float>(true, upper == 0, unit != 0, n, 1, View<const float>{A, ars, acs}.t(), {x, incx, 0});
}
void orc_trmm_f64(int upper, int unit, size_t m, size_t n, const double* A, ptrdiff_t ars, ptrdiff_t acs, double* B,
                  ptrdiff_t brs, ptrdiff_t bcs) {
	trmm<double>(upper != 0, unit != 0, m, n, {A, ars, acs}, {B, brs, bcs});
}
void orc_trmm_f32(int upper, int unit, size_t m, size_t n, const float* A, ptrdiff_t ars, ptrdiff_t acs, float* B,
                  ptrdiff_t brs, ptrdiff_t bcs) {
	trmm<float>(upper != 0, unit != 0, m, n, {A, ars, acs}, {B, brs, bcs});
}
size_t orc_potrf_f64(int upper, size_t n, double* A, ptrdiff_t rs, ptrdiff_t cs) {
	return potrf<double>(upper, n, {A, rs, cs});
}
size_t orc_potrf_f32(int upper, size_t n, float* A, ptrdiff_t rs, ptrdiff_t cs) {
	return potrf<float>(upper, n, {A, rs, cs});
}
size_t orc_getrf_f64(size_t n, double* A, ptrdiff_t rs, ptrdiff_t cs, int* piv) {
	for (size_t i = 0; i < n; ++i) piv[i] = (int)i;
	return getrf_rec<double>(n, {A, rs, cs}, piv, 0, n);
}
size_t orc_getrf_f32(size_t n, float* A, ptrdiff_t rs, ptrdiff_t cs, int* piv) {
	for (size_t i = 0; i < n; ++i) piv[i] = (int)i;
	return getrf_rec<float>(n, {A, rs, cs}, piv, 0, n);
}
size_t orc_pstrf_f64(size_t n, double* A, ptrdiff_t rs, ptrdiff_t cs, int* piv) {
	for (size_t i = 0; i < n; ++i) piv[i] = (int)i;
	return n ? pstrf_lower<double>(n, {A, rs, cs}, piv) : 0;
}
size_t orc_pstrf_f32(size_t n, float* A, ptrdiff_t rs, ptrdiff_t cs, int* piv) {
	for (size_t i = 0; i < n; ++i) piv[i] = (int)i;
	return n ? pstrf_lower<float>(n, {A, rs, cs}, piv) : 0;
}
size_t orc_cholesky_solve_f64(size_t n, size_t nrhs, const double* A, ptrdiff_t ars, ptrdiff_t acs,
                              double* B, ptrdiff_t brs, ptrdiff_t bcs) {
	// decompositions.hpp:81-84 (copy + potrf<lower>) and :101-105 (two left trsm).
	std::vector<double> L(n * n);
	View<double> Lv{L.data(), (ptrdiff_t)n, 1};
	for (size_t i = 0; i < n; ++i)
		for (size_t j = 0; j < n; ++j) Lv(i, j) = A[(ptrdiff_t)i * ars + (ptrdiff_t)j * acs];
	size_t r = potrf<double>(0, n, Lv);
	if (r) return r;
	View<double> Bv{B, brs, bcs};
	View<const double> Lc{L.data(), (ptrdiff_t)n, 1};
	trsm<double>(true, false, false, n, nrhs, Lc, Bv);
	trsm<double>(true, true, false, n, nrhs, Lc.t(), Bv);
	return 0;
}

}  // extern "C"
