// Test infrastructure: the oracle's input generator (std::mt19937 with the std
// distributions), the same calls the reference's CPU generator makes
// (include/remora/kernels/default/random.hpp:37-122). Kept in its own translation unit
// so it is compiled with the reference build's floating-point flags (oracle/Makefile):
// libstdc++'s distributions are header code, and contraction changes their last bit.
#include "rc_oracle.h"
#include <cmath>
#include <cstdlib>
#include <random>

namespace {
template<class T>
struct View {
	T* p;
	ptrdiff_t rs, cs;
	T& operator()(size_t i, size_t j) const { return p[(ptrdiff_t)i * rs + (ptrdiff_t)j * cs]; }
};

template<class T, class D>
void gen_fill(std::mt19937& g, D& dist, size_t rows, size_t cols, View<T> A) {
	// major-order traversal of kernels/default/random.hpp:57-63: along the storage's
	// contiguous direction inside each major index.
	bool row_major = std::abs(A.cs) <= std::abs(A.rs);
	size_t major = row_major ? rows : cols, minor = row_major ? cols : rows;
	for (size_t a = 0; a < major; ++a)
		for (size_t b = 0; b < minor; ++b) (row_major ? A(a, b) : A(b, a)) = dist(g);
}

}  // namespace

extern "C" {

void* orc_rng_create(uint32_t seed) { return new std::mt19937(seed); }
void orc_rng_destroy(void* rng) { delete static_cast<std::mt19937*>(rng); }
void orc_rng_key(void* rng, uint32_t key[4]) {
	// random.hpp:225-227
	std::uniform_int_distribution<uint32_t> dist(0, 0xffffffffu);
	for (int i = 0; i < 4; ++i) key[i] = dist(*static_cast<std::mt19937*>(rng));
}
void orc_generate_normal_f64(void* rng, size_t rows, size_t cols, double* A, ptrdiff_t rs, ptrdiff_t cs,
                             double mean, double variance) {
	std::normal_distribution<double> d(mean, std::sqrt(variance));
	gen_fill(*static_cast<std::mt19937*>(rng), d, rows, cols, View<double>{A, rs, cs});
}
void orc_generate_uniform_f64(void* rng, size_t rows, size_t cols, double* A, ptrdiff_t rs, ptrdiff_t cs,
                              double low, double high) {
	std::uniform_real_distribution<double> d(low, high);
	gen_fill(*static_cast<std::mt19937*>(rng), d, rows, cols, View<double>{A, rs, cs});
}
void orc_generate_normal_f32(void* rng, size_t rows, size_t cols, float* A, ptrdiff_t rs, ptrdiff_t cs,
                             float mean, float variance) {
	std::normal_distribution<float> d(mean, std::sqrt(variance));
	gen_fill(*static_cast<std::mt19937*>(rng), d, rows, cols, View<float>{A, rs, cs});
}
void orc_generate_uniform_f32(void* rng, size_t rows, size_t cols, float* A, ptrdiff_t rs, ptrdiff_t cs,
                              float low, float high) {
	std::uniform_real_distribution<float> d(low, high);
	gen_fill(*static_cast<std::mt19937*>(rng), d, rows, cols, View<float>{A, rs, cs});
}

}  // extern "C"
