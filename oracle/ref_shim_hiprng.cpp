// Test infrastructure, not product code: compiles the reference's device RNG functions
// (include/remora/kernels/hip/random.hpp:40-161) as HOST code, so that the reference's
// own Threefry-4x32 rounds, counter schedule and float transforms run here and pin the
// oracle restatement bit for bit. The reference has no CPU implementation of this
// stream; its HIP toolchain is absent, so a small host environment below stands in for
// the HIP vector types and launch macros the header names. Only the __device__ helper
// functions are called; the templated kernels are parsed but never instantiated.
//
// Floating-point contraction: the reference's generator is compiled by nvcc for NVIDIA
// GPUs, where `low + z * (high - low)` (random.hpp:113-116) and
// `mean + stddev * r * sin` (:127-130) are fused into FMAs by default (--fmad=true).
// oracle/Makefile builds this file with -mfma -ffp-contract=fast so the host build
// fuses the same expressions; the transcendental functions (logf, sincosf) are glibc's.
#include <cstddef>
#include <cstdint>
#include <cmath>
#include <algorithm>
#include <type_traits>

typedef unsigned int uint;
struct uint4 { uint x, y, z, w; };
struct float4 { float x, y, z, w; };
struct float2 { float x, y; };
static inline uint4 make_uint4(uint x, uint y, uint z, uint w) { return {x, y, z, w}; }
static inline float4 make_float4(float x, float y, float z, float w) { return {x, y, z, w}; }
static inline float2 make_float2(float x, float y) { return {x, y}; }
inline std::size_t min(std::size_t a, std::size_t b) { return a < b ? a : b; }
struct hipLaunchParm {};
#define __device__
#define __global__
#define hipBlockIdx_x 0u
#define hipBlockIdx_y 0u
#define hipBlockDim_x 1u
#define hipBlockDim_y 1u
#define hipThreadIdx_x 0u
#define hipThreadIdx_y 0u
#define hipLaunchKernel(...) ((void)0)

#include <remora/proxy_expressions.hpp>
#include <remora/detail/traits.hpp>
#include <remora/kernels/hip/random.hpp>

extern "C" {

// rng4_32_device: kernels/hip/random.hpp:44-108
void ref_hip_threefry(const std::uint32_t ctr[4], const std::uint32_t key[4], std::uint32_t out[4]) {
	uint4 r = remora::hip::rng4_32_device(make_uint4(ctr[0], ctr[1], ctr[2], ctr[3]),
	                                      make_uint4(key[0], key[1], key[2], key[3]));
	out[0] = r.x; out[1] = r.y; out[2] = r.z; out[3] = r.w;
}

// uniform4_32_device: kernels/hip/random.hpp:110-118
void ref_hip_uniform4(float low, float high, const std::uint32_t x[4], float out[4]) {
	float4 r = remora::hip::uniform4_32_device(low, high, make_uint4(x[0], x[1], x[2], x[3]));
	out[0] = r.x; out[1] = r.y; out[2] = r.z; out[3] = r.w;
}

// normal4_32_device: kernels/hip/random.hpp:119-132
void ref_hip_normal4(float mean, float stddev, const std::uint32_t x[4], float out[4]) {
	float4 r = remora::hip::normal4_32_device(mean, stddev, make_uint4(x[0], x[1], x[2], x[3]));
	out[0] = r.x; out[1] = r.y; out[2] = r.z; out[3] = r.w;
}

// discrete4_32_device: kernels/hip/random.hpp:133-161
void ref_hip_discrete4(const std::uint32_t key[4], const std::uint32_t ctr[4], std::uint32_t N, std::uint32_t out[4]) {
	uint4 r = remora::hip::discrete4_32_device(make_uint4(key[0], key[1], key[2], key[3]),
	                                           make_uint4(ctr[0], ctr[1], ctr[2], ctr[3]), N,
	                                           make_uint4(0, 0, 0, 0));
	out[0] = r.x; out[1] = r.y; out[2] = r.z; out[3] = r.w;
}

}  // extern "C"
