// Counter-based RNG fills (Threefry-4x32, 12 rounds) for Remora's cuda_tag.
//
// Replaces the reference's generate_{uniform,normal,discrete}32_kernel
// (include/remora/kernels/hip/random.hpp:163-210) and its launcher (:218-259). The
// stream is the reference's, bit for bit: same counter per (row, 4-column group)
// (:167, :181), same key schedule including the reference's third key injection
// (:102-106), same float transforms (:110-132) with the multiply-adds fused as nvcc
// compiles them. The layout differs: one thread per 4-element group, threads laid out
// along the storage's contiguous direction so each warp store is one or four 128-byte
// segments (16-byte vector stores for aligned row-major rows), a bounds check on both
// indices (the reference writes past the matrix when cols % 64 != 0, :172, :186), and
// a grid that strides over rows so row counts above 65535 launch.
#include "common.cuh"
#include <cmath>

namespace rc {
namespace {

__device__ __forceinline__ uint32_t rotl32(uint32_t v, unsigned r) { return __funnelshift_l(v, v, r); }

// Rotation amounts of the eight round slots (random.hpp:45-54).
__device__ __forceinline__ void mix_block(uint4& X, int slot_base) {
    const unsigned r0[8] = {10, 11, 13, 23, 6, 17, 25, 18};
    const unsigned r1[8] = {26, 21, 27, 5, 20, 11, 10, 20};
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const int s = slot_base + r;
        if ((r & 1) == 0) {
            X.x += X.y; X.y = rotl32(X.y, r0[s]) ^ X.x;
            X.z += X.w; X.w = rotl32(X.w, r1[s]) ^ X.z;
        } else {
            X.x += X.w; X.w = rotl32(X.w, r0[s]) ^ X.x;
            X.z += X.y; X.y = rotl32(X.y, r1[s]) ^ X.z;
        }
    }
}

__device__ __forceinline__ uint4 threefry(uint4 X, uint4 k) {
    const uint32_t k4 = 0x1BD11BDAu ^ k.x ^ k.y ^ k.z ^ k.w;
    X.x += k.x; X.y += k.y; X.z += k.z; X.w += k.w;
    mix_block(X, 0);
    X.x += k.y; X.y += k.z; X.z += k.w; X.w += k4 + 1u;
    mix_block(X, 4);
    X.x += k.z; X.y += k.w; X.z += k4; X.w += k.x + 2u;
    mix_block(X, 0);
    // Third injection as the reference has it: .z untouched, .w += k.x + k.y + 3.
    X.x += k.w; X.y += k4; X.w += k.x + k.y + 3u;
    return X;
}

__device__ __forceinline__ float unit_float(uint32_t x) {
    return __uint2float_rn(x) * 2.3283064365386963e-10f;  // * 2^-32, exact
}

__device__ __forceinline__ float uniform1(uint32_t x, float low, float range) {
    return nextafterf(__fmaf_rn(unit_float(x), range, low), low);
}

enum Kind { kBits = 0, kUniform = 1, kNormal = 2, kDiscreteF = 3, kDiscreteI = 4 };

template <int K>
struct Out { using type = float; };
template <> struct Out<kBits> { using type = uint32_t; };
template <> struct Out<kDiscreteI> { using type = int32_t; };

template <int K>
__device__ __forceinline__ void transform(uint4 x, float a, float b, int ia, uint32_t N,
                                          typename Out<K>::type v[4]) {
    if constexpr (K == kBits) {
        v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
    } else if constexpr (K == kUniform) {
        const float range = b - a;
        v[0] = uniform1(x.x, a, range); v[1] = uniform1(x.y, a, range);
        v[2] = uniform1(x.z, a, range); v[3] = uniform1(x.w, a, range);
    } else if constexpr (K == kNormal) {
        // Box-Muller on the four uniforms in [0,1] (random.hpp:119-132); a = mean, b = stddev.
        const float u0 = uniform1(x.x, 0.f, 1.f), u1 = uniform1(x.y, 0.f, 1.f);
        const float u2 = uniform1(x.z, 0.f, 1.f), u3 = uniform1(x.w, 0.f, 1.f);
        const float r0 = sqrtf(-2.0f * logf(u0));
        const float r1 = sqrtf(-2.0f * logf(u1));
        const float two_pi = 2.0f * 3.14159265358979323846f;
        float s0, c0, s1, c1;
        sincosf(two_pi * u2, &s0, &c0);
        sincosf(two_pi * u3, &s1, &c1);
        const float g0 = b * r0, g1 = b * r1;
        v[0] = __fmaf_rn(g0, s0, a); v[1] = __fmaf_rn(g0, c0, a);
        v[2] = __fmaf_rn(g1, s1, a); v[3] = __fmaf_rn(g1, c1, a);
    } else if constexpr (K == kDiscreteF) {
        const float lo = (float)ia;
        v[0] = lo + (float)(x.x % N); v[1] = lo + (float)(x.y % N);
        v[2] = lo + (float)(x.z % N); v[3] = lo + (float)(x.w % N);
    } else {
        v[0] = ia + (int32_t)(x.x % N); v[1] = ia + (int32_t)(x.y % N);
        v[2] = ia + (int32_t)(x.z % N); v[3] = ia + (int32_t)(x.w % N);
    }
}

// Row-major: thread x walks 4-column groups of one row (contiguous), grid.y strides rows.
template <int K>
__global__ void __launch_bounds__(256) fill_rowmajor(typename Out<K>::type* __restrict__ A, uint64_t ld,
                                                      uint64_t rows, uint64_t cols, uint4 key, float a,
                                                      float b, int ia, uint32_t N, bool vec_ok) {
    using T = typename Out<K>::type;
    const uint64_t groups = (cols + 3) / 4;
    for (uint64_t i = blockIdx.y; i < rows; i += gridDim.y) {
        T* row = A + i * ld;
        for (uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; g < groups;
             g += (uint64_t)gridDim.x * blockDim.x) {
            const uint64_t j = 4 * g;
            uint4 ctr = make_uint4((uint32_t)(i & 0xffffu), (uint32_t)(i >> 32), (uint32_t)(j & 0xffffu),
                                   (uint32_t)(j >> 32));
            T v[4];
            transform<K>(threefry(ctr, key), a, b, ia, N, v);
            if (vec_ok && j + 3 < cols) {
                uint4 packed;
                memcpy(&packed, v, sizeof(packed));
                reinterpret_cast<uint4*>(row + j)[0] = packed;
            } else {
#pragma unroll
                for (int c = 0; c < 4; ++c)
                    if (j + c < cols) row[j + c] = v[c];
            }
        }
    }
}

// Column-major: thread x walks rows (contiguous), each thread writes the 4 columns of its
// group, so every store instruction of a warp covers 32 consecutive elements of one column.
template <int K>
__global__ void __launch_bounds__(256) fill_colmajor(typename Out<K>::type* __restrict__ A, uint64_t ld,
                                                      uint64_t rows, uint64_t cols, uint4 key, float a,
                                                      float b, int ia, uint32_t N) {
    using T = typename Out<K>::type;
    const uint64_t groups = (cols + 3) / 4;
    for (uint64_t g = blockIdx.y; g < groups; g += gridDim.y) {
        const uint64_t j = 4 * g;
        for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < rows;
             i += (uint64_t)gridDim.x * blockDim.x) {
            uint4 ctr = make_uint4((uint32_t)(i & 0xffffu), (uint32_t)(i >> 32), (uint32_t)(j & 0xffffu),
                                   (uint32_t)(j >> 32));
            T v[4];
            transform<K>(threefry(ctr, key), a, b, ia, N, v);
#pragma unroll
            for (int c = 0; c < 4; ++c)
                if (j + c < cols) A[i + (j + c) * ld] = v[c];
        }
    }
}

template <int K>
int launch_fill(const uint32_t key[4], size_t rows, size_t cols, void* Av, size_t ld, int row_major,
                float a, float b, int ia, int ib, void* stream) {
    using T = typename Out<K>::type;
    if (!key || (rows && cols && !Av)) return RC_ERR_INVALID_ARGUMENT;
    if (rows == 0 || cols == 0) return RC_SUCCESS;
    if (row_major ? ld < cols : ld < rows) return RC_ERR_INVALID_ARGUMENT;
    uint32_t N = 1;
    if (K == kDiscreteF || K == kDiscreteI) {
        if (ib < ia) return RC_ERR_INVALID_ARGUMENT;
        const int64_t range = (int64_t)ib - (int64_t)ia + 1;
        if (range >= ((int64_t)1 << 32)) return RC_ERR_INVALID_ARGUMENT;
        N = (uint32_t)range;
    }
    T* A = static_cast<T*>(Av);
    const uint4 k = make_uint4(key[0], key[1], key[2], key[3]);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const unsigned threads = 256;
    if (row_major) {
        const uint64_t groups = (cols + 3) / 4;
        const bool vec_ok = (reinterpret_cast<uintptr_t>(A) % 16 == 0) && (ld % 4 == 0);
        dim3 grid(ceil_div(groups, threads) < 65535u ? ceil_div(groups, threads) : 65535u,
                  rows < 65535 ? (unsigned)rows : 65535u);
        fill_rowmajor<K><<<grid, threads, 0, s>>>(A, ld, rows, cols, k, a, b, ia, N, vec_ok);
    } else {
        const uint64_t groups = (cols + 3) / 4;
        dim3 grid(ceil_div(rows, threads) < 65535u ? ceil_div(rows, threads) : 65535u,
                  groups < 65535 ? (unsigned)groups : 65535u);
        fill_colmajor<K><<<grid, threads, 0, s>>>(A, ld, rows, cols, k, a, b, ia, N);
    }
    return check_launch();
}

}  // namespace
}  // namespace rc

extern "C" {

int rc_rng_bits_u32(const uint32_t key[4], size_t rows, size_t cols, uint32_t* A, size_t ld, int row_major,
                    void* stream) {
    return rc::launch_fill<rc::kBits>(key, rows, cols, A, ld, row_major, 0.f, 0.f, 0, 0, stream);
}
int rc_rng_uniform_f32(const uint32_t key[4], size_t rows, size_t cols, float* A, size_t ld, int row_major,
                       float low, float high, void* stream) {
    return rc::launch_fill<rc::kUniform>(key, rows, cols, A, ld, row_major, low, high, 0, 0, stream);
}
int rc_rng_normal_f32(const uint32_t key[4], size_t rows, size_t cols, float* A, size_t ld, int row_major,
                      float mean, float stddev, void* stream) {
    return rc::launch_fill<rc::kNormal>(key, rows, cols, A, ld, row_major, mean, stddev, 0, 0, stream);
}
int rc_rng_discrete_f32(const uint32_t key[4], size_t rows, size_t cols, float* A, size_t ld, int row_major,
                        int low, int high, void* stream) {
    return rc::launch_fill<rc::kDiscreteF>(key, rows, cols, A, ld, row_major, 0.f, 0.f, low, high, stream);
}
int rc_rng_discrete_i32(const uint32_t key[4], size_t rows, size_t cols, int32_t* A, size_t ld, int row_major,
                        int low, int high, void* stream) {
    return rc::launch_fill<rc::kDiscreteI>(key, rows, cols, A, ld, row_major, 0.f, 0.f, low, high, stream);
}

}  // extern "C"
