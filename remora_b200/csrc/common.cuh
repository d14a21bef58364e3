// Shared device/host helpers for the sm_100a kernels behind the C-ABI.
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include "../../include/remora_cuda.h"

namespace rc {

// A strided matrix view: element (i, j) at p[i * rs + j * cs]. Every dense Remora
// storage (detail/storage.hpp:71-91: values + leading_dimension, orientation giving
// the unit stride) is such a view with one of rs, cs equal to 1; transposition swaps
// the two strides.
template <class T>
struct View {
    T* p;
    int64_t rs, cs;
    __host__ __device__ T& operator()(int64_t i, int64_t j) const { return p[i * rs + j * cs]; }
    __host__ __device__ View sub(int64_t i, int64_t j) const { return {p + i * rs + j * cs, rs, cs}; }
    __host__ __device__ View t() const { return {p, cs, rs}; }
};

template <class T>
inline View<T> colmajor(T* p, int64_t ld) { return {p, 1, ld}; }

// Count of kernels this library has launched (every launch is followed by check_launch).
void count_launch();

inline int check_launch() {
    count_launch();
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? RC_SUCCESS : RC_ERR_CUDA;
}

#define RC_TRY(...)                           \
    do {                                      \
        int rc_status_ = (__VA_ARGS__);       \
        if (rc_status_ != RC_SUCCESS) return rc_status_; \
    } while (0)

// Count one device allocation made by the library for its own use (rc_allocation_count).
void note_allocation();

// Number of SMs of the current device (cached per device).
int sm_count();

// Library-managed device workspace, cached per (device, stream). Grows on demand; the
// stream is synchronised before a buffer it may still use is replaced. Returns nullptr
// on allocation failure. `slot` selects one of a few independent buffers.
void* workspace(cudaStream_t stream, size_t bytes, int slot = 0);

// Device int used as a per-call status word when the caller passes none.
int* scratch_info(cudaStream_t stream);

// The library's device error word of the current device (two ints, zero-initialised
// once): kernels whose bounded waits run out write RC_ERR_TIMEOUT to the first and the
// site of the first timeout to the second; rc_device_status reads and clears them. The
// word is sticky: while it is set, every tensor-core kernel returns at once.
int* error_word();

// Synchronise s and return the error word's status (RC_SUCCESS when clear) without
// clearing it; RC_ERR_CUDA / RC_ERR_ALLOC when it cannot be read.
int pending_error(cudaStream_t s);

// Wall-clock limit of every bounded device-side wait, in nanoseconds (default 2 s).
uint64_t wait_limit_ns();
void set_wait_limit_ns(uint64_t ns);

inline unsigned ceil_div(uint64_t a, uint64_t b) { return (unsigned)((a + b - 1) / b); }

}  // namespace rc
