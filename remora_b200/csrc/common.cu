// Library-wide host helpers: status strings, SM count and the cached workspaces.
#include "common.cuh"
#include <atomic>
#include <map>
#include <mutex>
#include <utility>

namespace rc {
namespace {

struct Buffer {
    void* ptr = nullptr;
    size_t bytes = 0;
};

std::mutex g_mutex;
// (device, stream, slot) -> buffer
std::map<std::tuple<int, cudaStream_t, int>, Buffer> g_buffers;
std::atomic<unsigned long long> g_allocations{0};

}  // namespace

void note_allocation() { g_allocations.fetch_add(1, std::memory_order_relaxed); }

int sm_count() {
    static int counts[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (counts[dev] == 0) {
        int c = 0;
        if (cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || c <= 0) c = 148;
        counts[dev] = c;
    }
    return counts[dev];
}

void* workspace(cudaStream_t stream, size_t bytes, int slot) {
    if (bytes == 0) bytes = 256;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    std::lock_guard<std::mutex> lock(g_mutex);
    Buffer& b = g_buffers[std::make_tuple(dev, stream, slot)];
    if (b.bytes >= bytes) return b.ptr;
    if (b.ptr) {
        // Work queued earlier on this stream may still read the old buffer.
        if (cudaStreamSynchronize(stream) != cudaSuccess) return nullptr;
        cudaFree(b.ptr);
        b.ptr = nullptr;
        b.bytes = 0;
    }
    size_t rounded = (bytes + (1u << 20) - 1) & ~(size_t)((1u << 20) - 1);
    if (cudaMalloc(&b.ptr, rounded) != cudaSuccess) {
        cudaGetLastError();
        b.ptr = nullptr;
        return nullptr;
    }
    note_allocation();
    b.bytes = rounded;
    return b.ptr;
}

int* scratch_info(cudaStream_t stream) { return static_cast<int*>(workspace(stream, 256, 15)); }

namespace {
std::map<int, int*> g_error_words;
uint64_t g_wait_limit_ns = 2000000000ull;
}  // namespace

int* error_word() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    std::lock_guard<std::mutex> lock(g_mutex);
    int*& w = g_error_words[dev];
    if (!w) {  // [status, site of the first timeout]
        if (cudaMalloc(&w, 2 * sizeof(int)) != cudaSuccess || cudaMemset(w, 0, 2 * sizeof(int)) != cudaSuccess) {
            cudaGetLastError();
            w = nullptr;
        } else {
            note_allocation();
        }
    }
    return w;
}

int pending_error(cudaStream_t s) {
    int* w = error_word();
    if (!w) return RC_ERR_ALLOC;
    int v = 0;
    if (cudaMemcpyAsync(&v, w, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return RC_ERR_CUDA;
    return v;
}

namespace {
std::atomic<unsigned long long> g_launches{0};
}
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

uint64_t wait_limit_ns() { return g_wait_limit_ns; }
void set_wait_limit_ns(uint64_t ns) { g_wait_limit_ns = ns; }

}  // namespace rc

extern "C" {

int rc_version(void) { return 100; }

unsigned long long rc_launch_count(void) { return rc::g_launches.load(std::memory_order_relaxed); }

unsigned long long rc_allocation_count(void) { return rc::g_allocations.load(std::memory_order_relaxed); }

int rc_set_wait_limit_ns(uint64_t ns) {
    if (ns == 0) return RC_ERR_INVALID_ARGUMENT;
    rc::set_wait_limit_ns(ns);
    return RC_SUCCESS;
}

const char* rc_error_string(int status) {
    switch (status) {
    case RC_SUCCESS: return "success";
    case RC_ERR_INVALID_ARGUMENT: return "invalid argument (size, leading dimension or flag out of range)";
    case RC_ERR_CUDA: return "CUDA runtime error or kernel launch failure";
    case RC_ERR_ALLOC: return "device workspace allocation failed";
    case RC_ERR_NOT_SUPPORTED: return "combination not supported";
    case RC_ERR_TIMEOUT: return "a bounded device-side wait gave up";
    case RC_ERR_NOT_CONVERGED: return "iterative refinement did not converge";
    case RC_ERR_SIZE_LIMIT: return "problem larger than the entry point's fixed scratch";
    default: return "unknown status";
    }
}

int rc_release_workspaces(void) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return RC_ERR_CUDA;
    if (cudaDeviceSynchronize() != cudaSuccess) return RC_ERR_CUDA;
    std::lock_guard<std::mutex> lock(rc::g_mutex);
    for (auto it = rc::g_buffers.begin(); it != rc::g_buffers.end();) {
        if (std::get<0>(it->first) == dev) {
            cudaFree(it->second.ptr);
            it = rc::g_buffers.erase(it);
        } else {
            ++it;
        }
    }
    return RC_SUCCESS;
}

}  // extern "C"
