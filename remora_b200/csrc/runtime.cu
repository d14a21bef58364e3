// Device runtime entry points for host code that is compiled without the CUDA toolkit
// (the header-only cuda_tag containers): device selection, allocation, 2-D copies,
// page-locked host staging, events and streams. They replace the HIP runtime calls of
// include/remora/hip/device.hpp:41-180 and include/remora/hip/buffer.hpp:41-102, and the
// mapped-memory transport of include/remora/hip/copy.hpp:131-410 (here: pitched
// cudaMemcpy2DAsync through double-buffered page-locked chunks).
#include "common.cuh"

namespace {
int status_of(cudaError_t e) {
    if (e == cudaSuccess) return RC_SUCCESS;
    cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? RC_ERR_ALLOC : RC_ERR_CUDA;
}
}  // namespace

extern "C" {

int rc_device_count(int* count) {
    if (!count) return RC_ERR_INVALID_ARGUMENT;
    return status_of(cudaGetDeviceCount(count));
}
int rc_set_device(int device) { return status_of(cudaSetDevice(device)); }
int rc_get_device(int* device) {
    if (!device) return RC_ERR_INVALID_ARGUMENT;
    return status_of(cudaGetDevice(device));
}

int rc_malloc(void** ptr, size_t bytes) {
    if (!ptr) return RC_ERR_INVALID_ARGUMENT;
    *ptr = nullptr;
    if (bytes == 0) return RC_SUCCESS;
    return status_of(cudaMalloc(ptr, bytes));
}
int rc_free(void* ptr) { return ptr ? status_of(cudaFree(ptr)) : RC_SUCCESS; }

int rc_memcpy2d(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width_bytes, size_t rows,
                int kind, void* stream) {
    if (width_bytes == 0 || rows == 0) return RC_SUCCESS;
    if (!dst || !src || dpitch < width_bytes || spitch < width_bytes) return RC_ERR_INVALID_ARGUMENT;
    cudaMemcpyKind k;
    switch (kind) {
    case RC_COPY_H2D: k = cudaMemcpyHostToDevice; break;
    case RC_COPY_D2H: k = cudaMemcpyDeviceToHost; break;
    case RC_COPY_D2D: k = cudaMemcpyDeviceToDevice; break;
    default: return RC_ERR_INVALID_ARGUMENT;
    }
    return status_of(cudaMemcpy2DAsync(dst, dpitch, src, spitch, width_bytes, rows, k,
                                       static_cast<cudaStream_t>(stream)));
}

int rc_host_alloc(void** ptr, size_t bytes) {
    if (!ptr) return RC_ERR_INVALID_ARGUMENT;
    *ptr = nullptr;
    if (bytes == 0) return RC_SUCCESS;
    return status_of(cudaHostAlloc(ptr, bytes, cudaHostAllocPortable));
}
int rc_host_free(void* ptr) { return ptr ? status_of(cudaFreeHost(ptr)) : RC_SUCCESS; }

int rc_event_create(void** event) {
    if (!event) return RC_ERR_INVALID_ARGUMENT;
    cudaEvent_t e = nullptr;
    const int r = status_of(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    *event = e;
    return r;
}
int rc_event_record(void* event, void* stream) {
    if (!event) return RC_ERR_INVALID_ARGUMENT;
    return status_of(cudaEventRecord(static_cast<cudaEvent_t>(event), static_cast<cudaStream_t>(stream)));
}
int rc_event_synchronize(void* event) {
    if (!event) return RC_ERR_INVALID_ARGUMENT;
    return status_of(cudaEventSynchronize(static_cast<cudaEvent_t>(event)));
}
int rc_event_destroy(void* event) { return event ? status_of(cudaEventDestroy(static_cast<cudaEvent_t>(event))) : RC_SUCCESS; }

int rc_stream_create(void** stream) {
    if (!stream) return RC_ERR_INVALID_ARGUMENT;
    cudaStream_t s = nullptr;
    const int r = status_of(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    *stream = s;
    return r;
}
int rc_stream_destroy(void* stream) {
    return stream ? status_of(cudaStreamDestroy(static_cast<cudaStream_t>(stream))) : RC_SUCCESS;
}
int rc_stream_synchronize(void* stream) { return status_of(cudaStreamSynchronize(static_cast<cudaStream_t>(stream))); }

}  // extern "C"
