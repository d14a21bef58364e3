// Batched uneven SPD solves: POTRF + the two triangular solves of many independent
// small systems (n <= 512) in ONE persistent launch, replayed as a CUDA graph.
//
// Extension on top of the reference's per-system path (cholesky_decomposition + solve,
// include/remora/decompositions.hpp:81-115; no batched counterpart exists there).
//
// Design:
//  * persistent CTAs (a multiple of the SM count) pull systems from an atomic work
//    counter over an order sorted by decreasing n, so the large systems start first and
//    the small ones fill the tail -- no inter-CTA waiting, only one atomicAdd per system;
//  * per system, a right-looking Cholesky in NB-column steps: the NB x NB diagonal block
//    is factored in shared memory (one element per thread-slot, one barrier per column),
//    the panel below is solved row-parallel against it and kept in shared memory, and the
//    trailing lower triangle is updated in 4 x 4 register tiles read from that panel;
//  * then the forward and backward substitutions for the right-hand side, in shared
//    memory;
//  * a failing pivot records its 1-based index in info[i] and the CTA moves on.
// The tile configuration (NB, threads) is chosen per (precision, size bucket) by a small
// autotuner that times every candidate on the caller's batch once and caches the winner.
#include <algorithm>
#include <map>
#include <memory>
#include <tuple>
#include <mutex>
#include <numeric>
#include <vector>

#include "common.cuh"

namespace rc {
namespace {

constexpr int kMaxN = 512;

template <class T, int NB>
struct BatchedSmem {
    static constexpr int LD = NB + 1;
    static constexpr size_t bytes = (size_t)(NB * LD + kMaxN * LD + kMaxN) * sizeof(T);
};

template <class T, int NB, int THREADS>
__global__ void __launch_bounds__(THREADS) batched_chol_solve(int count, const int* __restrict__ order,
                                                             const int* __restrict__ sizes, T* const* __restrict__ Aptr,
                                                             T* const* __restrict__ bptr, int* __restrict__ info,
                                                             int* __restrict__ next) {
    constexpr int LD = NB + 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* D = reinterpret_cast<T*>(smem_raw);  // NB x LD diagonal block, row-major
    T* P = D + NB * LD;                      // up to kMaxN x LD panel rows, row-major
    T* x = P + kMaxN * LD;                   // right-hand side / solution
    __shared__ int s_work, s_fail;
    const int tid = threadIdx.x;
    while (true) {
        __syncthreads();
        if (tid == 0) s_work = atomicAdd(next, 1);
        __syncthreads();
        const int w = s_work;
        if (w >= count) break;
        const int sys = order[w];
        const int n = sizes[sys];
        T* A = Aptr[sys];  // column-major, ld = n
        T* b = bptr[sys];
        if (tid == 0) s_fail = 0;
        for (int r = tid; r < n; r += THREADS) x[r] = b[r];
        __syncthreads();
        for (int k = 0; k < n; k += NB) {
            const int kb = min(NB, n - k);
            // 1. diagonal block into shared memory (lower part)
            for (int e = tid; e < kb * kb; e += THREADS) {
                const int r = e % kb, c = e / kb;
                D[r * LD + c] = c <= r ? A[(k + r) + (size_t)(k + c) * n] : T(0);
            }
            __syncthreads();
            // 2. factor it: per column, the pivot, the column scaling, the rank-1 update
            for (int j = 0; j < kb; ++j) {
                const T d = D[j * LD + j];
                if (!(d > T(0))) {
                    if (tid == 0) s_fail = k + j + 1;
                    break;  // uniform: every thread read the same d
                }
                const T sq = sqrt(d);
                __syncthreads();
                for (int r = j + tid; r < kb; r += THREADS) D[r * LD + j] = r == j ? sq : D[r * LD + j] / sq;
                __syncthreads();
                const int t = kb - j - 1;
                for (int e = tid; e < t * t; e += THREADS) {
                    const int r = j + 1 + e / t, c = j + 1 + e % t;
                    if (c <= r) D[r * LD + c] -= D[r * LD + j] * D[c * LD + j];
                }
                __syncthreads();
            }
            __syncthreads();
            if (s_fail) break;
            for (int e = tid; e < kb * kb; e += THREADS) {
                const int r = e % kb, c = e / kb;
                if (c <= r) A[(k + r) + (size_t)(k + c) * n] = D[r * LD + c];
            }
            // 3. panel rows below: solve x L_kk^T = a row by row (forward substitution)
            const int m = n - k - kb;
            for (int r = tid; r < m; r += THREADS) {
                T* pr = P + r * LD;
                for (int c = 0; c < kb; ++c) {
                    T v = A[(k + kb + r) + (size_t)(k + c) * n];
                    for (int q = 0; q < c; ++q) v -= pr[q] * D[c * LD + q];
                    pr[c] = v / D[c * LD + c];
                }
                for (int c = 0; c < kb; ++c) A[(k + kb + r) + (size_t)(k + c) * n] = pr[c];
            }
            __syncthreads();
            // 4. trailing update of the lower triangle, 4 x 4 tiles
            const int tiles = (m + 3) / 4;
            const int ntile = tiles * (tiles + 1) / 2;
            for (int t = tid; t < ntile; t += THREADS) {
                // t -> (tr, tc) with tc <= tr, row-major over the lower triangle of tiles
                int tr = (int)((sqrtf(8.f * t + 1.f) - 1.f) * 0.5f);
                while ((tr + 1) * (tr + 2) / 2 <= t) ++tr;
                while (tr * (tr + 1) / 2 > t) --tr;
                const int tc = t - tr * (tr + 1) / 2;
                const int r0 = 4 * tr, c0 = 4 * tc;
                T acc[4][4] = {};
                for (int q = 0; q < kb; ++q) {
                    T pr[4], pc[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        pr[u] = r0 + u < m ? P[(r0 + u) * LD + q] : T(0);
                        pc[u] = c0 + u < m ? P[(c0 + u) * LD + q] : T(0);
                    }
#pragma unroll
                    for (int u = 0; u < 4; ++u)
#pragma unroll
                        for (int v = 0; v < 4; ++v) acc[u][v] += pr[u] * pc[v];
                }
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    const int c = c0 + v;
                    if (c >= m) continue;
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int r = r0 + u;
                        if (r >= m || r < c) continue;
                        A[(k + kb + r) + (size_t)(k + kb + c) * n] -= acc[u][v];
                    }
                }
            }
            __syncthreads();
        }
        if (s_fail) {
            if (tid == 0) info[sys] = s_fail;
            continue;
        }
        // 5. L y = b, then L^T x = y (one barrier per column), x in shared memory
        for (int j = 0; j < n; ++j) {
            if (tid == 0) x[j] /= A[j + (size_t)j * n];
            __syncthreads();
            const T yj = x[j];
            for (int r = j + 1 + tid; r < n; r += THREADS) x[r] -= A[r + (size_t)j * n] * yj;
            __syncthreads();
        }
        for (int j = n - 1; j >= 0; --j) {
            // x_j = (y_j - sum_{r > j} L_rj x_r) / L_jj: a block reduction per column
            T part = T(0);
            for (int r = j + 1 + tid; r < n; r += THREADS) part += A[r + (size_t)j * n] * x[r];
            for (int off = 16; off > 0; off >>= 1) part += __shfl_down_sync(0xffffffffu, part, off);
            __shared__ T red[32];
            if ((tid & 31) == 0) red[tid >> 5] = part;
            __syncthreads();
            if (tid == 0) {
                T s = T(0);
                for (int q = 0; q < THREADS / 32; ++q) s += red[q];
                x[j] = (x[j] - s) / A[j + (size_t)j * n];
            }
            __syncthreads();
        }
        for (int r = tid; r < n; r += THREADS) b[r] = x[r];
        if (tid == 0) info[sys] = 0;
    }
}

struct Config {
    int nb, threads;
};

template <class T>
using KernelFn = void (*)(int, const int*, const int*, T* const*, T* const*, int*, int*);

template <class T>
KernelFn<T> kernel_for(Config c, size_t* smem) {
    if (c.nb == 32 && c.threads == 256) {
        *smem = BatchedSmem<T, 32>::bytes;
        return batched_chol_solve<T, 32, 256>;
    }
    if (c.nb == 32 && c.threads == 128) {
        *smem = BatchedSmem<T, 32>::bytes;
        return batched_chol_solve<T, 32, 128>;
    }
    if (c.nb == 16 && c.threads == 256) {
        *smem = BatchedSmem<T, 16>::bytes;
        return batched_chol_solve<T, 16, 256>;
    }
    *smem = BatchedSmem<T, 16>::bytes;
    return batched_chol_solve<T, 16, 128>;
}

const Config kCandidates[] = {{32, 256}, {32, 128}, {16, 256}, {16, 128}};

// A plan: the device copy of sizes and order, the chosen configuration, the captured
// graph (work-counter reset + the persistent kernel) for one set of pointer arrays.
struct Plan {
    int dev = -1;
    int count = 0;
    const void* A = nullptr;
    const void* b = nullptr;
    const int* info = nullptr;
    std::vector<int> sizes;
    int* d_buf = nullptr;  // [next | order (count) | sizes (count)]
    Config cfg{32, 256};
    cudaGraphExec_t exec = nullptr;
    ~Plan() {
        if (exec) cudaGraphExecDestroy(exec);
        if (d_buf) cudaFree(d_buf);
    }
};

std::mutex g_mutex;
// (device, element size, A pointer array, b pointer array, info, count) -> plan. The element
// size is part of the key: a plan's graph holds a kernel for one element type, and arrays of
// another type can come back at the same addresses.
std::map<std::tuple<int, int, const void*, const void*, const int*, int>, std::unique_ptr<Plan>> g_plans;
std::map<std::pair<int, int>, Config> g_tuned;  // (sizeof(T), bucket of the largest n) -> config

int size_bucket(const std::vector<int>& sizes) {
    const int mx = sizes.empty() ? 0 : *std::max_element(sizes.begin(), sizes.end());
    return mx <= 64 ? 0 : mx <= 128 ? 1 : mx <= 256 ? 2 : 3;
}

template <class T>
int launch_plain(const Plan& p, Config c, cudaStream_t s) {
    size_t smem = 0;
    auto fn = kernel_for<T>(c, &smem);
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return RC_ERR_CUDA;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, c.threads, smem) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    const int grid = std::min(sm_count() * per_sm, std::max(p.count, 1));
    if (cudaMemsetAsync(p.d_buf, 0, sizeof(int), s) != cudaSuccess) return RC_ERR_CUDA;
    fn<<<grid, c.threads, smem, s>>>(p.count, p.d_buf + 1, p.d_buf + 1 + p.count, (T* const*)p.A, (T* const*)p.b,
                                    const_cast<int*>(p.info), p.d_buf);
    return check_launch();
}

// Time each candidate once on the caller's batch (the factorisations happen in place, so
// the caller's matrices are first saved and restored around the tuning runs).
template <class T>
int autotune(Plan& p, cudaStream_t s) {
    const auto key = std::make_pair((int)sizeof(T), size_bucket(p.sizes));
    {
        auto it = g_tuned.find(key);
        if (it != g_tuned.end()) {
            p.cfg = it->second;
            return RC_SUCCESS;
        }
    }
    // Save the inputs: host copies of the pointer arrays give every system's storage.
    std::vector<T*> hA(p.count), hb(p.count);
    if (cudaMemcpy(hA.data(), p.A, p.count * sizeof(T*), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(hb.data(), p.b, p.count * sizeof(T*), cudaMemcpyDeviceToHost) != cudaSuccess)
        return RC_ERR_CUDA;
    size_t total = 0;
    for (int i = 0; i < p.count; ++i) total += (size_t)p.sizes[i] * p.sizes[i] + p.sizes[i];
    T* save = nullptr;
    if (cudaMalloc(&save, total * sizeof(T)) != cudaSuccess) return RC_ERR_ALLOC;
    note_allocation();
    auto copy_all = [&](bool to_save) {
        size_t off = 0;
        for (int i = 0; i < p.count; ++i) {
            const size_t nn = (size_t)p.sizes[i] * p.sizes[i], nb = p.sizes[i];
            if (to_save) {
                cudaMemcpyAsync(save + off, hA[i], nn * sizeof(T), cudaMemcpyDeviceToDevice, s);
                cudaMemcpyAsync(save + off + nn, hb[i], nb * sizeof(T), cudaMemcpyDeviceToDevice, s);
            } else {
                cudaMemcpyAsync(hA[i], save + off, nn * sizeof(T), cudaMemcpyDeviceToDevice, s);
                cudaMemcpyAsync(hb[i], save + off + nn, nb * sizeof(T), cudaMemcpyDeviceToDevice, s);
            }
            off += nn + nb;
        }
    };
    copy_all(true);
    float best = 1e30f;
    Config best_cfg = kCandidates[0];
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (const Config& c : kCandidates) {
        cudaEventRecord(e0, s);
        const int st = launch_plain<T>(p, c, s);
        cudaEventRecord(e1, s);
        copy_all(false);
        if (st != RC_SUCCESS) continue;
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) {
            best = ms;
            best_cfg = c;
        }
    }
    cudaStreamSynchronize(s);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(save);
    p.cfg = best_cfg;
    g_tuned[key] = best_cfg;
    return RC_SUCCESS;
}

template <class T>
int batched(size_t count, const int* h_n, T* const* d_A, T* const* d_b, int* d_info, int autotune_flag,
            cudaStream_t s) {
    if (count == 0) return RC_SUCCESS;
    if (!h_n || !d_A || !d_b || !d_info || count > (size_t)INT32_MAX) return RC_ERR_INVALID_ARGUMENT;
    for (size_t i = 0; i < count; ++i)
        if (h_n[i] < 1 || h_n[i] > kMaxN) return RC_ERR_NOT_SUPPORTED;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return RC_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_mutex);
    auto key = std::make_tuple(dev, (int)sizeof(T), (const void*)d_A, (const void*)d_b, (const int*)d_info, (int)count);
    std::unique_ptr<Plan>& slot = g_plans[key];
    std::vector<int> sizes(h_n, h_n + count);
    if (slot && slot->sizes != sizes) slot.reset();
    if (!slot) {
        auto p = std::make_unique<Plan>();
        p->dev = dev;
        p->count = (int)count;
        p->A = d_A;
        p->b = d_b;
        p->info = d_info;
        p->sizes = sizes;
        std::vector<int> order(count);
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return sizes[a] > sizes[b]; });
        std::vector<int> host(1 + 2 * count, 0);
        std::copy(order.begin(), order.end(), host.begin() + 1);
        std::copy(sizes.begin(), sizes.end(), host.begin() + 1 + count);
        if (cudaMalloc(&p->d_buf, host.size() * sizeof(int)) != cudaSuccess) return RC_ERR_ALLOC;
        note_allocation();
        if (cudaMemcpy(p->d_buf, host.data(), host.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
            return RC_ERR_CUDA;
        if (autotune_flag) RC_TRY(autotune<T>(*p, s));
        // Capture counter reset + kernel once; later calls replay the graph.
        cudaStream_t cs;
        if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) return RC_ERR_CUDA;
        cudaGraph_t g = nullptr;
        int st = cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed) == cudaSuccess ? RC_SUCCESS : RC_ERR_CUDA;
        if (st == RC_SUCCESS) st = launch_plain<T>(*p, p->cfg, cs);
        if (cudaStreamEndCapture(cs, &g) != cudaSuccess && st == RC_SUCCESS) st = RC_ERR_CUDA;
        cudaStreamDestroy(cs);
        if (st == RC_SUCCESS && cudaGraphInstantiate(&p->exec, g, 0) != cudaSuccess) st = RC_ERR_CUDA;
        if (g) cudaGraphDestroy(g);
        if (st != RC_SUCCESS) {
            cudaGetLastError();
            return st;
        }
        slot = std::move(p);
    }
    if (cudaGraphLaunch(slot->exec, s) != cudaSuccess) return RC_ERR_CUDA;
    count_launch();
    return RC_SUCCESS;
}

}  // namespace
}  // namespace rc

extern "C" {

int rc_potrf_trsm_batched_f64(size_t count, const int* h_n, double* const* d_A, double* const* d_b, int* d_info,
                              int autotune, void* stream) {
    return rc::batched<double>(count, h_n, d_A, d_b, d_info, autotune, static_cast<cudaStream_t>(stream));
}
int rc_potrf_trsm_batched_f32(size_t count, const int* h_n, float* const* d_A, float* const* d_b, int* d_info,
                              int autotune, void* stream) {
    return rc::batched<float>(count, h_n, d_A, d_b, d_info, autotune, static_cast<cudaStream_t>(stream));
}
int rc_batched_release_plans(void) {
    std::lock_guard<std::mutex> lock(rc::g_mutex);
    rc::g_plans.clear();
    return RC_SUCCESS;
}

}  // extern "C"
