// SPD solve that allocates no device memory: rc_spd_solve_f64_noalloc.
//
// Some callers cannot let a library allocate device memory while they run: services
// whose device memory is reserved up front by their own pool allocator (a cudaMalloc
// from the library would fail or escape their accounting), and latency-bound loops in
// which cudaMalloc/cudaFree, which can synchronise the whole device, are not allowed.
// For them this entry point runs the same Cholesky factorisation and the same two
// triangular solves as rc_spd_solve_f64, on scratch that lives in one file-scope
// __device__ array instead of the library's cached workspaces.
//
// The array holds 9.19 MiB: the n x n copy of A (n <= 1024), the inverse of one
// diagonal block for the factorisation and of the eight diagonal blocks for the solves,
// and one 128 x nrhs tile (nrhs <= 64). Every GPU that loads this library keeps it until
// the process exits. Larger problems are rejected with RC_ERR_SIZE_LIMIT.
#include <mutex>

#include "assign.cuh"
#include "factor.cuh"
#include "gemm.cuh"

namespace rc {
namespace {

constexpr int64_t kMaxN = 1024, kMaxRhs = 64;
constexpr int64_t kNblkMax = kMaxN / kNB;
constexpr size_t kCopyElems = (size_t)kMaxN * kMaxN;
constexpr size_t kDiagElems = (size_t)kNB * kNB;
constexpr size_t kTrsmElems = (size_t)kNblkMax * kNB * kNB;
constexpr size_t kTileElems = (size_t)kNB * kMaxRhs;
constexpr size_t kScratchElems = kCopyElems + kDiagElems + kTrsmElems + kTileElems;

// Shared by every call on a device; the contents of the previous call stay in it. Every
// region is fully written before it is read, so nothing needs clearing between calls.
// Calls whose work overlaps on the GPU (two streams, or two host threads) race on it.
static __device__ __align__(256) double g_noalloc_scratch[kScratchElems];

std::mutex g_mutex;
double* g_scratch_ptr[64] = {};

// Device address of the array for the current device: looked up with
// cudaGetSymbolAddress on the first call on each device (host code only sees a host-side
// stand-in under the array's name).
double* scratch_address() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        g_scratch_ptr[dev] = static_cast<double*>(p);
    }
    return g_scratch_ptr[dev];
}

// B <- L^-1 B (upper = false) or L^-T B (upper = true) with the diagonal-block inverses
// already in Winv (column-major blocks); the same block loop as the allocating solve.
int solve_with_inverses(bool upper, int64_t n, int64_t nrhs, View<const double> L, const double* Winv,
                        View<double> B, double* tile, cudaStream_t s, const int* abort) {
    const int64_t nblk = (n + kNB - 1) / kNB;
    const View<const double> A = upper ? L.t() : L;  // the triangle being solved with
    const View<double> Tv = colmajor(tile, (int64_t)kNB);
    for (int64_t step = 0; step < nblk; ++step) {
        const int64_t b = upper ? nblk - 1 - step : step;
        const int64_t r0 = b * kNB, sz = (n - r0 < kNB) ? n - r0 : kNB;
        const View<const double> X = {Winv + (size_t)b * kNB * kNB, 1, kNB};
        View<double> Bb = B.sub(r0, 0);
        const View<const double> Bc = {Bb.p, Bb.rs, Bb.cs};
        RC_TRY(gemm<double>(sz, nrhs, sz, 1.0, upper ? X.t() : X, Bc, 0.0, Tv, kFull, 0, s, abort));
        RC_TRY(copy2d<double, double>(sz, nrhs, 1.0, View<const double>{Tv.p, Tv.rs, Tv.cs}, Bb, s, abort));
        if (!upper && r0 + sz < n)
            RC_TRY(gemm<double>(n - r0 - sz, nrhs, sz, -1.0, A.sub(r0 + sz, r0), Bc, 1.0, B.sub(r0 + sz, 0), kFull, 0,
                                s, abort));
        if (upper && r0 > 0) RC_TRY(gemm<double>(r0, nrhs, sz, -1.0, A.sub(0, r0), Bc, 1.0, B, kFull, 0, s, abort));
    }
    return RC_SUCCESS;
}

}  // namespace
}  // namespace rc

extern "C" {

int rc_spd_solve_f64_noalloc(size_t n, size_t nrhs, const double* A, size_t lda, double* B, size_t ldb, int* d_info,
                             void* stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (!d_info) return RC_ERR_INVALID_ARGUMENT;
    if (n > (size_t)rc::kMaxN || nrhs > (size_t)rc::kMaxRhs) return RC_ERR_SIZE_LIMIT;
    if (n > 0 && (!A || lda < n || (nrhs > 0 && (!B || ldb < n)))) return RC_ERR_INVALID_ARGUMENT;
    double* base = rc::scratch_address();
    if (!base) return RC_ERR_CUDA;
    if (cudaMemsetAsync(d_info, 0, sizeof(int), s) != cudaSuccess) return RC_ERR_CUDA;
    if (n == 0) return RC_SUCCESS;
    double* L = base;
    double* Wdiag = L + rc::kCopyElems;
    double* Wtrsm = Wdiag + rc::kDiagElems;
    double* tile = Wtrsm + rc::kTrsmElems;
    const int64_t nn = (int64_t)n;
    const rc::View<double> Lv = rc::colmajor(L, nn);
    RC_TRY(rc::copy2d<double, double>(nn, nn, 1.0, rc::colmajor(A, (int64_t)lda), Lv, s));
    // Cholesky: per 128-column panel, the FP64 diagonal block (with its inverse), the
    // panel solve in place, the lower-masked trailing update.
    const rc::View<const double> Wt = {Wdiag, rc::kNB, 1};
    for (int64_t k0 = 0; k0 < nn; k0 += rc::kNB) {
        const int sz = (int)((nn - k0) < rc::kNB ? nn - k0 : rc::kNB);
        RC_TRY(rc::potrf_diag_block<double>(Lv.sub(k0, k0), sz, k0, Wdiag, false, d_info, s));
        const int64_t rows = nn - k0 - sz;
        if (rows <= 0) break;
        rc::View<double> P = Lv.sub(k0 + sz, k0);
        const rc::View<const double> Pc = {P.p, P.rs, P.cs};
        RC_TRY(rc::gemm<double>(rows, sz, sz, 1.0, Pc, Wt, 0.0, P, rc::kFull, 0, s, d_info));
        RC_TRY(rc::gemm<double>(rows, rows, sz, -1.0, Pc, Pc.t(), 1.0, Lv.sub(k0 + sz, k0 + sz), rc::kLower, 0, s,
                                d_info));
    }
    if (nrhs == 0) return RC_SUCCESS;
    const rc::View<const double> Lc = {L, 1, nn};
    const rc::View<double> Bv = rc::colmajor(B, (int64_t)ldb);
    // The inverses of L's diagonal blocks serve both solves (inv(L_bb^T) = inv(L_bb)^T).
    RC_TRY(rc::trtri_blocks_launch<double>(nn, Lc, false, Wtrsm, nullptr, d_info, s));
    RC_TRY(rc::solve_with_inverses(false, nn, (int64_t)nrhs, Lc, Wtrsm, Bv, tile, s, d_info));
    return rc::solve_with_inverses(true, nn, (int64_t)nrhs, Lc, Wtrsm, Bv, tile, s, d_info);
}

}  // extern "C"
