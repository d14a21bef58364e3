// LU with partial pivoting (getrf) and pivoted Cholesky (pstrf) on the GPU, in place on
// any strided view of the logical n x n matrix.
//
// getrf (kernels/getrf.hpp:50-59; CPU algorithm kernels/default/getrf.hpp:41-181):
// blocked right-looking LU with 64-column panels. One CTA factors a panel column by
// column -- pivot = the row of largest |A(i, j)| at or below the diagonal (the lowest
// row among equals, as the reference's strictly-larger scan), the swap of the two rows
// across the panel, the division of the column by the pivot (in double, as the
// reference), the rank-1 update of the panel -- then the panel's swaps are applied to
// the other columns in order, U12 = L11^-1 A12 (unit lower TRSM) and A22 -= L21 U12 (DMMA
// GEMM). piv[i] is the row swapped with row i at step i (LAPACK order, 0-based, as
// Remora's permutation_matrix). A zero pivot records its 1-based column in *info and
// stops every later kernel (the reference throws).
//
// pstrf (kernels/pstrf.hpp:62-70; CPU algorithm kernels/default/pstrf.hpp:40-147, the
// blocked pivoted Cholesky of LAWN 161): blocks of 32 columns. One CTA runs a block: the
// pivot values (the trailing diagonal, refreshed from the block's finished columns)
// choose the largest remaining pivot (the lowest index among equals, as std::max_element),
// rows and columns of the whole matrix are swapped, the factor stops with rank c when the
// pivot value is below n^2 eps max|A_ii| (the trailing square is cleared), else the
// column is finished by the dot products with the block's earlier columns and a division,
// and the row right of the diagonal is cleared. After the block the whole trailing square
// (both triangles, which later swaps read) is updated by a DMMA GEMM with the block's
// columns. piv as for getrf (identity where no swap happened); the rank goes to *rank.
#include <cfloat>
#include <cmath>

#include "factor.cuh"
#include "gemm.cuh"

namespace rc {
namespace {

constexpr int kLuNB = 64;       // getrf panel width
constexpr int kPsNB = 32;       // pstrf block width
constexpr int kLuThreads = 1024;

// Block-wide (value, index) reduction: larger value wins, the smaller index among equals.
__device__ __forceinline__ void argmax_pair(double& v, int64_t& i, double ov, int64_t oi) {
    if (ov > v || (ov == v && oi < i)) {
        v = ov;
        i = oi;
    }
}

__device__ void block_argmax(double& v, int64_t& i, double* sv, int64_t* si) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o; o >>= 1) argmax_pair(v, i, __shfl_xor_sync(0xffffffffu, v, o),
                                             __shfl_xor_sync(0xffffffffu, i, o));
    if (lane == 0) {
        sv[warp] = v;
        si[warp] = i;
    }
    __syncthreads();
    if (warp == 0) {
        v = lane < (int)(blockDim.x >> 5) ? sv[lane] : -DBL_MAX;
        i = lane < (int)(blockDim.x >> 5) ? si[lane] : INT64_MAX;
#pragma unroll
        for (int o = 16; o; o >>= 1) argmax_pair(v, i, __shfl_xor_sync(0xffffffffu, v, o),
                                                 __shfl_xor_sync(0xffffffffu, i, o));
        if (lane == 0) {
            sv[0] = v;
            si[0] = i;
        }
    }
    __syncthreads();
    v = sv[0];
    i = si[0];
    __syncthreads();
}

template <class T>
__global__ void __launch_bounds__(kLuThreads) getrf_panel_kernel(int64_t n, View<T> A, int64_t k0, int nb, int* piv,
                                                                 int* info) {
    __shared__ double sv[32];
    __shared__ int64_t si[32];
    if (*(volatile int*)info != 0) return;
    for (int j = 0; j < nb; ++j) {
        const int64_t c = k0 + j;
        double best = -1.0;
        int64_t bi = INT64_MAX;
        for (int64_t i = c + threadIdx.x; i < n; i += blockDim.x) {
            const double a = fabs((double)A(i, c));
            if (a > best) {
                best = a;
                bi = i;
            }
        }
        block_argmax(best, bi, sv, si);
        const int64_t p = bi;
        const double pv = (double)A(p, c);
        if (pv == 0.0) {  // also all-zero columns: the first row is the pivot, value 0
            if (threadIdx.x == 0) {
                piv[c] = (int)c;
                record_first(info, (int)(c + 1));
            }
            return;
        }
        if (threadIdx.x == 0) piv[c] = (int)p;
        if (p != c)
            for (int col = threadIdx.x; col < nb; col += blockDim.x) {
                const T t = A(c, k0 + col);
                A(c, k0 + col) = A(p, k0 + col);
                A(p, k0 + col) = t;
            }
        __syncthreads();
        for (int64_t i = c + 1 + threadIdx.x; i < n; i += blockDim.x) A(i, c) = (T)((double)A(i, c) / pv);
        __syncthreads();
        const int64_t rows = n - c - 1, cols = nb - j - 1;
        for (int64_t e = threadIdx.x; e < rows * cols; e += blockDim.x) {
            const int64_t i = c + 1 + e % rows, col = c + 1 + e / rows;
            A(i, col) -= A(i, c) * A(c, col);
        }
        __syncthreads();
    }
}

// The same panel factorisation spread over a cooperative grid: CTA b holds rows
// [k0 + b chunk, k0 + (b + 1) chunk) of the panel in shared memory (row stride nb + 1), and
// one bounded grid barrier per column exchanges what the next column needs. For column j
// (c = k0 + j), after the barrier every CTA reduces the published candidates in the same
// order (so all agree on the pivot p) and reads p's row; the owners of rows c and p swap
// them; then, with a look-ahead of one column:
//   1. every row below c is divided by the pivot and only its column j + 1 is updated;
//   2. the CTA's candidate for column j + 1 (largest |A(i, c + 1)|, i > c, the lowest row
//      among equals) and row c + 1 are updated in full and published;
//   3. the CTA arrives at the barrier, applies the rest of the rank-1 update to its other
//      rows while the others arrive, and waits.
// Each element sees exactly the operations of getrf_panel_kernel, in the same order.
constexpr int kCoopThreads = 256;
constexpr int kCoopMaxChunk = 384;  // rows per CTA (shared memory: 384 x 65 doubles)

struct CoopScratch {  // indexed by column j; the barrier words live separately
    double* cand_v;   // [nb][G]
    int64_t* cand_i;  // [nb][G]
    double* cand_row; // [nb][G][nb]
    double* crow;     // [nb][nb]: row c before the swap
};

// Grid barrier over nblocks co-resident CTAs (a cooperative launch), split into an arrival
// and a wait so that work can run in between: bar[0] counts arrivals, bar[1] is the
// generation. The wait is bounded by the SM's cycle counter (2 cycles per ns of the
// library's wait limit); a timeout records RC_ERR_TIMEOUT in the error word and the caller
// leaves.
__device__ void grid_arrive(unsigned* bar, unsigned nblocks, unsigned gen) {
    __syncthreads();  // every thread's stores before the arrival
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&bar[0], 1u) == nblocks - 1) {
            atomicExch(&bar[0], 0u);
            __threadfence();
            atomicExch(&bar[1], gen + 1u);
        }
    }
}
__device__ bool grid_wait(unsigned* bar, unsigned& gen, uint64_t limit_ns, int* err, int* pass) {
    if (threadIdx.x == 0) {
        int ok = 1;
        const long long t0 = clock64(), lim = (long long)(limit_ns * 2u);
        while (*(volatile unsigned*)&bar[1] == gen) {
            if (clock64() - t0 > lim) {
                ok = 0;
                if (err && atomicCAS(err, 0, RC_ERR_TIMEOUT) == 0) atomicExch(err + 1, 500);
                break;
            }
            __nanosleep(32);
        }
        __threadfence();
        *pass = ok;
    }
    __syncthreads();
    ++gen;
    return *pass != 0;
}

template <class T>
__global__ void __launch_bounds__(kCoopThreads, 1)
    getrf_panel_coop_kernel(int64_t n, View<T> A, int64_t k0, int nb, int chunk, int* piv, int* info,
                            CoopScratch sc, unsigned* bar, int* err, uint64_t limit_ns, T* linv) {
    extern __shared__ unsigned char coop_smem[];
    T* P = reinterpret_cast<T*>(coop_smem);  // chunk x (nb + 1)
    double* prow = reinterpret_cast<double*>(coop_smem) + ((size_t)chunk * (nb + 1) * sizeof(T) + 7) / 8;  // nb
    double* sv = prow + kLuNB;                                // 32
    int64_t* si = reinterpret_cast<int64_t*>(sv + 32);        // 32
    int* pass = reinterpret_cast<int*>(si + 32);
    const int ld = nb + 1, G = (int)gridDim.x, b = (int)blockIdx.x;
    if (*(volatile int*)info != 0) return;
    const int64_t base = k0 + (int64_t)b * chunk;
    const int myrows = (int)(n - base < chunk ? (n - base > 0 ? n - base : 0) : chunk);
    for (int e = threadIdx.x; e < myrows * nb; e += kCoopThreads) {
        const int r = e / nb, col = e % nb;
        P[r * ld + col] = A(base + r, k0 + col);
    }
    __syncthreads();
    // Publish the candidate for column j (rows >= k0 + j) and row k0 + j; both fully updated.
    auto publish = [&](int j, double best, int64_t bi) {
        const int64_t c = k0 + j;
        if (threadIdx.x == 0) {
            sc.cand_v[(size_t)j * G + b] = best;
            sc.cand_i[(size_t)j * G + b] = bi;
        }
        if (bi != INT64_MAX) {
            double* dst = sc.cand_row + ((size_t)j * G + b) * nb;
            for (int col = threadIdx.x; col < nb; col += kCoopThreads) dst[col] = (double)P[(bi - base) * ld + col];
        }
        if (c >= base && c < base + myrows)
            for (int col = threadIdx.x; col < nb; col += kCoopThreads)
                sc.crow[(size_t)j * nb + col] = (double)P[(c - base) * ld + col];
    };
    auto local_argmax = [&](int j, double& best, int64_t& bi) {
        const int64_t c = k0 + j;
        best = -1.0;
        bi = INT64_MAX;
        for (int r = threadIdx.x; r < myrows; r += kCoopThreads) {
            const int64_t i = base + r;
            if (i < c) continue;
            const double a = fabs((double)P[r * ld + j]);
            if (a > best || (a == best && i < bi)) {
                best = a;
                bi = i;
            }
        }
        block_argmax(best, bi, sv, si);
    };
    unsigned gen = 0;
    {  // column 0 needs no update first
        double best;
        int64_t bi;
        local_argmax(0, best, bi);
        publish(0, best, bi);
        grid_arrive(bar, (unsigned)G, gen);
        if (!grid_wait(bar, gen, limit_ns, err, pass)) return;
    }
    for (int j = 0; j < nb; ++j) {
        const int64_t c = k0 + j;
        // The pivot: every CTA reduces the G candidates in the same order.
        double best = -1.0;
        int64_t bi = INT64_MAX;
        for (int q = threadIdx.x; q < G; q += kCoopThreads) {
            const double v = __ldcg(sc.cand_v + (size_t)j * G + q);
            const int64_t i = __ldcg(sc.cand_i + (size_t)j * G + q);
            if (v > best || (v == best && i < bi)) {
                best = v;
                bi = i;
            }
        }
        block_argmax(best, bi, sv, si);
        const int64_t p = bi;
        const int owner = (int)((p - k0) / chunk);
        const double* pr = sc.cand_row + ((size_t)j * G + owner) * nb;
        for (int col = threadIdx.x; col < nb; col += kCoopThreads) prow[col] = __ldcg(pr + col);
        __syncthreads();
        const double pv = prow[j];
        if (pv == 0.0) {  // also all-zero columns: the first row is the pivot, value 0
            if (b == 0 && threadIdx.x == 0) {
                piv[c] = (int)c;
                record_first(info, (int)(c + 1));
            }
            return;
        }
        if (b == 0 && threadIdx.x == 0) piv[c] = (int)p;
        if (p != c) {
            if (c >= base && c < base + myrows)
                for (int col = threadIdx.x; col < nb; col += kCoopThreads) P[(c - base) * ld + col] = (T)prow[col];
            if (p >= base && p < base + myrows)
                for (int col = threadIdx.x; col < nb; col += kCoopThreads)
                    P[(p - base) * ld + col] = (T)__ldcg(sc.crow + (size_t)j * nb + col);
        }
        __syncthreads();
        // 1. divide, and update column j + 1 only
        for (int r = threadIdx.x; r < myrows; r += kCoopThreads) {
            if (base + r <= c) continue;
            T* row = P + r * ld;
            const T l = (T)((double)row[j] / pv);
            row[j] = l;
            if (j + 1 < nb) row[j + 1] -= l * (T)prow[j + 1];
        }
        __syncthreads();
        if (j + 1 == nb) break;
        // 2. the candidate for column j + 1 and row c + 1, updated in full and published
        local_argmax(j + 1, best, bi);
        const int64_t rc1 = c + 1;
        const bool own_c1 = rc1 >= base && rc1 < base + myrows;
        const int ra = bi != INT64_MAX ? (int)(bi - base) : -1;
        const int rb = own_c1 ? (int)(rc1 - base) : -1;
        for (int col = j + 2 + threadIdx.x; col < nb; col += kCoopThreads) {
            if (ra >= 0) P[ra * ld + col] -= P[ra * ld + j] * (T)prow[col];
            if (rb >= 0 && rb != ra) P[rb * ld + col] -= P[rb * ld + j] * (T)prow[col];
        }
        __syncthreads();
        publish(j + 1, best, bi);
        grid_arrive(bar, (unsigned)G, gen);
        // 3. the rest of the rank-1 update while the other CTAs arrive
        for (int r = threadIdx.x; r < myrows; r += kCoopThreads) {
            if (base + r <= c || r == ra || r == rb) continue;
            T* row = P + r * ld;
            const T l = row[j];
            for (int col = j + 2; col < nb; ++col) row[col] -= l * (T)prow[col];
        }
        if (!grid_wait(bar, gen, limit_ns, err, pass)) return;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < myrows * nb; e += kCoopThreads) {
        const int r = e / nb, col = e % nb;
        A(base + r, k0 + col) = P[r * ld + col];
    }
    if (b != 0) return;
    // CTA 0 holds L11 (rows k0 .. k0 + nb, unit lower): its inverse, in place over L11 in
    // shared memory, column by column from the last (X L = I gives, for q > j,
    // X(q, j) = -(L(q, j) + sum_{j < m < q} X(q, m) L(m, j)), columns m > j already final),
    // then to linv (row-major nb x nb) for the TRSM of the rows right of the panel.
    __syncthreads();
    for (int j = nb - 2; j >= 0; --j) {
        const int q = j + 1 + threadIdx.x;
        T v = 0;
        if (q < nb) {
            v = P[q * ld + j];
            for (int m = j + 1; m < q; ++m) v += P[q * ld + m] * P[m * ld + j];
        }
        __syncthreads();
        if (q < nb) P[q * ld + j] = -v;
        __syncthreads();
    }
    for (int e = threadIdx.x; e < nb * nb; e += kCoopThreads) {
        const int q = e / nb, m = e % nb;
        linv[e] = q > m ? P[q * ld + m] : (q == m ? T(1) : T(0));
    }
}

// The row swaps piv[k0 .. k0 + nb) in order, on the columns outside the panel.
template <class T>
__global__ void lu_swap_kernel(int64_t n, View<T> A, int64_t k0, int nb, const int* piv, const int* info) {
    if (*(volatile const int*)info != 0) return;
    for (int64_t col = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; col < n - nb;
         col += (int64_t)gridDim.x * blockDim.x) {
        const int64_t cc = col < k0 ? col : col + nb;
        for (int j = 0; j < nb; ++j) {
            const int64_t r = k0 + j, p = piv[r];
            if (p != r) {
                const T t = A(r, cc);
                A(r, cc) = A(p, cc);
                A(p, cc) = t;
            }
        }
    }
}

// eps = n^2 epsilon(T) max(A(0, 0), max_i |A(i, i)|); piv = identity; rank = n; stop = 0.
template <class T>
__global__ void pstrf_init_kernel(int64_t n, View<const T> A, double* eps, int* piv, int* rank, int* stop) {
    __shared__ double sv[32];
    __shared__ int64_t si[32];
    double mx = -DBL_MAX;
    int64_t dummy = 0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        mx = fmax(mx, i == 0 ? (double)A(0, 0) : fabs((double)A(i, i)));
        piv[i] = (int)i;
    }
    block_argmax(mx, dummy, sv, si);
    if (threadIdx.x == 0) {
        const double e = sizeof(T) == 8 ? DBL_EPSILON : (double)FLT_EPSILON;
        *eps = (double)(n * n) * e * mx;
        *rank = (int)n;
        *stop = 0;
    }
}

template <class T>
__global__ void __launch_bounds__(kLuThreads) pstrf_block_kernel(int64_t n, View<T> A, int64_t k, int cur, T* pv,
                                                                 const double* eps, int* piv, int* rank,
                                                                 int* stop) {
    __shared__ double sv[32];
    __shared__ int64_t si[32];
    if (*(volatile int*)stop != 0) return;
    const double epsv = *eps;
    for (int j = 0; j < cur; ++j) {
        const int64_t c = k + j;
        for (int64_t i = c + threadIdx.x; i < n; i += blockDim.x) {
            if (j == 0) pv[i] = A(i, i);
            else pv[i] -= A(i, c - 1) * A(i, c - 1);
        }
        __syncthreads();
        double best = -DBL_MAX;
        int64_t bi = INT64_MAX;
        for (int64_t i = c + threadIdx.x; i < n; i += blockDim.x)
            if ((double)pv[i] > best) {
                best = (double)pv[i];
                bi = i;
            }
        block_argmax(best, bi, sv, si);
        const int64_t p = bi;
        if (p != c) {
            if (threadIdx.x == 0) piv[c] = (int)p;
            for (int64_t t = threadIdx.x; t < n; t += blockDim.x) {
                const T x = A(c, t);
                A(c, t) = A(p, t);
                A(p, t) = x;
            }
            __syncthreads();
            for (int64_t t = threadIdx.x; t < n; t += blockDim.x) {
                const T x = A(t, c);
                A(t, c) = A(t, p);
                A(t, p) = x;
            }
            if (threadIdx.x == 0) {
                const T x = pv[c];
                pv[c] = pv[p];
                pv[p] = x;
            }
            __syncthreads();
        }
        const T v = pv[c];
        if ((double)v < epsv) {
            const int64_t m = n - c;
            for (int64_t e = threadIdx.x; e < m * m; e += blockDim.x) A(c + e % m, c + e / m) = T(0);
            if (threadIdx.x == 0) {
                *rank = (int)c;
                *stop = 1;
            }
            return;
        }
        const T d = sqrt(v);
        // Row c's block columns in shared memory; each row's block entries loaded 8 at a time
        // (independent loads in flight), the dot product accumulated in the same order.
        __shared__ T rowc[kPsNB];
        if (threadIdx.x < j) rowc[threadIdx.x] = A(c, k + threadIdx.x);
        __syncthreads();
        for (int64_t i = c + 1 + threadIdx.x; i < n; i += blockDim.x) {
            T s = A(i, c);
            for (int t0 = 0; t0 < j; t0 += 8) {
                T a[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) a[u] = t0 + u < j ? A(i, k + t0 + u) : T(0);
#pragma unroll
                for (int u = 0; u < 8; ++u)
                    if (t0 + u < j) s -= a[u] * rowc[t0 + u];
            }
            A(i, c) = s / d;
        }
        __syncthreads();
        if (threadIdx.x == 0) A(c, c) = d;
        for (int64_t t = c + 1 + threadIdx.x; t < n; t += blockDim.x) A(c, t) = T(0);
        __syncthreads();
    }
}

template <class T>
View<T> view_of(int row_major, T* A, int64_t lda) {
    return row_major ? View<T>{A, lda, 1} : View<T>{A, 1, lda};
}

// The panel on a cooperative grid of about 256 rows per CTA (a grid barrier costs more the
// more CTAs meet at it, the column work per CTA grows with its rows), at most one CTA per
// SM; on one CTA when the panel's rows do not fit the grid's shared memory (n above ~56K).
constexpr int kCoopRows = 256;
// linv (device, nb x nb): receives inv(L11) when the cooperative form ran (*have_inv).
template <class T>
int getrf_panel(int64_t n, View<T> A, int64_t k0, int nb, int* piv, int* info, T* linv, bool* have_inv,
                cudaStream_t s) {
    *have_inv = false;
    const int64_t rows = n - k0;
    const int sms = sm_count();
    int G = (int)((rows + kCoopRows - 1) / kCoopRows);
    if (G > sms) G = sms;
    const int chunk = (int)((rows + G - 1) / G);
    if (chunk > kCoopMaxChunk || sms <= 0) {
        getrf_panel_kernel<T><<<1, kLuThreads, 0, s>>>(n, A, k0, nb, piv, info);
        return check_launch();
    }
    const size_t panel_bytes = ((size_t)chunk * (nb + 1) * sizeof(T) + 7) / 8 * 8;
    const size_t smem = panel_bytes + (kLuNB + 32) * sizeof(double) + 32 * sizeof(int64_t) + 16;
    const size_t n_cand = (size_t)kLuNB * sms;
    const size_t bytes = 256 + n_cand * (sizeof(double) + sizeof(int64_t)) + n_cand * kLuNB * sizeof(double) +
                         (size_t)kLuNB * kLuNB * sizeof(double);
    char* ws = static_cast<char*>(workspace(s, bytes, 14));
    if (!ws) return RC_ERR_ALLOC;
    unsigned* bar = reinterpret_cast<unsigned*>(ws);
    CoopScratch sc;
    sc.cand_v = reinterpret_cast<double*>(ws + 256);
    sc.cand_i = reinterpret_cast<int64_t*>(sc.cand_v + n_cand);
    sc.cand_row = reinterpret_cast<double*>(sc.cand_i + n_cand);
    sc.crow = sc.cand_row + n_cand * kLuNB;
    if (cudaMemsetAsync(bar, 0, 2 * sizeof(unsigned), s) != cudaSuccess) return RC_ERR_CUDA;
    if (cudaFuncSetAttribute(getrf_panel_coop_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
        return RC_ERR_CUDA;
    int* err = error_word();
    uint64_t lim = wait_limit_ns();
    void* args[] = {&n, &A, &k0, &nb, const_cast<int*>(&chunk), &piv, &info, &sc, &bar, &err, &lim, &linv};
    if (cudaLaunchCooperativeKernel((const void*)getrf_panel_coop_kernel<T>, dim3((unsigned)G), dim3(kCoopThreads),
                                    args, smem, s) != cudaSuccess) {
        cudaGetLastError();
        return RC_ERR_CUDA;
    }
    count_launch();
    *have_inv = true;
    return RC_SUCCESS;
}

template <class T>
int getrf(int row_major, int64_t n, T* Ap, int64_t lda, int* piv, int* info, cudaStream_t s) {
    if (cudaMemsetAsync(info, 0, sizeof(int), s) != cudaSuccess) return RC_ERR_CUDA;
    const View<T> A = view_of(row_major, Ap, lda);
    T* linv = static_cast<T*>(workspace(s, (size_t)kLuNB * kLuNB * sizeof(T), 16));
    if (!linv) return RC_ERR_ALLOC;
    for (int64_t k0 = 0; k0 < n; k0 += kLuNB) {
        const int nb = (int)(n - k0 < kLuNB ? n - k0 : kLuNB);
        bool have_inv = false;
        RC_TRY(getrf_panel<T>(n, A, k0, nb, piv, info, linv, &have_inv, s));
        if (n > nb) {
            const int64_t cols = n - nb;
            lu_swap_kernel<T><<<ceil_div(cols, 256) < 1024u ? ceil_div(cols, 256) : 1024u, 256, 0, s>>>(n, A, k0, nb,
                                                                                                      piv, info);
            RC_TRY(check_launch());
        }
        const int64_t r = n - k0 - nb;
        if (r <= 0) continue;
        if (have_inv) {  // U12 = inv(L11) A12, in place (the GEMM's single row tile reads all of A12's k range first)
            const View<T> A12 = A.sub(k0, k0 + nb);
            RC_TRY(gemm<T>(nb, r, nb, T(1), View<const T>{linv, kLuNB, 1}, View<const T>{A12.p, A12.rs, A12.cs},
                           T(0), A12, kFull, 0, s, info));
        } else {
            const View<const T> L11{A.sub(k0, k0).p, A.rs, A.cs};
            RC_TRY(trsm_left<T>(false, true, nb, r, T(1), L11, A.sub(k0, k0 + nb), nullptr, s, info));
        }
        const View<const T> L21{A.sub(k0 + nb, k0).p, A.rs, A.cs}, U12{A.sub(k0, k0 + nb).p, A.rs, A.cs};
        RC_TRY(gemm<T>(r, r, nb, T(-1), L21, U12, T(1), A.sub(k0 + nb, k0 + nb), kFull, 0, s, info));
    }
    return RC_SUCCESS;
}

template <class T>
int pstrf(int row_major, int64_t n, T* Ap, int64_t lda, int* piv, int* rank, cudaStream_t s) {
    const size_t bytes = ((size_t)n * sizeof(T) + 255) / 256 * 256 + 256;
    char* ws = static_cast<char*>(workspace(s, bytes, 12));
    if (!ws) return RC_ERR_ALLOC;
    T* pv = reinterpret_cast<T*>(ws);
    double* eps = reinterpret_cast<double*>(ws + bytes - 256);
    int* stop = reinterpret_cast<int*>(ws + bytes - 128);
    const View<T> A = view_of(row_major, Ap, lda);
    pstrf_init_kernel<T><<<1, kLuThreads, 0, s>>>(n, View<const T>{A.p, A.rs, A.cs}, eps, piv, rank, stop);
    RC_TRY(check_launch());
    for (int64_t k = 0; k < n; k += kPsNB) {
        const int cur = (int)(n - k < kPsNB ? n - k : kPsNB);
        pstrf_block_kernel<T><<<1, kLuThreads, 0, s>>>(n, A, k, cur, pv, eps, piv, rank, stop);
        RC_TRY(check_launch());
        const int64_t r = n - k - cur;
        if (r <= 0) continue;
        const View<const T> L21{A.sub(k + cur, k).p, A.rs, A.cs};
        RC_TRY(gemm<T>(r, r, cur, T(-1), L21, L21.t(), T(1), A.sub(k + cur, k + cur), kFull, 0, s, stop));
    }
    return RC_SUCCESS;
}

}  // namespace
}  // namespace rc

extern "C" {

int rc_getrf_f64(int row_major, size_t n, double* A, size_t lda, int* piv, int* info, void* stream) {
    if (!info) return RC_ERR_INVALID_ARGUMENT;
    if (n == 0) return cudaMemsetAsync(info, 0, sizeof(int), static_cast<cudaStream_t>(stream)) == cudaSuccess
                           ? RC_SUCCESS
                           : RC_ERR_CUDA;
    if (!A || !piv || lda < n) return RC_ERR_INVALID_ARGUMENT;
    if (n > (size_t)INT32_MAX) return RC_ERR_NOT_SUPPORTED;
    return rc::getrf<double>(row_major, (int64_t)n, A, (int64_t)lda, piv, info, static_cast<cudaStream_t>(stream));
}

int rc_getrf_f32(int row_major, size_t n, float* A, size_t lda, int* piv, int* info, void* stream) {
    if (!info) return RC_ERR_INVALID_ARGUMENT;
    if (n == 0) return cudaMemsetAsync(info, 0, sizeof(int), static_cast<cudaStream_t>(stream)) == cudaSuccess
                           ? RC_SUCCESS
                           : RC_ERR_CUDA;
    if (!A || !piv || lda < n) return RC_ERR_INVALID_ARGUMENT;
    if (n > (size_t)INT32_MAX) return RC_ERR_NOT_SUPPORTED;
    return rc::getrf<float>(row_major, (int64_t)n, A, (int64_t)lda, piv, info, static_cast<cudaStream_t>(stream));
}

int rc_pstrf_f64(int row_major, size_t n, double* A, size_t lda, int* piv, int* rank, void* stream) {
    if (!rank) return RC_ERR_INVALID_ARGUMENT;
    if (n == 0) return cudaMemsetAsync(rank, 0, sizeof(int), static_cast<cudaStream_t>(stream)) == cudaSuccess
                           ? RC_SUCCESS
                           : RC_ERR_CUDA;
    if (!A || !piv || lda < n) return RC_ERR_INVALID_ARGUMENT;
    if (n > (size_t)INT32_MAX) return RC_ERR_NOT_SUPPORTED;
    return rc::pstrf<double>(row_major, (int64_t)n, A, (int64_t)lda, piv, rank, static_cast<cudaStream_t>(stream));
}

int rc_pstrf_f32(int row_major, size_t n, float* A, size_t lda, int* piv, int* rank, void* stream) {
    if (!rank) return RC_ERR_INVALID_ARGUMENT;
    if (n == 0) return cudaMemsetAsync(rank, 0, sizeof(int), static_cast<cudaStream_t>(stream)) == cudaSuccess
                           ? RC_SUCCESS
                           : RC_ERR_CUDA;
    if (!A || !piv || lda < n) return RC_ERR_INVALID_ARGUMENT;
    if (n > (size_t)INT32_MAX) return RC_ERR_NOT_SUPPORTED;
    return rc::pstrf<float>(row_major, (int64_t)n, A, (int64_t)lda, piv, rank, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
