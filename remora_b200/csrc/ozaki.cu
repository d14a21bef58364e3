// FP64 matrix products C = alpha A P + beta C on the int8 tensor cores (tcgen05.mma
// kind::i8, exact 32-bit integer accumulation), by error-free digit splitting: the
// splitting of Ozaki, Ogita, Oishi and Rump (Numer. Algorithms 2012) in the integer form
// of Ootomo, Ozaki and Yokota ("DGEMM on integer matrix multiplication unit", IJHPCA
// 2024).
//
//   A(i, j) = 2^e_i  sum_{t=1..8} a_t(i, j) 2^-7t  (+ r, |r| < 2^(e_i - 56))
//   P(j, c) = 2^f_c  sum_{u=1..8} b_u(j, c) 2^-7u  (+ r, |r| < 2^(f_c - 56))
//
// with 2^e_i above row i's largest |A(i, j)| and 2^f_c above column c's largest |P(j, c)|,
// and a_t, b_u signed 7-bit digits (int8). Then
//
//   (A P)(i, c) ~= 2^(e_i + f_c) sum_{d=2..9} 2^-7d  sum_{t+u=d} (a_t b_u)(i, c)
//
// where every a_t b_u is an exact int8 GEMM; pairs of weight 2^-70 and below are dropped.
// The 36 kept pairs fall into 8 accumulators (one per d) that live side by side in
// tensor memory (8 x 64 columns of 32-bit integers for 64 right-hand sides): one
// tcgen05.mma of A_t against [P_1 .. P_(9-t)] writes the accumulators d = t+1 .. 9 at
// once. The bound s * 127^2 * Kc < 2^31 on one accumulator caps a K chunk at 16384, so the
// K range is split over CTAs and their FP64 partials are summed in a fixed order.
//
// Data layout: the digits of A are stored once per left operand, K-major (row i of slice
// t at slices + (t * Mp + i) * ldk), in the 128B-swizzled tiles the TMA moves; the digits
// of P are rebuilt per product, K-major as well (row (u, c) of slice u, column c).
// Per CTA: warp 0 streams, per 128-wide K block, the 8 x 128-row slices of A through a
// 6-deep ring and the 8 x nr rows of P's digits through a 2-deep ring; warp 1 issues the
// MMAs; warps 2..5 combine the 8 integer accumulators of each row into one FP64 partial.
// Every mbarrier wait is bounded.
#include <climits>
#include <cudaTypedefs.h>

#include "gemm.cuh"
#include "ozaki.cuh"
#include "ozaki_digits.cuh"
#include "tc_common.cuh"
#include "tc_gemm.cuh"

namespace rc {
namespace {

using namespace tc;
constexpr int S = kOzSlices;
constexpr int OZ_THREADS = 192;
constexpr int A_STAGES = 6;  // 6 x 16 KB + 2 x 64 KB of P digits: the 227 KB limit
constexpr int A_TILE = 128 * 128;  // one 128-row x 128-byte slice tile
constexpr int KC_MAX = 16384;      // S * 127 * 127 * KC_MAX < 2^31
constexpr int kBadExp = kOzBadExp;

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
int64_t round_up(int64_t x, int64_t q) { return (x + q - 1) / q * q; }
int rhs_width(int64_t nrhs) { return nrhs > 32 ? 64 : (nrhs > 16 ? 32 : 16); }

// K chunking: the number of chunks z and their length (a multiple of 128, at most
// KC_MAX) that minimise (waves of one-CTA-per-SM tiles) x (chunk length + a fill cost).
void oz_split(int64_t Mp, int64_t k, int* z_out, int64_t* kc_out) {
    const int64_t tiles = Mp / 128, sms = sm_count();
    const int64_t zmin = (k + KC_MAX - 1) / KC_MAX;
    const int64_t zmax_k = (k + 127) / 128;
    int64_t best_z = zmin, best_kc = round_up((k + zmin - 1) / zmin, 128);
    double best = 1e300;
    for (int64_t z = zmin; z <= zmin + 7 && z <= zmax_k; ++z) {
        const int64_t kc = round_up((k + z - 1) / z, 128);
        if (kc > KC_MAX) continue;
        const int64_t zz = (k + kc - 1) / kc;  // chunks actually non-empty
        const double cost = (double)((tiles * zz + sms - 1) / sms) * (double)(kc + 512);
        if (cost < best) {
            best = cost;
            best_z = zz;
            best_kc = kc;
        }
    }
    *z_out = (int)best_z;
    *kc_out = best_kc;
}

// Symmetric scaling from the diagonal (SPD A): 2^e_i >= sqrt(A_ii), so that
// |A_ij| <= sqrt(A_ii A_jj) < 2^(e_i + e_j). flag is set for a diagonal entry that is not
// positive and finite.
__global__ void diag_exp_kernel(int64_t n, const double* A, int64_t lda, int64_t Mp, int* rexp, int* flag) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < Mp; i += (int64_t)gridDim.x * blockDim.x) {
        int e = 0;
        if (i < n) {
            const double d = A[i + i * lda];
            const int E = scale_exp((unsigned long long)__double_as_longlong(d));  // d < 2^E
            if (!(d > 0.0) || E == kBadExp) atomicOr(flag, 1);
            else e = (E + 1) >> 1;  // ceil(E / 2)
        }
        rexp[i] = e;
    }
}

// rowbits[i] = max over j of the bits of |A(i, j)| (IEEE order = value order; NaN above Inf).
__global__ void __launch_bounds__(256) row_absmax_kernel(int64_t m, int64_t k, const double* A, int64_t lda,
                                                         unsigned long long* rowbits) {
    const int64_t i = (int64_t)blockIdx.y * 256 + threadIdx.x;
    if (i >= m) return;
    const int64_t j0 = (int64_t)blockIdx.x * 512, j1 = j0 + 512 < k ? j0 + 512 : k;
    unsigned long long mx = 0;
    for (int64_t j = j0; j < j1; ++j) {
        const unsigned long long b = (unsigned long long)__double_as_longlong(A[i + j * lda]) & 0x7FFFFFFFFFFFFFFFull;
        mx = b > mx ? b : mx;
    }
    atomicMax(&rowbits[i], mx);
}

// Digits of a 32-row x 128-column tile of column-major A, written K-major (row i of
// slice t contiguous in j) through shared memory: reads walk i, writes walk j.
__global__ void __launch_bounds__(256) slice_a_kernel(int64_t m, int64_t k, const double* A, int64_t lda,
                                                      const unsigned long long* rowbits, int* rexp, int8_t* Sa,
                                                      int64_t Mp, int64_t ldk) {
    __shared__ uint32_t sm[S][32][33];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t i0 = (int64_t)blockIdx.y * 32, i = i0 + lane;
    const int64_t j0 = (int64_t)blockIdx.x * 128;
    const int e = i < m ? scale_exp(rowbits[i]) : 0;
    if (blockIdx.x == 0 && w == 0) rexp[i] = e;
    const bool live = i < m && e != kBadExp;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        uint32_t word[S] = {};
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int64_t j = j0 + w * 16 + q * 4 + c;
            const double x = (live && j < k) ? A[i + j * lda] : 0.0;
            digits(x, e, word, c);
        }
#pragma unroll
        for (int t = 0; t < S; ++t) sm[t][lane][w * 4 + q] = word[t];
    }
    __syncthreads();
    const int r = threadIdx.x >> 3, g = threadIdx.x & 7;
    const int64_t jw = j0 + g * 16;
    if (jw < ldk) {
#pragma unroll
        for (int t = 0; t < S; ++t) {
            const uint4 v = make_uint4(sm[t][r][4 * g], sm[t][r][4 * g + 1], sm[t][r][4 * g + 2], sm[t][r][4 * g + 3]);
            *reinterpret_cast<uint4*>(Sa + ((int64_t)t * Mp + i0 + r) * ldk + jw) = v;
        }
    }
}

// One block per column c < nr of P (k x nrhs): its scale exponent, then its digits,
// K-major: row (t * nr + c) of Ps holds digit t + 1 of column c. Columns c >= nrhs are 0.
// With pre (the diagonal scaling of A), the digits are those of 2^pre[j] P(j, c).
__global__ void __launch_bounds__(256) slice_p_kernel(int64_t k, int64_t nrhs, const double* P, int64_t ldp, int nr,
                                                      const int* pre, int* cexp, int8_t* Ps, int64_t ldk) {
    __shared__ unsigned long long red[8];
    const int c = blockIdx.x, lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    unsigned long long mx = 0;
    if (c < nrhs)
        for (int64_t j = threadIdx.x; j < k; j += 256) {
            const double x = pre ? ldexp(P[j + c * ldp], pre[j]) : P[j + c * ldp];
            const unsigned long long b = (unsigned long long)__double_as_longlong(x) & 0x7FFFFFFFFFFFFFFFull;
            mx = b > mx ? b : mx;
        }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        const unsigned long long y = __shfl_xor_sync(0xffffffffu, mx, o);
        mx = y > mx ? y : mx;
    }
    if (lane == 0) red[w] = mx;
    __syncthreads();
    mx = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) mx = red[q] > mx ? red[q] : mx;
    const int e = c < nrhs ? scale_exp(mx) : 0;
    if (threadIdx.x == 0) cexp[c] = e;
    const bool live = c < nrhs && e != kBadExp;
    for (int64_t j0 = 4 * (int64_t)threadIdx.x; j0 < ldk; j0 += 1024) {
        uint32_t word[S] = {};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int64_t j = j0 + q;
            const double x = (live && j < k) ? (pre ? ldexp(P[j + c * ldp], pre[j]) : P[j + c * ldp]) : 0.0;
            digits(x, e, word, q);
        }
#pragma unroll
        for (int t = 0; t < S; ++t) *reinterpret_cast<uint32_t*>(Ps + ((int64_t)t * nr + c) * ldk + j0) = word[t];
    }
}

__device__ __forceinline__ uint32_t i8_idesc(int n) {
    // D = S32 (bits 4-5), A and B signed 8-bit (bits 7-9, 10-12), K-major, N >> 3, M = 128.
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

// One CTA: rows [128 y, 128 y + 128) of the product over the K chunk x, all 36 digit pairs.
// part[(x * nr + c) * Mp + i] = sum_d 2^-7(d-2) acc_d(i, c).
__global__ void __launch_bounds__(OZ_THREADS, 1)
    ozaki_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, int64_t m,
                 int64_t k, int64_t Mp, int nr, int64_t kc_len, uint32_t tmem_cols, double* part, int* err,
                 uint64_t limit_ns) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int b_bytes = S * nr * 128;  // one K block of P's digits
    uint8_t* sA = smem;
    uint8_t* sB = smem + A_STAGES * A_TILE;
    uint64_t* afull = reinterpret_cast<uint64_t*>(sB + 2 * b_bytes);
    uint64_t* aempty = afull + A_STAGES;
    uint64_t* bfull = aempty + A_STAGES;
    uint64_t* bempty = bfull + 2;
    uint64_t* done = bempty + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
    volatile int* stop = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int64_t m0 = (int64_t)blockIdx.y * 128;
    const int64_t k0 = (int64_t)blockIdx.x * kc_len;
    const int64_t k1 = k0 + kc_len < k ? k0 + kc_len : k;
    const int KB = (int)((k1 - k0 + 127) / 128);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int brows = S * nr, bbox = brows < 256 ? brows : 256;
    if (aborted(err)) return;  // an earlier wait of the device timed out

    if (threadIdx.x == 0) {
        for (int q = 0; q < A_STAGES; ++q) {
            mbar_init(&afull[q], 1);
            mbar_init(&aempty[q], 1);
        }
        for (int q = 0; q < 2; ++q) {
            mbar_init(&bfull[q], 1);
            mbar_init(&bempty[q], 1);
        }
        mbar_init(done, 1);
        *stop = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(&tmA) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(&tmB) : "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(tmem_cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            int a_issued = 0, b_issued = 0;
            for (int kb = 0; kb < KB && !*stop; ++kb) {
                const int bs = kb & 1;
                const int w = mbar_wait_bounded(&bempty[bs], ((kb >> 1) & 1) ^ 1, stop, err, nullptr, limit_ns);
                if (w != kWaitOk) {
                    raise_stop(stop, err, w, kSiteOzaki * 100 + kRoleProducer * 10);
                    break;
                }
                const int kx = (int)(k0 + 128 * kb);
                mbar_expect_tx(&bfull[bs], (uint32_t)b_bytes);
                for (int r = 0; r < brows; r += bbox) tma_load_2d(sB + bs * b_bytes + r * 128, &tmB, &bfull[bs], kx, r);
                ++b_issued;
                for (int t = 0; t < S; ++t) {
                    const int as = a_issued % A_STAGES;
                    const int wa =
                        mbar_wait_bounded(&aempty[as], ((a_issued / A_STAGES) & 1) ^ 1, stop, err, nullptr, limit_ns);
                    if (wa != kWaitOk) {
                        raise_stop(stop, err, wa, kSiteOzaki * 100 + kRoleProducer * 10);
                        break;
                    }
                    mbar_expect_tx(&afull[as], (uint32_t)A_TILE);
                    tma_load_2d(sA + as * A_TILE, &tmA, &afull[as], kx, (int)(t * Mp + m0));
                    ++a_issued;
                }
            }
            if (*stop) {
                // Let the copies this thread started land before the CTA's shared memory goes away.
                volatile int never = 0;
                bool drained = true;
                for (int q = (a_issued > A_STAGES ? a_issued - A_STAGES : 0); q < a_issued; ++q)
                    drained &= mbar_wait_bounded(&afull[q % A_STAGES], (q / A_STAGES) & 1, &never, nullptr, nullptr,
                                                 limit_ns) == kWaitOk;
                for (int q = (b_issued > 2 ? b_issued - 2 : 0); q < b_issued; ++q)
                    drained &= mbar_wait_bounded(&bfull[q & 1], (q >> 1) & 1, &never, nullptr, nullptr, limit_ns) ==
                               kWaitOk;
                if (!drained) settle(kSettleNs);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // The tensor pipe idles through every instruction this thread runs between two
            // MMAs: the slices are unrolled with their shapes precomputed, and the A stage
            // and its phase are carried incrementally.
            uint32_t id1[S], id2[S];
#pragma unroll
            for (int t = 0; t < S; ++t) {
                const int n_all = nr * (S - t);
                id1[t] = i8_idesc(n_all < 256 ? n_all : 256);
                id2[t] = i8_idesc(n_all > 256 ? n_all - 256 : 16);
            }
            const uint64_t ad0 = sw128_kmajor_desc(sA);
            constexpr uint64_t kAStep = A_TILE >> 4;
            const uint64_t b0d0 = sw128_kmajor_desc(sB), b0d1 = sw128_kmajor_desc(sB + 256 * 128);
            const uint64_t b1d0 = sw128_kmajor_desc(sB + b_bytes), b1d1 = sw128_kmajor_desc(sB + b_bytes + 256 * 128);
            int as = 0;
            uint32_t aph = 0;
            bool ok = true;
            for (int kb = 0; kb < KB && ok; ++kb) {
                const int bs = kb & 1;
                int w = mbar_wait_bounded(&bfull[bs], (kb >> 1) & 1, stop, err, nullptr, limit_ns);
                if (w != kWaitOk) {
                    raise_stop(stop, err, w, kSiteOzaki * 100 + kRoleMma * 10);
                    break;
                }
                tc_fence_after();
                const uint64_t bd0 = bs ? b1d0 : b0d0, bd1 = bs ? b1d1 : b0d1;
#pragma unroll
                for (int t = 0; t < S; ++t) {
                    w = mbar_wait_bounded(&afull[as], aph, stop, err, nullptr, limit_ns);
                    if (w != kWaitOk) {
                        raise_stop(stop, err, w, kSiteOzaki * 100 + kRoleMma * 10);
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint64_t ad = ad0 + (uint64_t)as * kAStep;
                    // A_t x [P_1 .. P_(S-t)] -> accumulators d = t+2 .. S+1 (columns nr t ..)
                    const bool two = nr * (S - t) > 256;
                    const uint32_t col = (uint32_t)(nr * t);
#pragma unroll
                    for (int kk = 0; kk < 4; ++kk) {
                        const uint32_t acc = (kb | t | kk) != 0 ? 1u : 0u;
                        umma_i8(tmem + col, ad + 2 * kk, bd0 + 2 * kk, id1[t], acc);
                        if (two) umma_i8(tmem + col + 256, ad + 2 * kk, bd1 + 2 * kk, id2[t], acc);
                    }
                    umma_commit(&aempty[as]);
                    if (++as == A_STAGES) {
                        as = 0;
                        aph ^= 1u;
                    }
                }
                if (ok) umma_commit(&bempty[bs]);
            }
            umma_commit(done);
        }
    } else {
        const int q = warp & 3;  // TMEM lane quadrant this warp may access
        const int w = mbar_wait_bounded(done, 0, stop, err, nullptr, limit_ns);
        const bool ok = w == kWaitOk;
        if (!ok) raise_stop(stop, err, w, kSiteOzaki * 100 + kRoleEpilogue * 10);
        tc_fence_after();
        if (__all_sync(0xffffffffu, ok && !*stop)) {
            const int64_t i = m0 + 32 * q + lane;
            for (int cc = 0; cc < nr; cc += 16) {
                double acc[16];
#pragma unroll
                for (int x = 0; x < 16; ++x) acc[x] = 0.0;
                for (int dd = S - 1; dd >= 0; --dd) {  // Horner from the lightest accumulator
                    int v[16];
                    tmem_ld16i(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(dd * nr + cc), v);
#pragma unroll
                    for (int x = 0; x < 16; ++x) acc[x] = fma(acc[x], 0.0078125, (double)v[x]);
                }
                if (i < m) {
                    double* dst = part + ((int64_t)blockIdx.x * nr + cc) * Mp + i;
#pragma unroll
                    for (int x = 0; x < 16; ++x) dst[(int64_t)x * Mp] = acc[x];
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tmem_cols));
    }
}

// C(i, c) = alpha 2^(e_i + f_c - 14) sum_x part[x][c][i] + beta C(i, c), the chunks summed
// in a fixed order; NaN where row i of A or column c of P holds Inf or NaN.
__global__ void __launch_bounds__(256) ozaki_reduce_kernel(int64_t m, int z, int nr, const double* part, int64_t Mp,
                                                           const int* rexp, const int* cexp, double alpha,
                                                           double beta, double* C, int64_t ldc) {
    const int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x;
    const int c = blockIdx.y;
    if (i >= m) return;
    double s = 0.0;
    for (int x = 0; x < z; ++x) s += part[((int64_t)x * nr + c) * Mp + i];
    const int er = rexp[i], ec = cexp[c];
    const double v = (er == kBadExp || ec == kBadExp) ? __longlong_as_double(0x7FF8000000000000ll)
                                                       : ldexp(s, er + ec - 14);
    double* dst = C + i + (int64_t)c * ldc;
    *dst = beta != 0.0 ? fma(beta, *dst, alpha * v) : alpha * v;
}

bool make_u8_tmap(CUtensorMap* tm, const void* base, int64_t rows, int64_t kdim, int64_t ld, int box_rows) {
    auto enc = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(tensor_map_encoder());
    if (!enc) return false;
    cuuint64_t dims[2] = {(cuuint64_t)kdim, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)ld};
    cuuint32_t box[2] = {128u, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    return enc(tm, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void*>(base), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

size_t ozaki_a_bytes(int64_t m, int64_t k) {
    const int64_t Mp = round_up(m, 128), ldk = round_up(k, 16);
    return align256((size_t)S * Mp * ldk) + align256((size_t)Mp * 8) + align256((size_t)Mp * 4) + 256;
}

size_t ozaki_p_bytes(int64_t m, int64_t k, int64_t nrhs) {
    const int64_t Mp = round_up(m, 128), ldk = round_up(k, 16);
    const int nr = rhs_width(nrhs);
    int z = 1;
    int64_t kc = 0;
    oz_split(Mp, k, &z, &kc);
    return align256((size_t)S * nr * ldk) + align256((size_t)z * nr * Mp * 8) + align256(64 * 4);
}

int ozaki_layout_a(int64_t m, int64_t k, void* ws, bool diagonal, OzakiA* out) {
    if (m <= 0 || k <= 0 || !out || (diagonal && m != k)) return RC_ERR_INVALID_ARGUMENT;
    OzakiA a;
    a.m = m;
    a.k = k;
    a.Mp = round_up(m, 128);
    a.ldk = round_up(k, 16);
    if (a.Mp / 32 > 65535 || k > ((int64_t)1 << 30)) return RC_ERR_NOT_SUPPORTED;  // grid and TMA limits
    char* p = static_cast<char*>(ws);
    a.slices = reinterpret_cast<int8_t*>(p);
    p += align256((size_t)S * a.Mp * a.ldk);
    a.rowbits = reinterpret_cast<unsigned long long*>(p);
    p += align256((size_t)a.Mp * 8);
    a.rexp = reinterpret_cast<int*>(p);
    p += align256((size_t)a.Mp * 4);
    a.flag = reinterpret_cast<int*>(p);
    a.diagonal = diagonal;
    if (!make_u8_tmap(&a.tmap, a.slices, S * a.Mp, k, a.ldk, 128)) return RC_ERR_NOT_SUPPORTED;
    *out = a;
    return RC_SUCCESS;
}

int ozaki_diag_exponents(const OzakiA& a, const double* A, int64_t lda, cudaStream_t s) {
    if (!a.diagonal) return RC_ERR_INVALID_ARGUMENT;
    if (cudaMemsetAsync(a.flag, 0, sizeof(int), s) != cudaSuccess) return RC_ERR_CUDA;
    diag_exp_kernel<<<ceil_div(a.Mp, 256) < 1024u ? ceil_div(a.Mp, 256) : 1024u, 256, 0, s>>>(a.m, A, lda, a.Mp,
                                                                                               a.rexp, a.flag);
    return check_launch();
}

int ozaki_prepare_a(int64_t m, int64_t k, const double* A, int64_t lda, void* ws, OzakiA* out, cudaStream_t s) {
    OzakiA a;
    RC_TRY(ozaki_layout_a(m, k, ws, false, &a));
    if (cudaMemsetAsync(a.flag, 0, sizeof(int), s) != cudaSuccess ||
        cudaMemsetAsync(a.rowbits, 0, (size_t)a.Mp * 8, s) != cudaSuccess)
        return RC_ERR_CUDA;
    row_absmax_kernel<<<dim3(ceil_div(k, 512), ceil_div(m, 256)), 256, 0, s>>>(m, k, A, lda, a.rowbits);
    RC_TRY(check_launch());
    slice_a_kernel<<<dim3(ceil_div(k, 128), (unsigned)(a.Mp / 32)), 256, 0, s>>>(m, k, A, lda, a.rowbits, a.rexp,
                                                                                a.slices, a.Mp, a.ldk);
    RC_TRY(check_launch());
    *out = a;
    return RC_SUCCESS;
}

int ozaki_gemm(const OzakiA& a, int64_t nrhs, double alpha, const double* P, int64_t ldp, double beta, double* C,
               int64_t ldc, void* ws, cudaStream_t s) {
    if (nrhs <= 0 || a.m <= 0) return RC_SUCCESS;
    if (nrhs > 64) return RC_ERR_NOT_SUPPORTED;
    const int nr = rhs_width(nrhs);
    int z = 1;
    int64_t kc = 0;
    oz_split(a.Mp, a.k, &z, &kc);
    char* p = static_cast<char*>(ws);
    int8_t* Ps = reinterpret_cast<int8_t*>(p);
    p += align256((size_t)S * nr * a.ldk);
    double* part = reinterpret_cast<double*>(p);
    p += align256((size_t)z * nr * a.Mp * 8);
    int* cexp = reinterpret_cast<int*>(p);

    CUtensorMap tmB;
    if (!make_u8_tmap(&tmB, Ps, S * nr, a.k, a.ldk, S * nr < 256 ? S * nr : 256)) return RC_ERR_NOT_SUPPORTED;
    slice_p_kernel<<<nr, 256, 0, s>>>(a.k, nrhs, P, ldp, nr, a.diagonal ? a.rexp : nullptr, cexp, Ps, a.ldk);
    RC_TRY(check_launch());

    const size_t smem = 1024 + (size_t)A_STAGES * A_TILE + 2 * (size_t)S * nr * 128 + 256;
    if (cudaFuncSetAttribute(ozaki_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return RC_ERR_CUDA;
    const uint32_t cols = S * nr <= 128 ? 128u : (S * nr <= 256 ? 256u : 512u);
    ozaki_kernel<<<dim3((unsigned)z, (unsigned)(a.Mp / 128)), OZ_THREADS, smem, s>>>(
        a.tmap, tmB, a.m, a.k, a.Mp, nr, kc, cols, part, error_word(), wait_limit_ns());
    RC_TRY(check_launch());
    ozaki_reduce_kernel<<<dim3(ceil_div(a.m, 256), (unsigned)nrhs), 256, 0, s>>>(a.m, z, nr, part, a.Mp, a.rexp,
                                                                                  cexp, alpha, beta, C, ldc);
    return check_launch();
}

}  // namespace rc

extern "C" {

int rc_gemm_f64_sliced(size_t m, size_t n, size_t k, double alpha, const double* A, size_t lda, const double* B,
                       size_t ldb, double beta, double* C, size_t ldc, void* stream) {
    if (m == 0 || n == 0) return RC_SUCCESS;
    if (!A || !B || !C || lda < m || ldb < k || ldc < m) return RC_ERR_INVALID_ARGUMENT;
    if (n > 64 || m > ((size_t)1 << 21) - 128 || k > ((size_t)1 << 30)) return RC_ERR_NOT_SUPPORTED;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (k == 0)
        return rc::gemm<double>((int64_t)m, (int64_t)n, 0, alpha, rc::View<const double>{nullptr, 1, 1},
                                rc::View<const double>{nullptr, 1, 1}, beta, rc::colmajor(C, (int64_t)ldc),
                                rc::kFull, 0, s);
    const size_t ab = rc::ozaki_a_bytes((int64_t)m, (int64_t)k);
    const size_t pb = rc::ozaki_p_bytes((int64_t)m, (int64_t)k, (int64_t)n);
    char* ws = static_cast<char*>(rc::workspace(s, ab + pb, 11));
    if (!ws) return RC_ERR_ALLOC;
    rc::OzakiA a;
    RC_TRY(rc::ozaki_prepare_a((int64_t)m, (int64_t)k, A, (int64_t)lda, ws, &a, s));
    return rc::ozaki_gemm(a, (int64_t)n, alpha, B, (int64_t)ldb, beta, C, (int64_t)ldc, ws + ab, s);
}

}  // extern "C"
