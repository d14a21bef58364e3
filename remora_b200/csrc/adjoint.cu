// Reverse-mode adjoints of the Cholesky factorisation and of the triangular solve
// (extension; the reference has no derivatives of its decompositions).
//
// Cholesky A = L L^T (Murray 2016, "Differentiation of the Cholesky decomposition"):
// with dA = dL L^T + L dL^T, X = L^-1 dL is lower triangular and L^-1 dA L^-T = X + X^T,
// so dL = L Phi(L^-1 dA L^-T) with Phi = lower triangle, diagonal halved. For a scalar
// f(L) with adjoint Lbar = df/dL this gives, for symmetric perturbations dA,
//     Abar = 1/2 L^-T (P + P^T) L^-1,   P = Phi(L^T Lbar).
// Blocked evaluation on the library's kernels, from L alone (the backward pass stores no
// intermediate of the forward factorisation):
//     M = tril(L^T Lbar)          lower-masked GEMM (the upper triangle is never formed)
//     S = M + M^T - diag(M)       = P + P^T
//     T = L^-T S                  blocked TRSM
//     Abar = 1/2 T L^-1           blocked TRSM on the transposed view, then symmetrised.
// Triangular solve X = L^-1 B (and X = L^-T B): Bbar = L^-T Xbar (L^-1 Xbar) and
// Lbar -= tril(Bbar X^T) (tril(X Bbar^T)).
#include "adjoint.cuh"
#include "assign.cuh"
#include "factor.cuh"
#include "gemm.cuh"

namespace rc {
namespace {

// dst = tril(src) (upper triangle zeroed), both n x n.
__global__ void tril_copy_kernel(int64_t n, View<const double> src, View<double> dst) {
    for (int64_t j = blockIdx.y; j < n; j += gridDim.y)
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
            dst(i, j) = i >= j ? src(i, j) : 0.0;
}

// mode 0: S(i, j) = S(j, i) for i < j (mirror the lower triangle up);
// mode 1: S = (S + S^T) / 2.
__global__ void symmetrize_kernel(int64_t n, View<double> S, int mode) {
    for (int64_t j = blockIdx.y; j < n; j += gridDim.y)
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < j; i += (int64_t)gridDim.x * blockDim.x) {
            if (mode == 0) {
                S(i, j) = S(j, i);
            } else {
                const double v = 0.5 * (S(i, j) + S(j, i));
                S(i, j) = v;
                S(j, i) = v;
            }
        }
}

dim3 sq_grid(int64_t n) {
    return dim3(ceil_div(n, 256) < 256u ? ceil_div(n, 256) : 256u, n < 65535 ? (unsigned)n : 65535u);
}

}  // namespace

int potrf_backward(int64_t n, View<const double> L, View<const double> Lbar, View<double> Abar, cudaStream_t s) {
    if (n <= 0) return RC_SUCCESS;
    double* w = static_cast<double*>(workspace(s, (size_t)2 * n * n * sizeof(double), 8));
    if (!w) return RC_ERR_ALLOC;
    const View<double> L0 = colmajor(w, n), Lb0 = colmajor(w + (size_t)n * n, n);
    tril_copy_kernel<<<sq_grid(n), 256, 0, s>>>(n, L, L0);
    tril_copy_kernel<<<sq_grid(n), 256, 0, s>>>(n, Lbar, Lb0);
    RC_TRY(check_launch());
    const View<const double> Lc = {L0.p, L0.rs, L0.cs}, Lbc = {Lb0.p, Lb0.rs, Lb0.cs};
    // M = tril(L^T Lbar) into Abar (lower triangle), S = M + M^T - diag(M).
    RC_TRY(gemm<double>(n, n, n, 1.0, Lc.t(), Lbc, 0.0, Abar, kLower, 0, s));
    symmetrize_kernel<<<sq_grid(n), 256, 0, s>>>(n, Abar, 0);
    RC_TRY(check_launch());
    // T = L^-T S; Abar = 1/2 T L^-1, i.e. L^T Abar^T = 1/2 T^T.
    RC_TRY(trsm_left<double>(true, false, n, n, 1.0, Lc.t(), Abar, nullptr, s));
    RC_TRY(trsm_left<double>(true, false, n, n, 0.5, Lc.t(), Abar.t(), nullptr, s));
    symmetrize_kernel<<<sq_grid(n), 256, 0, s>>>(n, Abar, 1);
    return check_launch();
}

int trsm_backward(bool trans, int64_t n, int64_t nrhs, View<const double> L, View<const double> X, View<double> Xbar,
                  View<double> Lbar, cudaStream_t s) {
    if (n <= 0 || nrhs <= 0) return RC_SUCCESS;
    double* w = static_cast<double*>(workspace(s, (size_t)n * n * sizeof(double), 8));
    if (!w) return RC_ERR_ALLOC;
    const View<double> L0 = colmajor(w, n);
    tril_copy_kernel<<<sq_grid(n), 256, 0, s>>>(n, L, L0);
    RC_TRY(check_launch());
    const View<const double> Lc = {L0.p, L0.rs, L0.cs};
    const View<const double> Bb = {Xbar.p, Xbar.rs, Xbar.cs};
    if (!trans) {
        // X = L^-1 B: Bbar = L^-T Xbar, Lbar -= tril(Bbar X^T)
        RC_TRY(trsm_left<double>(true, false, n, nrhs, 1.0, Lc.t(), Xbar, nullptr, s));
        return gemm<double>(n, n, nrhs, -1.0, Bb, X.t(), 1.0, Lbar, kLower, 0, s);
    }
    // X = L^-T B: Bbar = L^-1 Xbar, Lbar -= tril(X Bbar^T)
    RC_TRY(trsm_left<double>(false, false, n, nrhs, 1.0, Lc, Xbar, nullptr, s));
    return gemm<double>(n, n, nrhs, -1.0, X, Bb.t(), 1.0, Lbar, kLower, 0, s);
}

}  // namespace rc

extern "C" {

int rc_potrf_backward_f64(size_t n, const double* L, size_t ldl, const double* Lbar, size_t ldlb, double* Abar,
                          size_t ldab, void* stream) {
    if (n == 0) return RC_SUCCESS;
    if (!L || !Lbar || !Abar || ldl < n || ldlb < n || ldab < n) return RC_ERR_INVALID_ARGUMENT;
    return rc::potrf_backward((int64_t)n, rc::colmajor(L, (int64_t)ldl), rc::colmajor(Lbar, (int64_t)ldlb),
                              rc::colmajor(Abar, (int64_t)ldab), static_cast<cudaStream_t>(stream));
}

int rc_trsm_backward_f64(int trans, size_t n, size_t nrhs, const double* L, size_t ldl, const double* X, size_t ldx,
                         double* Xbar, size_t ldxb, double* Lbar, size_t ldlb, void* stream) {
    if (n == 0 || nrhs == 0) return RC_SUCCESS;
    if (!L || !X || !Xbar || !Lbar || ldl < n || ldx < n || ldxb < n || ldlb < n) return RC_ERR_INVALID_ARGUMENT;
    return rc::trsm_backward(trans != 0, (int64_t)n, (int64_t)nrhs, rc::colmajor(L, (int64_t)ldl),
                             rc::colmajor(X, (int64_t)ldx), rc::colmajor(Xbar, (int64_t)ldxb),
                             rc::colmajor(Lbar, (int64_t)ldlb), static_cast<cudaStream_t>(stream));
}

}  // extern "C"

// ---------------------------------------------------------------------------------------
// RBF kernel matrix of a Gaussian process and the contraction of its adjoint with the
// lengthscale derivatives: the model around the differentiated Cholesky in the
// marginal-likelihood workload.
namespace rc {
namespace {

__global__ void rbf_kernel(int64_t n, int d, const double* X, const double* ls, double noise, View<double> K) {
    for (int64_t j = blockIdx.y; j < n; j += gridDim.y)
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
            double r2 = 0.0;
            for (int q = 0; q < d; ++q) {
                const double t = (X[i * d + q] - X[j * d + q]) / ls[q];
                r2 = fma(t, t, r2);
            }
            K(i, j) = exp(-0.5 * r2) + (i == j ? noise : 0.0);
        }
}

// g[q] = sum_ij Kbar(i, j) k(i, j) (x_iq - x_jq)^2 / ls_q^3, k without the noise term.
__global__ void __launch_bounds__(256) rbf_ls_grad_kernel(int64_t n, int d, const double* X, const double* ls,
                                                          View<const double> Kbar, double* g) {
    __shared__ double red[16][8];
    double acc[16];
    for (int q = 0; q < 16; ++q) acc[q] = 0.0;
    for (int64_t j = blockIdx.y; j < n; j += gridDim.y)
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
            double r2 = 0.0;
            for (int q = 0; q < d; ++q) {
                const double t = (X[i * d + q] - X[j * d + q]) / ls[q];
                r2 = fma(t, t, r2);
            }
            const double w = Kbar(i, j) * exp(-0.5 * r2);
            for (int q = 0; q < d; ++q) {
                const double dx = X[i * d + q] - X[j * d + q];
                acc[q] = fma(w, dx * dx / (ls[q] * ls[q] * ls[q]), acc[q]);
            }
        }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int q = 0; q < d; ++q) {
        double v = acc[q];
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if (lane == 0) red[q][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < d) {
        double v = 0.0;
        for (int w8 = 0; w8 < 8; ++w8) v += red[threadIdx.x][w8];
        atomicAdd(&g[threadIdx.x], v);
    }
}

}  // namespace
}  // namespace rc

extern "C" {

int rc_rbf_kernel_f64(size_t n, int d, const double* X, const double* ls, double noise, double* K, size_t ldk,
                      void* stream) {
    if (n == 0) return RC_SUCCESS;
    if (d < 1 || d > 16 || !X || !ls || !K || ldk < n) return RC_ERR_INVALID_ARGUMENT;
    dim3 grid(rc::ceil_div(n, 256) < 256u ? rc::ceil_div(n, 256) : 256u, n < 65535 ? (unsigned)n : 65535u);
    rc::rbf_kernel<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>((int64_t)n, d, X, ls, noise,
                                                                         rc::colmajor(K, (int64_t)ldk));
    return rc::check_launch();
}

int rc_rbf_lengthscale_grad_f64(size_t n, int d, const double* X, const double* ls, const double* Kbar, size_t ldk,
                                double* grad, void* stream) {
    if (n == 0) return RC_SUCCESS;
    if (d < 1 || d > 16 || !X || !ls || !Kbar || !grad || ldk < n) return RC_ERR_INVALID_ARGUMENT;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(grad, 0, d * sizeof(double), s) != cudaSuccess) return RC_ERR_CUDA;
    dim3 grid(rc::ceil_div(n, 256) < 32u ? rc::ceil_div(n, 256) : 32u, n < 4096 ? (unsigned)n : 4096u);
    rc::rbf_ls_grad_kernel<<<grid, 256, 0, s>>>((int64_t)n, d, X, ls, rc::View<const double>{Kbar, 1, (int64_t)ldk},
                                                 grad);
    return rc::check_launch();
}

}  // extern "C"
