// Drop-in test of the cuda_tag device: a Remora program in which only the device tag
// changes. Checks, against Remora's own CPU kernels on the same inputs, the hot path of
// the reference's HIP tests (Test/hip_prod.cpp, hip_syrk.cpp, hip_triangular_solve.cpp,
// hip_cholesky.cpp, hip_random.cpp) through the unchanged API: copy_to_device,
// noalias(C) (+)= alpha * prod(A, B) with trans() views, kernels::syrk, kernels::trsm,
// kernels::potrf, cholesky_decomposition + solve, solve(A, B, symm_pos_def(), left()),
// normal(...) fills, copy_to_cpu. Prints one line per check and exits non-zero on failure.
#include <remora/cuda.hpp>
#include <remora/remora.hpp>

#include <cmath>
#include <cstdio>
#include <random>

using namespace remora;

static int failures = 0;

template <class M1, class M2>
double rel_diff(M1 const& a, M2 const& b) {
    double num = 0, den = 0;
    for (std::size_t i = 0; i != a.size1(); ++i)
        for (std::size_t j = 0; j != a.size2(); ++j) {
            double d = double(a(i, j)) - double(b(i, j));
            num += d * d;
            den += double(b(i, j)) * double(b(i, j));
        }
    return std::sqrt(num / (den > 0 ? den : 1));
}

static void report(char const* what, double err, double tol) {
    bool ok = err <= tol;
    std::printf("%-58s rel err %.3e (tol %.0e) %s\n", what, err, tol, ok ? "ok" : "FAIL");
    if (!ok) ++failures;
}

// A host vector as a 1 x n matrix (for rel_diff).
template <class V>
matrix<double> to_matrix(V const& v, std::size_t, std::size_t n) {
    matrix<double> m(1, n);
    for (std::size_t j = 0; j != n; ++j) m(0, j) = v(j);
    return m;
}

// Test/hip_cholesky.cpp:13-33
matrix<double> createSymm(std::size_t n) {
    matrix<double> R(n, n, 0.0);
    for (std::size_t i = 0; i != n; ++i) {
        for (std::size_t j = 0; j < i; ++j) R(i, j) = 0.2 / std::abs((int)i - (int)j);
        R(i, i) = 1 + 0.5 / n * i + 1;
    }
    matrix<double> A = prod(R, trans(R));
    return A;
}

template <class OA, class OB, class OC>
void prod_test(char const* name) {
    std::size_t rows = 50, cols = 80, mid = 33;  // Test/hip_prod.cpp:131-150
    matrix<float, OA> a(rows, mid);
    matrix<float, OB> b(mid, cols);
    for (std::size_t i = 0; i != rows; ++i)
        for (std::size_t j = 0; j != mid; ++j) a(i, j) = 0.1 * i * mid + 0.2 * j;
    for (std::size_t i = 0; i != mid; ++i)
        for (std::size_t j = 0; j != cols; ++j) b(i, j) = 0.1 * i * cols + 1.5 * j;
    matrix<float, OA, cuda_tag> ad = copy_to_device(a, cuda_tag());
    matrix<float, OB, cuda_tag> bd = copy_to_device(b, cuda_tag());
    matrix<float, OC, cuda_tag> cd(rows, cols, 1.5f);
    noalias(cd) += -2 * prod(ad, bd);
    matrix<float, OC> c(rows, cols, 1.5f);
    noalias(c) += -2 * prod(a, b);
    matrix<float> got = copy_to_cpu(cd);
    report(name, rel_diff(got, c), 1e-5);
    noalias(cd) = prod(ad, bd);
    noalias(c) = prod(a, b);
    got = copy_to_cpu(cd);
    report("  ... and noalias(C) = prod(A, B)", rel_diff(got, c), 1e-5);
}

int main() {
    std::mt19937 rng(42);
    // --- gemm, all 8 orientation combinations, float (Test/hip_prod.cpp)
    prod_test<row_major, row_major, row_major>("prod rm*rm->rm, +=, alpha=-2");
    prod_test<row_major, column_major, row_major>("prod rm*cm->rm");
    prod_test<column_major, row_major, row_major>("prod cm*rm->rm");
    prod_test<column_major, column_major, row_major>("prod cm*cm->rm");
    prod_test<row_major, row_major, column_major>("prod rm*rm->cm");
    prod_test<row_major, column_major, column_major>("prod rm*cm->cm");
    prod_test<column_major, row_major, column_major>("prod cm*rm->cm");
    prod_test<column_major, column_major, column_major>("prod cm*cm->cm");
    {  // FP64 with a transposed view on the device
        matrix<double> a(300, 200), b(300, 150);
        kernels::generate_uniform(a, rng, -1.0, 1.0);
        kernels::generate_uniform(b, rng, -1.0, 1.0);
        matrix<double, column_major, cuda_tag> ad = copy_to_device(a, cuda_tag());
        matrix<double, row_major, cuda_tag> bd = copy_to_device(b, cuda_tag());
        matrix<double, column_major, cuda_tag> cd(200, 150, 0.0);
        noalias(cd) = prod(trans(ad), bd);
        matrix<double> c = prod(trans(a), b);
        matrix<double> got = copy_to_cpu(cd);
        report("prod(trans(A), B) FP64, A cm, B rm", rel_diff(got, c), 1e-13);
    }
    // --- syrk (Test/hip_syrk.cpp:52-93, smaller), both triangles, the other stays 3
    {
        std::size_t dims = 136, K = 109;
        matrix<float> arg(dims, K);
        for (std::size_t i = 0; i != dims; ++i)
            for (std::size_t j = 0; j != K; ++j) arg(i, j) = (1.0 / dims) * i + 0.2 / K * j + 1;
        matrix<float, column_major, cuda_tag> argd = copy_to_device(arg, cuda_tag());
        for (int upper = 0; upper < 2; ++upper) {
            matrix<float, row_major, cuda_tag> cd(dims, dims, 3.0f);
            matrix<float> c(dims, dims, 3.0f);
            if (upper) { kernels::syrk<true>(argd, cd, 2.0f); kernels::syrk<true>(arg, c, 2.0f); }
            else { kernels::syrk<false>(argd, cd, 2.0f); kernels::syrk<false>(arg, c, 2.0f); }
            matrix<float> got = copy_to_cpu(cd);
            report(upper ? "syrk<upper> float, C row-major" : "syrk<lower> float, C row-major", rel_diff(got, c), 1e-5);
            bool untouched = true;
            for (std::size_t i = 0; i != dims; ++i)
                for (std::size_t j = 0; j != dims; ++j)
                    if ((upper ? j < i : j > i) && got(i, j) != 3.0f) untouched = false;
            report("  ... other triangle untouched", untouched ? 0.0 : 1.0, 0.0);
        }
    }
    // --- trsm (Test/hip_triangular_solve.cpp:100-187 inputs)
    {
        std::size_t size = 139, k = 238;
        matrix<double, row_major> A(size, size, 1.0);
        for (std::size_t i = 0; i != size; ++i)
            for (std::size_t j = 0; j <= i; ++j) {
                A(i, j) = 0.3 * (0.1 / size * i - 0.05 / (i + 1.0) * j);
                if (i == j) A(i, j) += 10;
            }
        matrix<double, row_major> B(size, k);
        for (std::size_t i = 0; i != size; ++i)
            for (std::size_t j = 0; j != k; ++j) B(i, j) = (0.1 / size) * i + 0.1 / k * j;
        matrix<double, row_major, cuda_tag> Ad = copy_to_device(A, cuda_tag());
        matrix<double, column_major, cuda_tag> Bd = copy_to_device(B, cuda_tag());
        kernels::trsm<lower, left>(Ad, Bd);
        matrix<double> X = B;
        kernels::trsm<lower, left>(A, X);
        matrix<double> got = copy_to_cpu(Bd);
        report("trsm<lower,left> FP64, A rm, B cm", rel_diff(got, X), 1e-13);
        matrix<double, row_major, cuda_tag> Bt = copy_to_device(matrix<double>(trans(B)), cuda_tag());
        kernels::trsm<upper, right>(trans(Ad), Bt);
        matrix<double> Y = trans(B);
        kernels::trsm<upper, right>(trans(A), Y);
        got = copy_to_cpu(Bt);
        report("trsm<upper,right>(trans(A)) FP64, B rm", rel_diff(got, Y), 1e-13);
    }
    // --- potrf (Test/hip_cholesky.cpp:36-58), whole matrix compared
    {
        matrix<double> A = createSymm(123);
        for (int rm = 0; rm < 2; ++rm) {
            matrix<double> ref = A;
            kernels::potrf<lower>(ref);
            double err;
            if (rm) {
                matrix<double, row_major, cuda_tag> Ad = copy_to_device(A, cuda_tag());
                std::size_t st = kernels::potrf<lower>(Ad);
                err = st ? 1.0 : rel_diff(matrix<double>(copy_to_cpu(Ad)), ref);
            } else {
                matrix<double, column_major, cuda_tag> Ad = copy_to_device(A, cuda_tag());
                std::size_t st = kernels::potrf<lower>(Ad);
                err = st ? 1.0 : rel_diff(matrix<double>(copy_to_cpu(Ad)), ref);
            }
            report(rm ? "potrf<lower> n=123 row-major (whole matrix)" : "potrf<lower> n=123 column-major (whole matrix)",
                   err, 1e-13);
        }
        matrix<double> U = A;
        kernels::potrf<upper>(U);
        matrix<double, column_major, cuda_tag> Ud = copy_to_device(A, cuda_tag());
        kernels::potrf<upper>(Ud);
        report("potrf<upper> n=123 column-major", rel_diff(matrix<double>(copy_to_cpu(Ud)), U), 1e-13);
        matrix<double> bad = A;
        bad(70, 70) = -1.0;
        matrix<double, column_major, cuda_tag> Bd = copy_to_device(bad, cuda_tag());
        std::size_t st = kernels::potrf<lower>(Bd);
        report("potrf failing pivot reported as global index 71", st == 71 ? 0.0 : 1.0, 0.0);
    }
    // --- cholesky_decomposition + solve, and solve(A, B, symm_pos_def(), left())
    {
        std::size_t n = 1024, nrhs = 16;  // the plain FP64 SPD solve recipe
        std::mt19937 g(1);
        matrix<double> G(n, n), B(n, nrhs);
        kernels::generate_normal(G, g, 0.0, 1.0);
        kernels::generate_normal(B, g, 0.0, 1.0);
        matrix<double> A = prod(G, trans(G));
        A /= double(n);
        for (std::size_t i = 0; i != n; ++i) A(i, i) += 1e-2;
        matrix<double, column_major, cuda_tag> Ad = copy_to_device(A, cuda_tag());
        matrix<double, column_major, cuda_tag> Bd = copy_to_device(B, cuda_tag());
        cholesky_decomposition<matrix<double, column_major, cuda_tag>> chol(Ad);
        chol.solve(Bd, left());
        matrix<double> X = B;
        cholesky_decomposition<matrix<double>> cchol(A);
        cchol.solve(X, left());
        report("cholesky_decomposition + solve FP64 n=1024, 16 RHS", rel_diff(matrix<double>(copy_to_cpu(Bd)), X), 1e-13);
        matrix<double, column_major, cuda_tag> Bd2 = copy_to_device(B, cuda_tag());
        matrix<double, column_major, cuda_tag> Xd = solve(Ad, Bd2, symm_pos_def(), left());
        report("solve(A, B, symm_pos_def(), left())", rel_diff(matrix<double>(copy_to_cpu(Xd)), X), 1e-13);
    }
    // --- matrix-vector products and vector solves (Test/hip_prod.cpp matrix-vector
    // cases, Test/hip_triangular_prod.cpp:47-115, decompositions.hpp:111-115)
    {
        std::size_t rows = 301, cols = 177;
        std::mt19937 g(9);
        matrix<double> M(rows, cols);
        vector<double> x(cols), y0(rows), xt(rows);
        kernels::generate_uniform(M, g, -1.0, 1.0);
        kernels::generate_uniform(x, g, -1.0, 1.0);
        kernels::generate_uniform(y0, g, -1.0, 1.0);
        kernels::generate_uniform(xt, g, -1.0, 1.0);
        vector<double, cuda_tag> xd = copy_to_device(x, cuda_tag());
        vector<double, cuda_tag> yd = copy_to_device(y0, cuda_tag());
        matrix<double, row_major, cuda_tag> Mr = copy_to_device(M, cuda_tag());
        matrix<double, column_major, cuda_tag> Mc = copy_to_device(M, cuda_tag());
        noalias(yd) += -2.0 * prod(Mr, xd);
        vector<double> yref = y0;
        noalias(yref) += -2.0 * prod(M, x);
        vector<double> yh = copy_to_cpu(yd);
        report("noalias(y) += -2 prod(A, x)  row-major A (gemv)", rel_diff(matrix<double>(to_matrix(yh, 1, rows)),
                                                                        matrix<double>(to_matrix(yref, 1, rows))), 1e-13);
        vector<double, cuda_tag> yc = prod(Mc, xd);
        vector<double> ych = copy_to_cpu(yc);
        vector<double> yref2 = prod(M, x);
        report("y = prod(A, x)  column-major A", rel_diff(matrix<double>(to_matrix(ych, 1, rows)),
                                                          matrix<double>(to_matrix(yref2, 1, rows))), 1e-13);
        vector<double, cuda_tag> xtd = copy_to_device(xt, cuda_tag());
        vector<double, cuda_tag> zt = prod(trans(Mc), xtd);
        vector<double> zth = copy_to_cpu(zt);
        vector<double> ztref = prod(trans(M), xt);
        report("z = prod(trans(A), x) (transposed gemv)", rel_diff(matrix<double>(to_matrix(zth, 1, cols)),
                                                                  matrix<double>(to_matrix(ztref, 1, cols))), 1e-13);
        // vector Cholesky solve: two triangular solves with one right-hand side
        std::size_t n = 300;
        matrix<double> A = createSymm(n);
        vector<double> b(n);
        kernels::generate_uniform(b, g, -1.0, 1.0);
        matrix<double, column_major, cuda_tag> Ad = copy_to_device(A, cuda_tag());
        vector<double, cuda_tag> bd = copy_to_device(b, cuda_tag());
        cholesky_decomposition<matrix<double, column_major, cuda_tag>> chol(Ad);
        chol.solve(bd, left());
        vector<double> bref = b;
        cholesky_decomposition<matrix<double>> cchol(A);
        cchol.solve(bref, left());
        vector<double> bh = copy_to_cpu(bd);
        report("cholesky_decomposition::solve(vector) (trsv)", rel_diff(matrix<double>(to_matrix(bh, 1, n)),
                                                                         matrix<double>(to_matrix(bref, 1, n))), 1e-13);
        // triangular products (Test/hip_triangular_prod.cpp:84-109)
        matrix<double> Lm(n, n);
        kernels::generate_uniform(Lm, g, -1.0, 1.0);
        vector<double> v(n);
        kernels::generate_uniform(v, g, -1.0, 1.0);
        matrix<double, row_major, cuda_tag> Lr = copy_to_device(Lm, cuda_tag());
        vector<double, cuda_tag> vd = copy_to_device(v, cuda_tag());
        vector<double, cuda_tag> tv(n);
        noalias(tv) = triangular_prod<lower>(Lr, vd);
        vector<double> tvref(n);
        noalias(tvref) = triangular_prod<lower>(Lm, v);
        vector<double> tvh = copy_to_cpu(tv);
        report("triangular_prod<lower>(A, x) (trmv)", rel_diff(matrix<double>(to_matrix(tvh, 1, n)),
                                                               matrix<double>(to_matrix(tvref, 1, n))), 1e-13);
        matrix<double> Bm(n, 9);
        kernels::generate_uniform(Bm, g, -1.0, 1.0);
        matrix<double, column_major, cuda_tag> Lc = copy_to_device(Lm, cuda_tag());
        matrix<double, row_major, cuda_tag> Bd = copy_to_device(Bm, cuda_tag());
        matrix<double, row_major, cuda_tag> TB(n, 9);
        noalias(TB) = triangular_prod<upper>(Lc, Bd);
        matrix<double> TBref(n, 9);
        noalias(TBref) = triangular_prod<upper>(Lm, Bm);
        report("triangular_prod<upper>(A, B) (trmm)", rel_diff(matrix<double>(copy_to_cpu(TB)), TBref), 1e-13);
        // vector triangular solve through solve() (Test/hip_triangular_solve.cpp:19-60)
        matrix<double> T = Lm;
        for (std::size_t i = 0; i != n; ++i) T(i, i) += double(n);
        matrix<double, column_major, cuda_tag> Td = copy_to_device(T, cuda_tag());
        vector<double, cuda_tag> sd = copy_to_device(v, cuda_tag());
        kernels::trsv<lower, left>(Td, sd);
        vector<double> sref = v;
        kernels::trsv<lower, left>(T, sref);
        vector<double> sh = copy_to_cpu(sd);
        report("kernels::trsv<lower, left>(A, b)", rel_diff(matrix<double>(to_matrix(sh, 1, n)),
                                                            matrix<double>(to_matrix(sref, 1, n))), 1e-13);
    }
    // --- normal fill through the expression API (Test/hip_random.cpp:79-121): moments
    {
        std::mt19937 g(42);
        matrix<float, column_major, cuda_tag> m(377, 389);
        noalias(m) = normal(g, 377, 389, 1.0f, 4.0f, cuda_tag());
        matrix<float> h = copy_to_cpu(m);
        double mean = 0, var = 0, N = 377.0 * 389.0;
        for (std::size_t i = 0; i != h.size1(); ++i)
            for (std::size_t j = 0; j != h.size2(); ++j) mean += h(i, j);
        mean /= N;
        for (std::size_t i = 0; i != h.size1(); ++i)
            for (std::size_t j = 0; j != h.size2(); ++j) var += (h(i, j) - mean) * (h(i, j) - mean);
        var /= N;
        report("normal(g, r, c, 1, 4, cuda_tag()): |mean - 1|", std::fabs(mean - 1.0), 0.02);
        report("  ... |variance - 4|", std::fabs(var - 4.0), 0.05);
    }
    // --- reverse mode: GP negative log likelihood f = 1/2 y^T K^-1 y + 1/2 log det K.
    // Device: forward Cholesky + triangular solve, backward through the hand-written
    // adjoints. Reference: Kbar = 1/2 (inv(K, symm_pos_def()) - alpha alpha^T) composed
    // from Remora's CPU kernels (solve.hpp:472-493).
    {
        std::size_t n = 160;
        std::mt19937 g(5);
        matrix<double> X(n, 16);
        vector<double> ydat(n);
        kernels::generate_normal(X, g, 0.0, 1.0);
        kernels::generate_normal(ydat, g, 0.0, 1.0);
        matrix<double> K(n, n);
        for (std::size_t i = 0; i != n; ++i)
            for (std::size_t j = 0; j != n; ++j) {
                double r2 = 0;
                for (std::size_t q = 0; q != 16; ++q) r2 += (X(i, q) - X(j, q)) * (X(i, q) - X(j, q));
                K(i, j) = std::exp(-0.5 * r2 / 4.0) + (i == j ? 1e-2 : 0.0);
            }
        matrix<double> y(n, 1);
        for (std::size_t i = 0; i != n; ++i) y(i, 0) = ydat(i);
        matrix<double, column_major, cuda_tag> L = copy_to_device(K, cuda_tag());
        kernels::potrf<lower>(L);
        matrix<double, column_major, cuda_tag> z = copy_to_device(y, cuda_tag());
        kernels::trsm<lower, left>(L, z);  // z = L^-1 y
        matrix<double> Lh = copy_to_cpu(L), zh = copy_to_cpu(z);
        matrix<double, column_major, cuda_tag> zbar = z;  // d(1/2 z^T z)/dz = z
        matrix<double> Lbar0(n, n, 0.0);
        for (std::size_t i = 0; i != n; ++i) Lbar0(i, i) = 1.0 / Lh(i, i);  // d(sum log L_ii)/dL_ii
        matrix<double, column_major, cuda_tag> Lbar = copy_to_device(Lbar0, cuda_tag());
        cuda::trsm_backward(false, L, z, zbar, Lbar);
        matrix<double, column_major, cuda_tag> Kbar(n, n);
        cuda::potrf_backward(L, Lbar, Kbar);
        matrix<double> Kinv = inv(K, symm_pos_def());
        matrix<double> alpha = solve(K, y, symm_pos_def(), left());
        matrix<double> ref = Kinv - prod(alpha, trans(alpha));
        ref *= 0.5;
        report("GP NLL adjoint dF/dK vs Remora CPU 1/2(inv(K) - a a^T)", rel_diff(matrix<double>(copy_to_cpu(Kbar)), ref),
               1e-9);
    }
    std::printf("%s (%d failures)\n", failures ? "FAILED" : "PASSED", failures);
    return failures ? 1 : 0;
}
