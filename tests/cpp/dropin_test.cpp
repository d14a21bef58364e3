// Drop-in test of the cuda_tag device: a Remora program in which only the device tag
// changes. Checks, against Remora's own CPU kernels on the same inputs, the hot path of
// the reference's HIP tests (Test/hip_prod.cpp, hip_syrk.cpp, hip_triangular_solve.cpp,
// hip_cholesky.cpp, hip_random.cpp) through the unchanged API: copy_to_device,
// noalias(C) (+)= alpha * prod(A, B) with trans() views, kernels::syrk, kernels::trsm,
// kernels::potrf, cholesky_decomposition + solve, solve(A, B, symm_pos_def(), left()),
// normal(...) fills, copy_to_cpu. Prints one line per check and exits non-zero on failure.
#include <remora/cuda.hpp>
#include <remora/remora.hpp>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
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

// Test/getrf.cpp:16-30: a matrix whose partial pivoting always picks the next row.
matrix<double> createLU(std::size_t n) {
    matrix<double> L(n, n, 0.0), U(n, n, 0.0);
    for (std::size_t i = 0; i != n; ++i) {
        for (std::size_t j = 0; j < i; ++j) L(i, j) = 3 - 3.0 / n * std::abs((int)i - (int)j);
        U(i, i) = 0.5 / n * i + 1;
        L(i, i) = 1;
    }
    matrix<double> A = prod(L, U);
    return A;
}

// Test/symm_solve.cpp:17-36: symmetric positive semidefinite of the given rank.
matrix<double> createSymmRank(std::size_t n, std::size_t rank) {
    matrix<double> R(n, n, 0.0);
    for (std::size_t i = 0; i != n; ++i) {
        for (std::size_t j = 0; j < std::min(i, rank); ++j) R(i, j) = 0.2 / std::abs((int)i - (int)j);
        if (i < rank) R(i, i) = 0.5 / n * i + 1;
    }
    matrix<double> A = prod(R, trans(R));
    if (rank != n)
        for (std::size_t i = 0; i != rank / 2; ++i) {
            A.swap_rows(2 * i, n - i - 1);
            A.swap_columns(2 * i, n - i - 1);
        }
    return A;
}

// kernels::getrf, pivoting_lu_decomposition and symm_pos_semi_definite_solver on the
// device (decompositions.hpp:253-263, :321-328) against the same classes on the CPU.
template <class O>
void pivoting_tests(char const* tag) {
    char name[128];
    {
        const std::size_t n = 123;  // Test/getrf.cpp:38
        matrix<double, O> A = createLU(n);
        permutation_matrix P(n), Pd(n);
        matrix<double, O> dec = A;
        kernels::getrf(dec, P);
        matrix<double, O, cuda_tag> decd = copy_to_device(A, cuda_tag());
        kernels::getrf(decd, Pd);
        matrix<double> got = copy_to_cpu(decd);
        std::size_t same = 0;
        for (std::size_t i = 0; i != n; ++i) same += P(i) == Pd(i);
        std::snprintf(name, sizeof(name), "kernels::getrf n=123 %s: pivots as the CPU's", tag);
        report(name, double(n - same), 0.0);
        std::snprintf(name, sizeof(name), "kernels::getrf n=123 %s: factors", tag);
        report(name, rel_diff(got, dec), 1e-13);
        matrix<double> up(n, n, 0.0);
        for (std::size_t r = 0; r != n; ++r)
            for (std::size_t c = r; c != n; ++c) up(r, c) = got(r, c);
        matrix<double> testA = triangular_prod<unit_lower>(got, up);
        swap_rows_inverted(Pd, testA);
        std::snprintf(name, sizeof(name), "kernels::getrf n=123 %s: max|A - P L U| (Test/getrf.cpp)", tag);
        report(name, max(abs(A - testA)), 1e-12);
    }
    {
        const std::size_t n = 300, k = 7;
        std::mt19937 gen(31);
        std::uniform_real_distribution<double> u(0, 1);
        matrix<double, O> A(n, n), B(n, k), Br(k, n);
        for (std::size_t i = 0; i != n; ++i)
            for (std::size_t j = 0; j != n; ++j) A(i, j) = u(gen) + (i == j ? 0.1 : 0.0);
        for (std::size_t i = 0; i != n; ++i)
            for (std::size_t j = 0; j != k; ++j) B(i, j) = Br(j, i) = u(gen) - 0.5;
        pivoting_lu_decomposition<matrix<double, O>> lu(A);
        matrix<double, O, cuda_tag> Ad = copy_to_device(A, cuda_tag());
        pivoting_lu_decomposition<matrix<double, O, cuda_tag>> lud(Ad);
        matrix<double, O> X = B, Xr = Br;
        lu.solve(X, left());
        lu.solve(Xr, right());
        matrix<double, O, cuda_tag> Xd = copy_to_device(B, cuda_tag()), Xrd = copy_to_device(Br, cuda_tag());
        lud.solve(Xd, left());
        lud.solve(Xrd, right());
        std::snprintf(name, sizeof(name), "pivoting_lu_decomposition n=300 %s: A X = B", tag);
        report(name, rel_diff(matrix<double>(copy_to_cpu(Xd)), X), 1e-12);
        std::snprintf(name, sizeof(name), "pivoting_lu_decomposition n=300 %s: X A = B", tag);
        report(name, rel_diff(matrix<double>(copy_to_cpu(Xrd)), Xr), 1e-12);
        vector<double> b(n), bd_h(n);
        for (std::size_t i = 0; i != n; ++i) b(i) = B(i, 0);
        vector<double, cuda_tag> bd = copy_to_device(b, cuda_tag());
        lu.solve(b, left());
        lud.solve(bd, left());
        bd_h = copy_to_cpu(bd);
        std::snprintf(name, sizeof(name), "pivoting_lu_decomposition n=300 %s: vector solve", tag);
        report(name, rel_diff(to_matrix(bd_h, 1, n), to_matrix(b, 1, n)), 1e-12);
    }
    for (std::size_t rank : {std::size_t(128), std::size_t(50)}) {  // Test/symm_solve.cpp:191, :289
        const std::size_t n = 128, k = 151;
        matrix<double> A = createSymmRank(n, rank);
        matrix<double, O> B(n, k);
        for (std::size_t i = 0; i != n; ++i)
            for (std::size_t j = 0; j < k; ++j) B(i, j) = 0.1 * j + (1.0 / n) * i;
        symm_pos_semi_definite_solver<matrix<double, O>> cpu(A);
        matrix<double, O, cuda_tag> Ad = copy_to_device(matrix<double, O>(A), cuda_tag());
        symm_pos_semi_definite_solver<matrix<double, O, cuda_tag>> dev(Ad);
        std::snprintf(name, sizeof(name), "symm_pos_semi_definite_solver n=128 rank %zu %s: rank", rank, tag);
        report(name, std::abs(double(dev.rank()) - double(cpu.rank())), 0.0);
        matrix<double, O> X = B;
        cpu.solve(X, left());
        matrix<double, O, cuda_tag> Xd = copy_to_device(B, cuda_tag());
        dev.solve(Xd, left());
        matrix<double> Xh = copy_to_cpu(Xd);
        std::snprintf(name, sizeof(name), "symm_pos_semi_definite_solver n=128 rank %zu %s: X vs CPU", rank, tag);
        report(name, rel_diff(Xh, X), 1e-10);
        matrix<double> diff = prod(A, Xh) - B;
        std::snprintf(name, sizeof(name), "symm_pos_semi_definite_solver rank %zu %s: max|A(AX - B)|", rank, tag);
        report(name, max(abs(prod(A, diff))), 1e-12);
    }
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
    pivoting_tests<row_major>("row-major");
    pivoting_tests<column_major>("column-major");
    {
        // Transport through the page-locked chunks: several chunks per matrix, both
        // orientations on both sides, strided (subrange) targets and an expression source;
        // every element must arrive bit for bit.
        const std::size_t m = 3001, n = 1537;  // 36.9 MB of FP64: five 8 MiB chunks
        std::mt19937 gen(77);
        std::uniform_real_distribution<double> u(-1, 1);
        matrix<double> A(m, n), B(m, n);
        for (std::size_t i = 0; i != m; ++i)
            for (std::size_t j = 0; j != n; ++j) {
                A(i, j) = u(gen);
                B(i, j) = u(gen);
            }
        matrix<double, column_major, cuda_tag> Ac = copy_to_device(A, cuda_tag());
        matrix<double, row_major, cuda_tag> Ar = copy_to_device(A, cuda_tag());
        matrix<double> back_c = copy_to_cpu(Ac), back_r = copy_to_cpu(Ar);
        matrix<double, column_major> back_cc = copy_to_cpu(Ar);
        report("transport 3001x1537 FP64 to column-major and back", rel_diff(back_c, A), 0.0);
        report("transport 3001x1537 FP64 to row-major and back", rel_diff(back_r, A), 0.0);
        report("transport row-major device to column-major host", rel_diff(back_cc, A), 0.0);
        matrix<double, row_major, cuda_tag> E = copy_to_device(2.0 * A - B, cuda_tag());
        matrix<double> Eh = 2.0 * A - B;
        report("transport of a host expression (2 A - B)", rel_diff(matrix<double>(copy_to_cpu(E)), Eh), 0.0);
        matrix<double, column_major, cuda_tag> big(m + 40, n + 30, 0.0);
        noalias(subrange(big, 17, 17 + m, 5, 5 + n)) = copy_to_device(A, cuda_tag());
        matrix<double> bigh = copy_to_cpu(big);
        report("transport into a strided device view", rel_diff(matrix<double>(subrange(bigh, 17, 17 + m, 5, 5 + n)), A),
               0.0);
        double outside = 0;
        for (std::size_t i = 0; i != m + 40; ++i)
            for (std::size_t j = 0; j != n + 30; ++j)
                if (i < 17 || i >= 17 + m || j < 5 || j >= 5 + n) outside += std::abs(bigh(i, j));
        report("transport leaves the rest of the device matrix alone", outside, 0.0);
        matrix<double> hv(m + 3, n + 9, -1.0);
        noalias(subrange(hv, 2, 2 + m, 4, 4 + n)) = copy_to_cpu(Ac);
        report("transport into a strided host view", rel_diff(matrix<double>(subrange(hv, 2, 2 + m, 4, 4 + n)), A), 0.0);
        matrix<float, row_major, cuda_tag> Af = copy_to_device(matrix<float>(A), cuda_tag());
        report("transport FP32 round trip", rel_diff(matrix<float>(copy_to_cpu(Af)), matrix<float>(A)), 0.0);
    }
    {
        // Transport rates (reported, not checked): a 8192 x 8192 FP64 matrix (512 MiB) to the
        // device and back through the cuda_tag transports, next to one plain DMA of the same
        // bytes from page-locked host memory (the link's rate).
        const std::size_t n = 8192, bytes = n * n * sizeof(double);
        matrix<double> H(n, n);
        for (std::size_t i = 0; i != n; ++i)
            for (std::size_t j = 0; j != n; ++j) H(i, j) = double(i) - 0.5 * double(j);
        matrix<double, row_major, cuda_tag> D(n, n);
        cuda::device& dev = device_traits<cuda_tag>::default_queue();
        auto seconds = [](std::chrono::steady_clock::time_point t0) {
            return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        };
        noalias(D) = copy_to_device(H, cuda_tag());  // first use: staging chunks allocated
        auto t0 = std::chrono::steady_clock::now();
        noalias(D) = copy_to_device(H, cuda_tag());
        const double h2d = seconds(t0);
        matrix<double> H2(n, n);
        noalias(H2) = copy_to_cpu(D);
        t0 = std::chrono::steady_clock::now();
        noalias(H2) = copy_to_cpu(D);
        const double d2h = seconds(t0);
        report("transport 8192x8192 FP64 round trip exact", rel_diff(H2, H), 0.0);
        void* pinned = nullptr;
        cuda::check(rc_host_alloc(&pinned, bytes), "rc_host_alloc");
        std::memcpy(pinned, H.raw_storage().values, bytes);
        cuda::check(rc_memcpy2d(D.raw_storage().values, bytes, pinned, bytes, bytes, 1, RC_COPY_H2D, dev.stream()),
                    "rc_memcpy2d");
        dev.synchronize();
        t0 = std::chrono::steady_clock::now();
        cuda::check(rc_memcpy2d(D.raw_storage().values, bytes, pinned, bytes, bytes, 1, RC_COPY_H2D, dev.stream()),
                    "rc_memcpy2d");
        dev.synchronize();
        const double link_h2d = seconds(t0);
        t0 = std::chrono::steady_clock::now();
        cuda::check(rc_memcpy2d(pinned, bytes, D.raw_storage().values, bytes, bytes, 1, RC_COPY_D2H, dev.stream()),
                    "rc_memcpy2d");
        dev.synchronize();
        const double link_d2h = seconds(t0);
        rc_host_free(pinned);
        t0 = std::chrono::steady_clock::now();
        cuda::check(rc_memcpy2d(D.raw_storage().values, bytes, H.raw_storage().values, bytes, bytes, 1, RC_COPY_H2D,
                                dev.stream()),
                    "rc_memcpy2d");
        dev.synchronize();
        const double pageable_h2d = seconds(t0);
        std::printf("transport rate 512 MiB FP64: copy_to_device %.1f GB/s, copy_to_cpu %.1f GB/s; one DMA from "
                    "page-locked memory H2D %.1f GB/s, D2H %.1f GB/s; one DMA from pageable memory H2D %.1f GB/s\n",
                    bytes / h2d / 1e9, bytes / d2h / 1e9, bytes / link_h2d / 1e9, bytes / link_d2h / 1e9,
                    bytes / pageable_h2d / 1e9);
    }
    std::printf("%s (%d failures)\n", failures ? "FAILED" : "PASSED", failures);
    return failures ? 1 : 0;
}
