// remora/cuda/kernels.hpp -- definitions of the cuda_tag kernel overloads declared in
// fwd.hpp. Each maps Remora's orientation-typed views onto the column-major C-ABI the
// same way the reference's HIP backend maps them onto cuBLAS (a row-major matrix is the
// transpose of a column-major one: kernels/hip/gemm.hpp:46-88, kernels/hip/syrk.hpp:
// 61-67, kernels/hip/trsm.hpp:45-88) and enqueues on the result's device stream.
#ifndef REMORA_CUDA_KERNELS_HPP
#define REMORA_CUDA_KERNELS_HPP

#include <cmath>
#include <cstdint>
#include <random>
#include <stdexcept>
#include <type_traits>
#include <utility>
#include <vector>

#include "dense.hpp"

namespace remora {
namespace cuda {
namespace detail {

template <class O>
constexpr int trans_of() {  // 1 when a matrix of orientation O is the transpose of its column-major storage
    return std::is_same<typename O::orientation, row_major>::value ? 1 : 0;
}

template <class T>
struct blas;
template <>
struct blas<double> {
    static int gemm(int ta, int tb, std::size_t m, std::size_t n, std::size_t k, double alpha, double const* A,
                    std::size_t lda, double const* B, std::size_t ldb, double beta, double* C, std::size_t ldc,
                    void* s) {
        return rc_gemm_f64(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, s);
    }
    static int syrk(int up, int t, std::size_t n, std::size_t k, double alpha, double const* A, std::size_t lda,
                    double beta, double* C, std::size_t ldc, void* s) {
        return rc_syrk_f64(up, t, n, k, alpha, A, lda, beta, C, ldc, s);
    }
    static int trsm(int left, int up, int t, int unit, std::size_t m, std::size_t n, double const* A, std::size_t lda,
                    double* B, std::size_t ldb, void* s) {
        return rc_trsm_f64(left, up, t, unit, m, n, 1.0, A, lda, B, ldb, nullptr, s);
    }
    static int potrf(int up, std::size_t n, double* A, std::size_t lda, int* info, void* s) {
        return rc_potrf_f64(up, n, A, lda, info, s);
    }
    static int gemv(int t, std::size_t m, std::size_t n, double alpha, double const* A, std::size_t lda, double const* x,
                    std::size_t incx, double beta, double* y, std::size_t incy, void* s) {
        return rc_gemv_f64(t, m, n, alpha, A, lda, x, incx, beta, y, incy, s);
    }
    static int trsv(int up, int t, int unit, std::size_t n, double const* A, std::size_t lda, double* x, std::size_t incx,
                    void* s) {
        return rc_trsv_f64(up, t, unit, n, A, lda, x, incx, s);
    }
    static int trmv(int up, int t, int unit, std::size_t n, double const* A, std::size_t lda, double* x, std::size_t incx,
                    void* s) {
        return rc_trmv_f64(up, t, unit, n, A, lda, x, incx, s);
    }
    static int trmm(int left, int up, int t, int unit, std::size_t m, std::size_t n, double const* A, std::size_t lda,
                    double* B, std::size_t ldb, void* s) {
        return rc_trmm_f64(left, up, t, unit, m, n, A, lda, B, ldb, s);
    }
    static int axpby(std::size_t n, double alpha, double const* x, std::size_t incx, double beta, double* y, std::size_t incy,
                     void* s) {
        return rc_axpby_f64(n, alpha, x, incx, beta, y, incy, s);
    }
    static int copy2d(int t, std::size_t m, std::size_t n, double alpha, double const* A, std::size_t lda, double* B,
                      std::size_t ldb, void* s) {
        return rc_copy2d_f64(t, m, n, alpha, A, lda, B, ldb, s);
    }
    static int getrf(int rm, std::size_t n, double* A, std::size_t lda, int* piv, int* info, void* s) {
        return rc_getrf_f64(rm, n, A, lda, piv, info, s);
    }
    static int pstrf(int rm, std::size_t n, double* A, std::size_t lda, int* piv, int* rank, void* s) {
        return rc_pstrf_f64(rm, n, A, lda, piv, rank, s);
    }
    static int gather(std::size_t m, std::size_t n, int const* idx, double const* A, std::ptrdiff_t ars,
                      std::ptrdiff_t acs, double* B, std::ptrdiff_t brs, std::ptrdiff_t bcs, void* s) {
        return rc_gather_rows_f64(m, n, idx, A, ars, acs, B, brs, bcs, s);
    }
};
template <>
struct blas<float> {
    static int gemm(int ta, int tb, std::size_t m, std::size_t n, std::size_t k, float alpha, float const* A,
                    std::size_t lda, float const* B, std::size_t ldb, float beta, float* C, std::size_t ldc,
                    void* s) {
        return rc_gemm_f32(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, s);
    }
    static int syrk(int up, int t, std::size_t n, std::size_t k, float alpha, float const* A, std::size_t lda,
                    float beta, float* C, std::size_t ldc, void* s) {
        return rc_syrk_f32(up, t, n, k, alpha, A, lda, beta, C, ldc, s);
    }
    static int trsm(int left, int up, int t, int unit, std::size_t m, std::size_t n, float const* A, std::size_t lda,
                    float* B, std::size_t ldb, void* s) {
        return rc_trsm_f32(left, up, t, unit, m, n, 1.0f, A, lda, B, ldb, nullptr, s);
    }
    static int potrf(int up, std::size_t n, float* A, std::size_t lda, int* info, void* s) {
        return rc_potrf_f32(up, n, A, lda, info, s);
    }
    static int gemv(int t, std::size_t m, std::size_t n, float alpha, float const* A, std::size_t lda, float const* x,
                    std::size_t incx, float beta, float* y, std::size_t incy, void* s) {
        return rc_gemv_f32(t, m, n, alpha, A, lda, x, incx, beta, y, incy, s);
    }
    static int trsv(int up, int t, int unit, std::size_t n, float const* A, std::size_t lda, float* x, std::size_t incx,
                    void* s) {
        return rc_trsv_f32(up, t, unit, n, A, lda, x, incx, s);
    }
    static int trmv(int up, int t, int unit, std::size_t n, float const* A, std::size_t lda, float* x, std::size_t incx,
                    void* s) {
        return rc_trmv_f32(up, t, unit, n, A, lda, x, incx, s);
    }
    static int trmm(int left, int up, int t, int unit, std::size_t m, std::size_t n, float const* A, std::size_t lda,
                    float* B, std::size_t ldb, void* s) {
        return rc_trmm_f32(left, up, t, unit, m, n, A, lda, B, ldb, s);
    }
    static int axpby(std::size_t n, float alpha, float const* x, std::size_t incx, float beta, float* y, std::size_t incy,
                     void* s) {
        return rc_axpby_f32(n, alpha, x, incx, beta, y, incy, s);
    }
    static int copy2d(int t, std::size_t m, std::size_t n, float alpha, float const* A, std::size_t lda, float* B,
                      std::size_t ldb, void* s) {
        return rc_copy2d_f32(t, m, n, alpha, A, lda, B, ldb, s);
    }
    static int getrf(int rm, std::size_t n, float* A, std::size_t lda, int* piv, int* info, void* s) {
        return rc_getrf_f32(rm, n, A, lda, piv, info, s);
    }
    static int pstrf(int rm, std::size_t n, float* A, std::size_t lda, int* piv, int* rank, void* s) {
        return rc_pstrf_f32(rm, n, A, lda, piv, rank, s);
    }
    static int gather(std::size_t m, std::size_t n, int const* idx, float const* A, std::ptrdiff_t ars,
                      std::ptrdiff_t acs, float* B, std::ptrdiff_t brs, std::ptrdiff_t bcs, void* s) {
        return rc_gather_rows_f32(m, n, idx, A, ars, acs, B, brs, bcs, s);
    }
};

/// Per-device status word for potrf (read back to return the pivot, as the reference does).
inline int* status_word(device& dev) {
    thread_local std::map<int, std::shared_ptr<void>> words;
    auto& w = words[dev.id()];
    if (!w) {
        dev.set_device();
        void* p = nullptr;
        check(rc_malloc(&p, sizeof(int)), "rc_malloc");
        w = std::shared_ptr<void>(p, [](void* q) { rc_free(q); });
    }
    return static_cast<int*>(w.get());
}

// The order of rows after Remora's sequence of swaps P (include/remora/permutation.hpp:
// 51-104): forward, row i swapped with row P(i) for i = 0, 1, ...; inverted, the same
// swaps in reverse. Row i of the result is row order[i] of the input.
template <class VecP>
std::vector<int> swap_order(VecP const& P, bool inverted) {
    const std::size_t n = P.size();
    std::vector<int> order(n);
    for (std::size_t i = 0; i != n; ++i) order[i] = (int)i;
    if (!inverted)
        for (std::size_t i = 0; i != n; ++i) std::swap(order[i], order[(std::size_t)P(i)]);
    else
        for (std::size_t i = n; i != 0; --i) std::swap(order[i - 1], order[(std::size_t)P(i - 1)]);
    return order;
}

// Rows of the m x n strided device matrix X (element (i, j) at p + i rs + j cs) reordered
// to `order` in one gather: X -> a dense copy -> back through the row order.
template <class T>
void gather_rows(std::vector<int> const& order, T* p, std::ptrdiff_t rs, std::ptrdiff_t cs, std::size_t m,
                 std::size_t n, device& dev) {
    if (m == 0 || n == 0) return;
    buffer<int> idx(m, dev), ident(m, dev);
    buffer<T> tmp(m * n, dev);
    std::vector<int> id(m);
    for (std::size_t i = 0; i != m; ++i) id[i] = (int)i;
    check(rc_memcpy2d(idx.get(), m * sizeof(int), order.data(), m * sizeof(int), m * sizeof(int), 1, RC_COPY_H2D,
                      dev.stream()),
          "rc_memcpy2d");
    check(rc_memcpy2d(ident.get(), m * sizeof(int), id.data(), m * sizeof(int), m * sizeof(int), 1, RC_COPY_H2D,
                      dev.stream()),
          "rc_memcpy2d");
    check(blas<T>::gather(m, n, idx.get(), p, rs, cs, tmp.get(), 1, (std::ptrdiff_t)m, dev.stream()),
          "rc_gather_rows");
    check(blas<T>::gather(m, n, ident.get(), tmp.get(), 1, (std::ptrdiff_t)m, p, rs, cs, dev.stream()),
          "rc_gather_rows");
    dev.synchronize();
}

// Element strides (rs, cs) of a dense device matrix.
template <class M>
std::pair<std::ptrdiff_t, std::ptrdiff_t> strides_of(M const& A) {
    const std::ptrdiff_t ld = (std::ptrdiff_t)A.raw_storage().leading_dimension;
    return trans_of<typename M::orientation>() ? std::make_pair(ld, std::ptrdiff_t(1)) : std::make_pair(std::ptrdiff_t(1), ld);
}

}  // namespace detail
}  // namespace cuda

// Row and column swaps of cuda_tag matrices and vectors by a host permutation, the
// device counterparts of include/remora/permutation.hpp:51-104 (found by argument-
// dependent lookup from Remora's decompositions).
template <class VecP, class M>
void swap_rows(vector_expression<VecP, cpu_tag> const& P, matrix_expression<M, cuda_tag>& A) {
    auto st = cuda::detail::strides_of(A());
    cuda::detail::gather_rows(cuda::detail::swap_order(P(), false), A().raw_storage().values, st.first, st.second,
                              A().size1(), A().size2(), A().queue());
}
template <class VecP, class M>
void swap_rows_inverted(vector_expression<VecP, cpu_tag> const& P, matrix_expression<M, cuda_tag>& A) {
    auto st = cuda::detail::strides_of(A());
    cuda::detail::gather_rows(cuda::detail::swap_order(P(), true), A().raw_storage().values, st.first, st.second,
                              A().size1(), A().size2(), A().queue());
}
template <class VecP, class M>
void swap_columns(vector_expression<VecP, cpu_tag> const& P, matrix_expression<M, cuda_tag>& A) {
    auto st = cuda::detail::strides_of(A());
    cuda::detail::gather_rows(cuda::detail::swap_order(P(), false), A().raw_storage().values, st.second, st.first,
                              A().size2(), A().size1(), A().queue());
}
template <class VecP, class M>
void swap_columns_inverted(vector_expression<VecP, cpu_tag> const& P, matrix_expression<M, cuda_tag>& A) {
    auto st = cuda::detail::strides_of(A());
    cuda::detail::gather_rows(cuda::detail::swap_order(P(), true), A().raw_storage().values, st.second, st.first,
                              A().size2(), A().size1(), A().queue());
}
template <class VecP, class V>
void swap_rows(vector_expression<VecP, cpu_tag> const& P, vector_expression<V, cuda_tag>& v) {
    cuda::detail::gather_rows(cuda::detail::swap_order(P(), false), v().raw_storage().values,
                              (std::ptrdiff_t)v().raw_storage().stride, std::ptrdiff_t(0), v().size(), 1, v().queue());
}
template <class VecP, class V>
void swap_rows_inverted(vector_expression<VecP, cpu_tag> const& P, vector_expression<V, cuda_tag>& v) {
    cuda::detail::gather_rows(cuda::detail::swap_order(P(), true), v().raw_storage().values,
                              (std::ptrdiff_t)v().raw_storage().stride, std::ptrdiff_t(0), v().size(), 1, v().queue());
}

namespace kernels {

template <typename MatA, typename VecP>
void getrf(matrix_expression<MatA, cuda_tag>& A, vector_expression<VecP, cpu_tag>& P) {
    REMORA_SIZE_CHECK(A().size1() == A().size2());
    REMORA_SIZE_CHECK(P().size() == A().size1());
    typedef typename MatA::value_type T;
    const std::size_t n = A().size1();
    if (n == 0) return;
    auto sa = A().raw_storage();
    cuda::device& dev = A().queue();
    cuda::buffer<int> piv(n, dev), info(1, dev);
    cuda::check(cuda::detail::blas<T>::getrf(cuda::detail::trans_of<typename MatA::orientation>(), n, sa.values,
                                             sa.leading_dimension, piv.get(), info.get(), dev.stream()),
                "rc_getrf");
    std::vector<int> h(n);
    int hinfo = 0;
    cuda::check(rc_memcpy2d(h.data(), n * sizeof(int), piv.get(), n * sizeof(int), n * sizeof(int), 1, RC_COPY_D2H,
                            dev.stream()),
                "rc_memcpy2d");
    cuda::check(rc_memcpy2d(&hinfo, sizeof(int), info.get(), sizeof(int), sizeof(int), 1, RC_COPY_D2H, dev.stream()),
                "rc_memcpy2d");
    dev.synchronize();
    if (hinfo != 0)  // the reference's CPU kernel throws on a zero pivot (kernels/default/getrf.hpp:59)
        throw std::invalid_argument("[getrf] Matrix is rank deficient or numerically unstable");
    for (std::size_t i = 0; i != n; ++i) P()(i) = h[i];
}

template <class Triangular, class MatA, class VecP>
std::size_t pstrf(matrix_expression<MatA, cuda_tag>& A, vector_expression<VecP, cpu_tag>& P) {
    REMORA_SIZE_CHECK(A().size1() == A().size2());
    REMORA_SIZE_CHECK(P().size() == A().size1());
    typedef typename MatA::value_type T;
    const std::size_t n = A().size1();
    if (n == 0) return 0;
    auto sa = A().raw_storage();
    cuda::device& dev = A().queue();
    cuda::buffer<int> piv(n, dev), rank(1, dev);
    // The upper factor is the lower factor of the transpose (kernels/default/pstrf.hpp:152-160).
    const int rm = cuda::detail::trans_of<typename MatA::orientation>() ^ (Triangular::is_upper ? 1 : 0);
    cuda::check(cuda::detail::blas<T>::pstrf(rm, n, sa.values, sa.leading_dimension, piv.get(), rank.get(),
                                             dev.stream()),
                "rc_pstrf");
    std::vector<int> h(n);
    int hrank = 0;
    cuda::check(rc_memcpy2d(h.data(), n * sizeof(int), piv.get(), n * sizeof(int), n * sizeof(int), 1, RC_COPY_D2H,
                            dev.stream()),
                "rc_memcpy2d");
    cuda::check(rc_memcpy2d(&hrank, sizeof(int), rank.get(), sizeof(int), sizeof(int), 1, RC_COPY_D2H, dev.stream()),
                "rc_memcpy2d");
    dev.synchronize();
    for (std::size_t i = 0; i != n; ++i) P()(i) = h[i];
    return (std::size_t)hrank;
}

template <class MatA, class MatB, class MatC>
void gemm(matrix_expression<MatA, cuda_tag> const& A, matrix_expression<MatB, cuda_tag> const& B,
          matrix_expression<MatC, cuda_tag>& C, typename MatC::value_type const& alpha) {
    REMORA_SIZE_CHECK(A().size1() == C().size1());
    REMORA_SIZE_CHECK(B().size2() == C().size2());
    REMORA_SIZE_CHECK(A().size2() == B().size1());
    typedef typename MatC::value_type T;
    static_assert(std::is_same<typename MatA::value_type, T>::value, "[gemm] Arguments do not have same element type");
    static_assert(std::is_same<typename MatB::value_type, T>::value, "[gemm] Arguments do not have same element type");
    auto const& Ae = eval_expression(A);
    auto const& Be = eval_expression(B);
    auto sa = Ae.raw_storage();
    auto sb = Be.raw_storage();
    auto sc = C().raw_storage();
    const int ta = cuda::detail::trans_of<typename std::decay<decltype(Ae)>::type::orientation>();
    const int tb = cuda::detail::trans_of<typename std::decay<decltype(Be)>::type::orientation>();
    const int tc = cuda::detail::trans_of<typename MatC::orientation>();
    const std::size_t m = C().size1(), n = C().size2(), k = A().size2();
    void* s = C().queue().stream();
    if (!tc)
        cuda::check(cuda::detail::blas<T>::gemm(ta, tb, m, n, k, alpha, sa.values, sa.leading_dimension, sb.values,
                                                sb.leading_dimension, T(1), sc.values, sc.leading_dimension, s),
                    "rc_gemm");
    else  // C^T = B^T A^T
        cuda::check(cuda::detail::blas<T>::gemm(1 - tb, 1 - ta, n, m, k, alpha, sb.values, sb.leading_dimension,
                                                sa.values, sa.leading_dimension, T(1), sc.values,
                                                sc.leading_dimension, s),
                    "rc_gemm");
}

template <bool Upper, class MatA, class MatC>
void syrk(matrix_expression<MatA, cuda_tag> const& A, matrix_expression<MatC, cuda_tag>& C,
          typename MatC::value_type const& alpha) {
    REMORA_SIZE_CHECK(A().size1() == C().size1());
    REMORA_SIZE_CHECK(C().size1() == C().size2());
    typedef typename MatC::value_type T;
    auto const& Ae = eval_expression(A);
    auto sa = Ae.raw_storage();
    auto sc = C().raw_storage();
    const int ta = cuda::detail::trans_of<typename std::decay<decltype(Ae)>::type::orientation>();
    const int tc = cuda::detail::trans_of<typename MatC::orientation>();
    const int up = (Upper ? 1 : 0) ^ tc;  // a row-major C's upper triangle is its storage's lower one
    cuda::check(cuda::detail::blas<T>::syrk(up, ta, C().size1(), A().size2(), alpha, sa.values, sa.leading_dimension,
                                            T(1), sc.values, sc.leading_dimension, C().queue().stream()),
                "rc_syrk");
}

template <class Triangular, class Side, class MatA, class MatB>
void trsm(matrix_expression<MatA, cuda_tag> const& A, matrix_expression<MatB, cuda_tag>& B) {
    REMORA_SIZE_CHECK(A().size1() == A().size2());
    typedef typename MatB::value_type T;
    auto const& Ae = eval_expression(A);
    auto sa = Ae.raw_storage();
    auto sb = B().raw_storage();
    const int ta = cuda::detail::trans_of<typename std::decay<decltype(Ae)>::type::orientation>();
    const int tb = cuda::detail::trans_of<typename MatB::orientation>();
    const int up = (Triangular::is_upper ? 1 : 0) ^ ta;  // the triangle as stored
    int left = Side::is_left ? 1 : 0, trans = ta;
    std::size_t m = B().size1(), n = B().size2();
    if (tb) {  // B row-major: solve for B^T on the other side with op(A)^T
        left = 1 - left;
        trans = 1 - ta;
        std::swap(m, n);
    }
    cuda::check(cuda::detail::blas<T>::trsm(left, up, trans, Triangular::is_unit ? 1 : 0, m, n, sa.values,
                                            sa.leading_dimension, sb.values, sb.leading_dimension,
                                            B().queue().stream()),
                "rc_trsm");
}

template <class Triangular, class MatA>
std::size_t potrf(matrix_container<MatA, cuda_tag>& A) {
    REMORA_SIZE_CHECK(A().size1() == A().size2());
    typedef typename MatA::value_type T;
    auto sa = A().raw_storage();
    const int ta = cuda::detail::trans_of<typename MatA::orientation>();
    cuda::device& dev = A().queue();
    int* info = cuda::detail::status_word(dev);
    cuda::check(cuda::detail::blas<T>::potrf((Triangular::is_upper ? 1 : 0) ^ ta, A().size1(), sa.values,
                                             sa.leading_dimension, info, dev.stream()),
                "rc_potrf");
    int h = 0;
    cuda::check(rc_memcpy2d(&h, sizeof(int), info, sizeof(int), sizeof(int), 1, RC_COPY_D2H, dev.stream()),
                "rc_memcpy2d");
    dev.synchronize();
    return (std::size_t)h;  // 0, or the global 1-based index of the failing pivot
}

// v += alpha * A x (kernels/gemv.hpp:56-69; hip: kernels/hip/gemv.hpp:45-90).
template <class MatA, class VecX, class VecV>
void gemv(matrix_expression<MatA, cuda_tag> const& A, vector_expression<VecX, cuda_tag> const& x,
          vector_expression<VecV, cuda_tag>& v, typename VecV::value_type const& alpha) {
    REMORA_SIZE_CHECK(A().size1() == v().size());
    REMORA_SIZE_CHECK(A().size2() == x().size());
    typedef typename VecV::value_type T;
    auto const& Ae = eval_expression(A);
    auto const& xe = eval_expression(x);
    auto sa = Ae.raw_storage();
    auto sx = xe.raw_storage();
    auto sv = v().raw_storage();
    const int ta = cuda::detail::trans_of<typename std::decay<decltype(Ae)>::type::orientation>();
    std::size_t m = A().size1(), n = A().size2();
    if (ta) std::swap(m, n);  // the column-major storage of a row-major A is A^T
    cuda::check(cuda::detail::blas<T>::gemv(ta, m, n, alpha, sa.values, sa.leading_dimension, sx.values, sx.stride,
                                            T(1), sv.values, sv.stride, v().queue().stream()),
                "rc_gemv");
}

// b <- A^-1 b (left) or the solution of x A = b (right) (kernels/trsv.hpp:56-65; hip:
// kernels/hip/trsv.hpp:44-90).
template <class Triangular, class Side, class MatA, class VecV>
void trsv(matrix_expression<MatA, cuda_tag> const& A, vector_expression<VecV, cuda_tag>& v) {
    REMORA_SIZE_CHECK(A().size1() == A().size2());
    REMORA_SIZE_CHECK(A().size2() == v().size());
    typedef typename VecV::value_type T;
    auto const& Ae = eval_expression(A);
    auto sa = Ae.raw_storage();
    auto sv = v().raw_storage();
    const int ta = cuda::detail::trans_of<typename std::decay<decltype(Ae)>::type::orientation>();
    const int up = (Triangular::is_upper ? 1 : 0) ^ ta;  // the triangle as stored
    const int trans = Side::is_left ? ta : 1 - ta;       // x A = b is A^T x = b
    cuda::check(cuda::detail::blas<T>::trsv(up, trans, Triangular::is_unit ? 1 : 0, v().size(), sa.values,
                                            sa.leading_dimension, sv.values, sv.stride, v().queue().stream()),
                "rc_trsv");
}

// b <- A b for the named triangle of A (kernels/trmv.hpp:54-65; hip: kernels/hip/trmv.hpp:44-90).
template <bool Upper, bool Unit, class MatA, class VecV>
void trmv(matrix_expression<MatA, cuda_tag> const& A, vector_expression<VecV, cuda_tag>& v) {
    REMORA_SIZE_CHECK(A().size1() == A().size2());
    REMORA_SIZE_CHECK(A().size2() == v().size());
    typedef typename VecV::value_type T;
    auto const& Ae = eval_expression(A);
    auto sa = Ae.raw_storage();
    auto sv = v().raw_storage();
    const int ta = cuda::detail::trans_of<typename std::decay<decltype(Ae)>::type::orientation>();
    cuda::check(cuda::detail::blas<T>::trmv((Upper ? 1 : 0) ^ ta, ta, Unit ? 1 : 0, v().size(), sa.values,
                                            sa.leading_dimension, sv.values, sv.stride, v().queue().stream()),
                "rc_trmv");
}

// B <- A B for the named triangle of A (kernels/trmm.hpp:53-64; hip: kernels/hip/trmm.hpp:90-106).
template <bool Upper, bool Unit, class MatA, class MatB>
void trmm(matrix_expression<MatA, cuda_tag> const& A, matrix_expression<MatB, cuda_tag>& B) {
    REMORA_SIZE_CHECK(A().size1() == A().size2());
    REMORA_SIZE_CHECK(A().size2() == B().size1());
    typedef typename MatB::value_type T;
    auto const& Ae = eval_expression(A);
    auto sa = Ae.raw_storage();
    auto sb = B().raw_storage();
    const int ta = cuda::detail::trans_of<typename std::decay<decltype(Ae)>::type::orientation>();
    const int tb = cuda::detail::trans_of<typename MatB::orientation>();
    const int up = (Upper ? 1 : 0) ^ ta;
    int left = 1, trans = ta;
    std::size_t m = B().size1(), n = B().size2();
    if (tb) {  // B row-major: B^T <- B^T T^T on the right
        left = 0;
        trans = 1 - ta;
        std::swap(m, n);
    }
    cuda::check(cuda::detail::blas<T>::trmm(left, up, trans, Unit ? 1 : 0, m, n, sa.values, sa.leading_dimension,
                                            sb.values, sb.leading_dimension, B().queue().stream()),
                "rc_trmm");
}

}  // namespace kernels

namespace cuda {

/// Reverse mode of A = L L^T: the full symmetric adjoint Abar of A for the adjoint Lbar
/// of the lower factor L (all FP64, column-major, on the device). No reference
/// counterpart; see rc_potrf_backward_f64.
template <class ML, class MLb, class MAb>
void potrf_backward(matrix_expression<ML, cuda_tag> const& L, matrix_expression<MLb, cuda_tag> const& Lbar,
                    matrix_expression<MAb, cuda_tag>& Abar) {
    static_assert(std::is_same<typename MAb::orientation::orientation, column_major>::value &&
                      std::is_same<typename ML::orientation::orientation, column_major>::value &&
                      std::is_same<typename MLb::orientation::orientation, column_major>::value,
                  "potrf_backward takes column-major matrices");
    auto sl = L().raw_storage();
    auto slb = Lbar().raw_storage();
    auto sa = Abar().raw_storage();
    check(rc_potrf_backward_f64(L().size1(), sl.values, sl.leading_dimension, slb.values, slb.leading_dimension,
                                sa.values, sa.leading_dimension, Abar().queue().stream()),
          "rc_potrf_backward_f64");
}

/// Reverse mode of X = L^-1 B (trans = false) or X = L^-T B (trans = true): Xbar is
/// overwritten by Bbar and the lower triangle of Lbar accumulates the adjoint of L.
template <class ML, class MX, class MXb, class MLb>
void trsm_backward(bool trans, matrix_expression<ML, cuda_tag> const& L, matrix_expression<MX, cuda_tag> const& X,
                   matrix_expression<MXb, cuda_tag>& Xbar, matrix_expression<MLb, cuda_tag>& Lbar) {
    auto sl = L().raw_storage();
    auto sx = X().raw_storage();
    auto sxb = Xbar().raw_storage();
    auto slb = Lbar().raw_storage();
    check(rc_trsm_backward_f64(trans ? 1 : 0, X().size1(), X().size2(), sl.values, sl.leading_dimension, sx.values,
                               sx.leading_dimension, sxb.values, sxb.leading_dimension, slb.values,
                               slb.leading_dimension, Lbar().queue().stream()),
          "rc_trsm_backward_f64");
}

}  // namespace cuda

namespace bindings {

namespace cuda_detail {
// v <- alpha * e + beta * v for a device vector e with dense storage.
template <class V, class E>
void axpby_dense(vector_expression<V, cuda_tag>& v, E const& e, typename V::value_type alpha,
                 typename V::value_type beta) {
    typedef typename V::value_type T;
    auto se = e.raw_storage();
    auto sv = v().raw_storage();
    cuda::check(cuda::detail::blas<T>::axpby(v().size(), alpha, se.values, se.stride, beta, sv.values, sv.stride,
                                             v().queue().stream()),
                "rc_axpby");
}
template <class V, class E>
void assign_dense(vector_expression<V, cuda_tag>& v, E const& e, typename V::value_type scale) {
    axpby_dense(v, e, scale, typename V::value_type(0));
}
template <class V, class E>
void assign_dense(vector_expression<V, cuda_tag>& v, vector_scalar_multiply<E> const& e,
                  typename V::value_type scale) {
    assign_dense(v, e.expression(), scale * e.scalar());
}
}  // namespace cuda_detail

template <class F, class M, class Orientation>
void matrix_assign(matrix_expression<M, cuda_tag>& m, typename M::value_type t, Orientation) {
    typedef typename M::value_type T;
    static_assert(std::is_same<F, typename device_traits<cuda_tag>::template multiply<T>>::value,
                  "cuda_tag: only X *= t is provided as a scalar assignment");
    auto sm = m().raw_storage();
    const int tm = cuda::detail::trans_of<typename M::orientation>();
    const std::size_t rows = tm ? m().size2() : m().size1(), cols = tm ? m().size1() : m().size2();
    cuda::check(cuda::detail::blas<T>::copy2d(0, rows, cols, t, sm.values, sm.leading_dimension, sm.values,
                                              sm.leading_dimension, m().queue().stream()),
                "rc_copy2d");
}

template <class V, class E, class TagV, class TagE>
void vector_assign(vector_expression<V, cuda_tag>& v, vector_expression<E, cuda_tag> const& e, TagV, TagE) {
    cuda_detail::assign_dense(v, e(), typename V::value_type(1));
}

template <class V, class E, class F, class TagV, class TagE>
void vector_assign_functor(vector_expression<V, cuda_tag>& v, vector_expression<E, cuda_tag> const& e, F f, TagV,
                           TagE) {
    typedef typename V::value_type T;
    typedef typename device_traits<cuda_tag>::template multiply_assign<T> Assign;
    typedef typename device_traits<cuda_tag>::template multiply_and_add<T> AddAssign;
    static_assert(std::is_same<F, Assign>::value || std::is_same<F, AddAssign>::value,
                  "cuda_tag: only v = alpha e and v += alpha e are provided as functor assignments");
    cuda_detail::axpby_dense(v, e(), f.m_s, std::is_same<F, AddAssign>::value ? T(1) : T(0));
}

template <class M, class E, class EOrientation, class TagE, class TagM>
void matrix_assign(matrix_expression<M, cuda_tag>& m, matrix_expression<E, cuda_tag> const& e, row_major,
                   EOrientation, TagE, TagM) {
    typedef typename M::value_type T;
    auto const& Ee = eval_expression(e);
    auto se = Ee.raw_storage();
    auto sm = m().raw_storage();
    // m is row-major: its storage is the column-major size2 x size1 matrix m^T.
    const int te = cuda::detail::trans_of<typename std::decay<decltype(Ee)>::type::orientation>();
    cuda::check(cuda::detail::abi<T>::copy(te ? 0 : 1, m().size2(), m().size1(), T(1), se.values, se.leading_dimension,
                                           sm.values, sm.leading_dimension, m().queue().stream()),
                "rc_copy2d");
}

namespace cuda_detail {
template <class Rng>
void draw_key(Rng& rng, std::uint32_t key[4]) {
    // kernels/hip/random.hpp:225-227
    std::uniform_int_distribution<std::uint32_t> dist(0, 0xffffffff);
    for (int i = 0; i != 4; ++i) key[i] = dist(rng);
}
template <class M>
void fill_args(M const& m, float*& p, std::size_t& ld, int& row) {
    static_assert(std::is_same<typename M::value_type, float>::value,
                  "only 32 bit random number types are supported (as kernels/hip/random.hpp:222)");
    auto s = m.raw_storage();
    p = s.values;
    ld = s.leading_dimension;
    row = cuda::detail::trans_of<typename M::orientation>();
}
}  // namespace cuda_detail

template <class M, class Rng>
void generate_normal(matrix_expression<M, cuda_tag>& m, Rng& rng, typename M::value_type mean,
                     typename M::value_type variance) {
    std::uint32_t key[4];
    cuda_detail::draw_key(rng, key);
    float* p; std::size_t ld; int row;
    cuda_detail::fill_args(m(), p, ld, row);
    cuda::check(rc_rng_normal_f32(key, m().size1(), m().size2(), p, ld, row, mean, std::sqrt(variance),
                                  m().queue().stream()),
                "rc_rng_normal_f32");
}
template <class M, class Rng>
void generate_uniform(matrix_expression<M, cuda_tag>& m, Rng& rng, typename M::value_type low,
                      typename M::value_type high) {
    std::uint32_t key[4];
    cuda_detail::draw_key(rng, key);
    float* p; std::size_t ld; int row;
    cuda_detail::fill_args(m(), p, ld, row);
    cuda::check(rc_rng_uniform_f32(key, m().size1(), m().size2(), p, ld, row, low, high, m().queue().stream()),
                "rc_rng_uniform_f32");
}
template <class M, class Rng>
void generate_discrete(matrix_expression<M, cuda_tag>& m, Rng& rng, int low, int high) {
    std::uint32_t key[4];
    cuda_detail::draw_key(rng, key);
    float* p; std::size_t ld; int row;
    cuda_detail::fill_args(m(), p, ld, row);
    cuda::check(rc_rng_discrete_f32(key, m().size1(), m().size2(), p, ld, row, low, high, m().queue().stream()),
                "rc_rng_discrete_f32");
}
// A vector is filled as a 1 x n row-major matrix (kernels/hip/random.hpp:269).
template <class V, class Rng>
void generate_normal(vector_expression<V, cuda_tag>& v, Rng& rng, typename V::value_type mean,
                     typename V::value_type variance) {
    static_assert(std::is_same<typename V::value_type, float>::value, "only 32 bit random number types");
    std::uint32_t key[4];
    cuda_detail::draw_key(rng, key);
    auto s = v().raw_storage();
    cuda::check(rc_rng_normal_f32(key, 1, v().size(), s.values, v().size(), 1, mean, std::sqrt(variance),
                                  v().queue().stream()),
                "rc_rng_normal_f32");
}
template <class V, class Rng>
void generate_uniform(vector_expression<V, cuda_tag>& v, Rng& rng, typename V::value_type low,
                      typename V::value_type high) {
    static_assert(std::is_same<typename V::value_type, float>::value, "only 32 bit random number types");
    std::uint32_t key[4];
    cuda_detail::draw_key(rng, key);
    auto s = v().raw_storage();
    cuda::check(rc_rng_uniform_f32(key, 1, v().size(), s.values, v().size(), 1, low, high, v().queue().stream()),
                "rc_rng_uniform_f32");
}
template <class V, class Rng>
void generate_discrete(vector_expression<V, cuda_tag>& v, Rng& rng, int low, int high) {
    static_assert(std::is_same<typename V::value_type, float>::value, "only 32 bit random number types");
    std::uint32_t key[4];
    cuda_detail::draw_key(rng, key);
    auto s = v().raw_storage();
    cuda::check(rc_rng_discrete_f32(key, 1, v().size(), s.values, v().size(), 1, low, high, v().queue().stream()),
                "rc_rng_discrete_f32");
}

}  // namespace bindings
}  // namespace remora

#endif
