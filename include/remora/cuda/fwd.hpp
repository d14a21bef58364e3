// remora/cuda/fwd.hpp -- the cuda_tag device and the declarations of its kernel overloads.
//
// Remora binds its kernel calls by qualified name inside templates
// (e.g. kernels::gemm in detail/matrix_expression_classes.hpp:1004-1012,
// bindings::matrix_assign in kernels/matrix_assign.hpp, bindings::generate_normal in
// kernels/random.hpp:44-62), and qualified names are looked up where the template is
// defined. So every cuda_tag overload is declared here, before remora.hpp is parsed;
// remora/cuda.hpp includes this file first and the definitions after remora.hpp.
#ifndef REMORA_CUDA_FWD_HPP
#define REMORA_CUDA_FWD_HPP

#include <cstddef>

#include <remora/detail/traits.hpp>
#include <remora/expression_types.hpp>

namespace remora {

/// \brief Device tag of the B200 (sm_100a) backend; joins cpu_tag, opencl_tag and hip_tag
/// (expression_types.hpp:33-35).
struct cuda_tag {};

namespace cuda {
class device;
}

namespace bindings {
// Dense assignment X = E (X row-major after the dispatcher's transposition,
// kernels/matrix_assign.hpp:76-105).
template <class M, class E, class EOrientation, class TagE, class TagM>
void matrix_assign(matrix_expression<M, cuda_tag>& m, matrix_expression<E, cuda_tag> const& e, row_major,
                   EOrientation, TagE, TagM);

// Scalar assignment X = f(X, t) for the functors Remora's blockwise products issue
// (kernels/matrix_assign.hpp:58-66: X *= alpha after an in-place triangular product).
template <class F, class M, class Orientation>
void matrix_assign(matrix_expression<M, cuda_tag>& m, typename M::value_type t, Orientation);
// Vector assignment v = e for a dense e or alpha * (dense e) (kernels/vector_assign.hpp:
// 58-64), and v = alpha e / v += alpha e with a scalar functor (:72-78).
template <class V, class E, class TagV, class TagE>
void vector_assign(vector_expression<V, cuda_tag>& v, vector_expression<E, cuda_tag> const& e, TagV, TagE);
template <class V, class E, class F, class TagV, class TagE>
void vector_assign_functor(vector_expression<V, cuda_tag>& v, vector_expression<E, cuda_tag> const& e, F f, TagV,
                           TagE);
// RNG fills, the hip_tag overloads of kernels/hip/random.hpp:261-323.
template <class M, class Rng>
void generate_normal(matrix_expression<M, cuda_tag>& m, Rng& rng, typename M::value_type mean,
                     typename M::value_type variance);
template <class M, class Rng>
void generate_uniform(matrix_expression<M, cuda_tag>& m, Rng& rng, typename M::value_type low,
                      typename M::value_type high);
template <class M, class Rng>
void generate_discrete(matrix_expression<M, cuda_tag>& m, Rng& rng, int low, int high);
template <class V, class Rng>
void generate_normal(vector_expression<V, cuda_tag>& v, Rng& rng, typename V::value_type mean,
                     typename V::value_type variance);
template <class V, class Rng>
void generate_uniform(vector_expression<V, cuda_tag>& v, Rng& rng, typename V::value_type low,
                      typename V::value_type high);
template <class V, class Rng>
void generate_discrete(vector_expression<V, cuda_tag>& v, Rng& rng, int low, int high);
}  // namespace bindings

namespace kernels {
// C += alpha * A * B (kernels/gemm.hpp:85-106; hip: kernels/hip/gemm.hpp:90-112).
template <class MatA, class MatB, class MatC>
void gemm(matrix_expression<MatA, cuda_tag> const& A, matrix_expression<MatB, cuda_tag> const& B,
          matrix_expression<MatC, cuda_tag>& C, typename MatC::value_type const& alpha);
// Triangle of C += alpha * A * A^T (kernels/syrk.hpp:55-67; hip: kernels/hip/syrk.hpp:44-85).
template <bool Upper, class MatA, class MatC>
void syrk(matrix_expression<MatA, cuda_tag> const& A, matrix_expression<MatC, cuda_tag>& C,
          typename MatC::value_type const& alpha);
// B <- A^-1 B / B A^-1 (kernels/trsm.hpp:55-65; hip: kernels/hip/trsm.hpp:90-107).
template <class Triangular, class Side, class MatA, class MatB>
void trsm(matrix_expression<MatA, cuda_tag> const& A, matrix_expression<MatB, cuda_tag>& B);
// In-place Cholesky (kernels/potrf.hpp:56-62; hip: kernels/hip/potrf.hpp:131-141).
template <class Triangular, class MatA>
std::size_t potrf(matrix_container<MatA, cuda_tag>& A);
// v += alpha * A x (kernels/gemv.hpp:56-69; hip: kernels/hip/gemv.hpp:45-90).
template <class MatA, class VecX, class VecV>
void gemv(matrix_expression<MatA, cuda_tag> const& A, vector_expression<VecX, cuda_tag> const& x,
          vector_expression<VecV, cuda_tag>& v, typename VecV::value_type const& alpha);
// Triangular solve with one vector (kernels/trsv.hpp:56-65; hip: kernels/hip/trsv.hpp:44-90).
template <class Triangular, class Side, class MatA, class VecV>
void trsv(matrix_expression<MatA, cuda_tag> const& A, vector_expression<VecV, cuda_tag>& v);
// Triangular products b <- A b, B <- A B (kernels/trmv.hpp:54-65, kernels/trmm.hpp:53-64).
template <bool Upper, bool Unit, class MatA, class VecV>
void trmv(matrix_expression<MatA, cuda_tag> const& A, vector_expression<VecV, cuda_tag>& v);
template <bool Upper, bool Unit, class MatA, class MatB>
void trmm(matrix_expression<MatA, cuda_tag> const& A, matrix_expression<MatB, cuda_tag>& B);
// LU with partial pivoting A = P L U in place, P the host permutation Remora's
// pivoting_lu_decomposition keeps (kernels/getrf.hpp:50-59, decompositions.hpp:253-263).
template <typename MatA, typename VecP>
void getrf(matrix_expression<MatA, cuda_tag>& A, vector_expression<VecP, cpu_tag>& P);
// Pivoted Cholesky P^T A P = L L^T in place, returning the rank (kernels/pstrf.hpp:61-70,
// decompositions.hpp:321-328).
template <class Triangular, class MatA, class VecP>
std::size_t pstrf(matrix_expression<MatA, cuda_tag>& A, vector_expression<VecP, cpu_tag>& P);
}  // namespace kernels

}  // namespace remora

#endif
