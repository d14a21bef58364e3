// remora/cuda/copy.hpp -- host <-> device transport for the cuda_tag device:
// copy_to_device(cpu expression, cuda_tag()) and copy_to_cpu(cuda expression), the
// interface of include/remora/device_copy.hpp:33-64 and hip/copy.hpp:468-505.
//
// The reference page-locks the user's host memory and lets a kernel read or write it
// over the bus (hip/copy.hpp:131-410). Here a matrix moves in chunks of whole storage
// lines (rows of a row-major target, columns of a column-major one) through two
// page-locked staging chunks per (device, host thread): host threads evaluate the host
// expression straight into one chunk (or unpack it into the host target) while the DMA of
// the other chunk runs, so every element is touched once on the host and the copy engine
// moves page-locked memory at the link's rate. The device side is one dense staging
// matrix in the target's orientation; an orientation change or a strided target is a
// device-side assignment. Both directions synchronise the stream before returning, as the
// reference does.
#ifndef REMORA_CUDA_COPY_HPP
#define REMORA_CUDA_COPY_HPP

#include <algorithm>
#include <cstring>
#include <type_traits>

#include "dense.hpp"

namespace remora {
namespace cuda {

namespace detail {
// Lines [a, b) of an m x n expression in the orientation of its storage: rows of a
// row-major matrix, columns of a column-major one.
template <class E>
auto lines(E&& e, std::size_t a, std::size_t b, std::size_t m, std::size_t n, row_major)
    -> decltype(subrange(std::forward<E>(e), a, b, 0, n)) {
    return subrange(std::forward<E>(e), a, b, 0, n);
}
template <class E>
auto lines(E&& e, std::size_t a, std::size_t b, std::size_t m, std::size_t n, column_major)
    -> decltype(subrange(std::forward<E>(e), 0, m, a, b)) {
    return subrange(std::forward<E>(e), 0, m, a, b);
}
// A host matrix over `count` consecutive lines of a staging chunk.
template <class T, class O>
remora::dense_matrix_adaptor<T, O> chunk_view(T* p, std::size_t count, std::size_t m, std::size_t n) {
    const std::size_t minor = O::index_m(m, n);
    return std::is_same<O, row_major>::value ? remora::dense_matrix_adaptor<T, O>(p, count, n, minor)
                                             : remora::dense_matrix_adaptor<T, O>(p, m, count, minor);
}
// True when M has dense storage in orientation O (its lines can be copied as memory).
template <class M, class O>
struct dense_lines
    : std::integral_constant<bool, std::is_base_of<dense_tag, typename M::storage_type::storage_tag>::value &&
                                       std::is_same<typename M::orientation, O>::value> {};

// Lines [a, b) of the host expression e into the staging lines at buf.
template <class O, class E, class T>
void pack(E const& e, T* buf, std::size_t a, std::size_t b, std::size_t m, std::size_t n, std::true_type) {
    auto st = e.raw_storage();
    const std::size_t minor = O::index_m(m, n);
    for (std::size_t l = a; l != b; ++l)
        std::memcpy(buf + (l - a) * minor, st.values + l * st.leading_dimension, minor * sizeof(T));
}
template <class O, class E, class T>
void pack(E const& e, T* buf, std::size_t a, std::size_t b, std::size_t m, std::size_t n, std::false_type) {
    auto view = chunk_view<T, O>(buf, b - a, m, n);
    noalias(view) = lines(e, a, b, m, n, O());
}
// The staging lines at buf into lines [a, b) of the host target x.
template <class O, class X, class T>
void unpack(X& x, T const* buf, std::size_t a, std::size_t b, std::size_t m, std::size_t n, std::true_type) {
    auto st = x.raw_storage();
    const std::size_t minor = O::index_m(m, n);
    for (std::size_t l = a; l != b; ++l)
        std::memcpy(st.values + l * st.leading_dimension, buf + (l - a) * minor, minor * sizeof(T));
}
template <class O, class X, class T>
void unpack(X& x, T const* buf, std::size_t a, std::size_t b, std::size_t m, std::size_t n, std::false_type) {
    noalias(lines(x, a, b, m, n, O())) = chunk_view<T const, O>(buf, b - a, m, n);
}
}  // namespace detail

template <class E>
class matrix_transport_to_host : public matrix_expression<matrix_transport_to_host<E>, cpu_tag> {
public:
    typedef typename E::const_closure_type expression_closure_type;
    typedef typename E::value_type value_type;
    typedef typename E::size_type size_type;
    typedef value_type const& const_reference;
    typedef const_reference reference;
    typedef matrix_transport_to_host const_closure_type;
    typedef matrix_transport_to_host closure_type;
    typedef unknown_storage storage_type;
    typedef unknown_storage const_storage_type;
    typedef blockwise<typename E::evaluation_category::tag> evaluation_category;
    typedef typename E::orientation orientation;
    typedef no_iterator const_major_iterator;
    typedef no_iterator major_iterator;

    explicit matrix_transport_to_host(expression_closure_type const& e) : m_expression(e) {}
    size_type size1() const { return m_expression.size1(); }
    size_type size2() const { return m_expression.size2(); }
    typename device_traits<cpu_tag>::queue_type& queue() const { return device_traits<cpu_tag>::default_queue(); }
    no_functor elements() const { return no_functor(); }

    template <class MatX>
    void assign_to(matrix_expression<MatX, cpu_tag>& X) const {
        typedef typename MatX::orientation::orientation XO;
        const std::size_t m = size1(), n = size2();
        if (m == 0 || n == 0) return;
        // A dense device copy in X's orientation, then chunks of its lines through the
        // page-locked staging: the DMA of chunk k + 1 runs while chunk k is unpacked.
        matrix<value_type, XO, cuda_tag> staged(m_expression);
        device& dev = staged.queue();
        const std::size_t major = XO::index_M(m, n), minor = XO::index_m(m, n);
        const std::size_t line = minor * sizeof(value_type);
        const value_type* src = staged.raw_storage().values;
        if (line > host_staging::chunk_bytes) {  // a single line larger than a chunk
            remora::matrix<value_type, XO> host(m, n);
            check(rc_memcpy2d(host.raw_storage().values, line, src, line, line, major, RC_COPY_D2H, dev.stream()),
                  "rc_memcpy2d");
            dev.synchronize();
            noalias(X) = host;
            return;
        }
        host_staging& st = host_staging::of(dev);
        const std::size_t per = host_staging::chunk_bytes / line;
        const std::size_t chunks = (major + per - 1) / per;
        auto issue = [&](std::size_t k) {
            const int c = (int)(k & 1);
            const std::size_t l0 = k * per, nl = std::min(per, major - l0);
            st.wait(c);
            check(rc_memcpy2d(st.chunk(c), line, src + l0 * minor, line, line, nl, RC_COPY_D2H, dev.stream()),
                  "rc_memcpy2d");
            st.record(c, dev.stream());
        };
        issue(0);
        if (chunks > 1) issue(1);
        for (std::size_t k = 0; k < chunks; ++k) {
            const int c = (int)(k & 1);
            const std::size_t l0 = k * per, nl = std::min(per, major - l0);
            st.wait(c);
            value_type const* buf = static_cast<value_type const*>(st.chunk(c));
            parallel_lines(nl, [&](std::size_t b, std::size_t e) {
                detail::unpack<XO>(X(), buf + b * minor, l0 + b, l0 + e, m, n, detail::dense_lines<MatX, XO>());
            });
            if (k + 2 < chunks) issue(k + 2);
        }
        dev.synchronize();
    }
    template <class MatX>
    void plus_assign_to(matrix_expression<MatX, cpu_tag>& X) const {
        typename matrix_temporary<MatX>::type tmp(size1(), size2());
        assign_to(tmp);
        plus_assign(X, tmp);
    }

private:
    expression_closure_type m_expression;
};

template <class E>
class matrix_transport_to_device : public matrix_expression<matrix_transport_to_device<E>, cuda_tag> {
public:
    typedef typename E::const_closure_type expression_closure_type;
    typedef typename E::value_type value_type;
    typedef typename E::size_type size_type;
    typedef value_type const& const_reference;
    typedef const_reference reference;
    typedef matrix_transport_to_device const_closure_type;
    typedef matrix_transport_to_device closure_type;
    typedef unknown_storage storage_type;
    typedef unknown_storage const_storage_type;
    typedef blockwise<typename E::evaluation_category::tag> evaluation_category;
    typedef typename E::orientation orientation;
    typedef no_iterator const_major_iterator;
    typedef no_iterator major_iterator;

    matrix_transport_to_device(expression_closure_type const& e, device& queue) : m_expression(e), m_queue(&queue) {}
    size_type size1() const { return m_expression.size1(); }
    size_type size2() const { return m_expression.size2(); }
    device& queue() const { return *m_queue; }
    no_functor elements() const { return no_functor(); }

    template <class MatX>
    void assign_to(matrix_expression<MatX, cuda_tag>& X) const {
        typedef typename MatX::orientation::orientation XO;
        const std::size_t m = size1(), n = size2();
        if (m == 0 || n == 0) return;
        // Chunks of X-oriented lines of the host expression, evaluated by host threads into
        // a page-locked chunk while the other chunk's DMA runs, into a dense device staging
        // matrix; then a device assignment into X (which may be a strided view).
        matrix<value_type, XO, cuda_tag> staged(m, n, *m_queue);
        const std::size_t major = XO::index_M(m, n), minor = XO::index_m(m, n);
        const std::size_t line = minor * sizeof(value_type);
        value_type* dst = staged.raw_storage().values;
        if (line > host_staging::chunk_bytes) {  // a single line larger than a chunk
            remora::matrix<value_type, XO> host(m_expression);
            check(rc_memcpy2d(dst, line, host.raw_storage().values, line, line, major, RC_COPY_H2D,
                              m_queue->stream()),
                  "rc_memcpy2d");
            m_queue->synchronize();
        } else {
            host_staging& st = host_staging::of(*m_queue);
            const std::size_t per = host_staging::chunk_bytes / line;
            int c = 0;
            for (std::size_t l0 = 0; l0 < major; l0 += per, c ^= 1) {
                const std::size_t nl = std::min(per, major - l0);
                st.wait(c);
                value_type* buf = static_cast<value_type*>(st.chunk(c));
                parallel_lines(nl, [&](std::size_t b, std::size_t e) {
                    detail::pack<XO>(m_expression, buf + b * minor, l0 + b, l0 + e, m, n,
                                     detail::dense_lines<typename std::decay<expression_closure_type>::type, XO>());
                });
                check(rc_memcpy2d(dst + l0 * minor, line, buf, line, line, nl, RC_COPY_H2D, m_queue->stream()),
                      "rc_memcpy2d");
                st.record(c, m_queue->stream());
            }
        }
        assign(X, staged);
        m_queue->synchronize();
    }
    template <class MatX>
    void plus_assign_to(matrix_expression<MatX, cuda_tag>& X) const;  // not provided: device += host

private:
    expression_closure_type m_expression;
    device* m_queue;
};

/// Device vector (dense storage, any stride) -> host vector expression: one pitched copy.
template <class E>
class vector_transport_to_host : public vector_expression<vector_transport_to_host<E>, cpu_tag> {
public:
    typedef typename E::const_closure_type expression_closure_type;
    typedef typename E::value_type value_type;
    typedef typename E::size_type size_type;
    typedef value_type const& const_reference;
    typedef const_reference reference;
    typedef vector_transport_to_host const_closure_type;
    typedef vector_transport_to_host closure_type;
    typedef unknown_storage storage_type;
    typedef unknown_storage const_storage_type;
    typedef blockwise<typename E::evaluation_category::tag> evaluation_category;
    typedef no_iterator const_iterator;
    typedef no_iterator iterator;

    explicit vector_transport_to_host(expression_closure_type const& e) : m_expression(e) {}
    size_type size() const { return m_expression.size(); }
    typename device_traits<cpu_tag>::queue_type& queue() const { return device_traits<cpu_tag>::default_queue(); }

    template <class VecX>
    void assign_to(vector_expression<VecX, cpu_tag>& x) const {
        auto const& ev = eval_expression(m_expression);
        auto se = ev.raw_storage();
        auto sx = x().raw_storage();
        device& dev = ev.queue();
        if (size())
            check(rc_memcpy2d(sx.values, sx.stride * sizeof(value_type), se.values, se.stride * sizeof(value_type),
                              sizeof(value_type), size(), RC_COPY_D2H, dev.stream()),
                  "rc_memcpy2d");
        dev.synchronize();
    }
    template <class VecX>
    void plus_assign_to(vector_expression<VecX, cpu_tag>& x) const {
        remora::vector<value_type> tmp(size());
        assign_to(tmp);
        plus_assign(x, tmp);
    }

private:
    expression_closure_type m_expression;
};

/// Host vector expression -> device vector (dense storage, any stride): the values are
/// evaluated into a contiguous host vector, then one pitched copy.
template <class E>
class vector_transport_to_device : public vector_expression<vector_transport_to_device<E>, cuda_tag> {
public:
    typedef typename E::const_closure_type expression_closure_type;
    typedef typename E::value_type value_type;
    typedef typename E::size_type size_type;
    typedef value_type const& const_reference;
    typedef const_reference reference;
    typedef vector_transport_to_device const_closure_type;
    typedef vector_transport_to_device closure_type;
    typedef unknown_storage storage_type;
    typedef unknown_storage const_storage_type;
    typedef blockwise<typename E::evaluation_category::tag> evaluation_category;
    typedef no_iterator const_iterator;
    typedef no_iterator iterator;

    vector_transport_to_device(expression_closure_type const& e, device& queue) : m_expression(e), m_queue(&queue) {}
    size_type size() const { return m_expression.size(); }
    device& queue() const { return *m_queue; }

    template <class VecX>
    void assign_to(vector_expression<VecX, cuda_tag>& x) const {
        remora::vector<value_type> host(m_expression);
        auto sx = x().raw_storage();
        if (size())
            check(rc_memcpy2d(sx.values, sx.stride * sizeof(value_type), host.raw_storage().values,
                              sizeof(value_type), sizeof(value_type), size(), RC_COPY_H2D, m_queue->stream()),
                  "rc_memcpy2d");
        m_queue->synchronize();
    }
    template <class VecX>
    void plus_assign_to(vector_expression<VecX, cuda_tag>& x) const;  // not provided: device += host

private:
    expression_closure_type m_expression;
    device* m_queue;
};

}  // namespace cuda

template <class E>
cuda::vector_transport_to_host<E> copy_to_cpu(vector_expression<E, cuda_tag> const& e) {
    return cuda::vector_transport_to_host<E>(e());
}

template <class E>
cuda::vector_transport_to_device<E> copy_to_device(vector_expression<E, cpu_tag> const& e, cuda_tag,
                                                   cuda::device& queue = device_traits<cuda_tag>::default_queue()) {
    return cuda::vector_transport_to_device<E>(e(), queue);
}

template <class E>
E const& copy_to_device(vector_expression<E, cuda_tag> const& e, cuda_tag) {
    return e();
}

template <class E>
cuda::matrix_transport_to_host<E> copy_to_cpu(matrix_expression<E, cuda_tag> const& e) {
    return cuda::matrix_transport_to_host<E>(e());
}

template <class E>
cuda::matrix_transport_to_device<E> copy_to_device(matrix_expression<E, cpu_tag> const& e, cuda_tag,
                                                   cuda::device& queue = device_traits<cuda_tag>::default_queue()) {
    return cuda::matrix_transport_to_device<E>(e(), queue);
}

/// cuda -> cuda is the expression itself (the reference's hip twin forgets the return,
/// hip/copy.hpp:496-502).
template <class E>
E const& copy_to_device(matrix_expression<E, cuda_tag> const& e, cuda_tag) {
    return e();
}

}  // namespace remora

#endif
