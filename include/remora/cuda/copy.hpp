// remora/cuda/copy.hpp -- host <-> device transport for the cuda_tag device:
// copy_to_device(cpu expression, cuda_tag()) and copy_to_cpu(cuda expression), the
// interface of include/remora/device_copy.hpp:33-64 and hip/copy.hpp:468-505.
// Pitched copies (rc_memcpy2d) replace the reference's mapped host memory plus an
// assign kernel over PCIe (hip/copy.hpp:277-294); an orientation change is a transposing
// copy on the device. Both directions synchronise the stream before returning.
#ifndef REMORA_CUDA_COPY_HPP
#define REMORA_CUDA_COPY_HPP

#include "dense.hpp"

namespace remora {
namespace cuda {

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
        // A device copy with X's orientation, then one pitched device-to-host copy.
        matrix<value_type, XO, cuda_tag> staged(m_expression);
        device& dev = staged.queue();
        auto xs = X().raw_storage();
        const std::size_t major = XO::index_M(size1(), size2()), minor = XO::index_m(size1(), size2());
        check(rc_memcpy2d(xs.values, xs.leading_dimension * sizeof(value_type), staged.raw_storage().values,
                          minor * sizeof(value_type), minor * sizeof(value_type), major, RC_COPY_D2H, dev.stream()),
              "rc_memcpy2d");
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
        // Host values in X's orientation, one pitched host-to-device copy into a dense
        // staging matrix, then a device assignment into X (which may be a strided view).
        remora::matrix<value_type, XO> host(m_expression);
        matrix<value_type, XO, cuda_tag> staged(size1(), size2(), *m_queue);
        const std::size_t major = XO::index_M(size1(), size2()), minor = XO::index_m(size1(), size2());
        check(rc_memcpy2d(staged.raw_storage().values, minor * sizeof(value_type), host.raw_storage().values,
                          minor * sizeof(value_type), minor * sizeof(value_type), major, RC_COPY_H2D,
                          m_queue->stream()),
              "rc_memcpy2d");
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
