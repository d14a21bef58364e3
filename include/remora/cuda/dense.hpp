// remora/cuda/dense.hpp -- dense containers and proxies on the cuda_tag device.
//
// The same interface as the hip_tag containers (include/remora/hip/dense.hpp:54-740):
// matrix<T, Orientation, cuda_tag> owns device memory, dense_matrix_adaptor<..., cuda_tag>
// is the strided view that trans(), subrange(), rows() produce through the generic
// optimizers of dense.hpp:160-275, vector<T, cuda_tag> / dense_vector_adaptor for vectors.
// Storage is Remora's own dense_matrix_storage{values, leading_dimension}
// (detail/storage.hpp:71-91) holding a device pointer.
#ifndef REMORA_CUDA_DENSE_HPP
#define REMORA_CUDA_DENSE_HPP

#include <type_traits>

#include "device.hpp"

namespace remora {
namespace cuda {
namespace detail {

template <class T>
struct abi;
template <>
struct abi<double> {
    static int fill(std::size_t m, std::size_t n, double v, double* A, std::size_t lda, void* s) {
        return rc_fill_f64(m, n, v, A, lda, s);
    }
    static int copy(int trans, std::size_t m, std::size_t n, double alpha, double const* A, std::size_t lda, double* B,
                    std::size_t ldb, void* s) {
        return rc_copy2d_f64(trans, m, n, alpha, A, lda, B, ldb, s);
    }
};
template <>
struct abi<float> {
    static int fill(std::size_t m, std::size_t n, float v, float* A, std::size_t lda, void* s) {
        return rc_fill_f32(m, n, v, A, lda, s);
    }
    static int copy(int trans, std::size_t m, std::size_t n, float alpha, float const* A, std::size_t lda, float* B,
                    std::size_t ldb, void* s) {
        return rc_copy2d_f32(trans, m, n, alpha, A, lda, B, ldb, s);
    }
};

/// Fill a size1 x size2 strided device matrix of the given orientation.
template <class T, class Orientation>
void fill(T* values, std::size_t ld, std::size_t size1, std::size_t size2, T v, device& dev) {
    if (size1 == 0 || size2 == 0) return;
    const bool row = std::is_same<typename Orientation::orientation, row_major>::value;
    check(abi<T>::fill(row ? size2 : size1, row ? size1 : size2, v, values, ld, dev.stream()), "rc_fill");
}

}  // namespace detail
}  // namespace cuda

/// \brief Strided view of device memory (the cuda_tag specialisation of dense_matrix_adaptor).
template <class T, class Orientation, class Tag>
class dense_matrix_adaptor<T, Orientation, Tag, cuda_tag>
    : public matrix_expression<dense_matrix_adaptor<T, Orientation, Tag, cuda_tag>, cuda_tag> {
public:
    typedef std::size_t size_type;
    typedef typename std::remove_const<T>::type value_type;
    typedef value_type const& const_reference;
    typedef T& reference;
    typedef dense_matrix_adaptor closure_type;
    typedef dense_matrix_adaptor<value_type const, Orientation, Tag, cuda_tag> const_closure_type;
    typedef dense_matrix_storage<T, Tag> storage_type;
    typedef dense_matrix_storage<value_type const, Tag> const_storage_type;
    typedef Orientation orientation;
    typedef elementwise<dense_tag> evaluation_category;

    template <class U, class Tag2>
    dense_matrix_adaptor(dense_matrix_adaptor<U, Orientation, Tag2, cuda_tag> const& e)
        : m_storage(e.raw_storage()), m_queue(&e.queue()), m_size1(e.size1()), m_size2(e.size2()) {}
    dense_matrix_adaptor(storage_type storage, cuda::device& queue, size_type size1, size_type size2)
        : m_storage(storage), m_queue(&queue), m_size1(size1), m_size2(size2) {}
    dense_matrix_adaptor(matrix<value_type, Orientation, cuda_tag> const& m)
        : m_storage(m.raw_storage()), m_queue(&m.queue()), m_size1(m.size1()), m_size2(m.size2()) {}
    dense_matrix_adaptor(matrix<value_type, Orientation, cuda_tag>& m)
        : m_storage(m.raw_storage()), m_queue(&m.queue()), m_size1(m.size1()), m_size2(m.size2()) {}

    dense_matrix_adaptor& operator=(dense_matrix_adaptor const& e) {
        return assign(*this, typename matrix_temporary<dense_matrix_adaptor>::type(e));
    }
    template <class E>
    dense_matrix_adaptor& operator=(matrix_expression<E, cuda_tag> const& e) {
        return assign(*this, typename matrix_temporary<dense_matrix_adaptor>::type(e));
    }

    size_type size1() const { return m_size1; }
    size_type size2() const { return m_size2; }
    cuda::device& queue() const { return *m_queue; }
    storage_type raw_storage() const { return {m_storage.values, m_storage.leading_dimension}; }
    typename device_traits<cuda_tag>::template matrix_element<T> elements() const {
        return typename device_traits<cuda_tag>::template matrix_element<T>(
            dense_matrix_storage<T, dense_tag>(m_storage.values, m_storage.leading_dimension));
    }
    void clear() {
        cuda::detail::fill<value_type, Orientation>(m_storage.values, m_storage.leading_dimension, m_size1, m_size2,
                                                    value_type(), *m_queue);
    }

    typedef no_iterator major_iterator;
    typedef no_iterator const_major_iterator;

private:
    storage_type m_storage;
    cuda::device* m_queue;
    size_type m_size1;
    size_type m_size2;
};

/// \brief Dense matrix in device memory (the cuda_tag specialisation of matrix).
template <class T, class L>
class matrix<T, L, cuda_tag> : public matrix_container<matrix<T, L, cuda_tag>, cuda_tag> {
public:
    typedef T value_type;
    typedef value_type const& const_reference;
    typedef value_type& reference;
    typedef std::size_t size_type;
    typedef dense_matrix_adaptor<T const, L, continuous_dense_tag, cuda_tag> const_closure_type;
    typedef dense_matrix_adaptor<T, L, continuous_dense_tag, cuda_tag> closure_type;
    typedef dense_matrix_storage<T, continuous_dense_tag> storage_type;
    typedef dense_matrix_storage<T const, continuous_dense_tag> const_storage_type;
    typedef elementwise<dense_tag> evaluation_category;
    typedef L orientation;

    matrix(cuda::device& queue = device_traits<cuda_tag>::default_queue()) : m_storage(0, queue), m_size1(0), m_size2(0) {}
    explicit matrix(size_type size1, size_type size2, cuda::device& queue = device_traits<cuda_tag>::default_queue())
        : m_storage(size1 * size2, queue), m_size1(size1), m_size2(size2) {}
    matrix(size_type size1, size_type size2, value_type const& init,
           cuda::device& queue = device_traits<cuda_tag>::default_queue())
        : m_storage(size1 * size2, queue), m_size1(size1), m_size2(size2) {
        cuda::detail::fill<T, L>(m_storage.get(), L::index_m(size1, size2), size1, size2, init, queue);
    }
    matrix(matrix&& m) : m_storage(std::move(m.m_storage)), m_size1(m.m_size1), m_size2(m.m_size2) {}
    matrix(matrix const& m) : m_storage(m.m_storage), m_size1(m.m_size1), m_size2(m.m_size2) {}
    template <class E>
    matrix(matrix_expression<E, cuda_tag> const& e)
        : m_storage(e().size1() * e().size2(), e().queue()), m_size1(e().size1()), m_size2(e().size2()) {
        assign(*this, e);
    }

    matrix& operator=(matrix const& m) {
        if (size1() != m.size1() || size2() != m.size2()) resize(m.size1(), m.size2());
        return assign(*this, m);
    }
    matrix& operator=(matrix&& m) {
        swap(*this, m);
        return *this;
    }
    template <class C>
    matrix& operator=(matrix_container<C, cuda_tag> const& m) {
        if (size1() != m().size1() || size2() != m().size2()) resize(m().size1(), m().size2());
        return assign(*this, m);
    }
    template <class E>
    matrix& operator=(matrix_expression<E, cuda_tag> const& e) {
        matrix temporary(e);
        swap(*this, temporary);
        return *this;
    }

    size_type size1() const { return m_size1; }
    size_type size2() const { return m_size2; }
    cuda::device& queue() const { return m_storage.dev(); }
    const_storage_type raw_storage() const { return {m_storage.get(), L::index_m(m_size1, m_size2)}; }
    storage_type raw_storage() { return {m_storage.get(), L::index_m(m_size1, m_size2)}; }
    typename device_traits<cuda_tag>::template matrix_element<T> elements() {
        return typename device_traits<cuda_tag>::template matrix_element<T>(
            dense_matrix_storage<T, dense_tag>(m_storage.get(), L::index_m(m_size1, m_size2)));
    }
    void resize(size_type size1, size_type size2) {
        m_storage.resize(size1 * size2);
        m_size1 = size1;
        m_size2 = size2;
    }
    void clear() { cuda::detail::fill<T, L>(m_storage.get(), L::index_m(m_size1, m_size2), m_size1, m_size2, T(), queue()); }

    typedef no_iterator major_iterator;
    typedef no_iterator const_major_iterator;

    friend void swap(matrix& a, matrix& b) {
        std::swap(a.m_storage, b.m_storage);
        std::swap(a.m_size1, b.m_size1);
        std::swap(a.m_size2, b.m_size2);
    }
    template <class Archive>
    void serialize(Archive&, const unsigned int) {}

private:
    cuda::buffer<T> m_storage;
    size_type m_size1;
    size_type m_size2;
};

/// \brief A triangle of a strided device matrix (the cuda_tag specialisation of
/// dense_triangular_proxy, which to_triangular / triangular_prod build,
/// include/remora/dense.hpp:258-266): a view tagged with the triangle; kernels read it
/// through to_dense() and the tag.
template <class T, class Orientation, bool Upper, bool Unit>
class dense_triangular_proxy<T, Orientation, triangular_tag<Upper, Unit>, cuda_tag>
    : public matrix_expression<dense_triangular_proxy<T, Orientation, triangular_tag<Upper, Unit>, cuda_tag>, cuda_tag> {
public:
    typedef std::size_t size_type;
    typedef typename std::remove_const<T>::type value_type;
    typedef value_type result_type;
    typedef typename std::conditional<Unit, value_type const&, T&>::type reference;
    typedef value_type const& const_reference;
    typedef dense_triangular_proxy<value_type const, Orientation, triangular_tag<Upper, Unit>, cuda_tag>
        const_closure_type;
    typedef dense_triangular_proxy closure_type;
    typedef dense_matrix_storage<T, dense_tag> storage_type;
    typedef dense_matrix_storage<value_type const, dense_tag> const_storage_type;
    typedef elementwise<dense_tag> evaluation_category;
    typedef triangular<Orientation, triangular_tag<Upper, Unit>> orientation;

    template <class U>
    dense_triangular_proxy(dense_triangular_proxy<U, Orientation, triangular_tag<Upper, Unit>, cuda_tag> const& p)
        : m_storage(p.raw_storage()), m_queue(&p.queue()), m_size1(p.size1()), m_size2(p.size2()) {}
    dense_triangular_proxy(storage_type const& storage, cuda::device& queue, size_type size1, size_type size2)
        : m_storage(storage), m_queue(&queue), m_size1(size1), m_size2(size2) {}

    dense_matrix_adaptor<T, Orientation, dense_tag, cuda_tag> to_dense() const {
        return {m_storage, *m_queue, m_size1, m_size2};
    }
    size_type size1() const { return m_size1; }
    size_type size2() const { return m_size2; }
    storage_type raw_storage() const { return m_storage; }
    cuda::device& queue() const { return *m_queue; }
    typedef no_iterator major_iterator;
    typedef no_iterator const_major_iterator;

private:
    storage_type m_storage;
    cuda::device* m_queue;
    size_type m_size1, m_size2;
};

/// \brief Strided device vector view.
template <class T, class Tag>
class dense_vector_adaptor<T, Tag, cuda_tag> : public vector_expression<dense_vector_adaptor<T, Tag, cuda_tag>, cuda_tag> {
public:
    typedef std::size_t size_type;
    typedef typename std::remove_const<T>::type value_type;
    typedef value_type const& const_reference;
    typedef T& reference;
    typedef dense_vector_adaptor closure_type;
    typedef dense_vector_adaptor<value_type const, Tag, cuda_tag> const_closure_type;
    typedef dense_vector_storage<T, Tag> storage_type;
    typedef dense_vector_storage<value_type const, Tag> const_storage_type;
    typedef elementwise<dense_tag> evaluation_category;

    template <class U, class Tag2>
    dense_vector_adaptor(dense_vector_adaptor<U, Tag2, cuda_tag> const& v)
        : m_storage(v.raw_storage()), m_queue(&v.queue()), m_size(v.size()) {}
    dense_vector_adaptor(storage_type storage, cuda::device& queue, size_type size)
        : m_storage(storage), m_queue(&queue), m_size(size) {}
    dense_vector_adaptor(vector<value_type, cuda_tag> const& v)
        : m_storage(v.raw_storage()), m_queue(&v.queue()), m_size(v.size()) {}
    dense_vector_adaptor(vector<value_type, cuda_tag>& v)
        : m_storage(v.raw_storage()), m_queue(&v.queue()), m_size(v.size()) {}

    size_type size() const { return m_size; }
    cuda::device& queue() const { return *m_queue; }
    storage_type raw_storage() const { return m_storage; }
    typename device_traits<cuda_tag>::template vector_element<T> elements() const {
        return typename device_traits<cuda_tag>::template vector_element<T>(
            dense_vector_storage<T, dense_tag>(m_storage.values, m_storage.stride));
    }
    // A strided vector is the 1 x size column-major matrix with leading dimension = stride.
    void clear() {
        if (m_size)
            cuda::detail::fill<value_type, column_major>(const_cast<value_type*>(m_storage.values), m_storage.stride,
                                                         1, m_size, value_type(), *m_queue);
    }
    typedef no_iterator iterator;
    typedef no_iterator const_iterator;

private:
    storage_type m_storage;
    cuda::device* m_queue;
    size_type m_size;
};

/// \brief Dense vector in device memory.
template <class T>
class vector<T, cuda_tag> : public vector_container<vector<T, cuda_tag>, cuda_tag> {
public:
    typedef T value_type;
    typedef value_type const& const_reference;
    typedef value_type& reference;
    typedef std::size_t size_type;
    typedef dense_vector_adaptor<T const, continuous_dense_tag, cuda_tag> const_closure_type;
    typedef dense_vector_adaptor<T, continuous_dense_tag, cuda_tag> closure_type;
    typedef dense_vector_storage<T, continuous_dense_tag> storage_type;
    typedef dense_vector_storage<T const, continuous_dense_tag> const_storage_type;
    typedef elementwise<dense_tag> evaluation_category;

    vector(cuda::device& queue = device_traits<cuda_tag>::default_queue()) : m_storage(0, queue) {}
    explicit vector(size_type size, cuda::device& queue = device_traits<cuda_tag>::default_queue())
        : m_storage(size, queue) {}
    vector(size_type size, value_type const& init, cuda::device& queue = device_traits<cuda_tag>::default_queue())
        : m_storage(size, queue) {
        cuda::detail::fill<T, column_major>(m_storage.get(), 1, 1, size, init, queue);
    }
    /// From a device expression: a blockwise one (a transport from the host, a
    /// matrix-vector product, ...) assigns itself; a dense one is copied.
    template <class E>
    vector(vector_expression<E, cuda_tag> const& e) : m_storage(e().size(), e().queue()) {
        assign_from(e(), typename E::evaluation_category());
    }
    template <class E>
    vector& operator=(vector_expression<E, cuda_tag> const& e) {
        vector tmp(e);
        m_storage = std::move(tmp.m_storage);
        return *this;
    }
    vector(vector const& v) = default;
    vector(vector&& v) = default;
    vector& operator=(vector const& v) = default;
    vector& operator=(vector&& v) = default;

    size_type size() const { return m_storage.size(); }
    cuda::device& queue() const { return m_storage.dev(); }
    const_storage_type raw_storage() const { return {m_storage.get(), 1}; }
    storage_type raw_storage() { return {m_storage.get(), 1}; }
    typename device_traits<cuda_tag>::template vector_element<T const> elements() const {
        return typename device_traits<cuda_tag>::template vector_element<T const>(
            dense_vector_storage<T const, dense_tag>(m_storage.get(), 1));
    }
    void resize(size_type size) { m_storage.resize(size); }
    void clear() { cuda::detail::fill<T, column_major>(m_storage.get(), 1, 1, size(), T(), queue()); }
    typedef no_iterator iterator;
    typedef no_iterator const_iterator;

private:
    template <class E, class Tag>
    void assign_from(E const& e, blockwise<Tag>) {
        e.assign_to(*this);
    }
    template <class E, class Tag>
    void assign_from(E const& e, elementwise<Tag>) {  // dense device vector: one strided copy
        auto se = e.raw_storage();
        if (size())
            cuda::check(rc_memcpy2d(m_storage.get(), sizeof(T), se.values, se.stride * sizeof(T), sizeof(T), size(),
                                    RC_COPY_D2D, queue().stream()),
                        "rc_memcpy2d");
    }
    cuda::buffer<T> m_storage;
};

}  // namespace remora

#endif
