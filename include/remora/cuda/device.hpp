// remora/cuda/device.hpp -- device, stream, errors and owning buffers of the cuda_tag
// backend, over the C-ABI of libremora_cuda.so (no CUDA headers needed).
//
// Mirrors include/remora/hip/device.hpp:41-180 (device + a non-default stream per
// device and thread), include/remora/hip/exception.hpp:41-63 (errors become
// std::system_error) and include/remora/hip/buffer.hpp:41-102 (RAII allocation).
#ifndef REMORA_CUDA_DEVICE_HPP
#define REMORA_CUDA_DEVICE_HPP

#include <remora_cuda.h>

#include <algorithm>
#include <condition_variable>
#include <cstdint>
#include <cstddef>
#include <functional>
#include <map>
#include <mutex>
#include <memory>
#include <string>
#include <system_error>
#include <thread>
#include <utility>
#include <vector>

#include "fwd.hpp"

namespace remora {
namespace cuda {

class error_category_impl : public std::error_category {
public:
    const char* name() const noexcept override { return "remora_cuda"; }
    std::string message(int status) const override { return rc_error_string(status); }
};
inline std::error_category const& error_category() {
    static error_category_impl cat;
    return cat;
}

/// Throws std::system_error for a non-zero status of a C-ABI call.
inline void check(int status, char const* what) {
    if (status != RC_SUCCESS) throw std::system_error(status, error_category(), what);
}

/// A CUDA device with one non-default stream per host thread
/// (as hip::get_stream, include/remora/hip/device.hpp:158-173).
class device {
public:
    explicit device(int id) : m_id(id) {}
    int id() const { return m_id; }
    void set_device() const { check(rc_set_device(m_id), "rc_set_device"); }
    /// The calling thread's stream on this device (created on first use).
    void* stream() const {
        thread_local std::map<int, std::shared_ptr<void>> streams;
        auto& s = streams[m_id];
        if (!s) {
            set_device();
            void* h = nullptr;
            check(rc_stream_create(&h), "rc_stream_create");
            s = std::shared_ptr<void>(h, [](void* p) { rc_stream_destroy(p); });
        }
        return s.get();
    }
    void synchronize() const { check(rc_stream_synchronize(stream()), "rc_stream_synchronize"); }
    std::size_t warp_size() const { return 32; }

private:
    int m_id;
};

/// Two page-locked host chunks of `chunk_bytes` each, with an event per chunk, for the
/// transport between host expressions and device storage: the host side of chunk i is
/// filled (or drained) while the DMA of the other chunk runs on the device's stream. One
/// set per (device, host thread), allocated on first use, like the stream.
class host_staging {
public:
    static constexpr std::size_t chunk_bytes = std::size_t(32) << 20;

    static host_staging& of(device const& dev) {
        thread_local std::map<int, std::unique_ptr<host_staging>> sets;
        auto& s = sets[dev.id()];
        if (!s) s.reset(new host_staging(dev));
        return *s;
    }
    host_staging(host_staging const&) = delete;
    host_staging& operator=(host_staging const&) = delete;
    ~host_staging() {
        for (int c = 0; c < 2; ++c) {
            if (m_event[c]) {
                rc_event_synchronize(m_event[c]);
                rc_event_destroy(m_event[c]);
            }
            rc_host_free(m_buf[c]);
        }
    }
    void* chunk(int c) const { return m_buf[c]; }
    /// Wait until the DMA last recorded for chunk c has finished with it.
    void wait(int c) {
        if (m_used[c]) check(rc_event_synchronize(m_event[c]), "rc_event_synchronize");
        m_used[c] = false;
    }
    /// Mark chunk c busy until the work queued so far on `stream` has run.
    void record(int c, void* stream) {
        check(rc_event_record(m_event[c], stream), "rc_event_record");
        m_used[c] = true;
    }

private:
    explicit host_staging(device const& dev) {
        dev.set_device();
        for (int c = 0; c < 2; ++c) {
            check(rc_host_alloc(&m_buf[c], chunk_bytes), "rc_host_alloc");
            check(rc_event_create(&m_event[c]), "rc_event_create");
        }
    }
    void* m_buf[2] = {nullptr, nullptr};
    void* m_event[2] = {nullptr, nullptr};
    bool m_used[2] = {false, false};
};

/// A small pool of host threads (started on first use, half the hardware threads, at most
/// 7) that, with the calling thread, packs and unpacks the transport's staging chunks:
/// Remora's CPU assignment is single-threaded, and one thread moves far less than the
/// link's rate. One job at a time; a job is a set of parts run by whichever thread is free.
class host_workers {
public:
    static host_workers& instance() {
        static host_workers w;
        return w;
    }
    std::size_t threads() const { return m_threads.size() + 1; }
    /// f(part) for part in [0, parts), on the pool and the calling thread; returns when all
    /// parts are done.
    void run(std::size_t parts, std::function<void(std::size_t)> const& f) {
        std::lock_guard<std::mutex> one_job(m_run);
        {
            std::lock_guard<std::mutex> lock(m_mutex);
            m_job = &f;
            m_parts = parts;
            m_next = 0;
            m_finished = 0;
            ++m_generation;
        }
        m_wake.notify_all();
        work();
        std::unique_lock<std::mutex> lock(m_mutex);
        m_done.wait(lock, [&] { return m_finished == m_parts; });
        m_job = nullptr;
    }
    ~host_workers() {
        {
            std::lock_guard<std::mutex> lock(m_mutex);
            m_quit = true;
        }
        m_wake.notify_all();
        for (auto& t : m_threads) t.join();
    }

private:
    host_workers() {
        const unsigned hw = std::thread::hardware_concurrency();
        const unsigned n = std::min(7u, hw > 2 ? hw / 2 - 1 : 0u);
        for (unsigned i = 0; i < n; ++i) m_threads.emplace_back([this] { loop(); });
    }
    // Take parts of the current job until none is left.
    void work() {
        while (true) {
            std::size_t p;
            std::function<void(std::size_t)> const* job;
            {
                std::lock_guard<std::mutex> lock(m_mutex);
                if (!m_job || m_next >= m_parts) return;
                p = m_next++;
                job = m_job;
            }
            (*job)(p);
            std::lock_guard<std::mutex> lock(m_mutex);
            if (++m_finished == m_parts) m_done.notify_all();
        }
    }
    void loop() {
        std::uint64_t seen = 0;
        while (true) {
            {
                std::unique_lock<std::mutex> lock(m_mutex);
                m_wake.wait(lock, [&] { return m_quit || m_generation != seen; });
                if (m_quit) return;
                seen = m_generation;
            }
            work();
        }
    }
    std::vector<std::thread> m_threads;
    std::mutex m_run, m_mutex;
    std::condition_variable m_wake, m_done;
    std::function<void(std::size_t)> const* m_job = nullptr;
    std::size_t m_parts = 0, m_next = 0, m_finished = 0;
    std::uint64_t m_generation = 0;
    bool m_quit = false;
};

/// Run f(begin, end) over [0, count) in contiguous pieces on the host worker pool.
template <class F>
void parallel_lines(std::size_t count, F f) {
    host_workers& w = host_workers::instance();
    const std::size_t parts = std::min<std::size_t>(w.threads(), count);
    if (parts <= 1) {
        f(std::size_t(0), count);
        return;
    }
    const std::size_t step = (count + parts - 1) / parts;
    w.run((count + step - 1) / step, [&](std::size_t p) { f(p * step, std::min(count, (p + 1) * step)); });
}

/// All devices of the machine (hip/device.hpp:85-110).
class device_manager {
public:
    device_manager() {
        int n = 0;
        if (rc_device_count(&n) != RC_SUCCESS) n = 0;
        for (int i = 0; i < n; ++i) m_devices.emplace_back(new device(i));
    }
    std::size_t size() const { return m_devices.size(); }
    device& operator()(std::size_t i) {
        if (i >= m_devices.size()) throw std::system_error(RC_ERR_CUDA, error_category(), "no such CUDA device");
        return *m_devices[i];
    }

private:
    std::vector<std::unique_ptr<device>> m_devices;
};
inline device_manager& devices() {
    static device_manager m;
    return m;
}

/// Owning device allocation of n elements (hip/buffer.hpp:41-102).
template <class T>
class buffer {
public:
    buffer(std::size_t n, device& dev) : m_device(&dev), m_size(n) { allocate(); }
    buffer(buffer const& o) : m_device(o.m_device), m_size(o.m_size) {
        allocate();
        copy_from(o);
    }
    buffer(buffer&& o) noexcept : m_device(o.m_device), m_ptr(o.m_ptr), m_size(o.m_size) {
        o.m_ptr = nullptr;
        o.m_size = 0;
    }
    buffer& operator=(buffer const& o) {
        if (this != &o) {
            if (m_size != o.m_size) {
                release();
                m_size = o.m_size;
                allocate();
            }
            copy_from(o);
        }
        return *this;
    }
    buffer& operator=(buffer&& o) noexcept {
        std::swap(m_device, o.m_device);
        std::swap(m_ptr, o.m_ptr);
        std::swap(m_size, o.m_size);
        return *this;
    }
    ~buffer() { release(); }

    T* get() const { return m_ptr; }
    std::size_t size() const { return m_size; }
    device& dev() const { return *m_device; }
    /// Resizing discards the contents.
    void resize(std::size_t n) {
        if (n == m_size) return;
        release();
        m_size = n;
        allocate();
    }

private:
    void allocate() {
        m_device->set_device();
        void* p = nullptr;
        check(rc_malloc(&p, m_size * sizeof(T)), "rc_malloc");
        m_ptr = static_cast<T*>(p);
    }
    void release() {
        if (m_ptr) {
            m_device->synchronize();  // kernels queued on this buffer may still run
            rc_free(m_ptr);
        }
        m_ptr = nullptr;
    }
    void copy_from(buffer const& o) {
        if (m_size)
            check(rc_memcpy2d(m_ptr, m_size * sizeof(T), o.m_ptr, m_size * sizeof(T), m_size * sizeof(T), 1,
                              RC_COPY_D2D, m_device->stream()),
                  "rc_memcpy2d");
    }
    device* m_device;
    T* m_ptr = nullptr;
    std::size_t m_size;
};

}  // namespace cuda

/// device_traits for cuda_tag (hip/traits.hpp:40-411 for hip_tag). The element functors
/// exist so that the expression classes instantiate; elementwise device expressions
/// beyond dense assignment are not evaluated by this backend.
template <>
struct device_traits<cuda_tag> {
    typedef cuda::device queue_type;
    static queue_type& default_queue() { return cuda::devices()(0); }

    template <class Iterator, class Functor>
    struct transform_iterator { typedef no_iterator type; };
    template <class Iterator1, class Iterator2, class Functor>
    struct binary_transform_iterator { typedef no_iterator type; };
    template <class T>
    struct constant_iterator { typedef no_iterator type; };
    template <class T>
    struct one_hot_iterator { typedef no_iterator type; };
    template <class Closure>
    struct indexed_iterator { typedef no_iterator type; };

#define REMORA_CUDA_BINARY(name, expr)                                     \
    template <class T>                                                     \
    struct name {                                                          \
        typedef T result_type;                                             \
        T operator()(T x, T y) const { return expr; }                      \
    };
    REMORA_CUDA_BINARY(add, x + y)
    REMORA_CUDA_BINARY(subtract, x - y)
    REMORA_CUDA_BINARY(multiply, x * y)
    REMORA_CUDA_BINARY(divide, x / y)
    REMORA_CUDA_BINARY(safe_divide, y == T(0) ? T(0) : x / y)
    REMORA_CUDA_BINARY(min, x < y ? x : y)
    REMORA_CUDA_BINARY(max, x < y ? y : x)
#undef REMORA_CUDA_BINARY

    template <class T>
    struct identity {
        typedef T result_type;
        T operator()(T x) const { return x; }
    };
    template <class T>
    struct multiply_scalar {
        typedef T result_type;
        explicit multiply_scalar(T s) : m_s(s) {}
        T operator()(T x) const { return x * m_s; }
        T m_s;
    };
    template <class T>
    struct constant {
        typedef T result_type;
        explicit constant(T v) : m_v(v) {}
        T operator()(T) const { return m_v; }
        T m_v;
    };
    // Functors of the blockwise assignments Remora issues for scalar-scaled operands
    // (x = alpha e, x += alpha e); the cuda_tag bindings read their scalar.
    template <class T>
    struct multiply_assign {
        typedef T result_type;
        explicit multiply_assign(T s) : m_s(s) {}
        T m_s;
    };
    template <class T>
    struct multiply_and_add {
        typedef T result_type;
        explicit multiply_and_add(T s) : m_s(s) {}
        T m_s;
    };
    /// Element-functor composition: element functors are never evaluated by this backend
    /// (its bindings read dense storage), so the composition is an empty placeholder.
    template <class F, class G>
    static no_functor make_compose(F const&, G const&) {
        return no_functor();
    }
    template <class T>
    struct matrix_element {
        typedef T& result_type;
        explicit matrix_element(dense_matrix_storage<T, dense_tag> const& s) : storage(s) {}
        dense_matrix_storage<T, dense_tag> storage;
    };
    template <class T>
    struct vector_element {
        typedef T& result_type;
        explicit vector_element(dense_vector_storage<T, dense_tag> const& s) : storage(s) {}
        dense_vector_storage<T, dense_tag> storage;
    };
};

inline cuda::device& default_cuda_device() { return device_traits<cuda_tag>::default_queue(); }

}  // namespace remora

#endif
