// Builder-written no-op stand-in: serialization is out of scope for the oracle.
#pragma once
#include <cstddef>
namespace boost { namespace serialization {
template<class T> struct array_wrapper { T* p; std::size_t n; };
template<class T> array_wrapper<T> make_array(T* p, std::size_t n) { return {p, n}; }
}}
