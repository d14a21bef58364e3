// Builder-written no-op stand-in: serialization is out of scope for the oracle.
#pragma once
#include <cstddef>
namespace boost { namespace serialization {
struct collection_size_type {
	std::size_t t;
	collection_size_type(std::size_t v = 0) : t(v) {}
	operator std::size_t() const { return t; }
};
}}
