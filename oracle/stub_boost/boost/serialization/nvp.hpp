// Builder-written no-op stand-in: serialization is out of scope for the oracle.
#pragma once
namespace boost { namespace serialization {
template<class T> T& make_nvp(const char*, T& t) { return t; }
}}
