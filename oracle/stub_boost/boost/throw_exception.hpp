// Builder-written stand-in for Boost's throw_exception header (oracle build only).
#pragma once
namespace boost { template<class E> [[noreturn]] void throw_exception(E const& e) { throw e; } }
