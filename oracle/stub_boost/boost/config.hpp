// Builder-written stand-in for Boost's config header (oracle build only).
#pragma once
#define BOOST_CONSTEXPR constexpr
#define BOOST_NOEXCEPT noexcept
#define BOOST_NOEXCEPT_OR_NOTHROW noexcept
#define BOOST_STATIC_CONSTANT(type, assignment) static const type assignment
#define BOOST_GCC 1
#define BOOST_GCC_VERSION (__GNUC__ * 10000 + __GNUC_MINOR__ * 100 + __GNUC_PATCHLEVEL__)
#define BOOST_HAS_UNISTD_H 1
