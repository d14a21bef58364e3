// Builder-written stand-in for Boost's assert header (oracle build only).
#pragma once
#include <cassert>
#define BOOST_ASSERT(expr) assert(expr)
