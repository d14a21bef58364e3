// Builder-written stand-in for Boost's version header, used only to compile the
// reference's CPU path for the oracle. A version below 1.63 makes the reference
// use the aligned-allocator copy it ships (kernels/default/simd.hpp:33-44).
#pragma once
#define BOOST_VERSION 106200
