// Builder-written stand-in for Boost's static_assert header (oracle build only).
#pragma once
#define BOOST_STATIC_ASSERT(...) static_assert(__VA_ARGS__, #__VA_ARGS__)
