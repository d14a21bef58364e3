// Device helpers of the int8 digit split (shared by the kernels that write digits).
#pragma once
#include <climits>
#include <cstdint>

#include "ozaki.cuh"

namespace rc {

constexpr int kOzBadExp = INT_MIN;

// Exponent e with |x| < 2^e for every x of a row or column whose largest |x| has these
// bits (0 for an all-zero row; kOzBadExp when the largest is Inf or NaN).
__device__ __forceinline__ int scale_exp(unsigned long long bits) {
    if (bits == 0) return 0;
    if (bits >= 0x7FF0000000000000ull) return kOzBadExp;
    const int ex = (int)(bits >> 52);
    if (ex == 0) return (63 - __clzll((long long)bits)) - 1073;  // subnormal maximum
    return ex - 1022;
}

// The 8 signed base-128 digits of x / 2^e (|x| < 2^e), truncated: V = floor(|x| 2^(56-e))
// read 7 bits at a time, with x's sign, OR-ed into byte `byte` of word[t]. Returns false
// when |x| >= 2^e (the digits are then not x's).
__device__ __forceinline__ bool digits(double x, int e, uint32_t (&word)[kOzSlices], int byte) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(x);
    const int ex = (int)((b >> 52) & 0x7FF);
    const unsigned long long frac = b & 0xFFFFFFFFFFFFFull;
    const unsigned long long M = ex ? (frac | (1ull << 52)) : frac;
    const int sh = (ex ? ex : 1) - 1075 + 56 - e;
    unsigned long long V = 0;
    if (sh >= 0) V = M << (sh < 63 ? sh : 63);
    else if (sh > -64) V = M >> (-sh);
    const bool neg = (b >> 63) != 0;
#pragma unroll
    for (int t = 0; t < kOzSlices; ++t) {
        const int d = (int)((V >> (49 - 7 * t)) & 127);
        word[t] |= (uint32_t)(uint8_t)(int8_t)(neg ? -d : d) << (8 * byte);
    }
    return sh < 0 || M == 0 || (sh < 56 && (M >> (56 - sh)) == 0);  // M 2^sh < 2^56
}

}  // namespace rc
