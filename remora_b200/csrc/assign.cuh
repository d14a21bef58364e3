// Internal strided copy / fill helpers.
#pragma once
#include "common.cuh"

namespace rc {
// B <- alpha * A (both m x n views; converts the element type when S != D).
template <class S, class D>
int copy2d(int64_t m, int64_t n, D alpha, View<const S> A, View<D> B, cudaStream_t s, const int* abort = nullptr);
template <class T>
int fill(int64_t m, int64_t n, T value, View<T> A, cudaStream_t s);
}  // namespace rc
