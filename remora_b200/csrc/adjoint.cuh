// Internal entries of the reverse-mode adjoints.
#pragma once
#include "common.cuh"

namespace rc {
// Abar (full symmetric) = adjoint of A = L L^T for the adjoint Lbar of its lower factor.
int potrf_backward(int64_t n, View<const double> L, View<const double> Lbar, View<double> Abar, cudaStream_t s);
// Reverse mode of X = L^-1 B (trans = false) or X = L^-T B (trans = true): Xbar is
// overwritten by Bbar, Lbar (lower triangle) accumulates the adjoint of L.
int trsm_backward(bool trans, int64_t n, int64_t nrhs, View<const double> L, View<const double> X, View<double> Xbar,
                  View<double> Lbar, cudaStream_t s);
}  // namespace rc
