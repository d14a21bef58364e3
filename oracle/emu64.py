"""Test infrastructure: a CPU restatement of the emulated-FP64 lower SYRK (rc_syrk_emu64).

The reference has no counterpart (its products are FP64 BLAS calls); this restates the
digit-product method the kernel implements -- the Ozaki scheme in the integer form of
Ootomo, Ozaki and Yokota (IJHPCA 2024) -- with exact integer arithmetic, so the kernel can
be compared with it value by value:

  * per row i of P, e_i with max_k |P(i, k)| < 2^e_i (the frexp exponent of the row maximum);
  * per entry, V = floor(|P(i, k)| 2^(56 - e_i)) and the signed 7-bit digits
    a_t = sign(P) ((V >> (49 - 7 t)) & 127), t = 0..6 (weight 2^(-7 (t + 1)));
  * the digit pairs with t + u <= 6, summed per d = t + u into exact integers v_d;
  * h = (v_0 2^21 + v_1 2^14 + v_2 2^7 + v_3) 2^-21 + (v_4 2^14 + v_5 2^7 + v_6) 2^-42,
    rounded once to FP64 (the kernel's fused multiply-add of two exact partial sums);
  * C(i, j) = alpha * h * 2^(e_i + e_j - 14) for j <= i (beta = 0).

Only tests use this module. Inputs must be finite; the pairs are summed with numpy int64
(|v_d| <= 7 * 127^2 * k, exact for any k the kernel accepts).
"""
from __future__ import annotations

import math

import numpy as np

SLICES = 7


def row_exponents(P: np.ndarray) -> np.ndarray:
    """e_i with every |P(i, k)| < 2^e_i (0 for an all-zero row)."""
    mx = np.abs(P).max(axis=1)
    return np.array([math.frexp(float(m))[1] if m != 0.0 else 0 for m in mx], dtype=np.int64)


def digits(P: np.ndarray, e: np.ndarray) -> np.ndarray:
    """The SLICES signed digits of every entry, shape (SLICES, n, k), int64."""
    n, k = P.shape
    out = np.zeros((SLICES, n, k), dtype=np.int64)
    for i in range(n):
        for c in range(k):
            x = float(P[i, c])
            if x == 0.0:
                continue
            m, ex = math.frexp(abs(x))          # |x| = m 2^ex, m in [0.5, 1)
            M = int(m * (1 << 53))               # |x| = M 2^(ex - 53), exactly
            sh = ex - 53 + 56 - int(e[i])        # V = floor(M 2^sh)
            V = M << sh if sh >= 0 else M >> (-sh)
            s = -1 if x < 0 else 1
            for t in range(SLICES):
                out[t, i, c] = s * ((V >> (49 - 7 * t)) & 127)
    return out


def syrk_emu64(P: np.ndarray, alpha: float = 1.0) -> np.ndarray:
    """The lower triangle (zeros above) of alpha * P P^T as the kernel computes it with
    beta = 0."""
    P = np.asarray(P, dtype=np.float64)
    n, _ = P.shape
    e = row_exponents(P)
    D = digits(P, e)
    v = [np.zeros((n, n), dtype=np.int64) for _ in range(SLICES)]
    for t in range(SLICES):
        for u in range(SLICES - t):
            v[t + u] += D[t] @ D[u].T
    C = np.zeros((n, n))
    for i in range(n):
        for j in range(i + 1):
            vs = [int(v[d][i, j]) for d in range(SLICES)]
            hi = ((vs[0] * 128 + vs[1]) * 128 + vs[2]) * 128 + vs[3]
            lo = (vs[4] * 128 + vs[5]) * 128 + vs[6]
            h = math.ldexp(float(hi * (1 << 21) + lo), -42)  # int -> float rounds once, to nearest
            C[i, j] = alpha * math.ldexp(h, int(e[i] + e[j]) - 14)
    return C
