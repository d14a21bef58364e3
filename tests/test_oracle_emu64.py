"""The CPU restatement of the emulated-FP64 SYRK (oracle/emu64.py) checked on its own: on
entries that are 28-bit integers times a power of two per row (four nonzero digits) it must
return the correctly rounded exact product, computed here with Python integers; on general
FP64 rows it must stay within the method's truncation bound k 2^-44 m_i m_j."""
from __future__ import annotations

import math

import numpy as np

from oracle import emu64


def test_restatement_exact_on_four_digit_entries():
    rs = np.random.default_rng(11)
    n, k = 37, 53
    Pi = rs.integers(-(2 ** 28) + 1, 2 ** 28, size=(n, k))
    s = rs.integers(-30, 31, size=n)
    Pi[3] = 0
    P = Pi.astype(np.float64) * np.exp2(s)[:, None]
    C = emu64.syrk_emu64(P, alpha=-1.0)
    for i in range(n):
        for j in range(i + 1):
            exact = sum(int(Pi[i, c]) * int(Pi[j, c]) for c in range(k))
            assert C[i, j] == -math.ldexp(float(exact), int(s[i] + s[j]))
    assert np.all(np.triu(C, 1) == 0.0)


def test_restatement_within_truncation_bound():
    rs = np.random.default_rng(12)
    n, k = 41, 77
    P = rs.standard_normal((n, k)) * np.exp2(rs.integers(-25, 26, size=(n, 1)))
    C = emu64.syrk_emu64(P)
    m = np.abs(P).max(axis=1)
    err = np.abs(np.tril(C - P @ P.T))
    assert np.all(err <= k * 2.0 ** -44 * np.outer(m, m))


def test_row_exponents_bound_every_entry():
    rs = np.random.default_rng(13)
    P = rs.standard_normal((9, 5)) * np.exp2(rs.integers(-1000, 1000, size=(9, 1)))
    P[4] = 0.0
    e = emu64.row_exponents(P)
    assert e[4] == 0
    for i in (0, 1, 2, 3, 5, 6, 7, 8):
        top = np.abs(P[i]).max()
        assert top < math.ldexp(1.0, int(e[i])) and top >= math.ldexp(1.0, int(e[i]) - 1)
