"""FP64 products on the int8 tensor cores (rc_gemm_f64_sliced) against the oracle.

The product splits A by rows and B by columns into 8 signed 7-bit digits below a power of
two above the row / column maximum (2^e_i, 2^f_j) and multiplies the digits exactly, so
its error is bounded elementwise by the truncation of both operands plus the dropped
digit pairs: |C - AB|(i, j) <= 11 k 2^-56 2^(e_i + f_j), plus FP64 rounding of the result
(2^-50 |A||B|(i, j) here). Integer operands with at most 7 significant bits per row
maximum are represented exactly, so their products must match bit for bit."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from remora_b200 import ops

from helpers import to_dev, to_host

pytestmark = pytest.mark.gpu


def _pow2_above(x: np.ndarray) -> np.ndarray:
    """2^e with |x| < 2^e (1 for zero)."""
    out = np.ones_like(x)
    nz = x > 0
    out[nz] = np.ldexp(1.0, np.frexp(x[nz])[1])
    return out


def _bound(A, B):
    k = A.shape[1]
    ra = _pow2_above(np.abs(A).max(axis=1))[:, None]
    cb = _pow2_above(np.abs(B).max(axis=0))[None, :]
    return 11.0 * k * 2.0 ** -56 * ra * cb + 2.0 ** -50 * (np.abs(A) @ np.abs(B))


def _run(A, B, C0=None, alpha=1.0, beta=0.0):
    m, n = A.shape[0], B.shape[1]
    Cd = to_dev(C0 if C0 is not None else np.zeros((m, n)), False)
    ops.gemm_sliced(to_dev(A, False), to_dev(B, False), Cd, alpha=alpha, beta=beta)
    return to_host(Cd)


@pytest.mark.parametrize("m,k,n", [(1, 1, 1), (100, 37, 5), (1000, 1000, 8), (257, 129, 17), (777, 4097, 64),
                                   (4096, 300, 33), (300, 20000, 3)])
def test_sliced_matches_fp64(cuda, orc, m, k, n):
    rs = np.random.default_rng(m + 7 * k + n)
    A = rs.standard_normal((m, k)) * np.exp(rs.uniform(-3, 3, (m, 1)))
    B = rs.standard_normal((k, n)) * np.exp(rs.uniform(-3, 3, (1, n)))
    C = _run(A, B)
    ref = np.zeros((m, n))
    orc.gemm(A, B, ref)
    assert np.all(np.abs(C - ref) <= _bound(A, B))


def test_sliced_alpha_beta(cuda, orc):
    rs = np.random.default_rng(3)
    A, B, C0 = rs.standard_normal((513, 700)), rs.standard_normal((700, 9)), rs.standard_normal((513, 9))
    C = _run(A, B, C0, alpha=-1.0, beta=1.0)  # the residual form R = B - A X
    ref = C0.copy()
    orc.gemm(A, B, ref, alpha=-1.0)
    assert np.all(np.abs(C - ref) <= _bound(A, B) + 2.0 ** -52 * np.abs(C0))


def test_sliced_beta_zero_ignores_c(cuda, orc):
    rs = np.random.default_rng(4)
    A, B = rs.standard_normal((200, 50)), rs.standard_normal((50, 4))
    C = _run(A, B, np.full((200, 4), np.nan), beta=0.0)
    ref = np.zeros((200, 4))
    orc.gemm(A, B, ref)
    assert np.all(np.isfinite(C)) and np.all(np.abs(C - ref) <= _bound(A, B))


@pytest.mark.parametrize("k", [16, 3000, 40000])
def test_sliced_exact_on_small_integers(cuda, k):
    """7-bit integers are single digits: every product and sum is exact."""
    rs = np.random.default_rng(k)
    m, n = 384, 24
    A = rs.integers(-127, 128, (m, k)).astype(np.float64)
    B = rs.integers(-127, 128, (k, n)).astype(np.float64)
    C = _run(A, B)
    exact = (A.astype(np.int64) @ B.astype(np.int64)).astype(np.float64)
    assert np.array_equal(C, exact)


def test_sliced_nonfinite_and_zero(cuda, orc):
    rs = np.random.default_rng(5)
    A, B = rs.standard_normal((300, 200)), rs.standard_normal((200, 6))
    A[7, 11] = np.nan
    A[8, 3] = np.inf
    A[9, :] = 0.0
    B[5, 2] = -np.inf
    B[:, 4] = 0.0
    C = _run(A, B)
    assert np.all(np.isnan(C[[7, 8], :]))
    assert np.all(np.isnan(C[:, 2]))
    assert np.all(C[9, [0, 1, 3, 4, 5]] == 0.0) and np.all(C[[0, 1, 100], 4] == 0.0)
    keep_r = [i for i in range(300) if i not in (7, 8)]
    keep_c = [0, 1, 3, 4, 5]
    A2, B2 = A[keep_r], B[:, keep_c]
    ref = np.zeros((len(keep_r), len(keep_c)))
    orc.gemm(A2, B2, ref)
    assert np.all(np.abs(C[np.ix_(keep_r, keep_c)] - ref) <= _bound(A2, B2))


def test_sliced_wide_exponent_range(cuda, orc):
    """Rows and columns scaled over 2^-500 .. 2^500: the per-row / per-column exponents
    carry the range, the digits only the 56 bits below each maximum."""
    rs = np.random.default_rng(6)
    m, k, n = 256, 512, 8
    A = rs.standard_normal((m, k)) * np.ldexp(1.0, rs.integers(-500, 500, (m, 1)))
    B = rs.standard_normal((k, n)) * np.ldexp(1.0, rs.integers(-300, 300, (1, n)))
    C = _run(A, B)
    ref = np.zeros((m, n))
    orc.gemm(A, B, ref)
    assert np.all(np.abs(C - ref) <= _bound(A, B))


def test_sliced_rejects_wide_b(cuda):
    """More than 64 columns of B is RC_ERR_NOT_SUPPORTED (the DMMA GEMM covers it)."""
    from remora_b200._lib import RemoraCudaError

    def z(r, c):
        return torch.zeros((c, r), dtype=torch.float64, device="cuda").t()

    with pytest.raises(RemoraCudaError):
        ops.gemm_sliced(z(64, 64), z(64, 65), z(64, 65))
