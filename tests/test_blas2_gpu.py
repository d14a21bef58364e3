"""GEMV / TRSV / TRMV / TRMM on the GPU through the C-ABI against the oracle.

Tolerances (relative Frobenius norm against the oracle on the same inputs): FP64 <= 1e-13,
FP32 <= 1e-5. Triangular inputs are well conditioned with or without their diagonal
(off-diagonal U[-1,1] / n, diagonal 1 + U[0,1]), so the unit-diagonal solves do not grow."""
from __future__ import annotations

import itertools

import numpy as np
import pytest
import torch

import oracle
from remora_b200 import ops

from helpers import to_dev, to_host, with_ld

pytestmark = pytest.mark.gpu
TOL = {np.float64: 1e-13, np.float32: 1e-5}


def _vec_dev(v: np.ndarray, stride: int) -> torch.Tensor:
    """Device vector with element stride `stride` (a view into a larger buffer)."""
    big = torch.zeros(len(v) * stride, dtype=torch.from_numpy(v).dtype, device="cuda")
    big[::stride] = torch.from_numpy(np.ascontiguousarray(v)).cuda()
    return big[::stride]


def _tri(rs, n, dtype, upper):
    T = np.tril(rs.uniform(-1, 1, (n, n)), -1) / n + np.diag(1.0 + rs.uniform(0, 1, n))
    return (T.T.copy() if upper else T).astype(dtype)


def _rel(a, b):
    return oracle.rel_fro(np.asarray(a).reshape(len(a), -1), np.asarray(b).reshape(len(b), -1))


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("m,n", [(1, 1), (7, 300), (300, 7), (4097, 513), (1000, 1000)])
@pytest.mark.parametrize("a_rm", [False, True])
def test_gemv(cuda, orc, dtype, m, n, a_rm):
    rs = np.random.default_rng(m * 31 + n)
    A = rs.uniform(-1, 1, (m, n)).astype(dtype)
    x = rs.uniform(-1, 1, n).astype(dtype)
    y = rs.uniform(-1, 1, m).astype(dtype)
    yd = _vec_dev(y, 3)
    ops.gemv(with_ld(A, a_rm, 4), _vec_dev(x, 2), yd, alpha=0.5, beta=-2.0)
    y *= -2.0
    orc.gemv(A, x, y, alpha=0.5)
    assert _rel(to_host(yd), y) <= TOL[dtype]


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("upper,unit,left", list(itertools.product([False, True], repeat=3)))
@pytest.mark.parametrize("a_rm", [False, True])
@pytest.mark.parametrize("n", [1, 45, 300])
def test_trsv(cuda, orc, dtype, upper, unit, left, a_rm, n):
    rs = np.random.default_rng(n + 2 * upper + unit)
    T = _tri(rs, n, dtype, upper)
    b = rs.uniform(-1, 1, n).astype(dtype)
    xd = _vec_dev(b, 2)
    ops.trsv(with_ld(T, a_rm, 3), xd, upper=upper, unit=unit, left=left)
    assert orc.trsv(T, b, upper=upper, unit=unit, left=left) == 0
    assert _rel(to_host(xd), b) <= TOL[dtype]


def test_trsv_large(cuda, orc):
    """A solve longer than one 128 diagonal block chain (n = 1000)."""
    rs = np.random.default_rng(5)
    T = _tri(rs, 1000, np.float64, False)
    b = rs.uniform(-1, 1, 1000)
    xd = _vec_dev(b, 1)
    ops.trsv(to_dev(T, False), xd)
    assert orc.trsv(T, b) == 0
    assert _rel(to_host(xd), b) <= 1e-13


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("upper,unit", list(itertools.product([False, True], repeat=2)))
@pytest.mark.parametrize("a_rm,b_rm", [(False, False), (True, False), (False, True), (True, True)])
def test_trmm(cuda, orc, dtype, upper, unit, a_rm, b_rm):
    rs = np.random.default_rng(7 + upper + 2 * unit)
    n, k = 300, 17
    T = _tri(rs, n, dtype, upper)
    B = rs.uniform(-1, 1, (n, k)).astype(dtype)
    Bd = with_ld(B, b_rm, 5)
    ops.trmm(with_ld(T, a_rm, 3), Bd, upper=upper, unit=unit)
    orc.trmm(T, B, upper=upper, unit=unit)
    assert oracle.rel_fro(to_host(Bd), B) <= TOL[dtype]


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("upper,unit", list(itertools.product([False, True], repeat=2)))
@pytest.mark.parametrize("a_rm", [False, True])
def test_trmv(cuda, orc, dtype, upper, unit, a_rm):
    rs = np.random.default_rng(11 + upper + 2 * unit)
    n = 129
    T = _tri(rs, n, dtype, upper)
    v = rs.uniform(-1, 1, n).astype(dtype)
    vd = _vec_dev(v, 2)
    ops.trmv(with_ld(T, a_rm, 3), vd, upper=upper, unit=unit)
    orc.trmm(T, v[:, None], upper=upper, unit=unit)
    assert _rel(to_host(vd), v) <= TOL[dtype]
