"""GEMM / SYRK / TRSM on the GPU through the C-ABI against the oracle.

Tolerances (relative Frobenius norm against the oracle on the same inputs):
FP64 <= 1e-13, FP32 <= 1e-5 (the north-star parity bar)."""
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


def _u(rs, shape, dtype):
    return rs.uniform(-1, 1, shape).astype(dtype)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("a_rm,b_rm,c_rm", list(itertools.product([True, False], repeat=3)))
def test_gemm_orientations(cuda, orc, dtype, a_rm, b_rm, c_rm):
    """All 8 orientation combinations of Test/hip_prod.cpp (50x33 times 33x80), both
    `+=` with C initialised to 1.5 and `=`, alpha = -2."""
    rows, mid, cols = 50, 33, 80
    X = np.fromfunction(lambda i, j: 0.1 * i * mid + 0.2 * j, (rows, mid)).astype(dtype)
    Y = np.fromfunction(lambda i, j: 0.1 * i * cols + 1.5 * j, (mid, cols)).astype(dtype)
    for init in (1.5, 0.0):
        C = np.full((rows, cols), init, dtype=dtype)
        Cd = to_dev(C, c_rm)
        ops.gemm(to_dev(X, a_rm), to_dev(Y, b_rm), Cd, alpha=-2.0)
        orc.gemm(X, Y, C, alpha=-2.0)
        assert oracle.rel_fro(to_host(Cd), C) <= TOL[dtype]


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (7, 3, 300), (129, 257, 65), (300, 200, 1000), (512, 512, 512)])
@pytest.mark.parametrize("ta,tb", [(0, 0), (1, 0), (0, 1), (1, 1)])
def test_gemm_shapes(cuda, orc, dtype, m, n, k, ta, tb):
    rs = np.random.default_rng(m * 7 + n * 3 + k)
    A = _u(rs, (m, k), dtype)
    B = _u(rs, (k, n), dtype)
    C = _u(rs, (m, n), dtype)
    Cd = with_ld(C, False, 5)
    ops.gemm(with_ld(A, bool(ta), 3), with_ld(B, bool(tb), 2), Cd, alpha=0.75, beta=-1.25)
    C *= -1.25
    orc.gemm(A, B, C, alpha=0.75)
    assert oracle.rel_fro(to_host(Cd), C) <= TOL[dtype]


def test_gemm_beta_zero_ignores_nan(cuda):
    A = torch.ones((4, 4), dtype=torch.float64, device="cuda")
    C = torch.full((4, 4), float("nan"), dtype=torch.float64, device="cuda")
    ops.gemm(A, A, C, alpha=1.0, beta=0.0)
    assert torch.all(C == 4.0)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("a_rm", [True, False])
@pytest.mark.parametrize("c_rm", [True, False])
@pytest.mark.parametrize("upper", [False, True])
def test_syrk(cuda, orc, dtype, a_rm, c_rm, upper):
    """Test/hip_syrk.cpp: 936 x 1039 (not a block multiple), C initialised to 3, alpha 2;
    the other triangle must stay exactly 3."""
    dims, K = 936, 1039
    A = np.fromfunction(lambda i, j: (1.0 / dims) * i + 0.2 / K * j + 1, (dims, K)).astype(dtype)
    C = np.full((dims, dims), 3.0, dtype=dtype)
    Cd = to_dev(C, c_rm)
    ops.syrk(to_dev(A, a_rm), Cd, alpha=2.0, upper=upper)
    got = to_host(Cd)
    orc.syrk(A, C, alpha=2.0, upper=upper)
    tri = np.triu(np.ones_like(C, dtype=bool)) if upper else np.tril(np.ones_like(C, dtype=bool))
    assert np.all(got[~tri] == 3.0)
    assert oracle.rel_fro(got[tri], C[tri]) <= TOL[dtype]


def _tri_system(size, k, dtype):
    """Test/hip_triangular_solve.cpp:104-122 inputs."""
    A = np.ones((size, size))
    for i in range(size):
        for j in range(i + 1):
            A[i, j] = 0.3 * (0.1 / size * i - 0.05 / (i + 1.0) * j) + (10 if i == j else 0)
    B = np.fromfunction(lambda i, j: (0.1 / size) * i + 0.1 / k * j, (size, k))
    return np.tril(A).astype(dtype), B.astype(dtype)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("left", [True, False])
@pytest.mark.parametrize("upper", [False, True])
@pytest.mark.parametrize("unit", [False, True])
@pytest.mark.parametrize("a_rm,b_rm", [(True, True), (True, False), (False, True), (False, False)])
def test_trsm(cuda, orc, dtype, left, upper, unit, a_rm, b_rm):
    size, k = 139, 238
    L, B = _tri_system(size, k, dtype)
    T = L.T.copy() if upper else L
    Bm = B if left else B.T.copy()
    Bd = to_dev(Bm, b_rm)
    ops.trsm(to_dev(T, a_rm), Bd, upper=upper, unit=unit, left=left)
    X = np.array(Bm)
    assert orc.trsm(T, X, upper=upper, unit=unit, left=left) == 0
    assert oracle.rel_fro(to_host(Bd), X) <= TOL[dtype]


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_trsm_large_random(cuda, orc, dtype):
    """n = 700 (5.5 blocks) with 33 right-hand sides, L = tril(U[-1,1]) + n I, alpha = 2."""
    n, k = 700, 33
    rs = np.random.default_rng(11)
    L = np.tril(rs.uniform(-1, 1, (n, n))) + n * np.eye(n)
    L = L.astype(dtype)
    B = rs.uniform(-1, 1, (n, k)).astype(dtype)
    Bd = to_dev(B, False)
    ops.trsm(to_dev(L, False), Bd, alpha=2.0)
    X = 2.0 * B.astype(np.float64)
    orc.trsm(L.astype(np.float64), X)
    assert oracle.rel_fro(to_host(Bd), X) <= TOL[dtype]


def test_trsm_zero_diagonal_reports_index(cuda):
    L = torch.eye(300, dtype=torch.float64, device="cuda") * 2
    L[200, 200] = 0.0
    B = torch.ones((300, 4), dtype=torch.float64, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    ops.trsm(L, B, info=info)
    assert int(info.item()) == 201
