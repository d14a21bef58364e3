"""POTRF and the Cholesky solve on the GPU through the C-ABI against the oracle
(FP64 <= 1e-13, FP32 <= 1e-5 relative Frobenius; the untouched triangle bit-identical)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle
from remora_b200 import ops

from helpers import to_dev, to_host

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("row_major", [True, False])
@pytest.mark.parametrize("upper", [False, True])
def test_potrf_create_symm_123(cuda, orc, row_major, upper):
    """Test/hip_cholesky.cpp:36-58: n = 123, every layout, compared on the WHOLE matrix."""
    A = oracle.create_symm(123)
    Ad = to_dev(A, row_major)
    assert ops.potrf(Ad, upper=upper) == 0
    got = to_host(Ad)
    ref = np.array(A)
    assert orc.potrf(ref, upper=upper) == 0
    assert oracle.rel_fro(got, ref) <= 1e-13
    other = np.tril(np.ones_like(A, dtype=bool), -1) if upper else np.triu(np.ones_like(A, dtype=bool), 1)
    assert np.array_equal(got[other], A[other])


@pytest.mark.parametrize("n", [1, 2, 127, 128, 129, 300, 1000])
def test_potrf_random_spd(cuda, orc, n):
    rs = np.random.default_rng(n)
    G = rs.standard_normal((n, n))
    A = G @ G.T / n + 1e-2 * np.eye(n)
    Ad = to_dev(A, False)
    assert ops.potrf(Ad) == 0
    ref = np.array(A, order="F")
    assert orc.potrf(ref) == 0
    assert oracle.rel_fro(np.tril(to_host(Ad)), np.tril(ref)) <= 1e-13


@pytest.mark.parametrize("row_major,upper", [(True, False), (False, True), (True, True), (False, False)])
def test_potrf_f32(cuda, orc, row_major, upper):
    A = oracle.create_symm(200).astype(np.float32)
    Ad = to_dev(A, row_major)
    assert ops.potrf(Ad, upper=upper) == 0
    ref = A.astype(np.float64)
    orc.potrf(ref, upper=upper)
    tri = np.triu(np.ones_like(ref, dtype=bool)) if upper else np.tril(np.ones_like(ref, dtype=bool))
    assert oracle.rel_fro(to_host(Ad)[tri], ref[tri]) <= 1e-5


@pytest.mark.parametrize("bad", [0, 39, 127, 128, 250])
def test_potrf_failing_pivot_global_index(cuda, orc, bad):
    A = oracle.create_symm(300)
    A[bad, bad] = -1.0
    ref = np.array(A)
    expect = orc.potrf(ref)
    assert expect == bad + 1
    assert ops.potrf(to_dev(A, False)) == expect
    assert ops.potrf(to_dev(A, True), upper=True) == expect


def test_potrf_nan_is_reported(cuda):
    A = torch.eye(64, dtype=torch.float64, device="cuda")
    A[10, 10] = float("nan")
    assert ops.potrf(A) == 11


def test_cholesky_solve_config1(cuda, orc):
    """n = 1024, 16 RHS: G ~ N(0,1) from mt19937(seed), A = G G^T / n + 1e-2 I, B ~ N(0,1)."""
    n, nrhs = 1024, 16
    g = orc.rng(1)
    G = g.normal(n, n)
    B = g.normal(n, nrhs)
    A = np.zeros((n, n))
    orc.gemm(G, np.ascontiguousarray(G.T), A, alpha=1.0 / n)
    A += 1e-2 * np.eye(n)
    Ad = to_dev(A, False)
    Bd = to_dev(B, False)
    assert ops.cholesky_solve(Ad, Bd) == 0
    X = to_host(Bd)
    ref = np.array(B, order="F")
    assert orc.cholesky_solve(np.asfortranarray(A), ref) == 0
    assert oracle.rel_fro(X, ref) <= 1e-13
    bwd = np.linalg.norm(A @ X - B) / (np.linalg.norm(A) * np.linalg.norm(X))
    assert bwd <= 1e-15
    assert np.array_equal(to_host(Ad), A)  # A is not modified


def test_cholesky_solve_golden(cuda, golden):
    g = golden("solve")
    Bd = to_dev(g["B"], False)
    assert ops.cholesky_solve(to_dev(g["A"], False), Bd) == 0
    assert oracle.rel_fro(to_host(Bd), g["X"]) <= 1e-13


def test_cholesky_solve_failure_leaves_b(cuda):
    A = oracle.create_symm(200)
    A[150, 150] = -5.0
    B = np.ones((200, 3))
    Bd = to_dev(B, False)
    assert ops.cholesky_solve(to_dev(A, False), Bd) == 151
    assert np.array_equal(to_host(Bd), B)
