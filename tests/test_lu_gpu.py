"""LU with partial pivoting (rc_getrf) and pivoted Cholesky (rc_pstrf) on the GPU against
the oracle and the reference's own results (tests/golden/lu_pstrf.npz).

getrf: the same pivots as the reference, factors within 1e-13 (relative Frobenius) on
the reference's test matrices, and P L U = A within 1e-13 on random ones (whose factors
may differ by the growth factor times the rounding). pstrf: the same rank, the same
pivots before the rank, L's diagonal within 1e-13, zeros above the diagonal and from
the rank on, and P^T A P = L L^T within 1e-13. The pivot taken at the rank itself picks
among rounding-level remainders and is not compared."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle
from remora_b200 import ops

from helpers import to_dev, to_host

pytestmark = pytest.mark.gpu


def _swaps(A: np.ndarray, piv: np.ndarray, cols: bool) -> np.ndarray:
    B = A.copy()
    for i, p in enumerate(piv):
        if p != i:
            B[[i, p]] = B[[p, i]]
            if cols:
                B[:, [i, p]] = B[:, [p, i]]
    return B


def _lu_check(A: np.ndarray, F: np.ndarray, piv: np.ndarray, tol: float) -> None:
    n = len(piv)
    L, U = np.tril(F, -1) + np.eye(n), np.triu(F)
    assert oracle.rel_fro(L @ U, _swaps(A, piv, cols=False)) <= tol


@pytest.mark.parametrize("name", ["lu123", "lu61"])
@pytest.mark.parametrize("row_major", [False, True])
def test_getrf_golden(cuda, golden, name, row_major):
    g = golden("lu_pstrf")
    A = g[f"{name}_A"]
    Ad = to_dev(A, row_major)
    info, piv = ops.getrf(Ad)
    assert info == 0
    piv = piv.cpu().numpy()
    assert np.array_equal(piv, g[f"{name}_piv"])
    F = to_host(Ad)
    assert oracle.rel_fro(F, g[f"{name}_F"]) <= 1e-13
    _lu_check(A, F, piv, 1e-13)


@pytest.mark.parametrize("n", [1, 63, 64, 65, 300, 777])
def test_getrf_random(cuda, orc, n):
    rs = np.random.default_rng(n)
    A = rs.uniform(-1, 1, (n, n))
    Ad = to_dev(A, False)
    info, piv = ops.getrf(Ad)
    assert info == 0
    F2 = np.array(A, order="F")
    st, piv2 = orc.getrf(F2)
    assert st == 0 and np.array_equal(piv.cpu().numpy(), piv2)
    _lu_check(A, to_host(Ad), piv2, 1e-13)


def test_getrf_multi_cta_panel_2048(cuda, orc):
    """n = 2048: the panels run on a cooperative grid (up to one CTA per SM, one grid
    barrier per column); the pivots are the oracle's and P L U = A within 1e-13."""
    n = 2048
    rs = np.random.default_rng(2048)
    A = rs.uniform(-1, 1, (n, n))
    Ad = to_dev(A, True)
    info, piv = ops.getrf(Ad)
    assert info == 0
    F2 = np.array(A, order="F")
    st, piv2 = orc.getrf(F2)
    assert st == 0 and np.array_equal(piv.cpu().numpy(), piv2)
    _lu_check(A, to_host(Ad), piv2, 1e-13)


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-13), (torch.float32, 1e-4)])
def test_getrf_8192_residual(cuda, dtype, tol):
    """n = 8192 on the device: P L U = A (relative Frobenius) with the returned pivots."""
    n = 8192
    g = torch.Generator(device="cuda").manual_seed(81)
    A = torch.rand((n, n), generator=g, device="cuda", dtype=dtype) * 2 - 1
    F = A.clone()
    info, piv = ops.getrf(F)
    assert info == 0
    L = torch.tril(F.double(), -1) + torch.eye(n, device="cuda", dtype=torch.float64)
    U = torch.triu(F.double())
    PA = A.double().clone()
    p = piv.cpu().numpy()
    perm = np.arange(n)
    for i, q in enumerate(p):
        if q != i:
            perm[[i, q]] = perm[[q, i]]
    PA = PA[torch.from_numpy(perm).cuda()]
    rel = float(torch.linalg.norm(L @ U - PA) / torch.linalg.norm(PA))
    assert rel <= tol


def test_getrf_f32(cuda, golden):
    g = golden("lu_pstrf")
    A = g["lu123_A"]
    Ad = to_dev(A, False, dtype=np.float32)
    info, piv = ops.getrf(Ad)
    assert info == 0
    assert np.array_equal(piv.cpu().numpy(), g["lu123_piv"])
    assert oracle.rel_fro(to_host(Ad), g["lu123_F"]) <= 1e-5


def test_getrf_zero_pivot(cuda):
    rs = np.random.default_rng(9)
    A = rs.uniform(-1, 1, (200, 200))
    A[:, 70] = 0.0
    info, _ = ops.getrf(to_dev(A, False))
    assert info == 71


@pytest.mark.parametrize("name", ["ps60", "ps57r25", "ps45r44"])
@pytest.mark.parametrize("row_major", [False, True])
def test_pstrf_golden(cuda, golden, name, row_major):
    g = golden("lu_pstrf")
    A = g[f"{name}_A"]
    Ad = to_dev(A, row_major)
    rank, piv = ops.pstrf(Ad)
    r = int(g[f"{name}_rank"])
    assert rank == r
    piv = piv.cpu().numpy()
    assert np.array_equal(piv[:r], g[f"{name}_piv"][:r])
    F = to_host(Ad)
    d, dref = np.diag(F)[:r], np.diag(g[f"{name}_F"])[:r]
    assert np.max(np.abs(d - dref) / dref) <= 1e-13
    assert np.all(np.triu(F, 1) == 0.0) and np.all(F[:, r:] == 0.0)
    assert oracle.rel_fro(F @ F.T, _swaps(A, piv, cols=True)) <= 1e-13


def _semidef(n: int, rank: int) -> np.ndarray:
    """R R^T with R(i, j) = 0.2 / |i - j| below the diagonal (columns < rank) and
    R(i, i) = 1 + i / (2 n) for i < rank, rows and columns 2 i and n - 1 - i swapped for
    i < rank / 2 (the reference's semidefinite test recipe, Test/symm_solve.cpp:17-38)."""
    R = np.zeros((n, n))
    for i in range(n):
        for j in range(min(i, rank)):
            R[i, j] = 0.2 / abs(i - j)
        if i < rank:
            R[i, i] = 0.5 / n * i + 1
    A = R @ R.T
    if rank != n:
        for i in range(rank // 2):
            a, b = 2 * i, n - i - 1
            A[[a, b]] = A[[b, a]]
            A[:, [a, b]] = A[:, [b, a]]
    return A


@pytest.mark.parametrize("n,rank", [(200, 200), (333, 120)])
def test_pstrf_against_oracle(cuda, orc, n, rank):
    A = _semidef(n, rank)
    Ad = to_dev(A, False)
    r, piv = ops.pstrf(Ad)
    F2 = np.array(A, order="F")
    r2, piv2 = orc.pstrf(F2)
    assert r == r2
    assert np.array_equal(piv.cpu().numpy()[:r], piv2[:r])
    F = to_host(Ad)
    assert oracle.rel_fro(F @ F.T, _swaps(A, piv.cpu().numpy(), cols=True)) <= 1e-13
