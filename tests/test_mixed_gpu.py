"""Mixed-precision refined SPD solve against the FP64 oracle.

Inputs follow the mixed-precision configuration at reduced size: A = Q diag(lambda) Q^T
with Q from the QR of a seeded Gaussian matrix and lambda log-spaced from 1 to 1/kappa,
right-hand sides N(0,1) from the seeded host generator. Bars: normwise backward error
<= 1e-15 on every column (measured here independently in FP64), forward error against
the oracle's FP64 Cholesky solution <= 100 * kappa * 2^-53 (both are backward-stable
solutions of a kappa-conditioned system)."""
from __future__ import annotations

import numpy as np
import pytest

from remora_b200 import ops
from helpers import to_dev, to_host

pytestmark = pytest.mark.gpu
U64 = 2.0 ** -53


def spd_with_condition(n: int, kappa: float, seed: int) -> np.ndarray:
    rs = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(rs.standard_normal((n, n)))
    lam = np.logspace(0, -np.log10(kappa), n)
    A = (Q * lam) @ Q.T
    return (A + A.T) / 2


def backward_error(A, X, B):
    R = B - A @ X
    return np.max(np.abs(R).max(axis=0) / (np.abs(A).sum(axis=1).max() * np.abs(X).max(axis=0) + np.abs(B).max(axis=0)))


@pytest.mark.parametrize("precision", ["tf32", "bf16"])
@pytest.mark.parametrize("kappa", [1e2, 1e6])
def test_mixed_solve_conditioned(cuda, orc, precision, kappa):
    n, nrhs = 1000, 8
    A = spd_with_condition(n, kappa, seed=int(np.log10(kappa)))
    B = orc.rng(5).normal(n, nrhs)
    X, info, status = ops.spd_solve_mixed(to_dev(A, False), to_dev(B, False), precision, max_iter=400, outer=256)
    assert info["pivot"] == 0
    assert status == 0, info
    Xh = to_host(X)
    assert backward_error(A, Xh, B) <= 1e-15
    ref = np.array(B, order="F")
    assert orc.cholesky_solve(np.asfortranarray(A), ref) == 0
    fwd = np.linalg.norm(Xh - ref) / np.linalg.norm(ref)
    assert fwd <= max(1e-13, 100 * kappa * U64)


@pytest.mark.parametrize("precision", ["tf32", "bf16"])
def test_mixed_solve_kappa_1e10_reports_honestly(cuda, orc, precision):
    """At kappa = 1e10 a TF32/BF16 factor is too coarse a preconditioner: CG stalls near
    1e-9 (TF32) or the shifted BF16 factorisation breaks down. The solver must say so --
    RC_ERR_NOT_CONVERGED with the backward error it reached, or the failing pivot -- and
    never report convergence it did not reach."""
    n, nrhs = 1000, 8
    A = spd_with_condition(n, 1e10, seed=10)
    B = orc.rng(5).normal(n, nrhs)
    X, info, status = ops.spd_solve_mixed(to_dev(A, False), to_dev(B, False), precision, max_iter=60, outer=256)
    if info["pivot"]:
        assert status == 0 and info["converged"] == 0
        return
    measured = backward_error(A, to_host(X), B)
    if status == 0:
        assert info["converged"] == 1 and measured <= 1e-15
    else:
        assert status == 6 and info["converged"] == 0
        assert measured > 1e-15
        assert abs(measured - info["backward_error"]) <= 0.5 * measured


def test_mixed_solve_well_conditioned_few_iterations(cuda, orc):
    """SPD solve configuration recipe (A = G G^T / n + 1e-2 I) at n = 1536: converges in a
    handful of CG steps with either precision."""
    n, nrhs = 1536, 16
    g = orc.rng(11)
    G = g.normal(n, n)
    A = G @ G.T / n + 1e-2 * np.eye(n)
    B = g.normal(n, nrhs)
    for precision in ("tf32", "bf16"):
        X, info, status = ops.spd_solve_mixed(to_dev(A, False), to_dev(B, False), precision)
        assert status == 0 and info["converged"] == 1, info
        assert info["iterations"] <= 30
        assert backward_error(A, to_host(X), B) <= 1e-15


def test_mixed_solve_not_spd_reports_pivot(cuda):
    n = 300
    A = np.eye(n)
    A[200, 200] = -1.0
    X, info, status = ops.spd_solve_mixed(to_dev(A, False), to_dev(np.ones((n, 2)), False), "tf32")
    assert info["pivot"] == 201


@pytest.mark.parametrize("n,nrhs", [(3100, 70), (4096, 64), (2048, 1)])
def test_mixed_solve_block_steps_and_column_chunks(cuda, orc, n, nrhs):
    """Several diagonal blocks of the preconditioner solves (a ragged last block at
    n = 3100), right-hand sides spread over two 64-column chunks (nrhs = 70), exact
    multiples of both, and a single column."""
    A = spd_with_condition(n, 1e3, seed=n)
    B = orc.rng(n).normal(n, nrhs)
    X, info, status = ops.spd_solve_mixed(to_dev(A, False), to_dev(B, False), "tf32", max_iter=100)
    assert status == 0 and info["converged"] == 1, info
    Xh = to_host(X)
    assert backward_error(A, Xh, B) <= 1e-15
    ref = np.array(B, order="F")
    assert orc.cholesky_solve(np.asfortranarray(A), ref) == 0
    assert np.linalg.norm(Xh - ref) / np.linalg.norm(ref) <= 100 * 1e3 * U64


def _torch_spd(n: int, kappa: float, seed: int):
    """The headline inputs on the device: A = Q diag(lambda) Q^T (Q from the QR of a seeded
    Gaussian, lambda log-spaced 1 .. 1/kappa), exactly symmetric, column-major FP64."""
    import torch
    g = torch.Generator(device="cuda").manual_seed(seed)
    G = torch.randn((n, n), generator=g, device="cuda", dtype=torch.float64)
    Q, _ = torch.linalg.qr(G)
    lam = torch.logspace(0.0, -np.log10(kappa), n, device="cuda", dtype=torch.float64)
    A = (Q * lam) @ Q.T
    return (A + A.T) * 0.5


def _torch_backward_error(A, X, B) -> float:
    R = B - A @ X
    normA = A.abs().sum(dim=0).max()
    return float((R.abs().amax(dim=0) / (normA * X.abs().amax(dim=0) + B.abs().amax(dim=0))).max())


def test_mixed_solve_back_to_back_n8192(cuda):
    """Ten solves in a row at n = 8192 with 1024-column outer panels, so the look-ahead
    stream's panel chain runs beside the CTA-pair trailing updates on every panel; the
    device error word stays clear and every solve reaches the FP64 backward-error bar."""
    import ctypes
    import torch
    from remora_b200 import _lib
    n, nrhs = 8192, 64
    A = _torch_spd(n, 1e2, seed=81)
    B = torch.randn((nrhs, n), device="cuda", dtype=torch.float64).t()
    X = torch.empty((nrhs, n), device="cuda", dtype=torch.float64).t()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for _ in range(10):
        _, info, status = ops.spd_solve_mixed(A, B, "tf32", X=X)
        assert status == 0, info
        assert info["pivot"] == 0
        assert _torch_backward_error(A, X, B) <= 1e-15
    assert _lib.lib().rc_device_status(stream) == 0
