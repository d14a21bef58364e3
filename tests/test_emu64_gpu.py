"""The emulated-FP64 trailing update (rc_syrk_emu64: int8 digit products on the tcgen05
tensor cores) and the mixed-precision solve built on it (precision "emu64").

Bars:
  * exactness: entries that are 28-bit integers times a power of two per row have four
    nonzero digits, so every digit pair the kernel keeps is the whole product and the
    only error left is the FP64 combination of the seven int32 sums: |C - P P^T| <=
    16 * 2^-53 * (|P| |P|^T) elementwise against an exact reference (14-bit limbs, whose
    FP64 products and sums are exact). A digit pair in the wrong accumulator, with the
    wrong weight or the wrong sign moves an entry by 2^-42 of that bound's scale or more;
  * general FP64 inputs: within the kernel's truncation bound k 2^-44 m_i m_j (m_i the
    largest |P(i, :)|) of the FP64 product, and inside k 2^-46 m_i m_j everywhere (the
    digits truncate toward zero, so on the diagonal the dropped pairs add up with one
    sign: about 2^-48.5 per term there);
  * the solve: kappa = 1e10 systems reach normwise backward error <= 1e-15 on every
    column, forward error within 100 kappa 2^-53 of the oracle's FP64 Cholesky solution."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from remora_b200 import _lib, ops
from helpers import to_dev, to_host

pytestmark = pytest.mark.gpu
U64 = 2.0 ** -53


def _syrk_emu(P: torch.Tensor, C: torch.Tensor, alpha: float, beta: float) -> int:
    n, k = P.shape
    return _lib.lib().rc_syrk_emu64(n, k, alpha, ctypes.c_void_p(P.data_ptr()), P.stride(0), beta,
                                    ctypes.c_void_p(C.data_ptr()), C.stride(0),
                                    ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))


def _int_rows(n: int, k: int, signed: bool, seed: int):
    """28-bit integer entries, rows scaled by 2^s_i (s_i in [-40, 40]); two zero rows."""
    rs = np.random.default_rng(seed)
    lo = -(2 ** 28) + 1 if signed else 0
    Pi = rs.integers(lo, 2 ** 28, size=(n, k)).astype(np.float64)
    s = rs.integers(-40, 41, size=n).astype(np.float64)
    if n > 4:
        Pi[1] = 0.0
        Pi[n - 2] = 0.0
    return Pi, s


@pytest.mark.parametrize("n,k", [(1, 1), (130, 129), (300, 128), (1000, 700), (513, 2048)])
@pytest.mark.parametrize("signed", [False, True])
def test_syrk_emu64_exact_on_four_digit_entries(cuda, n, k, signed):
    Pi, s = _int_rows(n, k, signed, seed=n + 7 * k + signed)
    P = torch.from_numpy(Pi * np.exp2(s)[:, None]).cuda()
    H = np.floor(Pi / 2 ** 14)
    L = Pi - H * 2 ** 14
    Hd, Ld = torch.from_numpy(H).cuda(), torch.from_numpy(L).cuda()
    X, Y, Z = Hd @ Hd.T, Hd @ Ld.T + Ld @ Hd.T, Ld @ Ld.T  # exact: integers < 2^40
    scale = torch.from_numpy(np.exp2(s[:, None] + s[None, :])).cuda()
    ref = ((X * 2.0 ** 28 + Y * 2.0 ** 14) + Z) * scale
    Ha = Hd.abs() * 2.0 ** 14 + Ld.abs()
    bound = 16 * U64 * (Ha @ Ha.T) * scale
    C = torch.full((n, n), float("nan"), device="cuda", dtype=torch.float64)
    assert _syrk_emu(P, C, -1.0, 0.0) == 0  # beta = 0 must not read the NaNs
    torch.cuda.synchronize()
    low = torch.ones((n, n), device="cuda", dtype=torch.bool).tril()
    err = (C + ref).abs()
    assert bool(torch.all(err[low] <= bound[low]))
    assert bool(torch.all(torch.isnan(C[~low])))  # strictly upper: untouched
    assert _lib.lib().rc_device_status(None) == 0


@pytest.mark.parametrize("n,k", [(257, 64), (1024, 1024), (2000, 333)])
def test_syrk_emu64_general_fp64(cuda, n, k):
    g = torch.Generator(device="cuda").manual_seed(n + k)
    P = torch.randn((n, k), generator=g, device="cuda", dtype=torch.float64)
    P *= torch.exp2(torch.randint(-30, 31, (n, 1), generator=g, device="cuda").double())
    C0 = torch.randn((n, n), generator=g, device="cuda", dtype=torch.float64)
    C = C0.clone()
    assert _syrk_emu(P, C, 0.5, 1.5) == 0
    ref = 0.5 * (P @ P.T) + 1.5 * C0
    m = P.abs().amax(dim=1)
    mm = m[:, None] * m[None, :]
    low = torch.ones((n, n), device="cuda", dtype=torch.bool).tril()
    err = (C - ref).abs()
    bound = k * 2.0 ** -44 * mm + 8 * U64 * (0.5 * (P.abs() @ P.abs().T) + 1.5 * C0.abs())
    assert bool(torch.all(err[low] <= bound[low]))
    typical = (err / (mm * k + 1.5 * C0.abs()))[low].max().item()
    assert typical <= 2.0 ** -46
    assert torch.equal(C.triu(1), C0.triu(1))


def test_syrk_emu64_nonfinite_rows_and_k0(cuda):
    n, k = 300, 200
    g = torch.Generator(device="cuda").manual_seed(3)
    P = torch.randn((n, k), generator=g, device="cuda", dtype=torch.float64)
    P[17, 5] = float("inf")
    C = torch.zeros((n, n), device="cuda", dtype=torch.float64)
    assert _syrk_emu(P, C, 1.0, 0.0) == 0
    torch.cuda.synchronize()
    low = torch.ones((n, n), device="cuda", dtype=torch.bool).tril()
    bad = torch.zeros((n, n), device="cuda", dtype=torch.bool)
    bad[17, :] = True
    bad[:, 17] = True
    assert bool(torch.all(torch.isnan(C[low & bad])))
    assert bool(torch.all(torch.isfinite(C[low & ~bad])))
    C2 = torch.randn((n, n), generator=g, device="cuda", dtype=torch.float64)
    C2c = C2.clone()
    assert _syrk_emu(P[:, :0], C2, 1.0, -2.0) == 0  # k = 0: C <- beta C on the lower triangle
    torch.cuda.synchronize()
    assert torch.equal(C2.tril(), (-2.0 * C2c).tril())
    assert torch.equal(C2.triu(1), C2c.triu(1))


def spd_with_condition(n: int, kappa: float, seed: int) -> np.ndarray:
    rs = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(rs.standard_normal((n, n)))
    lam = np.logspace(0, -np.log10(kappa), n)
    A = (Q * lam) @ Q.T
    return (A + A.T) / 2


def backward_error(A, X, B):
    R = B - A @ X
    return np.max(np.abs(R).max(axis=0) / (np.abs(A).sum(axis=1).max() * np.abs(X).max(axis=0) + np.abs(B).max(axis=0)))


@pytest.mark.parametrize("kappa", [1e2, 1e10, 1e12])
@pytest.mark.parametrize("outer", [128, 256, 1024])
def test_mixed_solve_emu64_conditioned(cuda, orc, kappa, outer):
    n, nrhs = 1000, 8
    A = spd_with_condition(n, kappa, seed=int(np.log10(kappa)))
    B = orc.rng(5).normal(n, nrhs)
    X, info, status = ops.spd_solve_mixed(to_dev(A, False), to_dev(B, False), "emu64", max_iter=100, outer=outer)
    assert info["pivot"] == 0
    assert status == 0, info
    Xh = to_host(X)
    assert backward_error(A, Xh, B) <= 1e-15
    ref = np.array(B, order="F")
    assert orc.cholesky_solve(np.asfortranarray(A), ref) == 0
    fwd = np.linalg.norm(Xh - ref) / np.linalg.norm(ref)
    assert fwd <= max(1e-13, 100 * kappa * U64)
    assert _lib.lib().rc_device_status(None) == 0


def test_mixed_solve_emu64_not_spd_reports_pivot(cuda):
    n = 300
    A = np.eye(n)
    A[200, 200] = -1.0
    X, info, status = ops.spd_solve_mixed(to_dev(A, False), to_dev(np.ones((n, 2)), False), "emu64", outer=128)
    assert info["pivot"] == 201


def test_syrk_emu64_matches_the_restatement(cuda):
    """General FP64 rows against the CPU restatement of the same digit-product method
    (oracle/emu64.py: the same digits, the same 28 pairs, the same single rounding of their
    combination), which leaves the truncation out of the comparison: the two agree to the
    rounding of the combination (16 2^-53 (|P| |P|^T)), hundreds of times tighter than the
    truncation bound, so a slice, pair, weight or sign out of place cannot pass."""
    from oracle import emu64
    rs = np.random.default_rng(77)
    n, k = 200, 300
    Ph = rs.standard_normal((n, k)) * np.exp2(rs.integers(-20, 21, size=(n, 1)))
    ref = emu64.syrk_emu64(Ph)
    P = torch.from_numpy(Ph).cuda()
    C = torch.full((n, n), float("nan"), device="cuda", dtype=torch.float64)
    assert _syrk_emu(P, C, 1.0, 0.0) == 0
    Ch = to_host(C)
    low = np.tril(np.ones((n, n), dtype=bool))
    bound = 16 * U64 * (np.abs(Ph) @ np.abs(Ph).T)
    assert np.all(np.abs(Ch - ref)[low] <= bound[low])
    assert np.all(np.isnan(Ch[~low]))
