"""Parity at the benchmark configurations' own sizes.

The BLAS-3 sweep (GEMM M = N = K in {4096, 16384} in every transpose/layout mix, SYRK
n = 8192 with k = 4096, lower TRSM n = 8192 with 1024 right-hand sides, FP32 and FP64),
the mixed-precision refined solve at n = 16384, the batched configuration's 4096 uneven
systems and the differentiated GP likelihood at n = 8192.

At these sizes the CPU checker cannot redo every product in seconds, so each check is a
sampled block of the result: rows spread over the whole range (first, last and random),
recomputed by the reference's own CPU kernels (oracle/_ref, Remora's kernels::gemm /
trsm / potrf; the restatement where _ref is absent, on fewer rows), plus the
size-independent properties the operation has -- the untouched triangle of SYRK stays
bit-identical, the TRSM residual L X - B on sampled rows, the leading block of the TRSM
solution against a full CPU solve of that block, normwise backward error and forward
error against a known solution for the SPD solves. Tolerances: relative Frobenius FP64
<= 1e-13, FP32 <= 1e-5 (the reference's own HIP tests accept 1e-2 % for products,
Test/hip_prod.cpp:117-259, and 1e-5 absolute for triangular solves,
Test/hip_triangular_solve.cpp:100-187)."""
from __future__ import annotations

import itertools

import numpy as np
import pytest
import torch

import oracle
from remora_b200 import ops

pytestmark = pytest.mark.gpu
TOL = {torch.float64: 1e-13, torch.float32: 1e-5}
NP = {torch.float64: np.float64, torch.float32: np.float32}


@pytest.fixture(scope="module")
def cpu():
    """The reference's CPU kernels where built, else the restatement (fewer sampled rows)."""
    try:
        return oracle.Reference(), 24
    except FileNotFoundError:
        return oracle.Oracle(), 4


def sample_rows(n: int, count: int, seed: int) -> np.ndarray:
    rs = np.random.default_rng(seed)
    mid = rs.choice(np.arange(1, n - 1), size=max(count - 2, 0), replace=False)
    return np.unique(np.concatenate([[0, n - 1], mid]))


def uniform(shape, dtype, seed, row_major=True):
    """U[-1, 1] on the device in the requested storage order."""
    g = torch.Generator(device="cuda").manual_seed(seed)
    if row_major:
        return torch.rand(shape, generator=g, device="cuda", dtype=dtype) * 2 - 1
    return (torch.rand((shape[1], shape[0]), generator=g, device="cuda", dtype=dtype) * 2 - 1).t()


def host(t: torch.Tensor) -> np.ndarray:
    torch.cuda.synchronize()
    return np.ascontiguousarray(t.cpu().numpy())


def rel(x: np.ndarray, ref: np.ndarray) -> float:
    return oracle.rel_fro(x.astype(np.float64), ref.astype(np.float64))


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("a_rm,b_rm,c_rm", list(itertools.product([True, False], repeat=3)))
def test_gemm_4096_all_orientations(cuda, cpu, dtype, a_rm, b_rm, c_rm):
    """C = -0.75 A B + 1.25 C at M = N = K = 4096, U[-1, 1] entries; the four transpose
    combinations are the row/column-major mixes of A and B (a row-major operand is the
    transpose of a column-major one), times both layouts of C."""
    ref, count = cpu
    n = 4096
    seed = 17 + 4 * a_rm + 2 * b_rm + c_rm
    A, B, C = uniform((n, n), dtype, seed, a_rm), uniform((n, n), dtype, seed + 100, b_rm), \
        uniform((n, n), dtype, seed + 200, c_rm)
    C0 = C.clone()
    ops.gemm(A, B, C, alpha=-0.75, beta=1.25)
    rows = sample_rows(n, count, seed)
    Ah, Bh = host(A[rows]), host(B)
    Cs = (1.25 * host(C0[rows])).astype(NP[dtype])
    ref.gemm(Ah, Bh, Cs, alpha=-0.75)
    assert rel(host(C[rows]), Cs) <= TOL[dtype]


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_gemm_16384(cuda, cpu, dtype):
    ref, count = cpu
    n = 16384
    A, B = uniform((n, n), dtype, 5, True), uniform((n, n), dtype, 6, False)
    C = torch.empty((n, n), device="cuda", dtype=dtype)
    ops.gemm(A, B, C, alpha=1.0, beta=0.0)
    rows = sample_rows(n, max(count // 3, 2), 7)
    Cs = np.zeros((len(rows), n), dtype=NP[dtype])
    ref.gemm(host(A[rows]), host(B), Cs)
    assert rel(host(C[rows]), Cs) <= TOL[dtype]


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("upper", [False, True])
def test_syrk_8192_by_4096(cuda, cpu, dtype, upper):
    """C_tri = 0.5 A A^T - C_tri at n = 8192, k = 4096; the other triangle is untouched."""
    ref, count = cpu
    n, k = 8192, 4096
    A = uniform((n, k), dtype, 31 + upper, True)
    C = uniform((n, n), dtype, 41 + upper, False)
    C0 = C.clone()
    ops.syrk(A, C, alpha=0.5, upper=upper, beta=-1.0)
    other = torch.tril(C, -1) if upper else torch.triu(C, 1)
    other0 = torch.tril(C0, -1) if upper else torch.triu(C0, 1)
    assert torch.equal(other, other0)
    rows = sample_rows(n, count, 51)
    Ah = host(A)
    Cs = (-host(C0[rows])).astype(NP[dtype])
    ref.gemm(np.ascontiguousarray(Ah[rows]), np.ascontiguousarray(Ah.T), Cs, alpha=0.5)
    got = host(C[rows])
    mask = np.array([[(j >= i) if upper else (j <= i) for j in range(n)] for i in rows])
    assert rel(np.where(mask, got, 0), np.where(mask, Cs, 0)) <= TOL[dtype]


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_trsm_lower_8192_with_1024_rhs(cuda, cpu, dtype):
    """X = L^-1 B with L = tril(U[-1, 1]) + n I, n = 8192, 1024 right-hand sides: the
    leading 1024 rows against the CPU solve of that block, the residual L X - B on rows
    sampled over the whole range."""
    ref, count = cpu
    n, nrhs = 8192, 1024
    L = torch.tril(uniform((n, n), dtype, 61, False)) + n * torch.eye(n, device="cuda", dtype=dtype)
    B = uniform((n, nrhs), dtype, 62, False)
    X = B.clone()
    ops.trsm(L, X, upper=False)
    lead = 1024
    Lh = host(L)
    Xl = np.asfortranarray(host(B[:lead]))
    assert ref.trsm(np.asfortranarray(Lh[:lead, :lead]), Xl, upper=False) == 0
    Xh = host(X)
    assert rel(Xh[:lead], Xl) <= TOL[dtype]
    rows = sample_rows(n, count, 63)
    R = -host(B[rows]).astype(NP[dtype])
    ref.gemm(np.ascontiguousarray(Lh[rows]), Xh, R)
    res = np.linalg.norm(R.astype(np.float64)) / (np.linalg.norm(Lh[rows].astype(np.float64)) *
                                                   np.linalg.norm(Xh.astype(np.float64)))
    assert res <= (1e-15 if dtype == torch.float64 else 1e-7)


def _spd(n: int, kappa: float, seed: int):
    g = torch.Generator(device="cuda").manual_seed(seed)
    G = torch.randn((n, n), generator=g, device="cuda", dtype=torch.float64)
    Q, _ = torch.linalg.qr(G)
    lam = torch.logspace(0.0, -np.log10(kappa), n, device="cuda", dtype=torch.float64)
    A = (Q * lam) @ Q.T
    return (A + A.T) * 0.5


@pytest.mark.parametrize("precision", ["tf32", "bf16"])
@pytest.mark.parametrize("kappa", [1e2, 1e6])
def test_mixed_solve_16384(cuda, precision, kappa):
    """The mixed-precision configuration at n = 16384, 64 right-hand sides: normwise
    backward error <= 1e-15 per column, and the forward error against a known solution
    X* (B = A X*, formed in FP64) within 100 kappa 2^-53."""
    n, nrhs = 16384, 64
    A = _spd(n, kappa, seed=int(np.log10(kappa)) + 160)
    g = torch.Generator(device="cuda").manual_seed(7)
    Xs = torch.randn((nrhs, n), generator=g, device="cuda", dtype=torch.float64).t()
    B = (A @ Xs).t().contiguous().t()
    X, info, status = ops.spd_solve_mixed(A, B, precision, max_iter=400)
    assert status == 0, info
    R = B - A @ X
    eta = R.abs().amax(dim=0) / (A.abs().sum(dim=0).max() * X.abs().amax(dim=0) + B.abs().amax(dim=0))
    assert float(eta.max()) <= 1e-15
    fwd = float(torch.linalg.norm(X - Xs) / torch.linalg.norm(Xs))
    assert fwd <= max(1e-13, 100 * kappa * 2.0 ** -53)


def test_mixed_solve_16384_kappa_1e10_emu64(cuda):
    """kappa = 1e10 at n = 16384 with 64 right-hand sides: the emulated-FP64 factor (int8
    digit-product trailing updates) preconditions CG to backward error <= 1e-15 on every
    column, forward error within 100 kappa 2^-53 of the known solution."""
    n, nrhs, kappa = 16384, 64, 1e10
    A = _spd(n, kappa, seed=170)
    g = torch.Generator(device="cuda").manual_seed(8)
    Xs = torch.randn((nrhs, n), generator=g, device="cuda", dtype=torch.float64).t()
    B = (A @ Xs).t().contiguous().t()
    X, info, status = ops.spd_solve_mixed(A, B, "emu64", max_iter=100)
    assert status == 0, info
    R = B - A @ X
    eta = R.abs().amax(dim=0) / (A.abs().sum(dim=0).max() * X.abs().amax(dim=0) + B.abs().amax(dim=0))
    assert float(eta.max()) <= 1e-15
    fwd = float(torch.linalg.norm(X - Xs) / torch.linalg.norm(Xs))
    assert fwd <= 100 * kappa * 2.0 ** -53


def _rbf_batch(count: int, seed: int):
    rs = np.random.default_rng(seed)
    sizes = rs.integers(16, 513, count)
    mats, rhs = [], []
    for n in sizes:
        X = rs.standard_normal((n, 8))
        sq = (X * X).sum(1)
        d2 = np.maximum(sq[:, None] + sq[None, :] - 2 * X @ X.T, 0.0)
        np.fill_diagonal(d2, 0.0)
        mats.append(np.exp(-0.5 * d2) + 1e-2 * np.eye(n))
        rhs.append(rs.standard_normal(n))
    return mats, rhs


@pytest.mark.parametrize("dtype,btol,ftol", [(torch.float64, 1e-14, 1e-12), (torch.float32, 1e-5, 1e-4)])
def test_batched_4096_systems(cuda, cpu, dtype, btol, ftol):
    """The batched configuration: 4096 RBF systems, n ~ U{16..512}, one launch in a CUDA
    graph. Every solution's backward error; every 64th factor against the CPU potrf."""
    ref, _ = cpu
    mats, rhs = _rbf_batch(4096, seed=44)
    sysb = ops.BatchedSystems(mats, rhs, dtype=dtype)
    sysb.solve(autotune=True)
    torch.cuda.synchronize()
    assert torch.all(sysb.info == 0)
    for i in range(len(mats)):
        x = sysb.solution(i).double().cpu().numpy()
        A, b = mats[i], rhs[i]
        eta = np.abs(b - A @ x).max() / (np.abs(A).sum(axis=1).max() * np.abs(x).max() + np.abs(b).max())
        assert eta <= btol, i
    for i in range(0, len(mats), 64):
        L = np.tril(sysb.factor(i).double().cpu().numpy())
        R = np.array(mats[i], order="F")
        assert ref.potrf(R) == 0
        assert oracle.rel_fro(L, np.tril(R)) <= ftol, i


def test_gp_gradient_8192(cuda):
    """The differentiated GP configuration at n = 8192 (16-dimensional inputs, lengthscales
    U[0.5, 2], noise 1e-2): the adjoint-kernel gradient against central differences of
    the FP64 forward pass (h = 1e-6) on three lengthscales. At this size the forward value
    f ~ 1e4 carries rounding ~1e-12 |f|, so the differences are good to ~1e-4 relative
    at best; the bar is 1e-3."""
    n, d = 8192, 16
    rs = np.random.default_rng(8192)
    X = torch.from_numpy(rs.standard_normal((n, d))).cuda()
    y = torch.from_numpy(rs.standard_normal(n)).cuda()
    ls = torch.from_numpy(rs.uniform(0.5, 2.0, d)).cuda()
    f, g, _ = ops.gp_nll_and_grad(X, y, ls, 1e-2)
    g = g.cpu().numpy()
    h = 1e-6
    for q in (0, 7, 15):
        e = torch.zeros(d, dtype=torch.float64, device="cuda")
        e[q] = h
        fp, _, _ = ops.gp_nll_and_grad(X, y, ls + e, 1e-2)
        fm, _, _ = ops.gp_nll_and_grad(X, y, ls - e, 1e-2)
        fd = (fp - fm) / (2 * h)
        assert abs(fd - g[q]) <= 1e-3 * max(1.0, abs(g[q])), (q, fd, g[q])
