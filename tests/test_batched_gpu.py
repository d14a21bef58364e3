"""Batched uneven SPD solves (one persistent launch, CUDA graph) against the oracle.

Inputs follow the batched configuration at reduced count: systems of size n ~ U{16..512},
each an RBF kernel matrix exp(-|x - x'|^2 / 2) on points ~ N(0, I_8) plus 1e-2 I, one
N(0,1) right-hand side. Bars: the Cholesky factor against the oracle's (relative
Frobenius, FP64 <= 1e-12, FP32 <= 1e-4), the solution's normwise backward error (FP64
<= 1e-14, FP32 <= 1e-5), and failing pivots reported per system."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle
from remora_b200 import ops

pytestmark = pytest.mark.gpu


def rbf_systems(count: int, seed: int, lo: int = 16, hi: int = 512):
    rs = np.random.default_rng(seed)
    sizes = rs.integers(lo, hi + 1, count)
    mats, rhs = [], []
    for n in sizes:
        X = rs.standard_normal((n, 8))
        d2 = ((X[:, None, :] - X[None, :, :]) ** 2).sum(-1)
        mats.append(np.exp(-0.5 * d2) + 1e-2 * np.eye(n))
        rhs.append(rs.standard_normal(n))
    return mats, rhs


def bwd(A, x, b):
    return np.abs(b - A @ x).max() / (np.abs(A).sum(axis=1).max() * np.abs(x).max() + np.abs(b).max())


@pytest.mark.parametrize("dtype,ftol,btol", [(torch.float64, 1e-12, 1e-14), (torch.float32, 1e-4, 1e-5)])
def test_batched_uneven(cuda, orc, dtype, ftol, btol):
    mats, rhs = rbf_systems(96, seed=4)
    sys = ops.BatchedSystems(mats, rhs, dtype=dtype)
    sys.solve(autotune=True)
    torch.cuda.synchronize()
    assert torch.all(sys.info == 0)
    for i in range(len(mats)):
        x = sys.solution(i).double().cpu().numpy()
        assert bwd(mats[i], x, rhs[i]) <= btol, i
    for i in range(0, len(mats), 8):  # factors against the oracle on a subset
        L = np.tril(sys.factor(i).double().cpu().numpy())
        ref = np.array(mats[i])
        assert orc.potrf(ref) == 0
        assert oracle.rel_fro(L, np.tril(ref)) <= ftol, i


def test_batched_graph_replay_and_failures(cuda):
    mats, rhs = rbf_systems(40, seed=9, lo=16, hi=200)
    bad = {5: 3, 17: 100}
    for i, j in bad.items():
        j = min(j, mats[i].shape[0] - 1)
        bad[i] = j
        mats[i][j, j] = -1.0
    sys = ops.BatchedSystems(mats, rhs)
    # same pointer arrays twice: the second call replays the cached graph
    for _ in range(2):
        sys.A.copy_(torch.from_numpy(np.concatenate([m.T.reshape(-1) for m in mats])))
        sys.b.copy_(torch.from_numpy(np.concatenate(rhs)))
        sys.solve()
        torch.cuda.synchronize()
        info = sys.info.cpu().numpy()
        for i in range(len(mats)):
            if i in bad:
                assert info[i] == bad[i] + 1
            else:
                assert info[i] == 0
                assert bwd(mats[i], sys.solution(i).cpu().numpy(), rhs[i]) <= 1e-14


def test_batched_rejects_oversize(cuda):
    mats, rhs = [np.eye(513)], [np.ones(513)]
    sys = ops.BatchedSystems(mats, rhs)
    with pytest.raises(Exception):
        sys.solve()


def test_batched_plans_keep_element_types_apart(cuda):
    """An FP64 batch and then an FP32 batch passed through the SAME pointer-array, info
    buffers and sizes: the cached FP64 plan must not be replayed on FP32 storage."""
    mats, rhs = rbf_systems(24, seed=12, lo=16, hi=200)
    s64 = ops.BatchedSystems(mats, rhs, dtype=torch.float64)
    s64.solve(autotune=False)
    s32 = ops.BatchedSystems(mats, rhs, dtype=torch.float32)
    s64.a_ptrs.copy_(s32.a_ptrs)
    s64.b_ptrs.copy_(s32.b_ptrs)
    s32.a_ptrs, s32.b_ptrs, s32.info = s64.a_ptrs, s64.b_ptrs, s64.info
    s32.info.zero_()
    s32.solve(autotune=False)
    torch.cuda.synchronize()
    assert torch.all(s32.info == 0)
    for i in range(len(mats)):
        x = s32.solution(i).double().cpu().numpy()
        assert bwd(mats[i], x, rhs[i]) <= 1e-5, i
