"""Reverse-mode adjoints of Cholesky and TRSM, and the differentiated GP marginal
likelihood, against FP64 central finite differences (h = 1e-6, computed with the oracle)
and against the gradient composed from the oracle's Cholesky solves
(1/2 (K^-1 - alpha alpha^T), K^-1 by solving with the identity)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from remora_b200 import ops
from helpers import to_dev, to_host

pytestmark = pytest.mark.gpu
H = 1e-6


def spd(n, seed):
    rs = np.random.default_rng(seed)
    G = rs.standard_normal((n, n))
    return G @ G.T / n + np.eye(n)


def chol(orc, A):
    L = np.array(A, order="F")
    assert orc.potrf(L) == 0
    return np.tril(L)


@pytest.mark.parametrize("n", [50, 300])
def test_potrf_backward_vs_finite_differences(cuda, orc, n):
    A = spd(n, n)
    rs = np.random.default_rng(1)
    W = np.tril(rs.standard_normal((n, n)))  # f(L) = sum(W * L), so Lbar = W
    L = chol(orc, A)
    Abar = to_host(ops.potrf_backward(to_dev(L, False), to_dev(W, False)))
    assert np.allclose(Abar, Abar.T, atol=1e-12 * np.abs(Abar).max())
    for t in range(3):
        E = rs.standard_normal((n, n))
        E = (E + E.T) / 2
        fd = (np.sum(W * chol(orc, A + H * E)) - np.sum(W * chol(orc, A - H * E))) / (2 * H)
        an = np.sum(Abar * E)
        assert abs(fd - an) <= 1e-6 * max(1.0, abs(an)), (t, fd, an)


@pytest.mark.parametrize("trans", [False, True])
def test_trsm_backward_vs_finite_differences(cuda, orc, trans):
    n, k = 200, 7
    rs = np.random.default_rng(3)
    L = np.tril(rs.uniform(-1, 1, (n, n))) + n * np.eye(n) / 10
    B = rs.standard_normal((n, k))
    W = rs.standard_normal((n, k))  # f = sum(W * X)

    def solve(Lm, Bm):
        X = np.array(Bm, order="F")
        T = Lm.T.copy() if trans else Lm
        assert orc.trsm(T, X, upper=trans) == 0
        return X

    X = solve(L, B)
    Ld, Xd, Wd = to_dev(L, False), to_dev(X, False), to_dev(W, False)
    Lbar = torch.zeros((n, n), dtype=torch.float64, device="cuda").t()
    Bbar = to_host(ops.trsm_backward(Ld, Xd, Wd, Lbar, trans=trans))
    Lbar = np.tril(to_host(Lbar))
    EB = rs.standard_normal((n, k))
    fd = (np.sum(W * solve(L, B + H * EB)) - np.sum(W * solve(L, B - H * EB))) / (2 * H)
    assert abs(fd - np.sum(Bbar * EB)) <= 1e-6 * max(1.0, abs(fd))
    EL = np.tril(rs.standard_normal((n, n)))
    fd = (np.sum(W * solve(L + H * EL, B)) - np.sum(W * solve(L - H * EL, B))) / (2 * H)
    assert abs(fd - np.sum(Lbar * EL)) <= 1e-6 * max(1.0, abs(fd))


def gp_problem(n, seed=0):
    rs = np.random.default_rng(seed)
    X = rs.standard_normal((n, 16))
    y = rs.standard_normal(n)
    ls = rs.uniform(0.5, 2.0, 16)
    return X, y, ls, 1e-2


def rbf_np(X, ls, noise):
    Z = X / ls
    d2 = ((Z[:, None, :] - Z[None, :, :]) ** 2).sum(-1)
    return np.exp(-0.5 * d2) + noise * np.eye(X.shape[0])


def nll_oracle(orc, X, y, ls, noise):
    K = rbf_np(X, ls, noise)
    L = chol(orc, K)
    a = np.array(y.reshape(-1, 1), order="F")
    assert orc.cholesky_solve(np.asfortranarray(K), a) == 0
    return 0.5 * float(y @ a[:, 0]) + float(np.log(np.diag(L)).sum())


def test_gp_marginal_likelihood_gradient(cuda, orc):
    n = 256
    X, y, ls, noise = gp_problem(n)
    f, g, Kbar = ops.gp_nll_and_grad(torch.from_numpy(X).cuda(), torch.from_numpy(y).cuda(),
                                     torch.from_numpy(ls).cuda(), noise)
    g = g.cpu().numpy()
    # forward value against the oracle
    assert abs(f - nll_oracle(orc, X, y, ls, noise)) <= 1e-10 * abs(f)
    # gradient composed from the oracle's Cholesky solves: Kbar = 1/2 (K^-1 - alpha alpha^T)
    K = rbf_np(X, ls, noise)
    Kinv = np.eye(n, order="F")
    assert orc.cholesky_solve(np.asfortranarray(K), Kinv) == 0
    alpha = np.array(y.reshape(-1, 1), order="F")
    orc.cholesky_solve(np.asfortranarray(K), alpha)
    Kbar_ref = 0.5 * (Kinv - alpha @ alpha.T)
    assert np.linalg.norm(to_host(Kbar) - Kbar_ref) <= 1e-9 * np.linalg.norm(Kbar_ref)
    k = K - noise * np.eye(n)
    g_ref = np.array([np.sum(Kbar_ref * k * (X[:, None, q] - X[None, :, q]) ** 2) / ls[q] ** 3 for q in range(16)])
    assert np.allclose(g, g_ref, rtol=1e-9, atol=1e-12 * np.abs(g_ref).max())
    # central finite differences, h = 1e-6
    for q in (0, 5, 15):
        e = np.zeros(16)
        e[q] = H
        fd = (nll_oracle(orc, X, y, ls + e, noise) - nll_oracle(orc, X, y, ls - e, noise)) / (2 * H)
        assert abs(fd - g[q]) <= 1e-6 * max(1.0, abs(g[q])), (q, fd, g[q])
