"""The oracle restatement against the golden fixtures made by the reference's own code
(tests/golden/make_golden.py) and, where the reference is built here, against it live."""
from __future__ import annotations

import numpy as np
import pytest

import oracle


def test_threefry_words(orc, golden):
    g = golden("rng")
    key = g["key"].tolist()
    for ctr, words in zip(g["ctr"], g["words"]):
        assert orc.threefry(ctr.tolist(), key) == words.tolist()


def test_counter_mapping(orc, golden):
    g = golden("rng")
    pts = [(0, 0), (1, 0), (0, 4), (5, 12), (65535, 65532), (65536, 0), (65537, 65536), (70001, 131072),
           (2**32 + 3, 8), (7, 2**32 + 4), (2**33 + 65541, 2**34 + 65540)]
    for (i, j), ctr in zip(pts, g["ctr"]):
        assert orc.counter(i, j) == ctr.tolist()


@pytest.mark.parametrize("row_major", [True, False])
def test_rng_fills_bit_exact(orc, golden, row_major):
    g = golden("rng")
    key = g["key"].tolist()
    u = orc.rng_fill("uniform", key, 7, 13, row_major, -1.0, 1.0)
    assert np.array_equal(u.view(np.uint32), g["uniform"].view(np.uint32))
    n = orc.rng_fill("normal", key, 6, 10, row_major, 0.5, 2.0)
    assert np.array_equal(n.view(np.uint32), g["normal"].view(np.uint32))
    d = orc.rng_fill("discrete_f32", key, 5, 11, row_major, ia=-3, ib=6)
    assert np.array_equal(d, g["discrete"])


def test_input_generator(orc, golden):
    g = golden("generator")
    r = orc.rng(int(g["seed"]))
    assert np.array_equal(r.normal(5, 7, 0.0, 1.0, np.float64, True), g["normal64"])
    assert np.array_equal(r.uniform(4, 3, -1.0, 1.0, np.float64, False), g["uniform64"])
    assert np.array_equal(r.normal(3, 5, 1.0, 4.0, np.float32, True), g["normal32"])


@pytest.mark.parametrize("upper", [0, 1])
@pytest.mark.parametrize("rm", [0, 1])
def test_potrf_f64(orc, golden, upper, rm):
    g = golden("potrf")
    M = np.array(g["A"], order="C" if rm else "F")
    assert orc.potrf(M, upper=bool(upper)) == 0
    ref = g[f"L_u{upper}_r{rm}"]
    assert oracle.rel_fro(M, ref) <= 1e-14
    # the opposite triangle is untouched (Test/hip_cholesky.cpp:53-56 compares the whole matrix)
    other = np.tril(np.ones_like(M), -1) if upper else np.triu(np.ones_like(M), 1)
    assert np.array_equal(M[other == 1], g["A"][other == 1])


def test_potrf_f32(orc, golden):
    g = golden("potrf")
    A32 = g["A"].astype(np.float32)
    M = np.array(A32, order="C")
    assert orc.potrf(M, upper=False) == 0
    assert oracle.rel_fro(M, g["L32_u0_r1"]) <= 1e-6
    M = np.array(A32, order="F")
    assert orc.potrf(M, upper=True) == 0
    assert oracle.rel_fro(M, g["L32_u1_r0"]) <= 1e-6


def test_potrf_failing_pivot_is_global(orc, golden):
    g = golden("potrf")
    M = np.array(g["indef"], order="C")
    # The reference reports the index inside its recursive sub-block (61 -> 32 + 29, so
    # 40 - 32 = 8); the oracle and the CUDA kernels report the global index.
    assert int(g["indef_status"]) == 8
    assert orc.potrf(M, upper=False) == 40


@pytest.mark.parametrize("upper", [0, 1])
@pytest.mark.parametrize("unit", [0, 1])
def test_trsm(orc, golden, upper, unit):
    g = golden("trsm")
    T = g["L"] if not upper else g["L"].T.copy()
    X = np.array(g["B"], order="F")
    assert orc.trsm(T, X, upper=bool(upper), unit=bool(unit), left=True) == 0
    assert oracle.rel_fro(X, g[f"left_u{upper}_d{unit}"]) <= 1e-13
    Y = np.array(g["B"].T, order="C")
    assert orc.trsm(T, Y, upper=bool(upper), unit=bool(unit), left=False) == 0
    assert oracle.rel_fro(Y, g[f"right_u{upper}_d{unit}"]) <= 1e-13


def test_trsm_zero_diagonal(orc):
    L = np.tril(np.ones((5, 5)))
    L[3, 3] = 0.0
    assert orc.trsm(L, np.ones((5, 2))) == 1


def test_syrk_gemm(orc, golden):
    g = golden("syrk_gemm")
    for upper in (0, 1):
        C = np.full((37, 37), 3.0)
        orc.syrk(g["A"], C, alpha=2.0, upper=bool(upper))
        assert oracle.rel_fro(C, g[f"C_u{upper}"]) <= 1e-14
        untouched = np.tril(np.ones_like(C), -1) if upper else np.triu(np.ones_like(C), 1)
        assert np.all(C[untouched == 1] == 3.0)
    C = np.full((11, 13), 1.5)
    orc.gemm(np.asfortranarray(g["X"]), g["Y"], C, alpha=-2.0)
    assert oracle.rel_fro(C, g["G"]) <= 1e-14


def test_blas2(orc, golden):
    """gemv / trsv / trmv / trmm of the oracle against the reference's own kernels."""
    g = golden("blas2")
    for order in ("C", "F"):
        y = np.full(45, 0.25)
        orc.gemv(np.array(g["M"], order=order), g["x31"], y, alpha=-1.5)
        assert oracle.rel_fro(y[:, None], g[f"gemv_{order}"][:, None]) <= 1e-14
    for upper in (0, 1):
        T = g["L"] if not upper else g["L"].T.copy()
        for unit in (0, 1):
            for left in (1, 0):
                v = g["x"].copy()
                assert orc.trsv(T, v, upper=bool(upper), unit=bool(unit), left=bool(left)) == 0
                assert oracle.rel_fro(v[:, None], g[f"trsv_u{upper}_d{unit}_l{left}"][:, None]) <= 1e-13
            v = g["x"].copy()
            orc.trmm(T, v[:, None], upper=bool(upper), unit=bool(unit))
            assert oracle.rel_fro(v[:, None], g[f"trmv_u{upper}_d{unit}"][:, None]) <= 1e-14
            X = np.array(g["B"], order="F")
            orc.trmm(T, X, upper=bool(upper), unit=bool(unit))
            assert oracle.rel_fro(X, g[f"trmm_u{upper}_d{unit}"]) <= 1e-14


def _apply_swaps(A: np.ndarray, piv: np.ndarray, cols: bool) -> np.ndarray:
    """Row swaps i <-> piv[i] in order i = 0, 1, ... (and the same column swaps)."""
    B = A.copy()
    for i, p in enumerate(piv):
        if p != i:
            B[[i, p]] = B[[p, i]]
            if cols:
                B[:, [i, p]] = B[:, [p, i]]
    return B


@pytest.mark.parametrize("name", ["lu123", "lu61"])
@pytest.mark.parametrize("order", ["C", "F"])
def test_getrf(orc, golden, name, order):
    """LU with partial pivoting: the same pivots as the reference's kernels::getrf, factors
    within 1e-13, and P L U = A."""
    g = golden("lu_pstrf")
    A = g[f"{name}_A"]
    F = np.array(A, order=order)
    st, piv = orc.getrf(F)
    assert st == 0
    assert np.array_equal(piv, g[f"{name}_piv"])
    assert oracle.rel_fro(F, g[f"{name}_F"]) <= 1e-13
    L, U = np.tril(F, -1) + np.eye(len(piv)), np.triu(F)
    assert oracle.rel_fro(L @ U, _apply_swaps(A, piv, cols=False)) <= 1e-13


def test_getrf_f32_and_singular(orc):
    rs = np.random.default_rng(2)
    A = rs.uniform(-1, 1, (50, 50))
    F32 = np.array(A, dtype=np.float32)
    st, piv = orc.getrf(F32)
    F64 = A.copy()
    assert st == 0 and orc.getrf(F64)[0] == 0
    assert oracle.rel_fro(F32, F64) <= 1e-5
    S = A.copy()
    S[:, 7] = 0.0  # a zero column: the pivot search of column 7 finds only zeros
    assert orc.getrf(S)[0] == 8


@pytest.mark.parametrize("name", ["ps60", "ps57r25", "ps45r44"])
@pytest.mark.parametrize("order", ["C", "F"])
def test_pstrf(orc, golden, name, order):
    """Pivoted Cholesky against the reference's kernels::pstrf<lower>: the same rank, the
    same pivots before the rank, the same diagonal of L, and P^T A P = L L^T. (At the rank
    itself the reference swaps in the largest of the rounding-level remainders before it
    stops, so that one pivot depends on the summation order.)"""
    g = golden("lu_pstrf")
    A = g[f"{name}_A"]
    F = np.array(A, order=order)
    rank, piv = orc.pstrf(F)
    r = int(g[f"{name}_rank"])
    assert rank == r
    assert np.array_equal(piv[:r], g[f"{name}_piv"][:r])
    d, dref = np.diag(F)[:r], np.diag(g[f"{name}_F"])[:r]
    assert np.max(np.abs(d - dref) / dref) <= 1e-13
    assert np.all(np.triu(F, 1) == 0.0) and np.all(F[:, r:] == 0.0)
    assert oracle.rel_fro(F @ F.T, _apply_swaps(A, piv, cols=True)) <= 1e-13


def test_cholesky_solve(orc, golden):
    g = golden("solve")
    X = np.array(g["B"], order="F")
    assert orc.cholesky_solve(np.asfortranarray(g["A"]), X) == 0
    assert oracle.rel_fro(X, g["X"]) <= 1e-13


def test_against_live_reference(orc):
    """Wider random cases against the reference built here (skipped where it is absent)."""
    try:
        ref = oracle.Reference()
    except FileNotFoundError:
        pytest.skip("reference CPU path not built on this machine")
    rs = np.random.default_rng(3)
    key = rs.integers(0, 2**32, 4).tolist()
    for _ in range(500):
        ctr = rs.integers(0, 2**32, 4).tolist()
        assert orc.threefry(ctr, key) == ref.threefry(ctr, key)
    for n in (1, 31, 32, 33, 100, 130):
        A = oracle.create_symm(n)
        for upper in (False, True):
            for order in ("C", "F"):
                M1 = np.array(A, order=order)
                M2 = np.array(A, order=order)
                assert orc.potrf(M1, upper) == 0 and ref.potrf(M2, upper) == 0
                assert oracle.rel_fro(M1, M2) <= 1e-14
