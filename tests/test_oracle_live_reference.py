"""The oracle against the reference's own CPU kernels (oracle/_ref), on seeded random
shapes, orientations and element types beyond the committed golden fixtures.

Runs where the reference was built (skipped elsewhere). Tolerances: the two compute the same
sums, in orders that may differ, so FP64 agrees to ~1e-13 and FP32 to ~1e-5 relative
Frobenius; getrf's pivot sequence must be identical, and pstrf's up to the rank."""
from __future__ import annotations

import numpy as np
import pytest

import oracle

TOL = {np.float64: 1e-13, np.float32: 2e-5}


@pytest.fixture(scope="module")
def ref():
    try:
        return oracle.Reference()
    except FileNotFoundError:
        pytest.skip("reference CPU path not built on this machine")


@pytest.fixture(scope="module")
def orc():
    return oracle.Oracle()


def _arr(rs, shape, dtype, order, low=-1.0, high=1.0):
    return np.array(rs.uniform(low, high, shape), dtype=dtype, order=order)


CASES = [(dt, o) for dt in (np.float64, np.float32) for o in ("C", "F")]


@pytest.mark.parametrize("dtype,order", CASES)
def test_gemm_random_shapes(orc, ref, dtype, order):
    rs = np.random.default_rng(11)
    for m, n, k in ((1, 1, 1), (7, 130, 33), (129, 64, 257), (200, 3, 90)):
        A = _arr(rs, (m, k), dtype, order)
        B = _arr(rs, (k, n), dtype, "F" if order == "C" else "C")
        C1 = _arr(rs, (m, n), dtype, order)
        C2 = C1.copy(order="A")
        orc.gemm(A, B, C1, alpha=-0.75)
        ref.gemm(A, B, C2, alpha=-0.75)
        assert oracle.rel_fro(C1, C2) <= TOL[dtype], (m, n, k)


@pytest.mark.parametrize("dtype,order", CASES)
@pytest.mark.parametrize("upper", [False, True])
def test_syrk_random_shapes(orc, ref, dtype, order, upper):
    rs = np.random.default_rng(12)
    for n, k in ((1, 5), (33, 1), (130, 77), (97, 200)):
        A = _arr(rs, (n, k), dtype, order)
        C1 = _arr(rs, (n, n), dtype, order)
        C2 = C1.copy(order="A")
        orc.syrk(A, C1, alpha=0.5, upper=upper)
        ref.syrk(A, C2, alpha=0.5, upper=upper)
        assert oracle.rel_fro(C1, C2) <= TOL[dtype], (n, k)
        untouched = np.tril(np.ones((n, n), bool), -1) if upper else np.triu(np.ones((n, n), bool), 1)
        assert np.array_equal(C1[untouched], C2[untouched])


@pytest.mark.parametrize("dtype,order", CASES)
@pytest.mark.parametrize("upper,unit,left", [(u, d, s) for u in (False, True) for d in (False, True)
                                             for s in (True, False)])
def test_trsm_random_shapes(orc, ref, dtype, order, upper, unit, left):
    rs = np.random.default_rng(13)
    for n, r in ((1, 3), (45, 17), (150, 64)):
        T = _arr(rs, (n, n), dtype, order) + n * np.eye(n, dtype=dtype)
        T = np.array(np.triu(T) if upper else np.tril(T), dtype=dtype, order=order)
        shape = (n, r) if left else (r, n)
        B1 = _arr(rs, shape, dtype, order)
        B2 = B1.copy(order="A")
        assert orc.trsm(T, B1, upper=upper, unit=unit, left=left) == 0
        ref.trsm(T, B2, upper=upper, unit=unit, left=left)
        assert oracle.rel_fro(B1, B2) <= TOL[dtype], (n, r)


@pytest.mark.parametrize("dtype,order", CASES)
def test_getrf_random_pivots_identical(orc, ref, dtype, order):
    rs = np.random.default_rng(14)
    for n in (1, 2, 31, 65, 160):
        A = _arr(rs, (n, n), dtype, order)
        A1, A2 = A.copy(order="A"), A.copy(order="A")
        st1, p1 = orc.getrf(A1)
        st2, p2 = ref.getrf(A2)
        assert st1 == 0 and st2 == 0
        assert np.array_equal(p1, p2), n
        assert oracle.rel_fro(A1, A2) <= 10 * TOL[dtype], n


def _rows_in_original_order(L: np.ndarray, piv: np.ndarray) -> np.ndarray:
    """The rows of a pivoted factor put back in A's order: piv holds the swap made at each
    step (Remora's permutation_matrix order)."""
    perm = np.arange(L.shape[0])
    for i, q in enumerate(piv):
        perm[[i, q]] = perm[[q, i]]
    out = np.empty_like(L)
    out[perm] = L
    return out


@pytest.mark.parametrize("order", ["C", "F"])
def test_pstrf_random_rank_and_pivots(orc, ref, order):
    """FP64 only: the reference's FP32 pstrf does not compile (kernels/default/pstrf.hpp:78
    calls std::max(double&, float)). Past the rank, the last swap picks the largest of the
    remaining pivot values, which are rounding noise, so pivots are compared up to the rank
    and the factor's first rank columns with the rows put back in A's order."""
    rs = np.random.default_rng(15)
    for n, rank in ((1, 1), (40, 40), (96, 57), (130, 13)):
        G = rs.standard_normal((n, rank))
        A = np.array(G @ G.T, order=order)
        A1, A2 = A.copy(order="A"), A.copy(order="A")
        r1, p1 = orc.pstrf(A1)
        r2, p2 = ref.pstrf(A2)
        assert r1 == r2 == rank, (n, rank, r1, r2)
        assert np.array_equal(p1[:rank], p2[:rank]), (n, rank)
        L1 = _rows_in_original_order(np.tril(A1)[:, :rank], p1)
        L2 = _rows_in_original_order(np.tril(A2)[:, :rank], p2)
        assert oracle.rel_fro(L1, L2) <= 1e-12, (n, rank)


@pytest.mark.parametrize("order", ["C", "F"])
def test_cholesky_solve_random(orc, ref, order):
    rs = np.random.default_rng(16)
    for n, r in ((1, 1), (77, 5), (140, 33)):
        G = rs.standard_normal((n, n))
        A = np.array(G @ G.T / n + 1e-1 * np.eye(n), order=order)
        B = np.array(rs.standard_normal((n, r)), order=order)
        X1, X2 = B.copy(order="A"), B.copy(order="A")
        assert orc.cholesky_solve(A.copy(order="A"), X1) == 0
        assert ref.cholesky_solve(A.copy(order="A"), X2) == 0
        assert oracle.rel_fro(X1, X2) <= 1e-12, (n, r)


@pytest.mark.parametrize("dtype,order", CASES)
def test_blas2_and_trmm_random_shapes(orc, ref, dtype, order):
    rs = np.random.default_rng(17)
    for n, r in ((1, 1), (37, 5), (130, 40)):
        A = _arr(rs, (n, n + 3), dtype, order)
        x = _arr(rs, (n + 3,), dtype, "C")
        y1 = _arr(rs, (n,), dtype, "C")
        y2 = y1.copy()
        orc.gemv(A, x, y1, alpha=1.5)
        ref.gemv(A, x, y2, alpha=1.5)
        assert oracle.rel_fro(y1, y2) <= TOL[dtype], n
        for upper in (False, True):
            for unit in (False, True):
                T = _arr(rs, (n, n), dtype, order) + n * np.eye(n, dtype=dtype)
                T = np.array(np.triu(T) if upper else np.tril(T), dtype=dtype, order=order)
                for left in (True, False):
                    v1 = _arr(rs, (n,), dtype, "C")
                    v2 = v1.copy()
                    assert orc.trsv(T, v1, upper=upper, unit=unit, left=left) == 0
                    ref.trsv(T, v2, upper=upper, unit=unit, left=left)
                    assert oracle.rel_fro(v1, v2) <= TOL[dtype], (n, upper, unit, left)
                v1 = _arr(rs, (n,), dtype, "C")
                v2 = v1.copy()
                orc.trmm(T, v1.reshape(n, 1), upper=upper, unit=unit)
                ref.trmv(T, v2, upper=upper, unit=unit)
                assert oracle.rel_fro(v1, v2) <= TOL[dtype], (n, upper, unit)
                B1 = _arr(rs, (n, r), dtype, order)
                B2 = B1.copy(order="A")
                orc.trmm(T, B1, upper=upper, unit=unit)
                ref.trmm(T, B2, upper=upper, unit=unit)
                assert oracle.rel_fro(B1, B2) <= TOL[dtype], (n, r, upper, unit)


def test_rng_blocks_at_random_offsets(orc, ref):
    """Fills of 3 x 8 blocks at random row/column offsets (around the 16-bit counter masks
    and past 2^32) under random keys, against the reference's own per-group device functions
    compiled as host code (counter of group (i, j): kernels/hip/random.hpp:167). Host libm on
    both sides, so the float transforms are compared bit for bit as well."""
    rs = np.random.default_rng(18)
    offsets = [(0, 0), (65534, 65532), (2**32 - 1, 4), (12345, 2**32 + 8), (2**40 + 7, 2**33 + 65536)]
    offsets += [(int(rs.integers(0, 2**48)), 4 * int(rs.integers(0, 2**40))) for _ in range(6)]
    for row0, col0 in offsets:
        key = [int(v) for v in rs.integers(0, 2**32, 4)]
        got = {k: orc.rng_fill(k, key, 3, 8, True, -1.5, 2.5, ia=-4, ib=9, row0=row0, col0=col0)
               for k in ("uniform", "normal", "discrete_f32")}
        for i in range(3):
            for j in range(0, 8, 4):
                r, c = row0 + i, col0 + j
                ctr = [r & 0xFFFF, (r >> 32) & 0xFFFFFFFF, c & 0xFFFF, (c >> 32) & 0xFFFFFFFF]
                x = ref.threefry(ctr, key)
                want = {"uniform": ref.uniform4(-1.5, 2.5, x), "normal": ref.normal4(-1.5, 2.5, x),
                        "discrete_f32": [v - 4 for v in ref.discrete4(key, ctr, 14)]}
                for k, w in want.items():
                    a = np.asarray(got[k][i, j:j + 4], dtype=np.float32)
                    assert np.array_equal(a.view(np.uint32), np.asarray(w, np.float32).view(np.uint32)), (k, r, c)
