"""Generate the golden fixtures in this directory from the REFERENCE'S OWN CODE.

Runs Remora's CPU kernels and its device RNG functions (compiled for the host by
``oracle/Makefile`` into ``oracle/_ref/libremora_ref.so`` from the reference headers)
on the reference tests' own formula-built inputs, and stores inputs and outputs as
``.npz`` files. The oracle restatement is pinned against these fixtures by
``tests/test_oracle_golden.py``; the fixtures travel, the reference does not.

    python tests/golden/make_golden.py      # needs the reference headers and make
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402

OUT = Path(__file__).resolve().parent


def rng_fixture(ref: oracle.Reference) -> None:
    g = ref.rng(42)
    key = np.array(g.key(), dtype=np.uint32)  # kernels/hip/random.hpp:225-227
    # Counters of groups (i, j) that cover the 16-bit masks and the >> 32 halves of
    # random.hpp:167: small, around 2^16 and above 2^32.
    pts = [(0, 0), (1, 0), (0, 4), (5, 12), (65535, 65532), (65536, 0), (65537, 65536), (70001, 131072),
           (2**32 + 3, 8), (7, 2**32 + 4), (2**33 + 65541, 2**34 + 65540)]
    ctrs, words = [], []
    for i, j in pts:
        ctr = [i & 0xFFFF, (i >> 32) & 0xFFFFFFFF, j & 0xFFFF, (j >> 32) & 0xFFFFFFFF]
        ctrs.append(ctr)
        words.append(ref.threefry(ctr, key.tolist()))
    # Small fills assembled from the reference's per-group functions, row-major order.
    def fill(rows, cols, fn):
        out = np.zeros((rows, cols), dtype=np.float32)
        for i in range(rows):
            for j in range(0, cols, 4):
                ctr = [i & 0xFFFF, i >> 32, j & 0xFFFF, j >> 32]
                vals = fn(ref.threefry(ctr, key.tolist()), ctr)
                for c in range(4):
                    if j + c < cols:
                        out[i, j + c] = vals[c]
        return out
    uni = fill(7, 13, lambda x, c: ref.uniform4(-1.0, 1.0, x))
    nrm = fill(6, 10, lambda x, c: ref.normal4(0.5, 2.0, x))
    dsc = fill(5, 11, lambda x, c: [v - 3 for v in ref.discrete4(key.tolist(), c, 10)])  # low = -3, high = 6
    np.savez_compressed(OUT / "rng.npz", key=key, ctr=np.array(ctrs, dtype=np.uint32),
                        words=np.array(words, dtype=np.uint32), uniform=uni, normal=nrm, discrete=dsc)


def generator_fixture(ref: oracle.Reference) -> None:
    g = ref.rng(1234)
    n64 = g.normal(5, 7, 0.0, 1.0, np.float64, row_major=True)
    u64 = g.uniform(4, 3, -1.0, 1.0, np.float64, row_major=False)
    n32 = g.normal(3, 5, 1.0, 4.0, np.float32, row_major=True)
    np.savez_compressed(OUT / "generator.npz", seed=1234, normal64=n64, uniform64=u64, normal32=n32)


def potrf_fixture(ref: oracle.Reference) -> None:
    n = 61  # not a multiple of the reference's 32-block, so its recursion splits unevenly
    A = oracle.create_symm(n)
    res = {"A": A}
    for upper in (0, 1):
        for rm in (0, 1):
            M = np.array(A, order="C" if rm else "F")
            status = ref.potrf(M, upper=bool(upper))
            assert status == 0
            res[f"L_u{upper}_r{rm}"] = M
    # FP32: only the two layouts the reference can compile (kernels/default/potrf.hpp:74)
    A32 = A.astype(np.float32)
    M = np.array(A32, order="C")
    assert ref.potrf(M, upper=False) == 0
    res["L32_u0_r1"] = M
    M = np.array(A32, order="F")
    assert ref.potrf(M, upper=True) == 0
    res["L32_u1_r0"] = M
    # An indefinite matrix: pivot 40 (1-based) fails.
    B = A.copy()
    B[39, 39] = -1.0
    M = np.array(B, order="C")
    res["indef"] = B
    res["indef_status"] = np.array(ref.potrf(M, upper=False))
    np.savez_compressed(OUT / "potrf.npz", **res)


def trsm_fixture(ref: oracle.Reference) -> None:
    # Test/hip_triangular_solve.cpp:104-122 formulas at a smaller size.
    size, k = 45, 7
    A = np.ones((size, size), dtype=np.float64)
    for i in range(size):
        for j in range(i + 1):
            A[i, j] = 0.3 * (0.1 / size * i - 0.05 / (i + 1.0) * j) + (10 if i == j else 0)
    L = np.tril(A)
    B = np.fromfunction(lambda i, j: (0.1 / size) * i + 0.1 / k * j, (size, k))
    res = {"L": L, "B": B}
    for upper in (0, 1):
        for unit in (0, 1):
            T = L if not upper else L.T.copy()
            X = np.array(B, order="F")
            assert ref.trsm(np.array(T, order="C"), X, upper=bool(upper), unit=bool(unit), left=True) == 0
            res[f"left_u{upper}_d{unit}"] = X
            Y = np.array(B.T, order="C")
            assert ref.trsm(np.array(T, order="F"), Y, upper=bool(upper), unit=bool(unit), left=False) == 0
            res[f"right_u{upper}_d{unit}"] = Y
    np.savez_compressed(OUT / "trsm.npz", **res)


def syrk_gemm_fixture(ref: oracle.Reference) -> None:
    # Test/hip_syrk.cpp:57-62 at a smaller size (not a multiple of any block size).
    dims, K = 37, 29
    A = np.fromfunction(lambda i, j: (1.0 / dims) * i + 0.2 / K * j + 1, (dims, K))
    res = {"A": A}
    for upper in (0, 1):
        C = np.full((dims, dims), 3.0)
        ref.syrk(np.array(A, order="C"), C, alpha=2.0, upper=bool(upper))
        res[f"C_u{upper}"] = C
    # Test/hip_prod.cpp:131-150 formulas, C init 1.5, alpha = -2.
    rows, cols, mid = 11, 13, 9
    X = np.fromfunction(lambda i, j: 0.1 * i * mid + 0.2 * j, (rows, mid))
    Y = np.fromfunction(lambda i, j: 0.1 * i * cols + 1.5 * j, (mid, cols))
    C = np.full((rows, cols), 1.5)
    ref.gemm(np.array(X, order="F"), np.array(Y, order="C"), C, alpha=-2.0)
    res.update(X=X, Y=Y, G=C)
    np.savez_compressed(OUT / "syrk_gemm.npz", **res)


def blas2_fixture(ref: oracle.Reference) -> None:
    # Matrix-vector kernels on the Test/hip_triangular_solve.cpp:104-122 triangle (size 45)
    # and a formula-built general matrix: gemv (both orientations of A), trsv (left and
    # right, all triangles), trmv and trmm (all triangles).
    size, k = 45, 7
    A = np.ones((size, size), dtype=np.float64)
    for i in range(size):
        for j in range(i + 1):
            A[i, j] = 0.3 * (0.1 / size * i - 0.05 / (i + 1.0) * j) + (10 if i == j else 0)
    L = np.tril(A)
    M = np.fromfunction(lambda i, j: 0.01 * (i - 2 * j) + 0.5 * np.sin(i + j), (size, 31))
    x = np.fromfunction(lambda i: 0.1 * i - 1.0, (size,))
    x31 = np.fromfunction(lambda i: 0.05 * i + 0.3, (31,))
    B = np.fromfunction(lambda i, j: (0.1 / size) * i + 0.1 / k * j, (size, k))
    res = {"L": L, "M": M, "x": x, "x31": x31, "B": B}
    for order in ("C", "F"):
        y = np.full(size, 0.25)
        ref.gemv(np.array(M, order=order), x31, y, alpha=-1.5)
        res[f"gemv_{order}"] = y
    for upper in (0, 1):
        T = L if not upper else L.T.copy()
        for unit in (0, 1):
            for left in (1, 0):
                v = x.copy()
                ref.trsv(np.array(T, order="C"), v, upper=bool(upper), unit=bool(unit), left=bool(left))
                res[f"trsv_u{upper}_d{unit}_l{left}"] = v
            v = x.copy()
            ref.trmv(np.array(T, order="F"), v, upper=bool(upper), unit=bool(unit))
            res[f"trmv_u{upper}_d{unit}"] = v
            X = np.array(B, order="F")
            ref.trmm(np.array(T, order="C"), X, upper=bool(upper), unit=bool(unit))
            res[f"trmm_u{upper}_d{unit}"] = X
    np.savez_compressed(OUT / "blas2.npz", **res)


def lu_input(n: int) -> np.ndarray:
    """The getrf test matrix of Test/getrf.cpp:15-33: L U with L(i, j) = 3 - 3 |i - j| / n
    below a unit diagonal and U = diag(1 + i / (2 n)), built so that partial pivoting
    moves to the next row at every step."""
    L = np.eye(n)
    for i in range(n):
        for j in range(i):
            L[i, j] = 3 - 3.0 / n * abs(i - j)
    return L @ np.diag(0.5 / n * np.arange(n) + 1)


def semidef_input(n: int, rank: int = 0) -> np.ndarray:
    """The pivoted-Cholesky test matrix of Test/symm_solve.cpp:17-38: R R^T with
    R(i, j) = 0.2 / |i - j| (j < min(i, rank)), R(i, i) = 1 + i / (2 n) for i < rank, and
    for rank < n the rows and columns 2 i and n - 1 - i swapped (i < rank / 2)."""
    rank = rank or n
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


def lu_pstrf_fixture(ref: oracle.Reference) -> None:
    # kernels::getrf on the Test/getrf.cpp matrix (n = 123) and on a U[-1, 1] matrix from the
    # reference CPU generator (n = 61); kernels::pstrf<lower> on the Test/symm_solve.cpp
    # matrix at full rank (60) and rank-deficient (57 of rank 25, 45 of rank 44). Row-major
    # runs; for pstrf the pivot recorded at the rank itself picks among rounding-level
    # remainders and is not part of the parity contract.
    res = {}
    g = ref.rng(11)
    cases = {"lu123": lu_input(123), "lu61": g.uniform(61, 61, -1.0, 1.0)}
    for name, A in cases.items():
        F = np.array(A, order="C")
        st, piv = ref.getrf(F)
        assert st == 0
        res[f"{name}_A"], res[f"{name}_F"], res[f"{name}_piv"] = A, F, piv
    for name, (n, r) in {"ps60": (60, 0), "ps57r25": (57, 25), "ps45r44": (45, 44)}.items():
        A = semidef_input(n, r)
        F = np.array(A, order="C")
        rank, piv = ref.pstrf(F)
        res[f"{name}_A"], res[f"{name}_F"], res[f"{name}_piv"] = A, F, piv
        res[f"{name}_rank"] = np.array(rank)
    np.savez_compressed(OUT / "lu_pstrf.npz", **res)


def solve_fixture(ref: oracle.Reference) -> None:
    # The n = 1024 SPD solve recipe at n = 48: G ~ N(0,1) from mt19937(seed) through the
    # reference CPU generator, A = G G^T / n + 1e-2 I (reference gemm), B ~ N(0,1).
    n, nrhs = 48, 5
    g = ref.rng(7)
    G = g.normal(n, n)
    A = np.zeros((n, n))
    ref.gemm(G, np.array(G.T, order="C"), A, alpha=1.0 / n)
    A += 1e-2 * np.eye(n)
    B = g.normal(n, nrhs)
    X = np.array(B, order="F")
    assert ref.cholesky_solve(np.array(A, order="F"), X) == 0
    np.savez_compressed(OUT / "solve.npz", G=G, A=A, B=B, X=X)


def main() -> None:
    oracle.build(ref=True)
    ref = oracle.Reference()
    rng_fixture(ref)
    generator_fixture(ref)
    potrf_fixture(ref)
    trsm_fixture(ref)
    syrk_gemm_fixture(ref)
    blas2_fixture(ref)
    solve_fixture(ref)
    lu_pstrf_fixture(ref)
    for f in sorted(OUT.glob("*.npz")):
        print(f.name, f.stat().st_size)


if __name__ == "__main__":
    main()
