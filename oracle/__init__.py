"""Test infrastructure: ctypes views of the CPU oracle and of the reference's own CPU path.

* ``Oracle`` loads ``_build/liboracle.so`` -- the restatement in ``rc_oracle.cpp``;
* ``Reference`` loads ``_ref/libremora_ref.so`` -- Remora's CPU kernels compiled from
  the reference headers by ``oracle/Makefile`` (absent where the reference is absent).

Only tests, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use this module,
and only as the checker / the timed CPU baseline. The product never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import POINTER, c_double, c_float, c_int, c_size_t, c_ssize_t, c_uint32, c_uint64, c_void_p
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "liboracle.so"
REF_SO = HERE / "_ref" / "libremora_ref.so"
# Where the reference's headers lie (include/ of the Remora source tree): the environment
# variable REMORA_REF_INCLUDE, else the default of oracle/Makefile.
REF_INCLUDE = Path(os.environ.get("REMORA_REF_INCLUDE", "/root/reference/include"))


def reference_present() -> bool:
    """True where Remora's headers are on this machine (not on a machine that only runs the
    prebuilt libraries)."""
    return (REF_INCLUDE / "remora").is_dir()
_U4 = c_uint32 * 4


def build(ref: bool = True) -> None:
    """Compile the oracle (always) and the reference CPU shim (when its headers exist)."""
    subprocess.run(["make", "-s", "-C", str(HERE), "oracle"], check=True)
    if ref and reference_present():
        subprocess.run(["make", "-s", "-C", str(HERE), "ref", f"REF_INCLUDE={REF_INCLUDE}"], check=True)


def _p(a: np.ndarray) -> c_void_p:
    return a.ctypes.data_as(c_void_p)


def strides(a: np.ndarray) -> tuple[int, int]:
    """Element strides (rs, cs) of a 2-D numpy array."""
    return a.strides[0] // a.itemsize, a.strides[1] // a.itemsize


class Oracle:
    def __init__(self, path: Path = ORACLE_SO):
        if not path.exists():
            build(ref=False)
        self.lib = ctypes.CDLL(str(path))
        L = self.lib
        L.orc_rng_create.restype = c_void_p
        L.orc_rng_create.argtypes = [c_uint32]
        L.orc_rng_destroy.argtypes = [c_void_p]
        L.orc_rng_key.argtypes = [c_void_p, POINTER(c_uint32)]
        L.orc_threefry.argtypes = [POINTER(c_uint32), POINTER(c_uint32), POINTER(c_uint32)]
        L.orc_counter.argtypes = [c_uint64, c_uint64, POINTER(c_uint32)]
        L.orc_rng_fill.argtypes = [c_int, POINTER(c_uint32), c_size_t, c_size_t, c_void_p, c_ssize_t, c_ssize_t,
                                   c_float, c_float, c_int, c_int, c_int]
        L.orc_rng_fill_block.argtypes = [c_int, POINTER(c_uint32), c_uint64, c_uint64, c_size_t, c_size_t, c_void_p,
                                         c_ssize_t, c_ssize_t, c_float, c_float, c_int, c_int, c_int]
        for t, ct in (("f64", c_double), ("f32", c_float)):
            getattr(L, f"orc_generate_normal_{t}").argtypes = [c_void_p, c_size_t, c_size_t, c_void_p, c_ssize_t,
                                                               c_ssize_t, ct, ct]
            getattr(L, f"orc_generate_uniform_{t}").argtypes = [c_void_p, c_size_t, c_size_t, c_void_p, c_ssize_t,
                                                                c_ssize_t, ct, ct]
            getattr(L, f"orc_gemm_{t}").argtypes = [c_size_t, c_size_t, c_size_t, ct, c_void_p, c_ssize_t, c_ssize_t,
                                                    c_void_p, c_ssize_t, c_ssize_t, c_void_p, c_ssize_t, c_ssize_t]
            getattr(L, f"orc_syrk_{t}").argtypes = [c_int, c_size_t, c_size_t, ct, c_void_p, c_ssize_t, c_ssize_t,
                                                    c_void_p, c_ssize_t, c_ssize_t]
            getattr(L, f"orc_gemv_{t}").argtypes = [c_size_t, c_size_t, ct, c_void_p, c_ssize_t, c_ssize_t, c_void_p,
                                                   c_ssize_t, c_void_p, c_ssize_t]
            getattr(L, f"orc_trsv_{t}").argtypes = [c_int, c_int, c_int, c_size_t, c_void_p, c_ssize_t, c_ssize_t,
                                                   c_void_p, c_ssize_t]
            getattr(L, f"orc_trmm_{t}").argtypes = [c_int, c_int, c_size_t, c_size_t, c_void_p, c_ssize_t, c_ssize_t,
                                                   c_void_p, c_ssize_t, c_ssize_t]
            getattr(L, f"orc_trsm_{t}").argtypes = [c_int, c_int, c_int, c_size_t, c_size_t, c_void_p, c_ssize_t,
                                                    c_ssize_t, c_void_p, c_ssize_t, c_ssize_t]
            getattr(L, f"orc_potrf_{t}").argtypes = [c_int, c_size_t, c_void_p, c_ssize_t, c_ssize_t]
            getattr(L, f"orc_potrf_{t}").restype = c_size_t
            for f in ("getrf", "pstrf"):
                getattr(L, f"orc_{f}_{t}").argtypes = [c_size_t, c_void_p, c_ssize_t, c_ssize_t, c_void_p]
                getattr(L, f"orc_{f}_{t}").restype = c_size_t
        L.orc_cholesky_solve_f64.argtypes = [c_size_t, c_size_t, c_void_p, c_ssize_t, c_ssize_t, c_void_p, c_ssize_t,
                                             c_ssize_t]
        L.orc_cholesky_solve_f64.restype = c_size_t

    # -- RNG ------------------------------------------------------------------------------
    def threefry(self, ctr, key) -> list[int]:
        out = _U4()
        self.lib.orc_threefry(_U4(*ctr), _U4(*key), out)
        return list(out)

    def counter(self, i: int, j: int) -> list[int]:
        out = _U4()
        self.lib.orc_counter(i, j, out)
        return list(out)

    def rng_fill(self, kind: str, key, rows: int, cols: int, row_major: bool = True, a: float = 0.0,
                 b: float = 1.0, ia: int = 0, ib: int = 0, fused: bool = True, row0: int = 0,
                 col0: int = 0) -> np.ndarray:
        """Rows [row0, row0+rows) x columns [col0, col0+cols) of the fill (col0 % 4 == 0)."""
        code = {"bits": 0, "uniform": 1, "normal": 2, "discrete_f32": 3, "discrete_i32": 4}[kind]
        dt = {0: np.uint32, 4: np.int32}.get(code, np.float32)
        out = np.zeros((rows, cols), dtype=dt, order="C" if row_major else "F")
        rs, cs = strides(out)
        self.lib.orc_rng_fill_block(code, _U4(*key), row0, col0, rows, cols, _p(out), rs, cs, a, b, ia, ib,
                                    int(fused))
        return out

    # -- input generator (std::mt19937 + std distributions) --------------------------------
    def rng(self, seed: int) -> "HostRng":
        return HostRng(self.lib, seed)

    # -- BLAS-3 ----------------------------------------------------------------------------
    def gemm(self, A, B, C, alpha=1.0):
        t = "f64" if C.dtype == np.float64 else "f32"
        getattr(self.lib, f"orc_gemm_{t}")(C.shape[0], C.shape[1], A.shape[1], alpha, _p(A), *strides(A), _p(B),
                                           *strides(B), _p(C), *strides(C))

    def syrk(self, A, C, alpha=1.0, upper=False):
        t = "f64" if C.dtype == np.float64 else "f32"
        getattr(self.lib, f"orc_syrk_{t}")(int(upper), A.shape[0], A.shape[1], alpha, _p(A), *strides(A), _p(C),
                                           *strides(C))

    def trsm(self, A, B, upper=False, unit=False, left=True) -> int:
        t = "f64" if B.dtype == np.float64 else "f32"
        return getattr(self.lib, f"orc_trsm_{t}")(int(left), int(upper), int(unit), B.shape[0], B.shape[1], _p(A),
                                                  *strides(A), _p(B), *strides(B))

    def gemv(self, A, x, y, alpha=1.0):
        """y += alpha A x; x, y 1-D (any stride)."""
        t = "f64" if y.dtype == np.float64 else "f32"
        getattr(self.lib, f"orc_gemv_{t}")(A.shape[0], A.shape[1], alpha, _p(A), *strides(A), _p(x),
                                           x.strides[0] // x.itemsize, _p(y), y.strides[0] // y.itemsize)

    def trsv(self, A, x, upper=False, unit=False, left=True) -> int:
        t = "f64" if x.dtype == np.float64 else "f32"
        return getattr(self.lib, f"orc_trsv_{t}")(int(left), int(upper), int(unit), A.shape[0], _p(A), *strides(A),
                                                  _p(x), x.strides[0] // x.itemsize)

    def trmm(self, A, B, upper=False, unit=False):
        """B <- T B (B 2-D; a vector as an n x 1 array gives trmv)."""
        t = "f64" if B.dtype == np.float64 else "f32"
        getattr(self.lib, f"orc_trmm_{t}")(int(upper), int(unit), B.shape[0], B.shape[1], _p(A), *strides(A), _p(B),
                                           *strides(B))

    def potrf(self, A, upper=False) -> int:
        t = "f64" if A.dtype == np.float64 else "f32"
        return getattr(self.lib, f"orc_potrf_{t}")(int(upper), A.shape[0], _p(A), *strides(A))

    def getrf(self, A) -> tuple[int, np.ndarray]:
        """LU with partial pivoting in place; returns (status, piv)."""
        t = "f64" if A.dtype == np.float64 else "f32"
        piv = np.zeros(A.shape[0], dtype=np.int32)
        st = getattr(self.lib, f"orc_getrf_{t}")(A.shape[0], _p(A), *strides(A), _p(piv))
        return st, piv

    def pstrf(self, A) -> tuple[int, np.ndarray]:
        """Pivoted Cholesky (lower) in place; returns (rank, piv)."""
        t = "f64" if A.dtype == np.float64 else "f32"
        piv = np.zeros(A.shape[0], dtype=np.int32)
        rank = getattr(self.lib, f"orc_pstrf_{t}")(A.shape[0], _p(A), *strides(A), _p(piv))
        return rank, piv

    def cholesky_solve(self, A, B) -> int:
        return self.lib.orc_cholesky_solve_f64(A.shape[0], B.shape[1], _p(A), *strides(A), _p(B), *strides(B))


class HostRng:
    """std::mt19937(seed) with the reference CPU generator's fills on it."""

    def __init__(self, lib, seed: int):
        self.lib = lib
        self.h = c_void_p(lib.orc_rng_create(seed))

    def __del__(self):
        try:
            self.lib.orc_rng_destroy(self.h)
        except Exception:
            pass

    def key(self) -> list[int]:
        out = _U4()
        self.lib.orc_rng_key(self.h, out)
        return list(out)

    def normal(self, rows, cols, mean=0.0, variance=1.0, dtype=np.float64, row_major=True) -> np.ndarray:
        a = np.zeros((rows, cols), dtype=dtype, order="C" if row_major else "F")
        t = "f64" if dtype == np.float64 else "f32"
        getattr(self.lib, f"orc_generate_normal_{t}")(self.h, rows, cols, _p(a), *strides(a), mean, variance)
        return a

    def uniform(self, rows, cols, low=0.0, high=1.0, dtype=np.float64, row_major=True) -> np.ndarray:
        a = np.zeros((rows, cols), dtype=dtype, order="C" if row_major else "F")
        t = "f64" if dtype == np.float64 else "f32"
        getattr(self.lib, f"orc_generate_uniform_{t}")(self.h, rows, cols, _p(a), *strides(a), low, high)
        return a


class Reference:
    """Remora's own CPU kernels (oracle/_ref), where they were built."""

    def __init__(self, path: Path = REF_SO):
        if not path.exists():
            raise FileNotFoundError(f"{path} not built (the reference headers are needed to build it)")
        self.lib = ctypes.CDLL(str(path))
        L = self.lib
        L.ref_rng_create.restype = c_void_p
        L.ref_rng_create.argtypes = [c_uint32]
        L.ref_rng_destroy.argtypes = [c_void_p]
        L.ref_rng_key.argtypes = [c_void_p, POINTER(c_uint32)]
        L.ref_hip_threefry.argtypes = [POINTER(c_uint32)] * 3
        L.ref_hip_uniform4.argtypes = [c_float, c_float, POINTER(c_uint32), POINTER(c_float)]
        L.ref_hip_normal4.argtypes = [c_float, c_float, POINTER(c_uint32), POINTER(c_float)]
        L.ref_hip_discrete4.argtypes = [POINTER(c_uint32), POINTER(c_uint32), c_uint32, POINTER(c_uint32)]
        for t, ct in (("f64", c_double), ("f32", c_float)):
            getattr(L, f"ref_potrf_{t}").argtypes = [c_int, c_int, c_size_t, c_void_p, c_size_t]
            getattr(L, f"ref_potrf_{t}").restype = c_size_t
            getattr(L, f"ref_getrf_{t}").argtypes = [c_int, c_size_t, c_void_p, c_size_t, c_void_p]
            getattr(L, f"ref_getrf_{t}").restype = ctypes.c_long
            getattr(L, f"ref_pstrf_{t}").argtypes = [c_int, c_size_t, c_void_p, c_size_t, c_void_p]
            getattr(L, f"ref_pstrf_{t}").restype = c_size_t
            getattr(L, f"ref_trsm_{t}").argtypes = [c_int, c_int, c_int, c_int, c_int, c_size_t, c_size_t, c_void_p,
                                                    c_size_t, c_void_p, c_size_t]
            getattr(L, f"ref_syrk_{t}").argtypes = [c_int, c_int, c_int, c_size_t, c_size_t, ct, c_void_p, c_size_t,
                                                    c_void_p, c_size_t]
            getattr(L, f"ref_gemm_{t}").argtypes = [c_int, c_int, c_int, c_size_t, c_size_t, c_size_t, ct, c_void_p,
                                                    c_size_t, c_void_p, c_size_t, c_void_p, c_size_t]
            getattr(L, f"ref_generate_normal_{t}").argtypes = [c_void_p, c_int, c_size_t, c_size_t, c_void_p,
                                                               c_size_t, ct, ct]
            getattr(L, f"ref_generate_uniform_{t}").argtypes = [c_void_p, c_int, c_size_t, c_size_t, c_void_p,
                                                                c_size_t, ct, ct]
        for t, ct in (("f64", c_double), ("f32", c_float)):
            getattr(L, f"ref_gemv_{t}").argtypes = [c_int, c_size_t, c_size_t, ct, c_void_p, c_size_t, c_void_p,
                                                   c_void_p]
            getattr(L, f"ref_trsv_{t}").argtypes = [c_int, c_int, c_int, c_int, c_size_t, c_void_p, c_size_t, c_void_p]
            getattr(L, f"ref_trmv_{t}").argtypes = [c_int, c_int, c_int, c_size_t, c_void_p, c_size_t, c_void_p]
            getattr(L, f"ref_trmm_{t}").argtypes = [c_int, c_int, c_int, c_int, c_size_t, c_size_t, c_void_p, c_size_t,
                                                   c_void_p, c_size_t]
        L.ref_cholesky_solve_f64.argtypes = [c_int, c_int, c_size_t, c_size_t, c_void_p, c_size_t, c_void_p,
                                             c_size_t]

    @staticmethod
    def _ld(a: np.ndarray) -> tuple[int, int]:
        rs, cs = strides(a)
        return (1, rs) if cs == 1 else (0, cs)

    def threefry(self, ctr, key) -> list[int]:
        out = _U4()
        self.lib.ref_hip_threefry(_U4(*ctr), _U4(*key), out)
        return list(out)

    def uniform4(self, low, high, x) -> list[float]:
        out = (c_float * 4)()
        self.lib.ref_hip_uniform4(low, high, _U4(*x), out)
        return list(out)

    def normal4(self, mean, stddev, x) -> list[float]:
        out = (c_float * 4)()
        self.lib.ref_hip_normal4(mean, stddev, _U4(*x), out)
        return list(out)

    def discrete4(self, key, ctr, N) -> list[int]:
        out = _U4()
        self.lib.ref_hip_discrete4(_U4(*key), _U4(*ctr), N, out)
        return list(out)

    def getrf(self, A: np.ndarray) -> tuple[int, np.ndarray]:
        """The reference's kernels::getrf in place; (0 or -1 for its exception, piv)."""
        rm, ld = self._ld(A)
        t = "f64" if A.dtype == np.float64 else "f32"
        piv = np.zeros(A.shape[0], dtype=np.int32)
        return getattr(self.lib, f"ref_getrf_{t}")(rm, A.shape[0], _p(A), ld, _p(piv)), piv

    def pstrf(self, A: np.ndarray) -> tuple[int, np.ndarray]:
        """The reference's kernels::pstrf<lower> in place; (rank, piv)."""
        rm, ld = self._ld(A)
        t = "f64" if A.dtype == np.float64 else "f32"
        piv = np.zeros(A.shape[0], dtype=np.int32)
        return getattr(self.lib, f"ref_pstrf_{t}")(rm, A.shape[0], _p(A), ld, _p(piv)), piv

    def potrf(self, A: np.ndarray, upper=False) -> int:
        rm, ld = self._ld(A)
        t = "f64" if A.dtype == np.float64 else "f32"
        return getattr(self.lib, f"ref_potrf_{t}")(int(upper), rm, A.shape[0], _p(A), ld)

    def trsm(self, A, B, upper=False, unit=False, left=True) -> int:
        arm, lda = self._ld(A)
        brm, ldb = self._ld(B)
        t = "f64" if B.dtype == np.float64 else "f32"
        return getattr(self.lib, f"ref_trsm_{t}")(int(left), int(upper), int(unit), arm, brm, B.shape[0], B.shape[1],
                                                  _p(A), lda, _p(B), ldb)

    def gemv(self, A, x, y, alpha=1.0):
        """y += alpha A x (kernels::gemv); x, y contiguous 1-D arrays, y updated in place."""
        arm, lda = self._ld(A)
        t = "f64" if y.dtype == np.float64 else "f32"
        getattr(self.lib, f"ref_gemv_{t}")(arm, A.shape[0], A.shape[1], alpha, _p(A), lda, _p(x), _p(y))

    def trsv(self, A, x, upper=False, unit=False, left=True):
        """x <- A^-1 x (left) or x A^-1 (right) for the named triangle (kernels::trsv)."""
        arm, lda = self._ld(A)
        t = "f64" if x.dtype == np.float64 else "f32"
        getattr(self.lib, f"ref_trsv_{t}")(int(upper), int(unit), int(left), arm, A.shape[0], _p(A), lda, _p(x))

    def trmv(self, A, x, upper=False, unit=False):
        arm, lda = self._ld(A)
        t = "f64" if x.dtype == np.float64 else "f32"
        getattr(self.lib, f"ref_trmv_{t}")(int(upper), int(unit), arm, A.shape[0], _p(A), lda, _p(x))

    def trmm(self, A, B, upper=False, unit=False):
        arm, lda = self._ld(A)
        brm, ldb = self._ld(B)
        t = "f64" if B.dtype == np.float64 else "f32"
        getattr(self.lib, f"ref_trmm_{t}")(int(upper), int(unit), arm, brm, B.shape[0], B.shape[1], _p(A), lda, _p(B),
                                          ldb)

    def syrk(self, A, C, alpha=1.0, upper=False):
        arm, lda = self._ld(A)
        crm, ldc = self._ld(C)
        t = "f64" if C.dtype == np.float64 else "f32"
        getattr(self.lib, f"ref_syrk_{t}")(int(upper), arm, crm, A.shape[0], A.shape[1], alpha, _p(A), lda, _p(C), ldc)

    def gemm(self, A, B, C, alpha=1.0):
        arm, lda = self._ld(A)
        brm, ldb = self._ld(B)
        crm, ldc = self._ld(C)
        t = "f64" if C.dtype == np.float64 else "f32"
        getattr(self.lib, f"ref_gemm_{t}")(arm, brm, crm, C.shape[0], C.shape[1], A.shape[1], alpha, _p(A), lda,
                                           _p(B), ldb, _p(C), ldc)

    def cholesky_solve(self, A, B) -> int:
        arm, lda = self._ld(A)
        brm, ldb = self._ld(B)
        return self.lib.ref_cholesky_solve_f64(arm, brm, A.shape[0], B.shape[1], _p(A), lda, _p(B), ldb)

    def rng(self, seed: int) -> "RefRng":
        return RefRng(self.lib, seed)


class RefRng:
    def __init__(self, lib, seed):
        self.lib = lib
        self.h = c_void_p(lib.ref_rng_create(seed))

    def __del__(self):
        try:
            self.lib.ref_rng_destroy(self.h)
        except Exception:
            pass

    def key(self) -> list[int]:
        out = _U4()
        self.lib.ref_rng_key(self.h, out)
        return list(out)

    def normal(self, rows, cols, mean=0.0, variance=1.0, dtype=np.float64, row_major=True) -> np.ndarray:
        a = np.zeros((rows, cols), dtype=dtype, order="C" if row_major else "F")
        t = "f64" if dtype == np.float64 else "f32"
        ld = cols if row_major else rows
        getattr(self.lib, f"ref_generate_normal_{t}")(self.h, int(row_major), rows, cols, _p(a), ld, mean, variance)
        return a

    def uniform(self, rows, cols, low=0.0, high=1.0, dtype=np.float64, row_major=True) -> np.ndarray:
        a = np.zeros((rows, cols), dtype=dtype, order="C" if row_major else "F")
        t = "f64" if dtype == np.float64 else "f32"
        ld = cols if row_major else rows
        getattr(self.lib, f"ref_generate_uniform_{t}")(self.h, int(row_major), rows, cols, _p(a), ld, low, high)
        return a


def create_symm(n: int) -> np.ndarray:
    """createSymm of Test/hip_cholesky.cpp:13-33: R_ij = 0.2/|i-j| (j < i), R_ii = 1 + 0.5/n*i + 1, A = R R^T."""
    R = np.zeros((n, n))
    for i in range(n):
        for j in range(i):
            R[i, j] = 0.2 / abs(i - j)
        R[i, i] = 1 + 0.5 / n * i + 1
    return R @ R.T


def rel_fro(x: np.ndarray, ref: np.ndarray) -> float:
    d = np.linalg.norm(np.asarray(x, np.float64) - np.asarray(ref, np.float64))
    r = np.linalg.norm(np.asarray(ref, np.float64))
    return float(d / r) if r > 0 else float(d)
