"""Python view of the Remora kernel API on ``cuda`` tensors, through the C-ABI.

The functions mirror the reference's kernel entry points and their semantics:

=====================================  ==================================================
``gemm(A, B, C, alpha)``               ``kernels::gemm`` -- C += alpha * A * B
                                       (include/remora/kernels/gemm.hpp:85-106)
``syrk(A, C, alpha, upper)``           ``kernels::syrk<Upper>`` -- one triangle of C
                                       += alpha * A * A^T (kernels/syrk.hpp:55-67)
``trsm(A, B, upper, unit, left)``      ``kernels::trsm<Tri, Side>`` (kernels/trsm.hpp:55-65)
``potrf(A, upper) -> int``             ``kernels::potrf<Tri>`` (kernels/potrf.hpp:56-62),
                                       0 or the global 1-based failing pivot
``cholesky_solve(A, B)``               ``cholesky_decomposition(A).solve(B, left())``
                                       (decompositions.hpp:81-105)
``generate_normal/uniform/discrete``   ``kernels::generate_*`` for a device matrix
                                       (kernels/hip/random.hpp:262-323)
=====================================  ==================================================

Matrices are 2-D torch tensors on a CUDA device in row-major or column-major storage
(strided sub-matrices allowed); orientation is read from the strides, as Remora reads it
from the ``orientation`` type. Everything runs on the current torch stream.
"""
from __future__ import annotations

import ctypes
import math

import torch

from ._lib import call, key_array

_FP = {torch.float64: "f64", torch.float32: "f32"}


def _stream() -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t: torch.Tensor) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr())


def layout(X: torch.Tensor) -> tuple[int, int]:
    """(trans, ld) with X = op_trans(M), M column-major with leading dimension ld."""
    if X.dim() != 2:
        raise ValueError("expected a matrix")
    r, c = X.shape
    s0, s1 = X.stride()
    if s0 == 1 and (c <= 1 or s1 >= max(r, 1)):
        return 0, max(s1 if c > 1 else r, 1)
    if s1 == 1 and (r <= 1 or s0 >= max(c, 1)):
        return 1, max(s0 if r > 1 else c, 1)
    raise ValueError(f"matrix with strides {X.stride()} is neither row- nor column-major")


def is_row_major(X: torch.Tensor) -> bool:
    return layout(X)[0] == 1


def _sfx(*ts: torch.Tensor) -> str:
    dt = ts[0].dtype
    if any(t.dtype != dt for t in ts) or dt not in _FP:
        raise TypeError("arguments must share one element type, float32 or float64")
    return _FP[dt]


def gemm(A: torch.Tensor, B: torch.Tensor, C: torch.Tensor, alpha: float = 1.0, beta: float = 1.0,
         tf32: bool = False) -> None:
    """C <- alpha * A @ B + beta * C (beta = 1 is the reference's kernels::gemm)."""
    sfx = "tf32" if tf32 else _sfx(A, B, C)
    m, n = C.shape
    k = A.shape[1]
    if A.shape[0] != m or B.shape != (k, n):
        raise ValueError("gemm: shape mismatch")
    ta, lda = layout(A)
    tb, ldb = layout(B)
    tc, ldc = layout(C)
    if tc == 0:
        call(f"rc_gemm_{sfx}", ta, tb, m, n, k, alpha, _ptr(A), lda, _ptr(B), ldb, beta, _ptr(C), ldc, _stream())
    else:  # C^T = B^T A^T, column-major
        call(f"rc_gemm_{sfx}", 1 - tb, 1 - ta, n, m, k, alpha, _ptr(B), ldb, _ptr(A), lda, beta, _ptr(C), ldc,
             _stream())


def gemm_sliced(A: torch.Tensor, B: torch.Tensor, C: torch.Tensor, alpha: float = 1.0, beta: float = 1.0) -> None:
    """FP64 C <- alpha * A @ B + beta * C on the int8 tensor cores (digit-split operands),
    column-major A, B, C and at most 64 columns of B."""
    m, n = C.shape
    k = A.shape[1]
    if A.shape[0] != m or B.shape != (k, n):
        raise ValueError("gemm_sliced: shape mismatch")
    ta, lda = layout(A)
    tb, ldb = layout(B)
    tc, ldc = layout(C)
    if ta or tb or tc:
        raise ValueError("gemm_sliced: column-major operands only")
    call("rc_gemm_f64_sliced", m, n, k, alpha, _ptr(A), lda, _ptr(B), ldb, beta, _ptr(C), ldc, _stream())


def syrk(A: torch.Tensor, C: torch.Tensor, alpha: float = 1.0, upper: bool = False, beta: float = 1.0) -> None:
    """One triangle of C <- alpha * A @ A^T + beta * C; the other triangle is untouched."""
    sfx = _sfx(A, C)
    n, k = A.shape
    if C.shape != (n, n):
        raise ValueError("syrk: shape mismatch")
    ta, lda = layout(A)
    tc, ldc = layout(C)
    up = bool(upper) != bool(tc)  # a row-major C is the transpose of a column-major one
    call(f"rc_syrk_{sfx}", int(up), ta, n, k, alpha, _ptr(A), lda, beta, _ptr(C), ldc, _stream())


def syrk_emu64(P: torch.Tensor, C: torch.Tensor, alpha: float = 1.0, beta: float = 1.0) -> None:
    """Lower triangle of C <- alpha * P @ P^T + beta * C in emulated FP64 (7 int8 digits per
    entry of P, exact digit-pair products on the tensor cores): P and C row-major FP64 with
    any row strides. The strict upper triangle of C is untouched."""
    if P.dtype != torch.float64 or C.dtype != torch.float64:
        raise TypeError("syrk_emu64 takes FP64 matrices")
    n, k = P.shape
    if C.shape != (n, n) or P.stride(1) != 1 or C.stride(1) != 1:
        raise ValueError("syrk_emu64: P (n x k) and C (n x n) must be row-major")
    call("rc_syrk_emu64", n, k, alpha, _ptr(P), P.stride(0), beta, _ptr(C), C.stride(0), _stream())


def trsm(A: torch.Tensor, B: torch.Tensor, upper: bool = False, unit: bool = False, left: bool = True,
         alpha: float = 1.0, info: torch.Tensor | None = None) -> None:
    """B <- alpha * A^-1 B (left) or alpha * B A^-1 (right), A the named triangle."""
    sfx = _sfx(A, B)
    m, n = B.shape
    ta, lda = layout(A)
    tb, ldb = layout(B)
    up_stored = bool(upper) != bool(ta)
    if tb == 0:
        side, trans, mm, nn = left, ta, m, n
    else:  # B^T is column-major: X^T = B^T A^-T on the other side
        side, trans, mm, nn = not left, 1 - ta, n, m
    call(f"rc_trsm_{sfx}", int(side), int(up_stored), trans, int(unit), mm, nn, alpha, _ptr(A), lda, _ptr(B), ldb,
         _ptr(info) if info is not None else None, _stream())


def potrf(A: torch.Tensor, upper: bool = False, info: torch.Tensor | None = None, sync: bool = True):
    """In-place Cholesky; returns 0 or the global 1-based failing pivot (sync=True)."""
    sfx = _sfx(A)
    n = A.shape[0]
    ta, lda = layout(A)
    if info is None:
        info = torch.zeros(1, dtype=torch.int32, device=A.device)
    call(f"rc_potrf_{sfx}", int(bool(upper) != bool(ta)), n, _ptr(A), lda, _ptr(info), _stream())
    return int(info.item()) if sync else info


def getrf(A: torch.Tensor) -> tuple[int, torch.Tensor]:
    """LU with partial pivoting in place (A = P L U); returns (info, piv): info 0 or the
    1-based column of the first zero pivot, piv the device int32 swap sequence."""
    sfx = _sfx(A)
    n = A.shape[0]
    ta, lda = layout(A)
    piv = torch.empty(n, dtype=torch.int32, device=A.device)
    info = torch.zeros(1, dtype=torch.int32, device=A.device)
    call(f"rc_getrf_{sfx}", ta, n, _ptr(A), lda, _ptr(piv), _ptr(info), _stream())
    return int(info.item()), piv


def pstrf(A: torch.Tensor) -> tuple[int, torch.Tensor]:
    """Pivoted Cholesky P^T A P = L L^T in place (L lower); returns (rank, piv)."""
    sfx = _sfx(A)
    n = A.shape[0]
    ta, lda = layout(A)
    piv = torch.empty(n, dtype=torch.int32, device=A.device)
    rank = torch.zeros(1, dtype=torch.int32, device=A.device)
    call(f"rc_pstrf_{sfx}", ta, n, _ptr(A), lda, _ptr(piv), _ptr(rank), _stream())
    return int(rank.item()), piv


def cholesky_solve(A: torch.Tensor, B: torch.Tensor, info: torch.Tensor | None = None) -> int:
    """B <- A^-1 B for SPD A (FP64; A's lower triangle read, A unchanged)."""
    if A.dtype != torch.float64 or B.dtype != torch.float64:
        raise TypeError("cholesky_solve is FP64")
    n = A.shape[0]
    ta, lda = layout(A)  # A symmetric: a row-major A is the same matrix read column-major
    tb, ldb = layout(B)
    if tb != 0:
        raise ValueError("cholesky_solve: B must be column-major")
    if info is None:
        info = torch.zeros(1, dtype=torch.int32, device=A.device)
    call("rc_spd_solve_f64", n, B.shape[1], _ptr(A), lda, _ptr(B), ldb, _ptr(info), _stream())
    return int(info.item())


def _fill(kind: str, X: torch.Tensor, key, a, b) -> None:
    rows, cols = X.shape
    t, ld = layout(X)
    call(f"rc_rng_{kind}", key_array(key), rows, cols, _ptr(X), ld, t, a, b, _stream())


def generate_normal(X: torch.Tensor, key, mean: float = 0.0, variance: float = 1.0) -> None:
    """Normal fill; the reference passes sqrt(variance) as the scale (random.hpp:270, :280)."""
    _fill("normal_f32", X, key, mean, math.sqrt(variance))


def generate_uniform(X: torch.Tensor, key, low: float = 0.0, high: float = 1.0) -> None:
    _fill("uniform_f32", X, key, low, high)


def generate_discrete(X: torch.Tensor, key, low: int, high: int) -> None:
    _fill("discrete_i32" if X.dtype == torch.int32 else "discrete_f32", X, key, int(low), int(high))


def generate_bits(X: torch.Tensor, key) -> None:
    """Raw Threefry words (uint32 stored in an int32 tensor)."""
    rows, cols = X.shape
    t, ld = layout(X)
    call("rc_rng_bits_u32", key_array(key), rows, cols, _ptr(X), ld, t, _stream())


def spd_solve_mixed(A: torch.Tensor, B: torch.Tensor, precision: str = "tf32", tol: float = 1e-15,
                    max_iter: int = 100, outer: int = 1024, shift_factor: float = -1.0,
                    X: torch.Tensor | None = None):
    """Mixed-precision refined SPD solve (FP64 in/out; A full symmetric, column-major).

    precision: "tf32" or "bf16" (a reduced-precision factor, for condition numbers up to
    about 1e6..1e8) or "emu64" (an FP64 factor whose trailing updates are exact int8 digit
    products, for condition numbers up to about 1e12).

    Returns (X, info dict, status) -- status 0 on convergence, 6 (RC_ERR_NOT_CONVERGED) when
    max_iter ran out; info["pivot"] is the failing pivot of a low-precision breakdown."""
    from ._lib import RC_PREC_BF16, RC_PREC_EMU64, RC_PREC_TF32, MixedOptions, RefineInfo, lib
    if A.dtype != torch.float64 or B.dtype != torch.float64:
        raise TypeError("spd_solve_mixed takes FP64 matrices")
    n = A.shape[0]
    ta, lda = layout(A)
    tb, ldb = layout(B)
    if tb != 0:
        raise ValueError("B must be column-major")
    if X is None:
        X = torch.empty((B.shape[1], n), dtype=torch.float64, device=B.device).t()
    tx, ldx = layout(X)
    prec = {"tf32": RC_PREC_TF32, "bf16": RC_PREC_BF16, "emu64": RC_PREC_EMU64}[precision]
    opts = MixedOptions(tol, max_iter, outer, shift_factor)
    info = RefineInfo()
    d_info = torch.zeros(1, dtype=torch.int32, device=A.device)
    status = lib().rc_spd_solve_mixed(prec, n, B.shape[1], _ptr(A), lda, _ptr(B), ldb, _ptr(X), ldx,
                                      ctypes.byref(opts), _ptr(d_info), ctypes.byref(info), _stream())
    out = {f: getattr(info, f) for f, _ in RefineInfo._fields_}
    out["pivot"] = int(d_info.item())
    return X, out, status


class BatchedSystems:
    """Device storage for a batch of uneven SPD systems (one RHS each) laid out as
    consecutive column-major blocks, with the pointer arrays the batched C-ABI takes."""

    def __init__(self, mats, rhs, dtype=torch.float64, device="cuda"):
        import numpy as np
        self.sizes = np.array([m.shape[0] for m in mats], dtype=np.int32)
        offs = np.concatenate([[0], np.cumsum(self.sizes.astype(np.int64) ** 2)])
        self.A = torch.empty(int(offs[-1]), dtype=dtype, device=device)
        boffs = np.concatenate([[0], np.cumsum(self.sizes.astype(np.int64))])
        self.b = torch.empty(int(boffs[-1]), dtype=dtype, device=device)
        host_a = np.concatenate([np.asarray(m, dtype=np.float64).T.reshape(-1) for m in mats])  # column-major
        host_b = np.concatenate([np.asarray(v, dtype=np.float64).reshape(-1) for v in rhs])
        self.A.copy_(torch.from_numpy(host_a))
        self.b.copy_(torch.from_numpy(host_b))
        es = self.A.element_size()
        self.a_ptrs = torch.tensor([self.A.data_ptr() + int(o) * es for o in offs[:-1]], dtype=torch.int64,
                                   device=device)
        self.b_ptrs = torch.tensor([self.b.data_ptr() + int(o) * es for o in boffs[:-1]], dtype=torch.int64,
                                   device=device)
        self.info = torch.zeros(len(mats), dtype=torch.int32, device=device)
        self.offs, self.boffs = offs, boffs

    def solve(self, autotune: bool = True) -> None:
        from ._lib import lib
        fn = "rc_potrf_trsm_batched_f64" if self.A.dtype == torch.float64 else "rc_potrf_trsm_batched_f32"
        sizes = self.sizes.ctypes.data_as(ctypes.c_void_p)
        status = getattr(lib(), fn)(len(self.sizes), sizes, _ptr(self.a_ptrs), _ptr(self.b_ptrs), _ptr(self.info),
                                    int(autotune), _stream())
        if status != 0:
            from ._lib import RemoraCudaError
            raise RemoraCudaError(fn, status)

    def factor(self, i: int):
        n = int(self.sizes[i])
        return self.A[int(self.offs[i]):int(self.offs[i + 1])].view(n, n).t()  # column-major n x n

    def solution(self, i: int):
        return self.b[int(self.boffs[i]):int(self.boffs[i + 1])]


def potrf_backward(L: torch.Tensor, Lbar: torch.Tensor, Abar: torch.Tensor | None = None) -> torch.Tensor:
    """Adjoint of A = L L^T: the full symmetric Abar for the adjoint Lbar of the lower L
    (column-major FP64)."""
    n = L.shape[0]
    if Abar is None:
        Abar = torch.empty((n, n), dtype=torch.float64, device=L.device).t()
    _, ldl = layout(L)
    _, ldlb = layout(Lbar)
    _, ldab = layout(Abar)
    call("rc_potrf_backward_f64", n, _ptr(L), ldl, _ptr(Lbar), ldlb, _ptr(Abar), ldab, _stream())
    return Abar


def _vec(x: torch.Tensor) -> int:
    if x.dim() != 1:
        raise ValueError("expected a vector")
    return max(x.stride(0), 1)


def gemv(A: torch.Tensor, x: torch.Tensor, y: torch.Tensor, alpha: float = 1.0, beta: float = 1.0) -> None:
    """y <- alpha * A @ x + beta * y (beta = 1 is the reference's kernels::gemv)."""
    sfx = _sfx(A, x, y)
    ta, lda = layout(A)
    m, n = A.shape
    if x.shape[0] != n or y.shape[0] != m:
        raise ValueError("gemv: shape mismatch")
    if ta == 0:
        call(f"rc_gemv_{sfx}", 0, m, n, alpha, _ptr(A), lda, _ptr(x), _vec(x), beta, _ptr(y), _vec(y), _stream())
    else:  # A^T is column-major n x m
        call(f"rc_gemv_{sfx}", 1, n, m, alpha, _ptr(A), lda, _ptr(x), _vec(x), beta, _ptr(y), _vec(y), _stream())


def trsv(A: torch.Tensor, x: torch.Tensor, upper: bool = False, unit: bool = False, left: bool = True) -> None:
    """x <- A^-1 x (left) or solves x A = b in place (right), A the named triangle."""
    sfx = _sfx(A, x)
    ta, lda = layout(A)
    up_stored = bool(upper) != bool(ta)
    trans = ta if left else 1 - ta
    call(f"rc_trsv_{sfx}", int(up_stored), trans, int(unit), A.shape[0], _ptr(A), lda, _ptr(x), _vec(x), _stream())


def trmm(A: torch.Tensor, B: torch.Tensor, upper: bool = False, unit: bool = False) -> None:
    """B <- T B for the named triangle T of A (the reference's kernels::trmm)."""
    sfx = _sfx(A, B)
    ta, lda = layout(A)
    tb, ldb = layout(B)
    up_stored = bool(upper) != bool(ta)
    m, n = B.shape
    if tb == 0:
        call(f"rc_trmm_{sfx}", 1, int(up_stored), ta, int(unit), m, n, _ptr(A), lda, _ptr(B), ldb, _stream())
    else:  # B^T = B^T T^T, column-major n x m
        call(f"rc_trmm_{sfx}", 0, int(up_stored), 1 - ta, int(unit), n, m, _ptr(A), lda, _ptr(B), ldb, _stream())


def trmv(A: torch.Tensor, x: torch.Tensor, upper: bool = False, unit: bool = False) -> None:
    """x <- T x for the named triangle T of A (the reference's kernels::trmv)."""
    sfx = _sfx(A, x)
    ta, lda = layout(A)
    up_stored = bool(upper) != bool(ta)
    call(f"rc_trmv_{sfx}", int(up_stored), ta, int(unit), A.shape[0], _ptr(A), lda, _ptr(x), _vec(x), _stream())


def trsm_backward(L: torch.Tensor, X: torch.Tensor, Xbar: torch.Tensor, Lbar: torch.Tensor,
                  trans: bool = False) -> torch.Tensor:
    """Reverse mode of X = L^-1 B (trans: X = L^-T B): Xbar becomes Bbar (returned), Lbar
    accumulates the adjoint of L."""
    n, nrhs = X.shape
    call("rc_trsm_backward_f64", int(trans), n, nrhs, _ptr(L), layout(L)[1], _ptr(X), layout(X)[1], _ptr(Xbar),
         layout(Xbar)[1], _ptr(Lbar), layout(Lbar)[1], _stream())
    return Xbar


def rbf_kernel(X: torch.Tensor, ls: torch.Tensor, noise: float) -> torch.Tensor:
    n, d = X.shape
    K = torch.empty((n, n), dtype=torch.float64, device=X.device).t()
    call("rc_rbf_kernel_f64", n, d, _ptr(X.contiguous()), _ptr(ls), noise, _ptr(K), n, _stream())
    return K


def gp_nll_and_grad(X: torch.Tensor, y: torch.Tensor, ls: torch.Tensor, noise: float):
    """Negative log marginal likelihood of a GP with an RBF kernel (constant term
    dropped), f = 1/2 y^T K^-1 y + 1/2 log det K, and df/dls, all through the C-ABI:
    forward Cholesky + triangular solve, backward through the hand-written TRSM and
    Cholesky adjoints, then the lengthscale contraction."""
    n, d = X.shape
    Xc = X.contiguous()
    K = rbf_kernel(Xc, ls, noise)
    L = K.clone()
    info = potrf(L)
    if info:
        raise RuntimeError(f"K is not positive definite (pivot {info})")
    z = y.reshape(n, 1).clone().t().contiguous().t()
    trsm(L, z)  # z = L^-1 y
    Ld = torch.diagonal(L)
    f = 0.5 * float((z * z).sum()) + float(torch.log(Ld).sum())
    # backward: zbar = z; through z = L^-1 y; then d(sum log L_ii)/dL_ii = 1/L_ii
    Lbar = torch.zeros((n, n), dtype=torch.float64, device=X.device).t()
    zbar = z.clone()
    trsm_backward(L, z, zbar, Lbar, trans=False)
    Lbar.diagonal().add_(1.0 / Ld)
    Kbar = potrf_backward(L, Lbar)
    g = torch.empty(d, dtype=torch.float64, device=X.device)
    call("rc_rbf_lengthscale_grad_f64", n, d, _ptr(Xc), _ptr(ls), _ptr(Kbar), layout(Kbar)[1], _ptr(g), _stream())
    return f, g, Kbar
