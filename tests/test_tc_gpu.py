"""tcgen05 tensor-core GEMMs (TF32 and BF16 operands, FP32 accumulation) through the
C-ABI, and the bounded-wait failure path.

The TF32/BF16 products are compared against an FP64 product of the SAME reduced-precision
operands (TF32: low 13 mantissa bits cleared; BF16: rounded to nearest even), so the bar
(relative Frobenius <= 1e-5, the FP32 accumulation error of K <= 4096 terms) tests the kernel's data movement and accumulation exactly;
any layout or descriptor error shows as O(1)."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from remora_b200 import _lib, ops
from helpers import to_host

pytestmark = pytest.mark.gpu
TC_TOL = 1e-5


def _tf32(x: torch.Tensor) -> torch.Tensor:
    return (x.view(torch.int32) & ~0x1FFF).view(torch.float32)


def _rel(a: torch.Tensor, b: torch.Tensor) -> float:
    return ((a.double() - b.double()).norm() / b.double().norm()).item()


SHAPES = [(128, 128, 32), (1, 1, 1), (7, 300, 13), (256, 256, 256), (300, 500, 1000), (1000, 129, 77),
          (2048, 1024, 4096)]


@pytest.mark.parametrize("m,n,k", SHAPES)
@pytest.mark.parametrize("ta,tb", [(1, 0), (0, 0), (1, 1), (0, 1)])
def test_gemm_tf32(cuda, m, n, k, ta, tb):
    g = torch.Generator(device="cuda").manual_seed(m + 3 * n + 7 * k)
    A = torch.rand((m, k), generator=g, device="cuda") * 2 - 1
    B = torch.rand((k, n), generator=g, device="cuda") * 2 - 1
    C = torch.rand((m, n), generator=g, device="cuda") * 2 - 1
    Ad = A.t().contiguous().t() if not ta else A.contiguous()
    Bd = B.t().contiguous().t() if not tb else B.contiguous()
    ref = 0.5 * (_tf32(A).double() @ _tf32(B).double()) - 1.5 * C.double()
    Cd = C.t().contiguous().t()
    ops.gemm(Ad, Bd, Cd, alpha=0.5, beta=-1.5, tf32=True)
    assert _rel(Cd, ref) <= TC_TOL


@pytest.mark.parametrize("m,n,k", SHAPES)
def test_gemm_bf16(cuda, m, n, k):
    g = torch.Generator(device="cuda").manual_seed(m * 5 + n + k)
    A = torch.rand((m, k), generator=g, device="cuda") * 2 - 1
    B = torch.rand((k, n), generator=g, device="cuda") * 2 - 1
    ref = A.bfloat16().double() @ B.bfloat16().double()
    C = torch.zeros((n, m), device="cuda").t()
    Acm, Bcm = A.t().contiguous(), B.t().contiguous()  # column-major copies, kept alive across the call
    _lib.call("rc_gemm_bf16", 0, 0, m, n, k, 1.0, ctypes.c_void_p(Acm.data_ptr()), m,
              ctypes.c_void_p(Bcm.data_ptr()), k, 0.0, ctypes.c_void_p(C.data_ptr()), m,
              ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    assert _rel(C, ref) <= TC_TOL


def test_fp32_and_tf32_accuracy(cuda):
    """rc_gemm_f32 (FP32 FMA) is FP32-accurate against FP64; rc_gemm_tf32 carries the
    TF32 operand truncation (~2^-11 per operand), so its error sits between 1e-5 and 2e-3."""
    m = n = k = 2048
    g = torch.Generator(device="cuda").manual_seed(9)
    A = torch.rand((m, k), generator=g, device="cuda") * 2 - 1
    B = torch.rand((k, n), generator=g, device="cuda") * 2 - 1
    ref = A.double() @ B.double()
    C = torch.zeros((m, n), device="cuda")
    ops.gemm(A, B, C, alpha=1.0, beta=0.0)  # FP32 FMA
    assert _rel(C, ref) <= 1e-6
    ops.gemm(A, B, C, alpha=1.0, beta=0.0, tf32=True)
    assert 1e-5 < _rel(C, ref) < 2e-3


def test_bounded_wait_times_out_and_context_survives(cuda):
    lib = _lib.lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert lib.rc_device_status(stream) == 0
    assert lib.rc_selftest_wait_timeout(50_000_000, stream) == 0  # a 50 ms wait that nothing completes
    assert lib.rc_device_status(stream) == 5  # RC_ERR_TIMEOUT, read and cleared
    assert lib.rc_device_status(stream) == 0
    # the context is still usable
    A = torch.ones((256, 256), device="cuda")
    C = torch.zeros((256, 256), device="cuda")
    ops.gemm(A, A, C, alpha=1.0, beta=0.0, tf32=True)
    assert torch.all(C == 256.0)
    assert lib.rc_device_status(stream) == 0


def test_timeout_is_sticky_and_stops_every_tensor_core_kernel(cuda):
    """After a wait runs out, the device error word stays set until it is read: tcgen05
    kernels launched meanwhile return without touching C, the mixed solve returns
    RC_ERR_TIMEOUT instead of computing from a partial factor, and the site of the first
    timeout (the self-test kernel: 900) is reported. Clearing the word restores both."""
    lib = _lib.lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert lib.rc_device_status(stream) == 0
    assert lib.rc_selftest_wait_timeout(20_000_000, stream) == 0
    torch.cuda.synchronize()
    A = torch.ones((512, 512), device="cuda")
    C = torch.full((512, 512), 7.0, device="cuda")
    ops.gemm(A, A, C, alpha=1.0, beta=0.0, tf32=True)
    torch.cuda.synchronize()
    assert torch.all(C == 7.0)  # the tcgen05 kernel returned at once
    n = 600
    G = torch.randn((n, n), device="cuda", dtype=torch.float64)
    S = G @ G.T / n + torch.eye(n, device="cuda", dtype=torch.float64)
    B = torch.randn((4, n), device="cuda", dtype=torch.float64).t()
    _, _, status = ops.spd_solve_mixed(S, B, "tf32")
    assert status == 5  # RC_ERR_TIMEOUT: the sticky word is seen before any work
    site = ctypes.c_int(-1)
    assert lib.rc_device_error_site(stream, ctypes.byref(site)) == 5
    assert site.value == 900
    assert lib.rc_device_status(stream) == 0
    ops.gemm(A, A, C, alpha=1.0, beta=0.0, tf32=True)
    torch.cuda.synchronize()
    assert torch.all(C == 512.0)
    _, info, status = ops.spd_solve_mixed(S, B, "tf32")
    assert status == 0 and info["converged"] == 1
    assert lib.rc_device_status(stream) == 0


def _syrk_tc(prec: int, P: torch.Tensor, C: torch.Tensor, alpha: float, beta: float, flags: int = 0) -> None:
    """P is a row-major n x k view whose row stride is a multiple of 16 bytes (the TMA rule)."""
    n, k = P.shape
    _lib.call("rc_syrk_tc_ex", prec, n, k, alpha, ctypes.c_void_p(P.data_ptr()), P.stride(0), beta,
              ctypes.c_void_p(C.data_ptr()), n, flags, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))


@pytest.mark.parametrize("n,k", [(255, 64), (256, 32), (600, 100), (1024, 1024), (1500, 96), (2560, 512)])
@pytest.mark.parametrize("bf16", [False, True])
@pytest.mark.parametrize("flags", [0, 1])
def test_syrk_tc_lower(cuda, n, k, bf16, flags):
    """Lower SYRK C <- alpha P P^T + beta C on the tcgen05 tensor cores (n >= 256 runs on CTA
    pairs, 256 x 256 tiles; flags 1 = RC_SYRK_BESIDE, the factorisation's configuration; a
    multiple of 32 columns takes the reduce-add epilogue when beta = 1); the strict upper
    triangle of C stays bit-identical."""
    g = torch.Generator(device="cuda").manual_seed(n + k + int(bf16))
    P = torch.rand((n, k), generator=g, device="cuda") * 2 - 1
    C = torch.rand((n, n), generator=g, device="cuda") * 2 - 1
    Pq = P.bfloat16().float() if bf16 else _tf32(P)
    ld = (k + 15) // 16 * 16  # padded rows
    Pbuf = torch.zeros((n, ld), device="cuda", dtype=torch.bfloat16 if bf16 else torch.float32)
    Pbuf[:, :k] = P.bfloat16() if bf16 else P
    for beta in (1.25, 1.0):  # beta = 1: the reduce-add epilogue where the shape allows
        ref = (-0.75 * (Pq.double() @ Pq.double().t()) + beta * C.double()).tril()
        Cd = C.clone()
        _syrk_tc(1 if bf16 else 0, Pbuf[:, :k], Cd, -0.75, beta, flags)
        torch.cuda.synchronize()
        assert _rel(Cd.tril(), ref) <= TC_TOL
        assert torch.equal(Cd.triu(1), C.triu(1))
    assert _lib.lib().rc_device_status(None) == 0
