"""rc_spd_solve_f64_noalloc: the SPD solve for callers that cannot let the library
allocate device memory (their memory is reserved up front by their own allocator, or a
cudaMalloc's device-wide synchronisation is not allowed where they call it).

Two calls in a row through the C-ABI, each compared with the allocating entry point
rc_spd_solve_f64 on the same inputs, within the FP64 parity bar (relative Frobenius
<= 1e-13); neither call may add to the library's count of its own device allocations, and
the second leaves the device's free memory unchanged (the first may load the module that
holds the fixed scratch); sizes beyond the fixed scratch must be rejected. This file sorts
last so a run that stops at the first failure has run every other test already; it also
passes alone in a fresh process."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

import oracle
from remora_b200 import _lib
from helpers import to_dev, to_host

pytestmark = pytest.mark.gpu


def _solve(name: str, A: torch.Tensor, B: torch.Tensor) -> tuple[int, int, np.ndarray]:
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    X = B.clone()
    status = getattr(_lib.lib(), name)(A.shape[0], B.shape[1], ctypes.c_void_p(A.data_ptr()), A.stride(1),
                                       ctypes.c_void_p(X.data_ptr()), X.stride(1), ctypes.c_void_p(info.data_ptr()),
                                       ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    return status, int(info.item()), to_host(X)


def test_no_alloc_solve_matches_allocating_solve(cuda, orc):
    lib = _lib.lib()
    for call, (n, nrhs) in enumerate([(1024, 16), (700, 64)]):
        g = orc.rng(100 + call)
        G = g.normal(n, n)
        A = G @ G.T / n + 1e-2 * np.eye(n)
        B = g.normal(n, nrhs)
        Ad, Bd = to_dev(A, False), to_dev(B, False)
        info_d = torch.zeros(1, dtype=torch.int32, device="cuda")
        X = Bd.clone()
        torch.cuda.synchronize()
        count0, free0 = lib.rc_allocation_count(), torch.cuda.mem_get_info()[0]
        status = lib.rc_spd_solve_f64_noalloc(n, nrhs, ctypes.c_void_p(Ad.data_ptr()), Ad.stride(1),
                                              ctypes.c_void_p(X.data_ptr()), X.stride(1),
                                              ctypes.c_void_p(info_d.data_ptr()),
                                              ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        torch.cuda.synchronize()
        assert lib.rc_allocation_count() == count0
        if call > 0:
            assert torch.cuda.mem_get_info()[0] == free0
        assert status == 0 and int(info_d.item()) == 0
        X_static = to_host(X)
        status, info, X_alloc = _solve("rc_spd_solve_f64", Ad, Bd)
        assert status == 0 and info == 0
        assert oracle.rel_fro(X_static, X_alloc) <= 1e-13


def test_no_alloc_rejects_sizes_beyond_its_scratch(cuda):
    A = torch.eye(1025, dtype=torch.float64, device="cuda")
    B = torch.ones((1025, 2), dtype=torch.float64, device="cuda").t().contiguous().t()
    status, _, X = _solve("rc_spd_solve_f64_noalloc", A, B)
    assert status == 7  # RC_ERR_SIZE_LIMIT
    assert np.all(X == 1.0)
    A = torch.eye(64, dtype=torch.float64, device="cuda")
    B = torch.ones((65, 64), dtype=torch.float64, device="cuda").t()
    status, _, _ = _solve("rc_spd_solve_f64_noalloc", A, B)
    assert status == 7
