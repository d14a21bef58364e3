"""Helpers shared by the GPU parity tests: host<->device copies that keep a layout."""
from __future__ import annotations

import numpy as np
import torch


def to_dev(a: np.ndarray, row_major: bool = True, dtype=None) -> torch.Tensor:
    """Copy a 2-D array to cuda:0 in row-major (C) or column-major (F) storage."""
    a = np.asarray(a, dtype=dtype) if dtype is not None else np.asarray(a)
    if row_major:
        return torch.from_numpy(np.ascontiguousarray(a)).cuda()
    return torch.from_numpy(np.ascontiguousarray(a.T)).cuda().t()


def to_host(t: torch.Tensor) -> np.ndarray:
    torch.cuda.synchronize()
    return t.cpu().numpy()


def with_ld(a: np.ndarray, row_major: bool, pad: int, dtype=None) -> torch.Tensor:
    """Device copy embedded in a larger buffer so the leading dimension exceeds the size."""
    a = np.asarray(a, dtype=dtype) if dtype is not None else np.asarray(a)
    r, c = a.shape
    if row_major:
        big = torch.zeros((r, c + pad), dtype=torch.from_numpy(a).dtype, device="cuda")
        big[:, :c] = torch.from_numpy(np.ascontiguousarray(a)).cuda()
        return big[:, :c]
    big = torch.zeros((c, r + pad), dtype=torch.from_numpy(a).dtype, device="cuda")
    big[:, :r] = torch.from_numpy(np.ascontiguousarray(a.T)).cuda()
    return big[:, :r].t()
