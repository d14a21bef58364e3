"""RNG fills on the GPU through the C-ABI against the oracle (bit-exact for the Threefry
words, the uniform and the discrete fills; the normal fill within a stated bound because
its log/sincos come from CUDA's libm on one side and glibc's on the other)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from remora_b200 import ops

from helpers import to_host

pytestmark = pytest.mark.gpu

# Normal fill tolerance: |gpu - oracle| <= NORMAL_ATOL * stddev + NORMAL_RTOL * |oracle|.
# logf/sincosf differ by at most 2 ulp between the two libms; through sqrt and the scale
# by r <= ~6.7 this stays below 1e-6 absolute for stddev = 1.
NORMAL_ATOL = 4e-6
NORMAL_RTOL = 4e-6


def _mat(rows, cols, row_major, dtype):
    if row_major:
        return torch.empty((rows, cols), dtype=dtype, device="cuda")
    return torch.empty((cols, rows), dtype=dtype, device="cuda").t()


SHAPES = [(1, 1), (1, 7), (5, 3), (7, 13), (64, 64), (33, 130), (257, 1001)]


@pytest.mark.parametrize("row_major", [True, False])
@pytest.mark.parametrize("shape", SHAPES)
def test_bits_uniform_discrete_bit_exact(cuda, orc, row_major, shape):
    rows, cols = shape
    key = [0x12345678, 0x9ABCDEF0, 0x0F1E2D3C, 0x4B5A6978]
    X = _mat(rows, cols, row_major, torch.int32)
    ops.generate_bits(X, key)
    ref = orc.rng_fill("bits", key, rows, cols)
    assert np.array_equal(to_host(X).view(np.uint32), ref)
    U = _mat(rows, cols, row_major, torch.float32)
    ops.generate_uniform(U, key, -1.5, 2.5)
    ref = orc.rng_fill("uniform", key, rows, cols, a=-1.5, b=2.5)
    assert np.array_equal(to_host(U).view(np.uint32), ref.view(np.uint32))
    D = _mat(rows, cols, row_major, torch.int32)
    ops.generate_discrete(D, key, -3, 1000)
    assert np.array_equal(to_host(D), orc.rng_fill("discrete_i32", key, rows, cols, ia=-3, ib=1000))
    F = _mat(rows, cols, row_major, torch.float32)
    ops.generate_discrete(F, key, 2, 7)
    assert np.array_equal(to_host(F), orc.rng_fill("discrete_f32", key, rows, cols, ia=2, ib=7))


@pytest.mark.parametrize("row_major", [True, False])
def test_normal_within_bound(cuda, orc, row_major):
    rows, cols = 301, 517
    key = [1, 2, 3, 4]
    X = _mat(rows, cols, row_major, torch.float32)
    ops.generate_normal(X, key, 0.5, 4.0)  # stddev 2
    ref = orc.rng_fill("normal", key, rows, cols, a=0.5, b=2.0)
    got = to_host(X)
    fin = np.isfinite(ref)
    assert np.array_equal(np.isfinite(got), fin)
    err = np.abs(got[fin] - ref[fin])
    assert np.all(err <= NORMAL_ATOL * 2.0 + NORMAL_RTOL * np.abs(ref[fin]))
    # most elements agree to the last bit
    assert np.mean(got[fin].view(np.uint32) == ref[fin].view(np.uint32)) > 0.5


def test_key_from_host_generator(cuda, orc, golden):
    """The key is 4 draws of the seeded host mt19937 (kernels/hip/random.hpp:225-227)."""
    g = golden("rng")
    key = orc.rng(42).key()
    assert key == g["key"].tolist()
    U = _mat(7, 13, True, torch.float32)
    ops.generate_uniform(U, key, -1.0, 1.0)
    assert np.array_equal(to_host(U).view(np.uint32), g["uniform"].view(np.uint32))


def test_ld_padding_and_no_out_of_bounds_write(cuda, orc):
    rows, cols = 9, 10
    key = [7, 7, 7, 7]
    for row_major in (True, False):
        big = torch.full((40, 40), -7, dtype=torch.int32, device="cuda")
        X = big[:rows, :cols] if row_major else big[:cols, :rows].t()
        ops.generate_bits(X, key)
        h = to_host(big)
        sub = h[:rows, :cols] if row_major else h[:cols, :rows].T
        assert np.array_equal(sub.view(np.uint32), orc.rng_fill("bits", key, rows, cols))
        mask = np.ones_like(h, dtype=bool)
        if row_major:
            mask[:rows, :cols] = False
        else:
            mask[:cols, :rows] = False
        assert np.all(h[mask] == -7)


def test_counter_wrap_rows(cuda):
    """Rows i and i + 65536 share a counter (random.hpp:167 keeps 16 bits of the row)."""
    rows, cols = 65536 + 40, 8
    X = torch.empty((rows, cols), dtype=torch.int32, device="cuda")
    ops.generate_bits(X, [5, 6, 7, 8])
    h = to_host(X)
    assert np.array_equal(h[:40], h[65536:])
    assert not np.array_equal(h[0], h[1])


def test_full_size_fill_sampled(cuda, orc):
    """The 2^28-element normal fill as a 16384 x 16384 row-major matrix: sampled rows
    against the oracle, and moments of the whole fill."""
    n = 16384
    key = orc.rng(2024).key()
    X = torch.empty((n, n), dtype=torch.float32, device="cuda")
    ops.generate_normal(X, key, 0.0, 1.0)
    torch.cuda.synchronize()
    for i in (0, 1, 4097, 65535 % n, n - 1):
        ref = orc.rng_fill("normal", key, 1, n, a=0.0, b=1.0, row0=i)
        got = X[i:i + 1].cpu().numpy()
        fin = np.isfinite(ref)
        assert np.array_equal(np.isfinite(got), fin)
        assert np.all(np.abs(got[fin] - ref[fin]) <= NORMAL_ATOL + NORMAL_RTOL * np.abs(ref[fin]))
    fin = torch.isfinite(X)
    assert fin.float().mean().item() > 0.999
    vals = X[fin].double()
    assert abs(vals.mean().item()) < 1e-3
    assert abs(vals.std().item() - 1.0) < 1e-3
    del X
