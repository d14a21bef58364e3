"""The cuda_tag drop-in: a Remora C++ program (tests/cpp/dropin_test.cpp) written against
the unchanged API, with only the device tag switched, checked against Remora's own CPU
kernels in the same program (FP64 <= 1e-13, FP32 <= 1e-5 relative Frobenius)."""
from __future__ import annotations

import subprocess
from pathlib import Path

import pytest

BIN = Path(__file__).resolve().parent / "cpp" / "_build" / "dropin_test"


@pytest.mark.gpu
def test_dropin_program(cuda):
    assert BIN.exists(), f"{BIN} is not built (build() compiles it from tests/cpp/Makefile)"
    res = subprocess.run([str(BIN)], capture_output=True, text=True, timeout=600)
    print(res.stdout)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "PASSED" in res.stdout


def test_dropin_headers_compile_without_cuda_toolkit():
    """The cuda_tag headers compile with the host compiler alone (no CUDA headers on the
    include path) when Remora's headers are available."""
    import oracle
    if not oracle.reference_present():
        pytest.skip("Remora's headers are not on this machine")
    ref = oracle.REF_INCLUDE / "remora"
    root = Path(__file__).resolve().parents[1]
    src = "#include <remora/cuda.hpp>\n#include <remora/remora.hpp>\nint main(){return 0;}\n"
    res = subprocess.run(["g++", "-std=c++14", "-fsyntax-only", "-w", f"-I{root / 'include'}", f"-I{ref.parent}",
                          f"-I{root / 'oracle' / 'stub_boost'}", "-x", "c++", "-"], input=src, capture_output=True,
                         text=True)
    assert res.returncode == 0, res.stderr[-2000:]
