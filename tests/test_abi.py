"""The C-ABI library loads without a GPU and exports every entry point its header declares."""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

import pytest

import remora_b200
from remora_b200 import _lib

HEADERS = sorted((Path(__file__).resolve().parents[1] / "include").glob("*.h"))


def declared_symbols() -> set[str]:
    names = set()
    for h in HEADERS:
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(rc_\w+)\s*\(", text))
    return names


def test_library_loads_and_exports_header_symbols():
    lib = remora_b200.lib()
    names = declared_symbols()
    assert len(names) >= 20
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    assert declared_symbols() <= set(_lib.SIGNATURES)


def test_host_only_entry_points():
    lib = remora_b200.lib()
    assert lib.rc_version() >= 100
    assert lib.rc_error_string(0) == b"success"
    assert b"invalid" in lib.rc_error_string(1)


def test_argument_checks_need_no_device():
    """Size/leading-dimension checks return RC_ERR_INVALID_ARGUMENT before any CUDA call."""
    lib = remora_b200.lib()
    fake = ctypes.c_void_p(16)
    # lda < m
    assert lib.rc_gemm_f64(0, 0, 10, 10, 10, 1.0, fake, 5, fake, 10, 0.0, fake, 10, None) == 1
    # potrf without a status word
    assert lib.rc_potrf_f64(0, 10, fake, 10, None, None) == 1
    # discrete range reversed
    key = _lib.key_array([1, 2, 3, 4])
    assert lib.rc_rng_discrete_i32(key, 4, 4, fake, 4, 1, 5, 2, None) == 1
    # empty problems are no-ops
    assert lib.rc_gemm_f32(0, 0, 0, 5, 5, 1.0, None, 1, None, 1, 0.0, None, 1, None) == 0


def test_argument_checks_of_factorisations_and_sliced_product():
    """getrf / pstrf / the int8 FP64 product reject bad arguments before any CUDA call."""
    lib = remora_b200.lib()
    fake = ctypes.c_void_p(16)
    assert lib.rc_getrf_f64(0, 10, fake, 10, fake, None, None) == 1  # no status word
    assert lib.rc_getrf_f32(1, 10, fake, 5, fake, fake, None) == 1  # lda < n
    assert lib.rc_pstrf_f64(0, 10, fake, 10, fake, None, None) == 1  # no rank word
    assert lib.rc_pstrf_f32(0, 10, None, 10, fake, fake, None) == 1  # no matrix
    assert lib.rc_gemm_f64_sliced(10, 4, 10, 1.0, None, 10, fake, 10, 0.0, fake, 10, None) == 1
    assert lib.rc_gemm_f64_sliced(10, 4, 10, 1.0, fake, 9, fake, 10, 0.0, fake, 10, None) == 1  # lda < m
    assert lib.rc_gemm_f64_sliced(10, 65, 10, 1.0, fake, 10, fake, 10, 0.0, fake, 10, None) == 4  # > 64 columns
    assert lib.rc_gemm_f64_sliced(0, 4, 10, 1.0, None, 1, None, 1, 0.0, None, 1, None) == 0  # empty


def test_mixed_workspace_sizes_without_a_gpu():
    """rc_spd_solve_mixed_workspace is host arithmetic: the EMU64 solve keeps an FP64 working
    copy (8 n^2 bytes) where TF32 keeps an FP32 one (4 n^2), panel widths above 4096 fall
    back to 1024 for EMU64, and every size grows with the right-hand sides."""
    lib = remora_b200.lib()

    def size(prec, n, nrhs, outer=1024):
        o = _lib.MixedOptions(1e-15, 100, outer, -1.0)
        out = ctypes.c_size_t(0)
        assert lib.rc_spd_solve_mixed_workspace(prec, n, nrhs, ctypes.byref(o), ctypes.byref(out)) == 0
        return out.value

    n = 4096
    tf32, emu = size(_lib.RC_PREC_TF32, n, 64), size(_lib.RC_PREC_EMU64, n, 64)
    assert emu - tf32 >= 3 * n * n  # FP64 instead of FP32 working copy (less the FP32-only buffers)
    assert size(_lib.RC_PREC_EMU64, n, 64, outer=8192) == size(_lib.RC_PREC_EMU64, n, 64, outer=1024)
    assert size(_lib.RC_PREC_EMU64, n, 64) > size(_lib.RC_PREC_EMU64, n, 8)


@pytest.mark.parametrize("compiler,std", [("gcc", "-std=c99"), ("g++", "-std=c++14")])
def test_c_abi_header_is_plain_c_and_cpp(tmp_path, compiler, std):
    """include/remora_cuda.h compiles on its own as C99 and as C++14 (no CUDA headers, no
    torch types), which is what an FFI binding or a g++-built Remora program includes."""
    import shutil
    import subprocess
    if shutil.which(compiler) is None:
        pytest.skip(f"{compiler} not installed")
    src = tmp_path / ("t.c" if compiler == "gcc" else "t.cpp")
    src.write_text('#include <remora_cuda.h>\nint main(void) { return rc_version() > 0 ? 0 : 1; }\n')
    inc = Path(__file__).resolve().parent.parent / "include"
    subprocess.run([compiler, std, "-Wall", "-Werror", "-pedantic", "-fsyntax-only", f"-I{inc}", str(src)],
                   check=True)


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    """Without the built library every entry point raises (the ops wrappers all load it
    through _lib.lib()): there is no CPU fallback."""
    monkeypatch.setattr(_lib, "LIB_PATH", tmp_path / "libremora_cuda.so")
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(RuntimeError, match="is missing"):
        _lib.lib()
    with pytest.raises(RuntimeError, match="is missing"):
        _lib.call("rc_potrf_f64", 0, 4, None, 4, None, None)
