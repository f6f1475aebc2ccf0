"""CPU tests of the drop-in boundary: the C-ABI library loads without a GPU and
exports every symbol include/*.h declares, including every launcher name the
reference's Rust FFI binds (crates/cuda-kernels/src/lib.rs:16-186) for the
projection path."""
from __future__ import annotations

import ctypes
import glob
import os
import re

import pytest

from boilingsim_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# Launcher names of the reference's projection path (crates/cuda-kernels/src/*.cu).
REFERENCE_LAUNCHERS = [
    "jacobi_pressure_launch", "pressure_solve_launch", "laplacian_spmv_launch",
    "diag_inverse_apply_launch", "dot_launch", "axpy_device_launch", "scaled_axpy_launch",
    "divide_scalars_launch", "compute_b_launch", "zero_buffer_launch",
    "pressure_solve_pcg_launch", "scale_inplace_launch",
]


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\(", text,
                             flags=re.M):
            if m.group(1) not in ("defined",):
                names.add(m.group(1))
    return names


def test_library_loads_and_exports_every_declared_symbol():
    lib = _lib.lib()
    decl = declared_symbols()
    assert len(decl) >= 20
    missing = [n for n in sorted(decl) if not hasattr(lib, n)]
    assert not missing, missing


def test_header_declares_every_reference_launcher():
    decl = declared_symbols()
    assert set(REFERENCE_LAUNCHERS) <= decl


def test_python_signatures_cover_header():
    assert declared_symbols() <= set(_lib.SIGNATURES)


def test_version_and_error_strings():
    lib = _lib.lib()
    assert b"sm_100a" in lib.bsp_version()
    assert b"BSP_ERR_SHAPE" in lib.bsp_error_string(10001)
    assert b"NOT_CONVERGED" in lib.bsp_error_string(10005)


def test_product_library_does_not_link_the_oracle():
    """The product .so must not depend on or embed the CPU oracle."""
    blob = open(_lib.LIB_PATH, "rb").read()
    assert b"or_jacobi_step_f32" not in blob and b"liboracle" not in blob


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "absent.so"))
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(ImportError):
        _lib.lib()


def test_pointer_conversion():
    class CAI:
        __cuda_array_interface__ = {"data": (1234, False)}

    assert _lib.ptr(CAI()) == 1234
    assert _lib.ptr(None) == 0
    assert _lib.ptr(77) == 77
    with pytest.raises(TypeError):
        _lib.ptr(object())
    assert isinstance(ctypes.c_void_p(_lib.ptr(5)).value, int)
