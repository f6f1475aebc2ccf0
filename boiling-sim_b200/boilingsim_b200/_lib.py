"""ctypes binding of libbsproj.so (the C ABI declared in include/bsproj.h).

The product path has no CPU fallback: if the library is missing or no CUDA
device is present, every call raises.  Argument conversion accepts torch
tensors and any object exposing ``__cuda_array_interface__`` (the reference
passes Warp arrays that way, python/boilingsim/fluid.py:649-652).
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libbsproj.so")

_P = ctypes.c_void_p
_I = ctypes.c_int
_L = ctypes.c_int64
_F = ctypes.c_float

# name -> (restype, argtypes); mirrors include/bsproj.h
SIGNATURES = {
    # reference-compatible launchers
    "jacobi_pressure_launch": (_I, [_P, _P, _P, _P, _I, _I, _I, _F, _F, _F, _I, _I]),
    "pressure_solve_launch": (_I, [_P, _P, _P, _P, _I, _I, _I, _F, _F, _F, _I, _I, _I]),
    "laplacian_spmv_launch": (_I, [_P, _P, _P, _I, _I, _I, _I, _I]),
    "diag_inverse_apply_launch": (_I, [_P, _P, _P, _I, _I, _I, _I, _I]),
    "dot_launch": (_I, [_P, _P, _I, _P, _P]),
    "axpy_device_launch": (_I, [_P, _P, _P, _I, _I]),
    "scaled_axpy_launch": (_I, [_P, _P, _P, _P, _I]),
    "divide_scalars_launch": (_I, [_P, _P, _P]),
    "compute_b_launch": (_I, [_P, _P, _P, _I, _I, _I, _F, _I]),
    "zero_buffer_launch": (_I, [_P, _I]),
    "scale_inplace_launch": (_I, [_P, _I, _F]),
    "pressure_solve_pcg_launch": (_I, [_P, _P, _P, _I, _I, _I, _F, _F, _F, _I, _I, _F, _I]
                                  + [_P] * 13 + [ctypes.POINTER(ctypes.c_int)]),
    # B200-native
    "bsp_version": (ctypes.c_char_p, []),
    "bsp_error_string": (ctypes.c_char_p, [_I]),
    "bsp_mask_from_mat": (_I, [_P, _P, _I, _I, _I, _I, _I, _P]),
    "bsp_jacobi_sweep": (_I, [_P, _P, _P, _P, _I, _I, _I, _F, _F, _F, _P]),
    "bsp_jacobi_solve": (_I, [_P, _P, _P, _P, _P, _I, _I, _I, _F, _F, _F, _I, _I, _P]),
    "bsp_set_tuning": (_I, [_I, _I]),
    "bsp_sweep2_error": (_I, [_P]),
    "bsp_autotune_jacobi": (_I, [_P, _P, _P, _P, _P, _I, _I, _I, _F, _F, _F, _I, _P, _I, _P, _P]),
    "bsp_autotune_solve": (_I, [_P, _P, _P, _I, _I, _I, _F, _F, _F, _P, _P, ctypes.c_size_t, _P,
                                _I, _P, _P]),
    "bsp_solve_batch": (_I, [_I, _P, _P, _P, _P]),
    "bsp_dot_noalloc": (_I, [_P, _P, _L, _P, _P]),
    "bsp_profile_enable": (_I, [_I]),
    "bsp_profile_read": (_I, [_P, _P, _I]),
    "bsp_coarse_trace_read": (_I, [_P, _I]),
    "bsp_divergence": (_I, [_P, _P, _P, _P, _P, _I, _I, _I, _F, _P, _P]),
    "bsp_subtract_gradient": (_I, [_P, _P, _P, _P, _P, _I, _I, _I, _F, _F, _F, _P]),
    "bsp_enforce_no_slip": (_I, [_P, _P, _P, _P, _I, _I, _I, _P]),
    "bsp_projection_jacobi": (_I, [_P, _P, _P, _P, _P, _P, _P, _I, _I, _I, _F, _F, _F, _I, _I,
                                   _P, _P]),
    "bsp_step_projection_jacobi": (_I, [_P, _P, _P, _P, _P, _P, _P, _I, _I, _I, _F, _F, _F, _I,
                                        _I, _P, _P]),
    "bsp_noslip_divergence": (_I, [_P, _P, _P, _P, _P, _I, _I, _I, _F, _P]),
    # semi-Lagrangian advection (advect.cu)
    "bsp_extend_temperature": (_I, [_P, _P, _P, _I, _I, _I, _P]),
    "bsp_advect_temperature": (_I, [_P, _P, _P, _P, _P, _P, _P, _I, _I, _I, _F, _F, _F, _F, _F,
                                    _P]),
    "bsp_advect_velocity": (_I, [_I, _P, _P, _P, _P, _P, _I, _I, _I, _F, _F, _F, _F, _F, _P]),
    "bsp_advect_all": (_I, [_P] * 10 + [_I, _I, _I, _F, _F, _F, _F, _F, _I, _P]),
    # backward-Euler conduction (conduction.cu)
    "bsp_conduction_sweep": (_I, [_P, _P, _P, _P, _I, _I, _I, _P, _P, _P, _I, _F, _F, _F, _F, _I,
                                  _P]),
    "bsp_conduction_sweep_u8": (_I, [_P, _P, _P, _P, _I, _I, _I, _P, _P, _P, _I, _F, _F, _F, _F,
                                     _I, _P]),
    "bsp_conduction_be": (_I, [_P, _P, _P, _P, _I, _I, _I, _P, _P, _P, _I, _F, _F, _F, _F, _I, _I,
                               _P]),
    "bsp_conduction_be_u8": (_I, [_P, _P, _P, _P, _I, _I, _I, _P, _P, _P, _I, _F, _F, _F, _F, _I,
                                  _I, _P]),
    "bsp_material_ids": (_I, [_P, _P, _L, _I, _P, _P]),
    "bsp_conduction_prepare_workspace_bytes": (ctypes.c_size_t, []),
    "bsp_conduction_error": (_I, [_P]),
    "bsp_conduction_prepare": (_I, [_P, _P, ctypes.POINTER(ctypes.c_int), _P, _I, _I, _I, _I, _I,
                                    _P, ctypes.c_size_t, _P]),
    "bsp_conduction_tile_flags_bytes": (ctypes.c_size_t, [_I, _I, _I]),
    "bsp_conduction_tile_flags": (_I, [_P, _P, _I, _I, _I, _P]),
    "bsp_conduction_sweep_cls": (_I, [_P, _P, _P, _P, _P, _I, _P, _I, _I, _I, _P, _P, _P, _I, _F,
                                      _F, _F, _F, _I, _P]),
    "bsp_conduction_be_cls": (_I, [_P, _P, _P, _P, _P, _I, _P, _I, _I, _I, _P, _P, _P, _I, _F, _F,
                                   _F, _F, _I, _I, _P]),
    # learned warm start (unet.cu)
    "bsp_unet_conv3_fwd": (_I, [_P, _P, _P, _P, _I, _I, _I, _I, _I, _I, _P]),
    "bsp_unet_wgrad_workspace_bytes": (ctypes.c_size_t, [_I, _I, _I, _I, _I]),
    "bsp_unet_conv3_wgrad": (_I, [_P, _P, _P, _P, _I, _I, _I, _I, _I, _P, ctypes.c_size_t, _P]),
    "bsp_unet_flip_weights": (_I, [_P, _P, _I, _I, _P]),
    "bsp_unet_relu_bwd": (_I, [_P, _P, _L, _P]),
    "bsp_unet_pool": (_I, [_P, _P, _I, _I, _I, _I, _I, _I, _P]),
    "bsp_unet_up": (_I, [_P, _P, _I, _I, _I, _I, _I, _P]),
    "bsp_unet_add": (_I, [_P, _P, _L, _P]),
    "bsp_unet_pack_input": (_I, [_P, _P, _P, _L, _F, _P]),
    "bsp_unet_head_fwd": (_I, [_P, _P, _P, _P, _P, _L, _F, _P]),
    "bsp_unet_head_loss": (_I, [_P, _P, _I, _P, _P, _P, _P, _P, _L, _F, _F, _P]),
    "bsp_unet_sum_partials": (_I, [_P, _P, _I, _I, _P]),
    "bsp_unet_head_bwd": (_I, [_P, _P, _I, _P, _P, _P, _P, _L, _P]),
    "bsp_unet_adam": (_I, [_P, _P, _P, _P, _P, _L, _F, _F, _F, _F, _I, _P]),
    # tensor-core (tcgen05) inference path on the padded layout (unet_tc.cu)
    "bsp_unet_tc_rows": (_L, [_I, _I, _I]),
    "bsp_unet_tc_weights": (_I, [_P, _P, _I, _I, _P]),
    "bsp_unet_tc_conv3": (_I, [_P, _P, _P, _P, _P, _I, _I, _I, _I, _I, _I, _P]),
    "bsp_unet_tc_error": (_I, [_P]),
    "bsp_unet_tc_trace": (_I, [_P, _I]),
    "bsp_unet_tc_pack": (_I, [_P, _P, _P, _I, _I, _I, _P, _P]),
    "bsp_unet_scale_workspace_bytes": (ctypes.c_size_t, []),
    "bsp_unet_input_scale": (_I, [_P, _P, _P, _I, _I, _I, _P, ctypes.c_size_t, _P]),
    "bsp_unet_tc_pool": (_I, [_P, _P, _I, _I, _I, _I, _P]),
    "bsp_unet_tc_up": (_I, [_P, _P, _I, _I, _I, _I, _P]),
    "bsp_unet_tc_head": (_I, [_P, _P, _P, _P, _P, _I, _I, _I, _P, _F, _P]),
    "bsp_unet_restrict_div": (_I, [_P, _P, _P, _P, _I, _I, _I, _P]),
    "bsp_unet_prolong": (_I, [_P, _P, _P, _I, _I, _I, _P]),
    "bsp_unet_energy_scale": (_I, [_P, _P, _P, _P, _I, _I, _I, _F, _P, ctypes.c_size_t, _P, _P]),
    "bsp_unet_energy_scale_keep": (_I, [_P, _P, _P, _P, _I, _I, _I, _F, _F, _P, ctypes.c_size_t,
                                        _P, _P, _P]),
    "bsp_spmv": (_I, [_P, _P, _P, _I, _I, _I, _P]),
    "bsp_selftest_div6": (_I, [_P, _P]),
    "bsp_selftest_waits": (_I, [_P, _P, _P]),
    "bsp_solve_params_default": (None, [_P]),
    "bsp_solver_workspace_bytes": (ctypes.c_size_t, [_I, _I, _I, _I]),
    "bsp_solve_tol": (_I, [_P, _P, _P, _I, _I, _I, _F, _F, _F, _P, _P, ctypes.c_size_t, _P, _P,
                           _P]),
}


class BspSolveParams(ctypes.Structure):
    """include/bsproj.h: BspSolveParams."""

    _fields_ = [("tol", ctypes.c_double), ("inner_tol", ctypes.c_double),
                ("max_outer", ctypes.c_int), ("max_inner", ctypes.c_int),
                ("storage", ctypes.c_int), ("warm_start", ctypes.c_int),
                ("check_every", ctypes.c_int), ("reuse_setup", ctypes.c_int),
                ("use_graph", ctypes.c_int)]


class BspBatchItem(ctypes.Structure):
    """include/bsproj.h: BspBatchItem."""

    _fields_ = [("p", ctypes.c_void_p), ("div", ctypes.c_void_p), ("mask", ctypes.c_void_p),
                ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("dx", ctypes.c_float), ("dt", ctypes.c_float), ("rho", ctypes.c_float),
                ("workspace", ctypes.c_void_p), ("workspace_bytes", ctypes.c_size_t)]


class BspTuneChoice(ctypes.Structure):
    """include/bsproj.h: BspTuneChoice."""

    _fields_ = [("key", ctypes.c_int), ("value", ctypes.c_int), ("ms", ctypes.c_float),
                ("status", ctypes.c_int)]


class BspSolveInfo(ctypes.Structure):
    """include/bsproj.h: BspSolveInfo."""

    _fields_ = [("outer_iterations", ctypes.c_int), ("inner_iterations", ctypes.c_int),
                ("levels", ctypes.c_int), ("pad", ctypes.c_int),
                ("rel_residual", ctypes.c_double)]

_lib = None


class BspError(RuntimeError):
    """A non-zero status from the native library (cudaError_t or BSP_ERR_*)."""

    def __init__(self, fn: str, code: int, msg: str):
        super().__init__(f"{fn} failed with status {code}: {msg}")
        self.code = code


def lib() -> ctypes.CDLL:
    """Load libbsproj.so once; raise loudly if it is absent (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python boiling-sim_b200/build.py` "
                "(there is no CPU fallback for the projection path)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(fn: str, code: int) -> None:
    if code != 0:
        msg = lib().bsp_error_string(int(code)).decode()
        raise BspError(fn, int(code), msg)


def call(fn: str, *args) -> int:
    """Call ``fn`` and raise BspError on a non-zero status."""
    code = getattr(lib(), fn)(*args)
    if fn not in ("bsp_version", "bsp_error_string"):
        check(fn, code)
    return code


def ptr(x) -> int:
    """Device address of a torch tensor / CUDA-array-interface object / int."""
    if x is None:
        return 0
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        return int(x.data_ptr())
    cai = getattr(x, "__cuda_array_interface__", None)
    if cai is not None:
        return int(cai["data"][0])
    raise TypeError(f"cannot take a device pointer of {type(x)!r}")


def stream_handle(stream=None) -> int:
    """cudaStream_t of ``stream`` or of torch's current stream."""
    import torch

    if stream is None:
        stream = torch.cuda.current_stream()
    if isinstance(stream, int):
        return stream
    return int(stream.cuda_stream)
