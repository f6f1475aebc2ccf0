"""CPU oracle for the pressure-projection path and the two steps widened
around it, backward-Euler conduction and semi-Lagrangian advection (TEST
INFRASTRUCTURE ONLY).

Only tests/, ``__graft_entry__.smoke()`` and the cpu_baseline / reference arm
of ``bench.py`` import this module.  It is the checker, never the product:
the product library (``boilingsim_b200``) does not import it and has no CPU
fallback.

The arithmetic lives in ``proj_oracle.c`` (a plain-C restatement of the
reference's ``python/boilingsim/fluid.py:201-330, 612-734`` and
``crates/cuda-kernels/src/{jacobi_pressure,laplacian_spmv,diag_inverse_apply,
axpy_device,pressure_solve_pcg}.cu``); this module is a ctypes wrapper over it
that takes and returns numpy arrays, plus:

* ``ref_library(fma=True)`` -- the reference's own CUDA sources compiled from
  source into ``oracle/_ref/`` by ``oracle/Makefile`` (GPU comparator);
* ``analytic_*`` -- closed-form known answers from
  ``python/tests/test_pressure_cg.py:62-69``.

Parity pin: the FP32 restatement is checked bit-for-bit against outputs of
the reference CUDA kernels (``tests/golden/*.npz``, generated on a B200 by
``tests/golden/make_golden.py`` from ``oracle/_ref``).  The conduction
(``conduction_*``, ``thermal.py:259-388, 647-658``) and advection
(``extend_temperature``, ``advect_*``, ``fluid.py:39-104, 338-498, 737-776``)
restatements are parity unpinned against reference outputs (the reference
runs them only as Warp code, which cannot run here); they are checked against
closed-form answers and the reference's own drift test instead.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

MAT_FLUID, MAT_POT_WALL, MAT_AIR, MAT_CARROT = 0, 1, 2, 3

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_I, _F, _D, _L = ctypes.c_int, ctypes.c_float, ctypes.c_double, ctypes.c_int64


# Where the reference's hot-path CUDA sources lie when the reference tree is
# mounted (the build recipe compiles them in place into oracle/_ref); override
# with BOILINGSIM_REFERENCE_SRC.
_REF_SRC_DEFAULT = "/root/reference/crates/cuda-kernels/src"


def build() -> None:
    """Compile liboracle.so, and oracle/_ref when the reference sources are
    present."""
    src = os.environ.get("BOILINGSIM_REFERENCE_SRC", _REF_SRC_DEFAULT)
    cmd = ["make", "-s", "-C", _HERE]
    if os.path.isdir(src):
        cmd.append(f"REF_SRC={src}")
    subprocess.run(cmd, check=True)


def lib() -> ctypes.CDLL:
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        sig = {
            "or_num_threads": (_I, []),
            "or_set_num_threads": (None, [_I]),
            "or_divergence_f32": (None, [_f32p, _f32p, _f32p, _f32p, _i32p, _I, _I, _I, _F, _I]),
            "or_jacobi_step_f32": (None, [_f32p, _f32p, _f32p, _i32p, _I, _I, _I, _F, _F, _F, _I, _I]),
            "or_pressure_solve_f32": (None, [_f32p, _f32p, _f32p, _i32p, _I, _I, _I, _F, _F, _F, _I, _I, _I]),
            "or_subtract_gradient_f32": (None, [_f32p, _f32p, _f32p, _f32p, _i32p, _I, _I, _I, _F, _F, _F, _I]),
            "or_enforce_no_slip_f32": (None, [_f32p, _f32p, _f32p, _i32p, _I, _I, _I, _I]),
            "or_max_abs_f32": (_F, [_f32p, _L]),
            "or_projection_jacobi_f32": (_F, [_f32p, _f32p, _f32p, _f32p, _f32p, _f32p, _i32p,
                                              _I, _I, _I, _F, _F, _F, _I, _I, _I]),
            "or_spmv_f32": (None, [_f32p, _f32p, _i32p, _I, _I, _I, _I, _I, _I]),
            "or_diag_inverse_f32": (None, [_f32p, _f32p, _i32p, _I, _I, _I, _I, _I]),
            "or_compute_b_f32": (None, [_f32p, _f32p, _i32p, _I, _I, _I, _F, _F, _F, _I]),
            "or_dot_f32_f64": (_D, [_f32p, _f32p, _L]),
            "or_axpy_f32": (None, [_f32p, _f32p, _F, _L, _I]),
            "or_scaled_axpy_f32": (None, [_f32p, _f32p, _f32p, _F, _L]),
            "or_divide_f32": (_F, [_F, _F]),
            "or_scale_f32": (None, [_f32p, _L, _F]),
            "or_pcg_f32": (_I, [_f32p, _f32p, _i32p, _I, _I, _I, _F, _F, _F, _I, _I, _F, _I]),
            "or_apply_A_f64": (None, [_f64p, _f64p, _i32p, _I, _I, _I, _I, _I]),
            "or_rhs_f64": (None, [_f64p, _f32p, _i32p, _L, _D, _D, _D, _I]),
            "or_cg_f64": (_I, [_f64p, _f64p, _i32p, _I, _I, _I, _I, _I, _D, _I,
                               ctypes.POINTER(ctypes.c_double)]),
            "or_rel_residual_f64": (_D, [_f32p, _f32p, _i32p, _I, _I, _I, _D, _D, _D, _I, _I]),
            "or_conduction_sweep_f32": (None, [_f32p, _f32p, _f32p, _i32p, _I, _I, _I, _f32p,
                                               _f32p, _f32p, _F, _F, _F, _F, _I]),
            "or_conduction_be_f32": (None, [_f32p, _f32p, _f32p, _i32p, _I, _I, _I, _f32p,
                                            _f32p, _f32p, _F, _F, _F, _F, _I, _I]),
            "or_extend_temperature_f32": (None, [_f32p, _f32p, _i32p, _I, _I, _I, _I]),
            "or_advect_temperature_f32": (None, [_f32p, _f32p, _f32p, _f32p, _f32p, _f32p,
                                                 _i32p, _I, _I, _I, _f32p, _F, _F, _I]),
            "or_advect_velocity_f32": (None, [_I, _f32p, _f32p, _f32p, _f32p, _i32p, _I, _I, _I,
                                              _f32p, _F, _F, _I]),
            "or_advect_all_f32": (None, [_f32p] * 9 + [_i32p, _I, _I, _I, _f32p, _F, _F, _I]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def set_threads(n: int) -> None:
    lib().or_set_num_threads(int(n))


def num_threads() -> int:
    return int(lib().or_num_threads())


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


# ---------------------------------------------------------------------------
# FP32 restatement
# ---------------------------------------------------------------------------

def divergence(ux, uy, uz, mat, dx, mat_fluid=MAT_FLUID):
    mat = _c(mat, np.int32)
    nx, ny, nz = mat.shape
    out = np.empty((nx, ny, nz), np.float32)
    lib().or_divergence_f32(out, _c(ux, np.float32), _c(uy, np.float32), _c(uz, np.float32),
                            mat, nx, ny, nz, np.float32(dx), mat_fluid)
    return out


def jacobi_step(p_old, div, mat, dx, dt, rho, mat_fluid=MAT_FLUID, mat_air=MAT_AIR):
    mat = _c(mat, np.int32)
    nx, ny, nz = mat.shape
    out = np.empty((nx, ny, nz), np.float32)
    lib().or_jacobi_step_f32(out, _c(p_old, np.float32), _c(div, np.float32), mat,
                             nx, ny, nz, np.float32(dx), np.float32(dt), np.float32(rho),
                             mat_fluid, mat_air)
    return out


def pressure_solve(p0, div, mat, dx, dt, rho, n_iter, mat_fluid=MAT_FLUID, mat_air=MAT_AIR):
    """``n_iter`` ping-pong sweeps starting from ``p0``; returns p (new array)."""
    mat = _c(mat, np.int32)
    nx, ny, nz = mat.shape
    p = np.array(p0, dtype=np.float32, order="C", copy=True)
    tmp = np.zeros_like(p)
    lib().or_pressure_solve_f32(p, tmp, _c(div, np.float32), mat, nx, ny, nz,
                                np.float32(dx), np.float32(dt), np.float32(rho),
                                int(n_iter), mat_fluid, mat_air)
    return p


def subtract_gradient(ux, uy, uz, p, mat, dx, dt, rho, mat_fluid=MAT_FLUID):
    """Returns new (ux, uy, uz) after the gradient subtract."""
    mat = _c(mat, np.int32)
    nx, ny, nz = mat.shape
    ux, uy, uz = (np.array(a, np.float32, order="C", copy=True) for a in (ux, uy, uz))
    lib().or_subtract_gradient_f32(ux, uy, uz, _c(p, np.float32), mat, nx, ny, nz,
                                   np.float32(dx), np.float32(dt), np.float32(rho), mat_fluid)
    return ux, uy, uz


def enforce_no_slip(ux, uy, uz, mat, mat_fluid=MAT_FLUID):
    mat = _c(mat, np.int32)
    nx, ny, nz = mat.shape
    ux, uy, uz = (np.array(a, np.float32, order="C", copy=True) for a in (ux, uy, uz))
    lib().or_enforce_no_slip_f32(ux, uy, uz, mat, nx, ny, nz, mat_fluid)
    return ux, uy, uz


def projection_jacobi(ux, uy, uz, mat, dx, dt, rho, n_iter, mat_fluid=MAT_FLUID,
                      mat_air=MAT_AIR):
    """fluid.py:612-734 (Jacobi back-end).  Returns dict with p, div (the
    diagnostic divergence), ux, uy, uz (corrected) and max_div."""
    mat = _c(mat, np.int32)
    nx, ny, nz = mat.shape
    ux, uy, uz = (np.array(a, np.float32, order="C", copy=True) for a in (ux, uy, uz))
    p = np.empty((nx, ny, nz), np.float32)
    tmp = np.empty_like(p)
    div = np.empty_like(p)
    m = lib().or_projection_jacobi_f32(p, tmp, div, ux, uy, uz, mat, nx, ny, nz,
                                       np.float32(dx), np.float32(dt), np.float32(rho),
                                       int(n_iter), mat_fluid, mat_air)
    return {"p": p, "div": div, "ux": ux, "uy": uy, "uz": uz, "max_div": float(m)}


def spmv(p, mat, fused=True, mat_fluid=MAT_FLUID, mat_air=MAT_AIR):
    mat = _c(mat, np.int32)
    nx, ny, nz = mat.shape
    out = np.empty((nx, ny, nz), np.float32)
    lib().or_spmv_f32(out, _c(p, np.float32), mat, nx, ny, nz, mat_fluid, mat_air,
                      1 if fused else 0)
    return out


def diag_inverse(r, mat, mat_fluid=MAT_FLUID, mat_air=MAT_AIR):
    mat = _c(mat, np.int32)
    nx, ny, nz = mat.shape
    out = np.empty((nx, ny, nz), np.float32)
    lib().or_diag_inverse_f32(out, _c(r, np.float32), mat, nx, ny, nz, mat_fluid, mat_air)
    return out


def compute_b(div, mat, dx, dt, rho, mat_fluid=MAT_FLUID):
    mat = _c(mat, np.int32)
    nx, ny, nz = mat.shape
    out = np.empty((nx, ny, nz), np.float32)
    lib().or_compute_b_f32(out, _c(div, np.float32), mat, nx, ny, nz, np.float32(dx),
                           np.float32(dt), np.float32(rho), mat_fluid)
    return out


def dot_f64(x, y):
    x = _c(x, np.float32).ravel()
    y = _c(y, np.float32).ravel()
    return float(lib().or_dot_f32_f64(x, y, x.size))


def axpy(y, x, alpha, negate=False):
    """axpy_device.cu:20-31 (FMA build): returns alpha x + y, alpha negated
    first when ``negate``."""
    out = _c(y, np.float32).copy()
    lib().or_axpy_f32(out, _c(x, np.float32), np.float32(alpha), out.size, 1 if negate else 0)
    return out


def scaled_axpy(z, p_old, beta):
    """axpy_device.cu:51-63 (FMA build): z + beta p_old."""
    z = _c(z, np.float32)
    out = np.empty_like(z)
    lib().or_scaled_axpy_f32(out, z, _c(p_old, np.float32), np.float32(beta), z.size)
    return out


def divide_scalars(num, den):
    """axpy_device.cu:84-91: num / den, 0 when den == 0."""
    return np.float32(lib().or_divide_f32(np.float32(num), np.float32(den)))


def scale(x, s):
    """scale.cu:11-17: x * s."""
    out = _c(x, np.float32).copy()
    lib().or_scale_f32(out, out.size, np.float32(s))
    return out


def pcg(div, mat, dx, dt, rho, tol, max_iter, mat_fluid=MAT_FLUID, mat_air=MAT_AIR):
    """Reference PCG (pressure_solve_pcg.cu:89-243) with FP64 inner products.
    Returns (p, iterations)."""
    mat = _c(mat, np.int32)
    nx, ny, nz = mat.shape
    p = np.empty((nx, ny, nz), np.float32)
    it = lib().or_pcg_f32(p, _c(div, np.float32), mat, nx, ny, nz, np.float32(dx),
                          np.float32(dt), np.float32(rho), mat_fluid, mat_air,
                          np.float32(tol), int(max_iter))
    return p, int(it)


# ---------------------------------------------------------------------------
# FP64 system
# ---------------------------------------------------------------------------

def apply_A_f64(p, mat, mat_fluid=MAT_FLUID, mat_air=MAT_AIR):
    mat = _c(mat, np.int32)
    nx, ny, nz = mat.shape
    out = np.empty((nx, ny, nz), np.float64)
    lib().or_apply_A_f64(out, _c(p, np.float64), mat, nx, ny, nz, mat_fluid, mat_air)
    return out


def rhs_f64(div, mat, dx, dt, rho, mat_fluid=MAT_FLUID):
    mat = _c(mat, np.int32)
    out = np.empty(mat.shape, np.float64)
    lib().or_rhs_f64(out, _c(div, np.float32), mat, mat.size, float(np.float32(dx)),
                     float(np.float32(dt)), float(np.float32(rho)), mat_fluid)
    return out


def solve_f64(div, mat, dx, dt, rho, tol=1e-12, max_iter=100000, mat_fluid=MAT_FLUID,
              mat_air=MAT_AIR):
    """FP64 oracle solve p* of A p = b.  Returns (p*, iterations, rel_residual)."""
    mat = _c(mat, np.int32)
    nx, ny, nz = mat.shape
    b = rhs_f64(div, mat, dx, dt, rho, mat_fluid)
    p = np.empty_like(b)
    rel = ctypes.c_double(0.0)
    it = lib().or_cg_f64(p, b, mat, nx, ny, nz, mat_fluid, mat_air, float(tol), int(max_iter),
                         ctypes.byref(rel))
    return p, int(it), float(rel.value)


def rel_residual(p, div, mat, dx, dt, rho, mat_fluid=MAT_FLUID, mat_air=MAT_AIR):
    """||b - A p||_2 / ||b||_2 in FP64 (dx, dt, rho rounded to f32 first)."""
    mat = _c(mat, np.int32)
    nx, ny, nz = mat.shape
    return float(lib().or_rel_residual_f64(_c(p, np.float32), _c(div, np.float32), mat,
                                           nx, ny, nz, float(np.float32(dx)),
                                           float(np.float32(dt)), float(np.float32(rho)),
                                           mat_fluid, mat_air))


def rel_residual64(p64, div, mat, dx, dt, rho, mat_fluid=MAT_FLUID, mat_air=MAT_AIR):
    """||b - A p||_2 / ||b||_2 in FP64 for an FP64 pressure (non-fluid ignored)."""
    mat = _c(mat, np.int32)
    p = np.where(mat == mat_fluid, np.asarray(p64, np.float64), 0.0)
    b = rhs_f64(div, mat, dx, dt, rho, mat_fluid)
    r = b - apply_A_f64(p, mat, mat_fluid, mat_air)
    bn = float(np.sqrt((b * b).sum()))
    return float(np.sqrt((r * r).sum())) / bn if bn > 0 else 0.0


def rel_error(p, p_star, mat, mat_fluid=MAT_FLUID):
    """||p - p*||_2 / ||p*||_2 over fluid cells."""
    f = np.asarray(mat) == mat_fluid
    d = np.asarray(p, np.float64)[f] - np.asarray(p_star, np.float64)[f]
    den = np.linalg.norm(np.asarray(p_star, np.float64)[f])
    return float(np.linalg.norm(d) / den) if den > 0 else float(np.linalg.norm(d))


# ---------------------------------------------------------------------------
# Known answers (python/tests/test_pressure_cg.py:62-69)
# ---------------------------------------------------------------------------

def analytic_linear_field(shape):
    """p = i + j + k: A p = 0 at interior all-fluid cells."""
    i, j, k = np.indices(shape)
    return (i + j + k).astype(np.float32)


def analytic_quadratic_field(shape):
    """p = i^2: A p = -2 at interior all-fluid cells."""
    i = np.indices(shape)[0]
    return (i * i).astype(np.float32)


# ---------------------------------------------------------------------------
# The reference's own CUDA, compiled from source (oracle/_ref)
# ---------------------------------------------------------------------------

# ---------------------------------------------------------------------------
# Backward-Euler conduction (thermal.py:259-388, 647-658)
# ---------------------------------------------------------------------------

def conduction_sweep(T_dst, T_iter, T_old, mat, props, dx, dt, h_conv_air, T_amb,
                     mat_air=MAT_AIR):
    """One Jacobi sweep; returns a new array (T_dst's contents kept on air cells).
    ``props`` = (k, rho, cp), float32 arrays indexed by material id."""
    out = _c(T_dst, np.float32).copy()
    k, rho, cp = (_c(a, np.float32) for a in props)
    nx, ny, nz = out.shape
    lib().or_conduction_sweep_f32(out, _c(T_iter, np.float32), _c(T_old, np.float32),
                                  _c(mat, np.int32), nx, ny, nz, k, rho, cp, float(dx),
                                  float(dt), float(h_conv_air), float(T_amb), int(mat_air))
    return out


def conduction_be(T, T_alt, mat, props, dx, dt, h_conv_air, T_amb, n_iter, mat_air=MAT_AIR):
    """The backward-Euler conduction step: returns (T, T_alt, T_old) after it."""
    T = _c(T, np.float32).copy()
    T_alt = _c(T_alt, np.float32).copy()
    T_old = np.empty_like(T)
    k, rho, cp = (_c(a, np.float32) for a in props)
    nx, ny, nz = T.shape
    lib().or_conduction_be_f32(T, T_alt, T_old, _c(mat, np.int32), nx, ny, nz, k, rho, cp,
                               float(dx), float(dt), float(h_conv_air), float(T_amb),
                               int(mat_air), int(n_iter))
    return T, T_alt, T_old


# ---------------------------------------------------------------------------
# Semi-Lagrangian advection (fluid.py:39-104, 338-498, 737-776)
# ---------------------------------------------------------------------------

def _org(origin):
    return np.ascontiguousarray(origin, dtype=np.float32).reshape(3)


def extend_temperature(T, mat, mat_fluid=MAT_FLUID):
    T = _c(T, np.float32)
    out = np.empty_like(T)
    nx, ny, nz = T.shape
    lib().or_extend_temperature_f32(out, T, _c(mat, np.int32), nx, ny, nz, int(mat_fluid))
    return out


def advect_temperature(T_true, T_ext, ux, uy, uz, mat, origin, dx, dt, mat_fluid=MAT_FLUID):
    T_true = _c(T_true, np.float32)
    out = np.empty_like(T_true)
    nx, ny, nz = T_true.shape
    lib().or_advect_temperature_f32(out, T_true, _c(T_ext, np.float32), _c(ux, np.float32),
                                    _c(uy, np.float32), _c(uz, np.float32), _c(mat, np.int32),
                                    nx, ny, nz, _org(origin), float(dx), float(dt),
                                    int(mat_fluid))
    return out


def advect_velocity(axis, ux, uy, uz, mat, origin, dx, dt, mat_fluid=MAT_FLUID):
    """advect_ux / advect_uy / advect_uz: returns the new component ``axis``."""
    nx, ny, nz = mat.shape
    src = (ux, uy, uz)[axis]
    out = np.empty(src.shape, np.float32)
    lib().or_advect_velocity_f32(int(axis), out, _c(ux, np.float32), _c(uy, np.float32),
                                 _c(uz, np.float32), _c(mat, np.int32), nx, ny, nz, _org(origin),
                                 float(dx), float(dt), int(mat_fluid))
    return out


def advect_all(ux, uy, uz, T, mat, origin, dx, dt, mat_fluid=MAT_FLUID):
    """advect_all: returns (ux, uy, uz, T, T_ext) after the step."""
    ux, uy, uz, T = (_c(a, np.float32).copy() for a in (ux, uy, uz, T))
    tmp = [np.empty_like(a) for a in (ux, uy, uz, T)]
    T_ext = np.empty_like(T)
    nx, ny, nz = T.shape
    lib().or_advect_all_f32(ux, uy, uz, T, *tmp, T_ext, _c(mat, np.int32), nx, ny, nz,
                            _org(origin), float(dx), float(dt), int(mat_fluid))
    return ux, uy, uz, T, T_ext


def ref_library_path(fma: bool = True) -> str:
    return os.path.join(_HERE, "_ref", "libref_fma.so" if fma else "libref_nofma.so")


def ref_library(fma: bool = True):
    """ctypes handle on the reference's CUDA launchers, or None if not built."""
    path = ref_library_path(fma)
    if not os.path.exists(path):
        return None
    return ctypes.CDLL(path)
