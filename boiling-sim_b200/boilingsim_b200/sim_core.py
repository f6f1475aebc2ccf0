"""``SimCore`` -- mirror of the reference's PyO3 class ``sim_core.cuda.SimCore``
(``crates/sim-core/src/cuda.rs:17-412``) for the projection methods.

Arguments are raw device addresses (``u64``), as the reference passes them
(``python/boilingsim/fluid.py:649-688``).  Sizes are checked to fit in i32
(``crates/cuda-kernels/src/lib.rs:250-252``) and a non-zero status raises
``RuntimeError`` (``lib.rs:267-269``, ``cuda.rs:123``).
"""
from __future__ import annotations

import ctypes

import torch

from ._lib import call

_I32_MAX = 2**31 - 1
_PCG_WS: dict = {"key": None, "buffers": None}


def _check_i32(*vals):
    for v in vals:
        if v < 0 or v > _I32_MAX:
            raise RuntimeError(f"size {v} does not fit in i32")


class SimCore:
    def __init__(self, device_id: int = 0):
        if not torch.cuda.is_available():
            raise RuntimeError("no CUDA device: the projection library has no CPU path")
        self.device_id = int(device_id)
        torch.cuda.set_device(self.device_id)

    def device_info(self) -> str:
        p = torch.cuda.get_device_properties(self.device_id)
        return f"{p.name} (sm_{p.major}{p.minor}, {p.multi_processor_count} SMs)"

    def scale_array(self, device_ptr: int, n: int, scale: float) -> None:
        _check_i32(n)
        call("scale_inplace_launch", device_ptr, n, float(scale))

    def jacobi_pressure_step(self, p_new_ptr, p_old_ptr, div_u_ptr, mat_ptr, nx, ny, nz, dx,
                             dt, rho, mat_fluid=0, mat_air=2) -> None:
        _check_i32(nx, ny, nz, nx * ny * nz)
        call("jacobi_pressure_launch", p_new_ptr, p_old_ptr, div_u_ptr, mat_ptr, nx, ny, nz,
             float(dx), float(dt), float(rho), mat_fluid, mat_air)

    def pressure_solve(self, p_ptr, p_tmp_ptr, div_u_ptr, mat_ptr, nx, ny, nz, dx, dt, rho,
                       n_iter, mat_fluid=0, mat_air=2) -> None:
        _check_i32(nx, ny, nz, nx * ny * nz, n_iter)
        call("pressure_solve_launch", p_ptr, p_tmp_ptr, div_u_ptr, mat_ptr, nx, ny, nz,
             float(dx), float(dt), float(rho), n_iter, mat_fluid, mat_air)

    def pressure_solve_pcg(self, p_out_ptr, div_u_ptr, mat_ptr, nx, ny, nz, dx, dt, rho,
                           pressure_tol, max_iter, ws_b_ptr, ws_r_ptr, ws_z_ptr,
                           ws_p_search_ptr, ws_ap_ptr, dot_workspace_ptr, dev_alpha_ptr,
                           dev_beta_ptr, dev_rzold_ptr, dev_rznew_ptr, dev_bsq_ptr,
                           dev_rsq_ptr, dev_pap_ptr, mat_fluid=0, mat_air=2) -> int:
        _check_i32(nx, ny, nz, nx * ny * nz, max_iter)
        it = ctypes.c_int(0)
        call("pressure_solve_pcg_launch", p_out_ptr, div_u_ptr, mat_ptr, nx, ny, nz, float(dx),
             float(dt), float(rho), mat_fluid, mat_air, float(pressure_tol), int(max_iter),
             ws_b_ptr, ws_r_ptr, ws_z_ptr, ws_p_search_ptr, ws_ap_ptr, dot_workspace_ptr,
             dev_alpha_ptr, dev_beta_ptr, dev_rzold_ptr, dev_rznew_ptr, dev_bsq_ptr,
             dev_rsq_ptr, dev_pap_ptr, ctypes.byref(it))
        return int(it.value)

    def __repr__(self) -> str:
        return f"SimCore(device_id={self.device_id})"


def pcg_workspace(shape, device) -> dict:
    """Cached PCG workspace (``fluid.py:554-582``): 5 field vectors, a 1024-float
    dot workspace and 7 device scalars, rebuilt on shape change."""
    key = (tuple(shape), str(device))
    if _PCG_WS["key"] == key:
        return _PCG_WS["buffers"]
    z = lambda *s: torch.zeros(s, dtype=torch.float32, device=device)  # noqa: E731
    bufs = {k: z(*shape) for k in ("b", "r", "z", "p_search", "Ap")}
    bufs["dot_ws"] = z(1024)
    for k in ("alpha", "beta", "rzold", "rznew", "bsq", "rsq", "pAp"):
        bufs[k] = z(1)
    _PCG_WS.update(key=key, buffers=bufs)
    return bufs
