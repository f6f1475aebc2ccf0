"""Pressure projection on the MAC grid -- host-side mirror of the reference API.

Drop-in for ``python/boilingsim/fluid.py`` (the projection part): the same
function names, arguments and results, backed by the sm_100a kernels of
libbsproj.so instead of Warp.  Fields are torch CUDA tensors (or any object
with ``__cuda_array_interface__`` of the right dtype and layout):

* ``Grid``:  p (nx,ny,nz) f32, mat (nx,ny,nz) int32, ux (nx+1,ny,nz),
  uy (nx,ny+1,nz), uz (nx,ny,nz+1) f32 -- ``geometry.py:253-314``;
* ``FluidWorkspace``: div_u, p_tmp (nx,ny,nz) f32 -- ``fluid.py:500-528``.

Solver selection follows ``_select_pressure_solver`` (``fluid.py:585-609``):
``BOILINGSIM_PRESSURE_SOLVER`` = ``jacobi`` (default; fixed
``pressure_max_iter`` sweeps), ``cg-rust`` (Jacobi-preconditioned CG to
``pressure_tol``), ``b200-jacobi`` (the uint8-mask sweep path), and
``BOILINGSIM_USE_RUST_PRESSURE=1`` selects the fused fixed-count Jacobi
launcher; ``b200-mg`` / ``b200-mixed`` / ``b200-bf16`` are the to-tolerance
solver with FP32 / FP16 / BF16 iterate storage, and ``b200-learned`` starts
the FP16 solve from the learned warm start (learned.py).  Every back-end runs
on the GPU; there is no CPU path.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field

import torch

from . import _lib
from ._lib import call, ptr, stream_handle

MAT_FLUID, MAT_POT_WALL, MAT_AIR, MAT_CARROT = 0, 1, 2, 3


@dataclass
class SolverConfig:
    """The projection knobs of ``config.py:161-182``."""

    pressure_tol: float = 1e-5
    pressure_max_iter: int = 200
    # B200 extension, to-tolerance back-ends only: start each solve from the
    # previous time step's pressure instead of zero (the reference always
    # zeroes p, fluid.py:628-629).
    pressure_warm_start: bool = False


@dataclass
class ScenarioConfig:
    """The part of ``ScenarioConfig`` (``config.py:808``) the projection reads."""

    solver: SolverConfig = field(default_factory=SolverConfig)


@dataclass
class Grid:
    nx: int
    ny: int
    nz: int
    dx: float
    p: torch.Tensor
    mat: torch.Tensor
    ux: torch.Tensor
    uy: torch.Tensor
    uz: torch.Tensor
    mask: torch.Tensor | None = None  # uint8 cell classes, derived once from mat
    T: torch.Tensor | None = None      # (nx, ny, nz) f32 cell temperature (advection)
    origin: tuple = (0.0, 0.0, 0.0)    # world position of the grid corner (advection)

    @property
    def shape(self):
        return (self.nx, self.ny, self.nz)

    @classmethod
    def from_numpy(cls, mat, ux, uy, uz, dx, device="cuda:0"):
        nx, ny, nz = mat.shape
        t = lambda a, dt: torch.as_tensor(a, dtype=dt).contiguous().to(device)  # noqa: E731
        return cls(nx, ny, nz, float(dx), torch.zeros((nx, ny, nz), dtype=torch.float32,
                                                      device=device),
                   t(mat, torch.int32), t(ux, torch.float32), t(uy, torch.float32),
                   t(uz, torch.float32))


@dataclass
class FluidWorkspace:
    div_u: torch.Tensor
    p_tmp: torch.Tensor
    max_div: torch.Tensor  # (1,) device float: max|div| of the last projection
    # semi-Lagrangian advection buffers (fluid.py:500-528); allocated on first use
    ux_tmp: torch.Tensor | None = None
    uy_tmp: torch.Tensor | None = None
    uz_tmp: torch.Tensor | None = None
    T_tmp: torch.Tensor | None = None
    T_ext: torch.Tensor | None = None


def allocate_fluid_workspace(grid: Grid, device: str = "cuda:0") -> FluidWorkspace:
    shp = grid.shape
    return FluidWorkspace(torch.zeros(shp, dtype=torch.float32, device=device),
                          torch.zeros(shp, dtype=torch.float32, device=device),
                          torch.zeros(1, dtype=torch.float32, device=device))


def _advection_buffers(grid: Grid, ws: FluidWorkspace) -> None:
    nx, ny, nz = grid.shape
    dev = grid.mat.device
    z = lambda *shp: torch.zeros(shp, dtype=torch.float32, device=dev)  # noqa: E731
    if ws.ux_tmp is None:
        ws.ux_tmp, ws.uy_tmp, ws.uz_tmp = z(nx + 1, ny, nz), z(nx, ny + 1, nz), z(nx, ny, nz + 1)
    if ws.T_tmp is None:
        ws.T_tmp, ws.T_ext = z(nx, ny, nz), z(nx, ny, nz)


def cell_mask(mat: torch.Tensor, mat_fluid: int = MAT_FLUID, mat_air: int = MAT_AIR,
              stream=None) -> torch.Tensor:
    """uint8 cell mask of an int32 material grid: bit 7 fluid, bit 6 solid
    (air: neither), bits 0-2 the number of solid face neighbours."""
    if mat.dtype != torch.int32 or not mat.is_contiguous():
        raise TypeError("mat must be a contiguous int32 CUDA tensor")
    out = torch.empty(mat.shape, dtype=torch.uint8, device=mat.device)
    nx, ny, nz = mat.shape
    call("bsp_mask_from_mat", ptr(out), ptr(mat), nx, ny, nz, mat_fluid, mat_air,
         stream_handle(stream))
    return out


def grid_mask(grid: Grid) -> torch.Tensor:
    if grid.mask is None:
        grid.mask = cell_mask(grid.mat)
    return grid.mask


_TOL_SOLVERS: dict = {}


def _tol_solver(grid: Grid, storage: str):
    """Per (grid, storage) cached solver: the workspace is allocated once."""
    from .solver import TolSolver

    key = (id(grid), grid.shape, storage)
    if key not in _TOL_SOLVERS:
        _TOL_SOLVERS.clear()
        _TOL_SOLVERS[key] = TolSolver(grid_mask(grid), storage)
    return _TOL_SOLVERS[key]


def _select_pressure_solver() -> str:
    """``fluid.py:585-609`` with the B200 back-ends added."""
    use_rust_jacobi = os.environ.get("BOILINGSIM_USE_RUST_PRESSURE") == "1"
    solver = os.environ.get("BOILINGSIM_PRESSURE_SOLVER", "jacobi").lower()
    valid = ("jacobi", "cg-rust", "b200-jacobi", "b200-mg", "b200-mixed", "b200-bf16",
             "b200-learned")
    if solver not in valid:
        raise ValueError(f"BOILINGSIM_PRESSURE_SOLVER={solver!r} is not recognised; "
                         f"valid values are {', '.join(repr(v) for v in valid)}.")
    if use_rust_jacobi and solver == "cg-rust":
        raise ValueError("BOILINGSIM_USE_RUST_PRESSURE=1 and BOILINGSIM_PRESSURE_SOLVER=cg-rust "
                         "are mutually exclusive -- they route through different code paths.")
    if solver == "cg-rust":
        return "cg-rust"
    if use_rust_jacobi:
        return "rust-jacobi"
    return solver


# ---------------------------------------------------------------------------
# kernel-level calls (Warp kernel signatures of fluid.py, launched on torch's
# current stream)
# ---------------------------------------------------------------------------

def compute_divergence(div_u, ux, uy, uz, mask, dx, max_abs_div=None, stream=None):
    nx, ny, nz = div_u.shape
    call("bsp_divergence", ptr(div_u), ptr(ux), ptr(uy), ptr(uz), ptr(mask), nx, ny, nz,
         float(dx), ptr(max_abs_div), stream_handle(stream))


def jacobi_pressure_step(p_new, p_old, div_u, mat, dx, dt, rho, mat_fluid=MAT_FLUID,
                         mat_air=MAT_AIR, stream=None):
    """One sweep.  ``mat`` may be the int32 material grid (reference layout) or
    the uint8 class mask."""
    nx, ny, nz = p_new.shape
    if mat.dtype == torch.uint8:
        call("bsp_jacobi_sweep", ptr(p_new), ptr(p_old), ptr(div_u), ptr(mat), nx, ny, nz,
             float(dx), float(dt), float(rho), stream_handle(stream))
    else:
        # reference launcher: legacy default stream, as jacobi_pressure.cu:203
        call("jacobi_pressure_launch", ptr(p_new), ptr(p_old), ptr(div_u), ptr(mat), nx, ny,
             nz, float(dx), float(dt), float(rho), mat_fluid, mat_air)


def subtract_pressure_gradient(ux, uy, uz, p, mask, dx, dt, rho, stream=None):
    nx, ny, nz = p.shape
    call("bsp_subtract_gradient", ptr(ux), ptr(uy), ptr(uz), ptr(p), ptr(mask), nx, ny, nz,
         float(dx), float(dt), float(rho), stream_handle(stream))


def enforce_no_slip(grid: Grid, device: str = "cuda:0", stream=None) -> None:
    """``fluid.py:154-165``."""
    call("bsp_enforce_no_slip", ptr(grid.ux), ptr(grid.uy), ptr(grid.uz), ptr(grid_mask(grid)),
         grid.nx, grid.ny, grid.nz, stream_handle(stream))


# ---------------------------------------------------------------------------
# the projection (fluid.py:612-734)
# ---------------------------------------------------------------------------

def pressure_projection(grid: Grid, ws: FluidWorkspace, cfg: ScenarioConfig, dt: float,
                        rho: float, device: str = "cuda:0") -> float:
    """Enforce incompressibility: solve the pressure Poisson problem, correct u.

    Returns max |div u| after the correction (a diagnostic), as the reference.
    The reference reads the whole divergence field back to the host for this
    (fluid.py:733-734); here it is reduced on the device and 4 bytes are read.
    """
    nx, ny, nz = grid.shape
    dx = float(grid.dx)
    mask = grid_mask(grid)
    s = stream_handle()
    solver = _select_pressure_solver()
    n_iter = int(cfg.solver.pressure_max_iter)
    if solver in ("jacobi", "b200-jacobi"):
        call("bsp_projection_jacobi", ptr(grid.p), ptr(ws.p_tmp), ptr(ws.div_u), ptr(grid.ux),
             ptr(grid.uy), ptr(grid.uz), ptr(mask), nx, ny, nz, dx, float(dt), float(rho),
             n_iter, 0, ptr(ws.max_div), s)
    elif solver.startswith("b200-"):
        compute_divergence(ws.div_u, grid.ux, grid.uy, grid.uz, mask, dx)
        _tol_projection(grid, ws, cfg, solver, dt, rho)
    else:
        grid.p.zero_()
        ws.p_tmp.zero_()
        compute_divergence(ws.div_u, grid.ux, grid.uy, grid.uz, mask, dx)
        # the reference launchers run on the legacy default stream
        torch.cuda.current_stream().synchronize()
        if solver == "rust-jacobi":
            call("pressure_solve_launch", ptr(grid.p), ptr(ws.p_tmp), ptr(ws.div_u),
                 ptr(grid.mat), nx, ny, nz, dx, float(dt), float(rho), n_iter, MAT_FLUID,
                 MAT_AIR)
        else:
            from .sim_core import pcg_workspace, SimCore
            w = pcg_workspace(grid.shape, grid.p.device)
            SimCore(0).pressure_solve_pcg(
                ptr(grid.p), ptr(ws.div_u), ptr(grid.mat), nx, ny, nz, dx, float(dt),
                float(rho), float(cfg.solver.pressure_tol), n_iter, *[ptr(w[k]) for k in (
                    "b", "r", "z", "p_search", "Ap", "dot_ws", "alpha", "beta", "rzold",
                    "rznew", "bsq", "rsq", "pAp")], MAT_FLUID, MAT_AIR)
        torch.cuda.synchronize()
        subtract_pressure_gradient(grid.ux, grid.uy, grid.uz, grid.p, mask, dx, dt, rho)
        compute_divergence(ws.div_u, grid.ux, grid.uy, grid.uz, mask, dx, ws.max_div)
    return float(ws.max_div.item())


_STORAGE = {"b200-mg": "fp32", "b200-mixed": "fp16", "b200-bf16": "bf16",
            "b200-learned": "fp16"}


def _tol_projection(grid: Grid, ws: FluidWorkspace, cfg: ScenarioConfig, solver: str,
                    dt: float, rho: float, tol_solver=None, warm_start=None,
                    wait: bool = True, want_x64: bool = True) -> None:
    """Solve, gradient and diagnostic divergence of the to-tolerance back-ends
    (multigrid-preconditioned CG inside FP64 refinement, stopping at
    ||b - A p|| <= pressure_tol ||b|| in FP64); ws.div_u holds the divergence.
    tol_solver / warm_start: the caller's own objects (else the per-grid
    caches).  wait=False: the solve is only enqueued (no host synchronisation
    once its graph exists); want_x64=False: the solver's FP64 iterate is not
    copied out (its ``last.p64`` is then stale)."""
    mask = grid_mask(grid)
    dx = float(grid.dx)
    if tol_solver is None:
        tol_solver = _tol_solver(grid, _STORAGE[solver])
    warm = bool(cfg.solver.pressure_warm_start)
    if solver == "b200-learned" and all(d % 8 == 0 for d in grid.shape):
        # the network's pressure is the starting guess; the solve finishes it
        # to the same tolerance (grids not divisible by 8 start from zero)
        (warm_start or _warm_start(grid, mask)).guess(ws.div_u, dx, dt, rho, out=grid.p)
        warm = True
    tol_solver.solve(ws.div_u, dx, dt, rho, tol=float(cfg.solver.pressure_tol), p=grid.p,
                     warm_start=warm, raise_on_fail=False, graph=True, wait=wait,
                     want_x64=want_x64)
    subtract_pressure_gradient(grid.ux, grid.uy, grid.uz, grid.p, mask, dx, dt, rho)
    compute_divergence(ws.div_u, grid.ux, grid.uy, grid.uz, mask, dx, ws.max_div)


class ProjectionPipeline:
    """Independent pressure projections of one geometry with host velocity
    buffers, ``depth`` of them in flight.

    Each slot owns its device fields, workspace, solver, learned warm start
    (with its own network buffers) and CUDA stream.  ``submit`` enqueues on
    the slot's stream the host->device copy of the velocities (pinned host
    tensors), the projection (``pressure_projection``'s operations: the
    divergence, the solve to ``pressure_tol``, the gradient subtraction and
    the diagnostic divergence) and the device->host copies of the corrected
    velocities, the pressure and max |div u|, and returns a ticket at once;
    ``result`` waits for that projection and returns its max |div u|.  The
    copy engines then move one projection's fields while another computes.
    The host buffers given to ``submit`` must stay untouched until its
    ``result`` is taken.  Back-ends: the to-tolerance ones (``b200-mg``,
    ``b200-mixed``, ``b200-bf16``, ``b200-learned``) and ``b200-jacobi``,
    chosen as ``pressure_projection`` chooses (BOILINGSIM_PRESSURE_SOLVER)."""

    def __init__(self, mat: torch.Tensor, dx: float, cfg: ScenarioConfig, depth: int = 2):
        from .solver import TolSolver

        if mat.dtype != torch.int32 or not mat.is_cuda:
            raise TypeError("mat must be an int32 CUDA tensor")
        if depth < 1:
            raise ValueError("depth must be >= 1")
        self.solver = _select_pressure_solver()
        if self.solver not in ("b200-jacobi", "jacobi") and self.solver not in _STORAGE:
            raise ValueError(f"{self.solver!r} launches on the legacy default stream; "
                             "ProjectionPipeline needs a stream-ordered back-end")
        self.cfg = cfg
        self.dx = float(dx)
        nx, ny, nz = mat.shape
        dev = mat.device
        mask = cell_mask(mat)
        z = lambda *shp: torch.zeros(shp, dtype=torch.float32, device=dev)  # noqa: E731
        self.slots = []
        for _ in range(depth):
            grid = Grid(nx, ny, nz, self.dx, z(nx, ny, nz), mat, z(nx + 1, ny, nz),
                        z(nx, ny + 1, nz), z(nx, ny, nz + 1), mask=mask)
            ws = FluidWorkspace(z(nx, ny, nz), z(nx, ny, nz), z(1))
            slot = {"grid": grid, "ws": ws, "stream": torch.cuda.Stream(device=dev),
                    "done": None, "max_div": torch.zeros(1, dtype=torch.float32).pin_memory(),
                    "tol": None, "warm": None}
            if self.solver in _STORAGE:
                slot["tol"] = TolSolver(mask, _STORAGE[self.solver], device=dev)
                if self.solver == "b200-learned" and all(d % 8 == 0 for d in grid.shape):
                    from .learned import UNet, WarmStart

                    slot["warm"] = WarmStart(UNet.load(device=dev), mat, mask)
            self.slots.append(slot)
        # the mask, weights and buffers above were made on the current stream;
        # the slots' streams start after them
        torch.cuda.synchronize(dev)
        self.issued = 0

    def submit(self, ux_h, uy_h, uz_h, ux_out, uy_out, uz_out, p_out, dt: float,
               rho: float) -> int:
        slot = self.slots[self.issued % len(self.slots)]
        if slot["done"] is not None:
            slot["done"].synchronize()  # the slot's previous projection has left the device
        grid, ws = slot["grid"], slot["ws"]
        with torch.cuda.stream(slot["stream"]):
            for d, h in zip((grid.ux, grid.uy, grid.uz), (ux_h, uy_h, uz_h)):
                d.copy_(h, non_blocking=True)
            if self.solver in ("b200-jacobi", "jacobi"):
                nx, ny, nz = grid.shape
                call("bsp_projection_jacobi", ptr(grid.p), ptr(ws.p_tmp), ptr(ws.div_u),
                     ptr(grid.ux), ptr(grid.uy), ptr(grid.uz), ptr(grid.mask), nx, ny, nz,
                     self.dx, float(dt), float(rho), int(self.cfg.solver.pressure_max_iter), 0,
                     ptr(ws.max_div), stream_handle())
            else:
                compute_divergence(ws.div_u, grid.ux, grid.uy, grid.uz, grid.mask, self.dx)
                _tol_projection(grid, ws, self.cfg, self.solver, dt, rho,
                                tol_solver=slot["tol"], warm_start=slot["warm"], wait=False,
                                want_x64=False)
            p_out.copy_(grid.p, non_blocking=True)
            for h, d in zip((ux_out, uy_out, uz_out), (grid.ux, grid.uy, grid.uz)):
                h.copy_(d, non_blocking=True)
            slot["max_div"].copy_(ws.max_div, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record()
        slot["done"] = ev
        slot["ticket"] = self.issued
        self.issued += 1
        return self.issued - 1

    def result(self, ticket: int) -> float:
        slot = self.slots[ticket % len(self.slots)]
        if slot.get("ticket") != ticket:
            raise ValueError("that projection's slot has been reused; take results in order")
        slot["done"].synchronize()
        return float(slot["max_div"].item())


_NET = None
_WARM_STARTS: dict = {}


def _warm_start(grid: Grid, mask: torch.Tensor):
    """The learned warm start of this grid (network resolution chosen by the
    grid size, boilingsim_b200.learned.WarmStart), built once per grid."""
    key = (id(grid), grid.shape)
    if key not in _WARM_STARTS:
        from .learned import WarmStart

        _WARM_STARTS[key] = WarmStart(_learned_net(), grid.mat, mask)
    return _WARM_STARTS[key]


def _learned_net():
    """The trained warm-start network (boilingsim_b200/data/unet_warmstart.npz)."""
    global _NET
    if _NET is None:
        from .learned import UNet

        _NET = UNet.load()
    return _NET


def autotune_jacobi(grid: Grid, ws: FluidWorkspace, dt: float, rho: float, sweeps: int = 20,
                    stream=None) -> list[dict]:
    """Time the sweep plane chunk x sweeps per HBM pass on this grid
    (bsp_autotune_jacobi, on the workspace's buffers) and keep the fastest for
    later Jacobi solves.  Returns one row per candidate (ms per sweep)."""
    import ctypes

    nx, ny, nz = grid.shape
    mask = grid_mask(grid)
    compute_divergence(ws.div_u, grid.ux, grid.uy, grid.uz, mask, grid.dx)
    rhs = torch.empty_like(ws.div_u)
    p = torch.empty_like(ws.div_u)
    rows = (_lib.BspTuneChoice * 32)()
    n = ctypes.c_int(0)
    call("bsp_autotune_jacobi", ptr(p), ptr(ws.p_tmp), ptr(ws.div_u), ptr(rhs), ptr(mask), nx, ny,
         nz, float(grid.dx), float(dt), float(rho), int(sweeps),
         ctypes.cast(rows, ctypes.c_void_p), 32, ctypes.byref(n), stream_handle(stream))
    return [{"plane_chunk": r.value & 0xFFFF, "sweeps_per_pass": r.value >> 16,
             "ms_per_sweep": r.ms, "status": r.status} for r in rows[:min(n.value, 32)]]


def noslip_divergence(div_u, ux, uy, uz, mask, dx, stream=None):
    """``enforce_no_slip`` then ``compute_divergence`` in one pass (bit-identical)."""
    nx, ny, nz = div_u.shape
    call("bsp_noslip_divergence", ptr(div_u), ptr(ux), ptr(uy), ptr(uz), ptr(mask), nx, ny, nz,
         float(dx), stream_handle(stream))


def projection_step(grid: Grid, ws: FluidWorkspace, cfg: ScenarioConfig, dt: float,
                    rho: float, device: str = "cuda:0") -> float:
    """Steps 5-7 of a time step (``pipeline.py:605-619``): no-slip, pressure
    projection, no-slip; returns the projection's max |div u|.

    On the B200 back-ends the first no-slip is fused into the divergence pass
    and the second is skipped: the gradient subtract writes only faces between
    two fluid cells, which no-slip leaves alone, so it would change nothing.
    The reference launchers (``rust-jacobi``, ``cg-rust``) run the three calls
    as written.  The result equals the reference sequence bit for bit on the
    Jacobi back-ends.
    """
    nx, ny, nz = grid.shape
    dx = float(grid.dx)
    mask = grid_mask(grid)
    solver = _select_pressure_solver()
    if solver in ("jacobi", "b200-jacobi"):
        call("bsp_step_projection_jacobi", ptr(grid.p), ptr(ws.p_tmp), ptr(ws.div_u),
             ptr(grid.ux), ptr(grid.uy), ptr(grid.uz), ptr(mask), nx, ny, nz, dx, float(dt),
             float(rho), int(cfg.solver.pressure_max_iter), 0, ptr(ws.max_div), stream_handle())
        return float(ws.max_div.item())
    if solver.startswith("b200-"):
        noslip_divergence(ws.div_u, grid.ux, grid.uy, grid.uz, mask, dx)
        _tol_projection(grid, ws, cfg, solver, dt, rho)
        return float(ws.max_div.item())
    enforce_no_slip(grid, device)
    out = pressure_projection(grid, ws, cfg, dt, rho, device)
    enforce_no_slip(grid, device)
    return out


# ---------------------------------------------------------------------------
# Semi-Lagrangian advection (fluid.py:338-498, 737-776)
# ---------------------------------------------------------------------------

def extend_temperature_into_solids(T_ext, T, mask, stream=None) -> None:
    """fluid.py:338-382 on the uint8 cell mask (``cell_mask``)."""
    nx, ny, nz = T.shape
    call("bsp_extend_temperature", ptr(T_ext), ptr(T), ptr(mask), nx, ny, nz,
         stream_handle(stream))


def advect_temperature(T_new, T_true, T_ext, ux, uy, uz, mask, origin, dx, dt,
                       stream=None) -> None:
    """fluid.py:385-411."""
    nx, ny, nz = T_true.shape
    call("bsp_advect_temperature", ptr(T_new), ptr(T_true), ptr(T_ext), ptr(ux), ptr(uy),
         ptr(uz), ptr(mask), nx, ny, nz, *(float(o) for o in origin), float(dx), float(dt),
         stream_handle(stream))


def advect_velocity(axis: int, u_new, ux, uy, uz, mask, origin, dx, dt, stream=None) -> None:
    """advect_ux / advect_uy / advect_uz (fluid.py:414-498) for axis 0 / 1 / 2."""
    nx, ny, nz = mask.shape
    call("bsp_advect_velocity", int(axis), ptr(u_new), ptr(ux), ptr(uy), ptr(uz), ptr(mask),
         nx, ny, nz, *(float(o) for o in origin), float(dx), float(dt), stream_handle(stream))


def advect_all(grid: Grid, ws: FluidWorkspace, dt: float, device: str = "cuda:0",
               stream=None) -> None:
    """``advect_all`` (fluid.py:737-776): semi-Lagrangian advection of ux, uy,
    uz and T from the old fields into the workspace, then copied back into
    the grid -- bit-identical to the reference arithmetic."""
    del device
    if grid.T is None:
        raise ValueError("advect_all needs grid.T")
    _advection_buffers(grid, ws)
    nx, ny, nz = grid.shape
    call("bsp_advect_all", ptr(grid.ux), ptr(grid.uy), ptr(grid.uz), ptr(grid.T),
         ptr(ws.ux_tmp), ptr(ws.uy_tmp), ptr(ws.uz_tmp), ptr(ws.T_tmp), ptr(ws.T_ext),
         ptr(grid_mask(grid)), nx, ny, nz, *(float(o) for o in grid.origin), float(grid.dx),
         float(dt), 1, stream_handle(stream))


def main(argv=None):
    """``python -m boilingsim_b200.fluid sweeps --dims NX NY NZ --tblock T --sweeps N``:
    N Jacobi sweeps of the reference contract (bsp_jacobi_solve, T sweeps per
    HBM pass) on a synthetic pot of the given size, timed with CUDA events
    after one untimed solve; prints ms per sweep and the effective bandwidth
    at 13 bytes per cell per sweep."""
    import argparse
    import json

    import numpy as np

    from . import scenes

    ap = argparse.ArgumentParser(description="time the Jacobi sweep kernels")
    ap.add_argument("cmd", choices=["sweeps"])
    ap.add_argument("--dims", type=int, nargs=3, default=[256, 256, 192])
    ap.add_argument("--tblock", type=int, default=1, choices=[1, 2])
    ap.add_argument("--sweeps", type=int, default=40)
    ap.add_argument("--reps", type=int, default=3)
    args = ap.parse_args(argv)
    nx, ny, nz = args.dims
    spec = scenes.PotSpec(nx, ny, nz, r_in=nx / 2 - 6, t_w=3, water_line=int(0.55 * nz),
                          carrot_r=max(3, nx // 12), carrot_len=nx // 2)
    mat = scenes.pot_mat(spec)
    ux, uy, uz = scenes.velocity_field(mat, seed=7)
    dev = torch.device("cuda", 0)
    mask = cell_mask(torch.as_tensor(mat).to(dev))
    u = [torch.as_tensor(a).to(dev) for a in (ux, uy, uz)]
    dx, dt, rho = 0.002, 0.01, 997.0
    div = torch.zeros(mat.shape, device=dev)
    compute_divergence(div, *u, mask, dx)
    p, q, rhs = (torch.zeros_like(div) for _ in range(3))
    st = stream_handle()

    def solve():
        p.zero_()
        call("bsp_jacobi_solve", ptr(p), ptr(q), ptr(div), ptr(rhs), ptr(mask), nx, ny, nz,
             dx, dt, rho, args.sweeps, args.tblock, st)

    solve()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ms = []
    for _ in range(args.reps):
        e0.record()
        solve()
        e1.record()
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1) / args.sweeps)
    best = float(np.min(ms))
    n = nx * ny * nz
    print(json.dumps({"dims": [nx, ny, nz], "tblock": args.tblock, "sweeps": args.sweeps,
                      "ms_per_sweep": round(best, 5),
                      "effective_GBs": round(13.0 * n / (best * 1e-3) / 1e9, 1)}))


if __name__ == "__main__":
    main()
