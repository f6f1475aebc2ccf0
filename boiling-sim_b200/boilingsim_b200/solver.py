"""To-tolerance pressure solve (host side of ``bsp_solve_tol``).

Solves the reference's projection system A p = b (pressure_solve_pcg.cu:129-139)
to a relative FP64 residual ``tol`` with FP64 iterative refinement around a
multigrid-preconditioned CG whose inner vectors are stored in FP32, FP16 or
BF16.  The workspace is allocated once per (shape, storage) by the caller-side
cache below and passed to the library, which itself never allocates.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._lib import BspSolveInfo, BspSolveParams, call, ptr, stream_handle

STORAGE = {"fp32": 0, "fp16": 1, "bf16": 2}


@dataclass
class SolveResult:
    p: torch.Tensor            # float32 pressure (0 on non-fluid cells)
    p64_dev: torch.Tensor      # FP64 iterate on the device
    status: int
    outer_iterations: int
    inner_iterations: int
    levels: int
    rel_residual: float        # the device's FP64 relative residual

    @property
    def iterations(self) -> int:
        return self.inner_iterations

    @property
    def p64(self) -> np.ndarray:
        return self.p64_dev.cpu().numpy()


class TolSolver:
    """Reusable solver for one grid shape: owns the workspace and the mask."""

    def __init__(self, mask: torch.Tensor, storage: str = "fp32", device="cuda:0"):
        if mask.dtype != torch.uint8 or not mask.is_cuda:
            raise TypeError("mask must be the uint8 cell mask on the GPU")
        self.mask = mask.contiguous()
        self.shape = tuple(mask.shape)
        self.storage = STORAGE[storage]
        nx, ny, nz = self.shape
        nbytes = int(_lib.lib().bsp_solver_workspace_bytes(nx, ny, nz, self.storage))
        # 256-byte alignment: torch's caching allocator hands out 512-byte aligned blocks
        self.ws = torch.empty(nbytes, dtype=torch.uint8, device=mask.device)
        self.x64 = torch.empty(self.shape, dtype=torch.float64, device=mask.device)
        self.params = BspSolveParams()
        _lib.lib().bsp_solve_params_default(ctypes.byref(self.params))
        self.params.storage = self.storage
        # the mask is fixed for this solver's lifetime: build the multigrid
        # levels on the first solve (never trust a record left by an earlier
        # workspace at the same address), reuse them afterwards
        self.params.reuse_setup = 0
        self._setup_done = False
        self.last: SolveResult | None = None  # result of the latest solve

    def solve(self, div: torch.Tensor, dx: float, dt: float, rho: float, tol: float = 1e-6,
              p: torch.Tensor | None = None, warm_start: bool = False, inner_tol: float | None = None,
              max_outer: int | None = None, max_inner: int | None = None,
              check_every: int | None = None, stream=None, raise_on_fail: bool = True,
              graph: bool = False, wait: bool = True, want_x64: bool = True) -> SolveResult:
        """Solve A p = b for the divergence ``div``.  ``graph=True`` runs the
        whole solve as one device-driven CUDA graph (built on the first call
        with this set of buffers, replayed afterwards).  ``wait=False`` (with
        ``graph``, after the first solve on these buffers) only enqueues the
        graph: p is written when the stream reaches it and the returned
        result carries no iteration counts (status 0, counts -1).
        ``want_x64=False`` skips the copy of the FP64 iterate out of the
        workspace (a device-to-device pass over n doubles); the result's
        ``p64`` is then not this solve's."""
        nx, ny, nz = self.shape
        if p is None:
            p = torch.zeros(self.shape, dtype=torch.float32, device=self.mask.device)
        prm = BspSolveParams.from_buffer_copy(self.params)
        prm.tol = float(tol)
        prm.warm_start = 1 if warm_start else 0
        prm.reuse_setup = 1 if self._setup_done else 0
        prm.use_graph = 1 if graph else 0
        if inner_tol is not None:
            prm.inner_tol = float(inner_tol)
        if max_outer is not None:
            prm.max_outer = int(max_outer)
        if max_inner is not None:
            prm.max_inner = int(max_inner)
        if check_every is not None:
            prm.check_every = int(check_every)
        info = BspSolveInfo()
        enqueue_only = graph and not wait and self._setup_done
        code = _lib.lib().bsp_solve_tol(ptr(p), ptr(div), ptr(self.mask), nx, ny, nz, float(dx),
                                         float(dt), float(rho), ctypes.byref(prm), ptr(self.ws),
                                         self.ws.numel(), ptr(self.x64) if want_x64 else None,
                                         None if enqueue_only else ctypes.byref(info),
                                         stream_handle(stream))
        if code not in (0, 10005) or (raise_on_fail and code != 0):
            _lib.check("bsp_solve_tol", code)
        self._setup_done = True
        if enqueue_only:
            self.last = SolveResult(p, self.x64, code, -1, -1, -1, float("nan"))
        else:
            self.last = SolveResult(p, self.x64, code, info.outer_iterations,
                                    info.inner_iterations, info.levels, info.rel_residual)
        return self.last


    def autotune(self, div: torch.Tensor, dx: float, dt: float, rho: float, tol: float = 1e-6,
                 graph: bool = True, stream=None) -> list[dict]:
        """Time the level-0 tile plane chunk x the one-launch coarse cycle on
        this problem (bsp_autotune_solve) and keep the fastest for later solves.
        Returns one row per candidate."""
        nx, ny, nz = self.shape
        prm = BspSolveParams.from_buffer_copy(self.params)
        prm.tol = float(tol)
        prm.use_graph = 1 if graph else 0
        p = torch.zeros(self.shape, dtype=torch.float32, device=self.mask.device)
        rows = (_lib.BspTuneChoice * 32)()
        n = ctypes.c_int(0)
        _lib.call("bsp_autotune_solve", ptr(p), ptr(div), ptr(self.mask), nx, ny, nz, float(dx),
                  float(dt), float(rho), ctypes.byref(prm), ptr(self.ws), self.ws.numel(),
                  ctypes.cast(rows, ctypes.c_void_p), 32, ctypes.byref(n), stream_handle(stream))
        self._setup_done = False  # the tile geometry may have changed
        return [{"key": r.key, "plane_chunk": r.value & 0xFFFF, "coarse_fused": r.value >> 16,
                 "ms": r.ms, "status": r.status} for r in rows[:min(n.value, 32)]]


class BatchSolver:
    """Many independent pot scenes (uneven sizes) solved by one graph launch
    (``bsp_solve_batch``).  Each instance owns its workspace; the masks are
    fixed for the solver's lifetime."""

    def __init__(self, masks, storage: str = "fp32"):
        self.masks = [m.contiguous() for m in masks]
        self.storage = STORAGE[storage]
        lib = _lib.lib()
        self.ws = []
        for m in self.masks:
            nx, ny, nz = m.shape
            nbytes = int(lib.bsp_solver_workspace_bytes(nx, ny, nz, self.storage))
            self.ws.append(torch.empty(nbytes, dtype=torch.uint8, device=m.device))
        self.params = BspSolveParams()
        lib.bsp_solve_params_default(ctypes.byref(self.params))
        self.params.storage = self.storage
        self.params.use_graph = 1
        self._setup_done = False

    def solve(self, divs, ps, dx, dt, rho, tol: float = 1e-6, wait: bool = True, stream=None):
        """Solve every instance; ``ps`` (float32 tensors) receive the pressures.
        With ``wait`` the call returns one BspSolveInfo per instance."""
        n = len(self.masks)
        items = (_lib.BspBatchItem * n)()
        for q, (m, d, p, w) in enumerate(zip(self.masks, divs, ps, self.ws)):
            nx, ny, nz = m.shape
            items[q] = _lib.BspBatchItem(ptr(p), ptr(d), ptr(m), nx, ny, nz, float(dx),
                                         float(dt), float(rho), ptr(w), w.numel())
        prm = BspSolveParams.from_buffer_copy(self.params)
        prm.tol = float(tol)
        prm.reuse_setup = 1 if self._setup_done else 0
        infos = (BspSolveInfo * n)() if wait else None
        code = _lib.lib().bsp_solve_batch(
            n, ctypes.cast(items, ctypes.c_void_p), ctypes.byref(prm),
            ctypes.cast(infos, ctypes.c_void_p) if wait else None, stream_handle(stream))
        self._items = items  # keep the item array alive until the launch completes
        _lib.check("bsp_solve_batch", code)
        self._setup_done = True
        return list(infos) if wait else None


def solve_tolerance(div, mat, dx, dt, rho, tol=1e-6, storage="fp32", **kw) -> SolveResult:
    """Convenience wrapper on numpy inputs (int32 material ids, float32 div)."""
    from .fluid import cell_mask

    mat_t = torch.as_tensor(np.ascontiguousarray(mat, np.int32)).cuda()
    div_t = torch.as_tensor(np.ascontiguousarray(div, np.float32)).cuda()
    solver = TolSolver(cell_mask(mat_t), storage)
    return solver.solve(div_t, dx, dt, rho, tol=tol, **kw)


def main(argv=None):
    """``python -m boilingsim_b200.solver solve [--storage fp16] [--max-inner N]
    [--graph]``: one tolerance solve on the 384x384x256 benchmark pot
    (synthetic velocities, seed 7); prints iterations, residual and time.
    With a small ``--max-inner`` and host-driven launches it is the small,
    repeatable run the level-0 kernels are profiled on."""
    import argparse
    import json
    import time

    from . import scenes
    from .fluid import cell_mask, compute_divergence

    ap = argparse.ArgumentParser(description="one tolerance solve on the benchmark pot")
    ap.add_argument("cmd", choices=["solve"])
    ap.add_argument("--storage", default="fp16", choices=["fp32", "fp16", "bf16"])
    ap.add_argument("--max-inner", type=int, default=200)
    ap.add_argument("--max-outer", type=int, default=10)
    ap.add_argument("--graph", action="store_true")
    args = ap.parse_args(argv)
    dx = 0.0005
    mat = scenes.pot_mat(scenes.POT_384)
    ux, uy, uz = scenes.velocity_field(mat, seed=7)
    mask = cell_mask(torch.as_tensor(mat).cuda())
    u = [torch.as_tensor(a).cuda() for a in (ux, uy, uz)]
    div = torch.zeros(mat.shape, device="cuda")
    compute_divergence(div, *u, mask, dx)
    s = TolSolver(mask, args.storage)
    p = torch.zeros_like(div)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    r = s.solve(div, dx, 0.01, 997.0, tol=1e-6, p=p, max_outer=args.max_outer,
                max_inner=args.max_inner, graph=args.graph, raise_on_fail=False)
    torch.cuda.synchronize()
    print(json.dumps({"status": r.status, "inner": r.inner_iterations, "outer": r.outer_iterations,
                      "rel_residual": r.rel_residual,
                      "ms_host_clock": round((time.perf_counter() - t0) * 1e3, 3)}))


if __name__ == "__main__":
    main()
