"""Failure paths of the solvers, tested without faulting, trapping or hanging
the GPU.

* A right-hand side with NaN or inf: the to-tolerance solve and the
  reference-compatible PCG return BSP_ERR_NONFINITE (the reference guards only
  ||b|| == 0, pressure_solve_pcg.cu:151-155), and the next call on good input
  succeeds.
* A closed Neumann island (fluid sealed by solid, no air contact): the system
  is singular there; the solves return a defined status within their
  iteration caps.
* Bounded device waits: a grid barrier that one block never reaches and an
  mbarrier nothing arrives at give up with BSP_ERR_TIMEOUT (selftest), and a
  solve whose coarse-cycle barrier reports a timeout returns BSP_ERR_TIMEOUT
  while the next solve on the same workspace succeeds (the barrier's control
  words are cleared by every solve).
"""
from __future__ import annotations

import time

import numpy as np
import pytest
import torch

import oracle as O
from boilingsim_b200 import _lib, scenes as S
from boilingsim_b200._lib import BspError, call, ptr
from boilingsim_b200.fluid import cell_mask
from boilingsim_b200.sim_core import SimCore
from boilingsim_b200.solver import TolSolver

pytestmark = pytest.mark.gpu

DX, DT, RHO = 0.002, 0.01, 997.0
NONFINITE, NOT_CONVERGED, TIMEOUT = 10006, 10005, 10007
BSP_TUNE_TEST_BARRIER_ERROR = 11
BSP_TUNE_COARSE_CLUSTER = 24


def _pot(spec=S.POT_64, seed=7):
    mat = S.pot_mat(spec)
    ux, uy, uz = S.velocity_field(mat, seed=seed)
    return mat, O.divergence(ux, uy, uz, mat, DX)


def _pcg(mat, div, tol=1e-6, max_iter=200):
    shape = mat.shape
    z = lambda *s: torch.zeros(s, dtype=torch.float32, device="cuda")  # noqa: E731
    ws = [z(*shape) for _ in range(5)] + [z(1024)] + [z(1) for _ in range(7)]
    p = torch.zeros(shape, device="cuda")
    # named tensors: a temporary freed after ptr() could hand its memory to the
    # next argument's allocation before the kernel reads it
    div_d, mat_d = torch.as_tensor(div).cuda(), torch.as_tensor(mat).cuda()
    it = SimCore(0).pressure_solve_pcg(ptr(p), ptr(div_d), ptr(mat_d), *shape, DX, DT, RHO,
                                       tol, max_iter, *[ptr(w) for w in ws])
    return it, p


@pytest.mark.parametrize("bad", [np.nan, np.inf, -np.inf])
@pytest.mark.parametrize("graph", [False, True])
def test_nonfinite_rhs_tolerance_solve(cuda, bad, graph):
    mat, div = _pot()
    fl = np.argwhere(mat == 0)
    d = div.copy()
    d[tuple(fl[len(fl) // 2])] = bad
    solver = TolSolver(cell_mask(torch.as_tensor(mat).cuda()), "fp16")
    with pytest.raises(BspError) as e:
        solver.solve(torch.as_tensor(d).cuda(), DX, DT, RHO, tol=1e-6, graph=graph)
    assert e.value.code == NONFINITE
    res = solver.solve(torch.as_tensor(div).cuda(), DX, DT, RHO, tol=1e-6, graph=graph)
    assert res.status == 0
    assert O.rel_residual64(res.p64, div, mat, DX, DT, RHO) <= 1.0001e-6


@pytest.mark.parametrize("bad", [np.nan, np.inf])
def test_nonfinite_rhs_reference_pcg(cuda, bad):
    mat, div = _pot()
    fl = np.argwhere(mat == 0)
    d = div.copy()
    d[tuple(fl[0])] = bad
    with pytest.raises(BspError) as e:
        _pcg(mat, d)
    assert e.value.code == NONFINITE
    it, p = _pcg(mat, div, tol=1e-3)
    assert 0 < it <= 200 and np.isfinite(p.cpu().numpy()).all()


def _sealed_island():
    """A 48x32x32 block of solid holding a sealed 20x20x20 fluid cavity and,
    beside it, a separate open tank with a free surface (air above): the
    cavity has no Dirichlet cell, so A is singular on it."""
    mat = np.full((48, 32, 32), 1, np.int32)          # solid everywhere
    mat[2:22, 6:26, 6:26] = 0                         # sealed cavity (island)
    mat[26:46, 4:28, 2:20] = 0                        # open tank ...
    mat[26:46, 4:28, 20:32] = 2                       # ... with air above it
    mat[0, :, :] = 2                                  # an air ring on the outer layer
    mat[-1, :, :] = 2
    return mat


def test_closed_neumann_island_consistent_rhs(cuda):
    """Physically derived divergence (no-slip velocities): its sum over the
    sealed cavity is zero, so the singular system is consistent.  The solve
    ends within its caps with a finite pressure and a defined status."""
    mat = _sealed_island()
    ux, uy, uz = S.velocity_field(mat, seed=3)
    div = O.divergence(ux, uy, uz, mat, DX)
    solver = TolSolver(cell_mask(torch.as_tensor(mat).cuda()), "fp32")
    res = solver.solve(torch.as_tensor(div).cuda(), DX, DT, RHO, tol=1e-6, max_outer=4,
                       max_inner=100, raise_on_fail=False)
    assert res.status in (0, NOT_CONVERGED)
    assert res.outer_iterations <= 4 and res.inner_iterations <= 4 * 100
    assert np.isfinite(res.p64).all()
    assert O.rel_residual64(res.p64, div, mat, DX, DT, RHO) <= 1e-3


def test_closed_neumann_island_inconsistent_rhs(cuda):
    """A constant divergence inside the sealed cavity has no solution there:
    the solve stops at its caps with BSP_NOT_CONVERGED, or BSP_ERR_NONFINITE
    when the iterate overflows, and never hangs; the reference-compatible PCG
    runs to max_iter."""
    mat = _sealed_island()
    div = np.where(mat == 0, np.float32(0.5), np.float32(0.0)).astype(np.float32)
    solver = TolSolver(cell_mask(torch.as_tensor(mat).cuda()), "fp32")
    t0 = time.time()
    res = solver.solve(torch.as_tensor(div).cuda(), DX, DT, RHO, tol=1e-6, max_outer=3,
                       max_inner=50, raise_on_fail=False)
    assert time.time() - t0 < 60
    assert res.status in (NOT_CONVERGED, NONFINITE)
    assert res.outer_iterations <= 3 and res.inner_iterations <= 3 * 50
    if res.status == NOT_CONVERGED:
        assert np.isfinite(res.p64).all()
    # the reference algorithm has no in-loop finiteness check: it runs to its cap
    it, _ = _pcg(mat, div, tol=1e-6, max_iter=120)
    assert it == 120


def test_bounded_waits_give_up_and_context_survives(cuda):
    codes = torch.zeros(2, dtype=torch.int32, device="cuda")
    scratch = torch.zeros(16, dtype=torch.int32, device="cuda")
    t0 = time.time()
    call("bsp_selftest_waits", ptr(codes), ptr(scratch), 0)
    torch.cuda.synchronize()
    assert time.time() - t0 < 60
    assert codes.cpu().tolist() == [TIMEOUT, TIMEOUT]
    # the context is intact: a solve afterwards succeeds
    mat, div = _pot()
    res = TolSolver(cell_mask(torch.as_tensor(mat).cuda())).solve(
        torch.as_tensor(div).cuda(), DX, DT, RHO, tol=1e-6)
    assert res.status == 0


def test_coarse_barrier_timeout_then_next_solve_succeeds(cuda):
    """A coarse-cycle barrier that gave up leaves its error word set; that
    solve returns BSP_ERR_TIMEOUT, and the next solve on the same workspace
    (setup reused) starts from clean barrier words and succeeds.  The
    software grid barrier belongs to the cooperative form of the coarse
    cycle (BSP_TUNE_COARSE_CLUSTER = 0); the cluster form waits in the
    hardware cluster barrier."""
    spec = S.PotSpec(96, 96, 64, r_in=42, t_w=2, water_line=50, carrot_r=6, carrot_len=30)
    mat, div = _pot(spec)
    call("bsp_set_tuning", BSP_TUNE_COARSE_CLUSTER, 0)
    try:
        solver = TolSolver(cell_mask(torch.as_tensor(mat).cuda()), "fp16")
        div_t = torch.as_tensor(div).cuda()
        assert solver.solve(div_t, DX, DT, RHO, tol=1e-6).status == 0  # builds the setup
        call("bsp_set_tuning", BSP_TUNE_TEST_BARRIER_ERROR, 1)
        with pytest.raises(BspError) as e:
            solver.solve(div_t, DX, DT, RHO, tol=1e-6)
        assert e.value.code == TIMEOUT
        res = solver.solve(div_t, DX, DT, RHO, tol=1e-6)
        assert res.status == 0
        assert O.rel_residual64(res.p64, div, mat, DX, DT, RHO) <= 1.0001e-6
    finally:
        call("bsp_set_tuning", BSP_TUNE_COARSE_CLUSTER, 16)
