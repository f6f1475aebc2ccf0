"""The projection part of a time step (pipeline.py:605-619): no-slip,
projection, no-slip, with the first no-slip fused into the divergence and the
second dropped -- checked bit for bit against the oracle running the three
reference calls in sequence -- and the warm start across time steps of the
to-tolerance solver."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle as O
from boilingsim_b200 import fluid as F, scenes as S
from boilingsim_b200._lib import call, ptr

pytestmark = pytest.mark.gpu


def dev(a, dt=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dt).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def raw_velocity(mat, seed):
    """Face velocities with nonzero values on every face (no no-slip applied),
    so the fused no-slip has work to do on walls, air and the domain edge."""
    return S.velocity_field(mat, seed=seed, apply_no_slip=False)


CASES = [(seed, shape) for seed, shape in S.PARITY_CASES] + [
    (11, (5, 7, 132)), (12, (1, 1, 1)), (13, (2, 3, 1))]


@pytest.mark.parametrize("seed,shape", CASES)
def test_noslip_divergence_bit_exact(cuda, seed, shape):
    rng = np.random.default_rng(seed)
    if min(shape) < 3:
        # all fluid: only the domain-edge faces are zeroed
        mat = np.zeros(shape, np.int32)
        ux, uy, uz = (rng.standard_normal(s).astype(np.float32) for s in (
            (shape[0] + 1, shape[1], shape[2]), (shape[0], shape[1] + 1, shape[2]),
            (shape[0], shape[1], shape[2] + 1)))
    else:
        mat, _, _ = S.parity_random_grid(rng, shape)
        ux, uy, uz = raw_velocity(mat, seed)
    dx = float(rng.uniform(0.0005, 0.004))
    wu = O.enforce_no_slip(ux, uy, uz, mat)
    want = O.divergence(*wu, mat, dx)
    nx, ny, nz = shape
    mask = F.cell_mask(dev(mat, torch.int32))
    U = [dev(a) for a in (ux, uy, uz)]
    div = torch.full(shape, 7.0, dtype=torch.float32, device="cuda")
    call("bsp_noslip_divergence", ptr(div), *[ptr(u) for u in U], ptr(mask), nx, ny, nz, dx, 0)
    assert np.array_equal(bits(host(div)), bits(want))
    for got, w in zip(U, wu):
        assert np.array_equal(bits(host(got)), bits(w))


@pytest.mark.parametrize("spec", [S.POT_64])
def test_step_projection_jacobi_bit_exact(cuda, spec, monkeypatch):
    """projection_step (Jacobi back-end) equals no_slip; pressure_projection;
    no_slip of the oracle on every output: p, the diagnostic divergence, the
    three velocity components and max |div|."""
    monkeypatch.setenv("BOILINGSIM_PRESSURE_SOLVER", "jacobi")
    monkeypatch.delenv("BOILINGSIM_USE_RUST_PRESSURE", raising=False)
    mat = S.pot_mat(spec)
    ux, uy, uz = raw_velocity(mat, 5)
    dx, dt, rho = 0.002, 0.01, 997.0
    wu = O.enforce_no_slip(ux, uy, uz, mat)
    want = O.projection_jacobi(*wu, mat, dx, dt, rho, 200)
    wf = O.enforce_no_slip(want["ux"], want["uy"], want["uz"], mat)
    grid = F.Grid.from_numpy(mat, ux, uy, uz, dx)
    ws = F.allocate_fluid_workspace(grid)
    cfg = F.ScenarioConfig(F.SolverConfig(pressure_max_iter=200))
    got_max = F.projection_step(grid, ws, cfg, dt, rho)
    assert np.array_equal(bits(host(grid.p)), bits(want["p"]))
    assert np.array_equal(bits(host(ws.div_u)), bits(want["div"]))
    for got, w in zip((grid.ux, grid.uy, grid.uz), wf):
        assert np.array_equal(bits(host(got)), bits(w))
    assert got_max == pytest.approx(want["max_div"], rel=0, abs=0)


def test_step_projection_tolerance_matches_unfused(cuda, monkeypatch):
    """On a to-tolerance back-end, projection_step gives the same fields as
    enforce_no_slip + pressure_projection + enforce_no_slip (same solver on
    bit-identical inputs)."""
    monkeypatch.setenv("BOILINGSIM_PRESSURE_SOLVER", "b200-mg")
    monkeypatch.delenv("BOILINGSIM_USE_RUST_PRESSURE", raising=False)
    mat = S.pot_mat(S.POT_64)
    ux, uy, uz = raw_velocity(mat, 9)
    cfg = F.ScenarioConfig(F.SolverConfig(pressure_tol=1e-6))
    outs = []
    for fused in (True, False):
        grid = F.Grid.from_numpy(mat, ux, uy, uz, 0.002)
        ws = F.allocate_fluid_workspace(grid)
        if fused:
            m = F.projection_step(grid, ws, cfg, 0.01, 997.0)
        else:
            F.enforce_no_slip(grid)
            m = F.pressure_projection(grid, ws, cfg, 0.01, 997.0)
            F.enforce_no_slip(grid)
        outs.append([host(t) for t in (grid.p, grid.ux, grid.uy, grid.uz, ws.div_u)] + [m])
    for a, b in zip(outs[0][:5], outs[1][:5]):
        assert np.array_equal(bits(a), bits(b))
    assert outs[0][5] == outs[1][5]


def _step_velocities(mat, n_steps, seed=21):
    """A slowly varying sequence of pre-projection velocity fields: a fixed
    plume flow growing by 1 % per step plus a small random part per step."""
    base = S.velocity_field(mat, seed=seed, apply_no_slip=False)
    out = []
    for t in range(n_steps):
        kick = S.velocity_field(mat, seed=seed + 1 + t, amp=0.0005, plume=0.0,
                                apply_no_slip=False)
        out.append([np.float32(1.0 + 0.01 * t) * b + k for b, k in zip(base, kick)])
    return out


@pytest.mark.parametrize("storage", ["b200-mg", "b200-mixed"])
def test_warm_start_across_steps(cuda, monkeypatch, storage):
    """Starting each solve from the previous step's pressure reaches the same
    tolerance with fewer inner iterations than starting from zero."""
    monkeypatch.setenv("BOILINGSIM_PRESSURE_SOLVER", storage)
    monkeypatch.delenv("BOILINGSIM_USE_RUST_PRESSURE", raising=False)
    mat = S.pot_mat(S.POT_64)
    seq = _step_velocities(mat, 6)
    dx, dt, rho, tol = 0.002, 0.01, 997.0, 1e-6
    iters = {}
    for warm in (False, True):
        cfg = F.ScenarioConfig(F.SolverConfig(pressure_tol=tol, pressure_warm_start=warm))
        grid = F.Grid.from_numpy(mat, *seq[0], dx)
        ws = F.allocate_fluid_workspace(grid)
        total = []
        for t, vel in enumerate(seq):
            for dst, src in zip((grid.ux, grid.uy, grid.uz), vel):
                dst.copy_(torch.as_tensor(src))
            F.projection_step(grid, ws, cfg, dt, rho)
            res = F._TOL_SOLVERS[next(iter(F._TOL_SOLVERS))]
            info = res.last
            assert info.status == 0, (warm, t, info)
            # the solve's own FP64 residual check, repeated on the CPU in FP64
            # from the solver's FP64 iterate
            nsv = O.enforce_no_slip(*vel, mat)
            div = O.divergence(*nsv, mat, dx)
            rel = O.rel_residual64(host(info.p64_dev), div, mat, dx, dt, rho)
            assert rel <= tol * 1.01, (warm, t, rel)
            total.append(info.inner_iterations)
        iters[warm] = total
    # the first step is a cold start either way
    assert iters[True][0] == iters[False][0]
    assert sum(iters[True][1:]) < 0.85 * sum(iters[False][1:]), iters
