"""Semi-Lagrangian advection on the GPU (fluid.py:39-104, 338-498, 737-776):
the extension of T into solids, the T and face-velocity advection and
advect_all, each compared bit for bit with the CPU oracle -- random material
grids with a non-zero origin, velocities large enough to push backtraces
onto the clamped domain edge, the pot scenes at 192x192x128 and 384x384x256,
and the argument checks."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle as O
from boilingsim_b200 import fluid as F
from boilingsim_b200 import scenes as S
from boilingsim_b200._lib import BspError, call, ptr

pytestmark = pytest.mark.gpu


def dev(a, dt=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dt).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def faces(shape):
    nx, ny, nz = shape
    return (nx + 1, ny, nz), (nx, ny + 1, nz), (nx, ny, nz + 1)


def case(seed, shape, amp):
    rng = np.random.default_rng(seed)
    mat, _, _ = S.parity_random_grid(rng, shape)
    u = [(amp * rng.standard_normal(s)).astype(np.float32) for s in faces(shape)]
    T = (280 + 40 * rng.random(shape)).astype(np.float32)
    org = (float(rng.uniform(-0.02, 0.0)), float(rng.uniform(-0.02, 0.0)),
           float(rng.uniform(-0.01, 0.01)))
    return mat, u, T, org


SHAPES = [(6, 7, 9), (12, 10, 16), (20, 17, 33), (5, 5, 130)]
AMPS = [0.05, 3.0]  # a few cells of backtrace / far past the domain edge (clamped)
DX, DT = 0.002, 0.01


@pytest.mark.parametrize("amp", AMPS)
@pytest.mark.parametrize("shape", SHAPES)
def test_kernels_bit_exact(cuda, shape, amp):
    mat, u, T, org = case(sum(shape) + int(amp * 10), shape, amp)
    mask = F.cell_mask(dev(mat, torch.int32))
    U = [dev(a) for a in u]
    Td = dev(T)
    ext = torch.full(shape, -1.0, device="cuda")
    F.extend_temperature_into_solids(ext, Td, mask)
    want_ext = O.extend_temperature(T, mat)
    assert np.array_equal(bits(host(ext)), bits(want_ext))
    Tn = torch.empty_like(Td)
    F.advect_temperature(Tn, Td, ext, *U, mask, org, DX, DT)
    want_T = O.advect_temperature(T, want_ext, *u, mat, org, DX, DT)
    assert np.array_equal(bits(host(Tn)), bits(want_T))
    for ax in range(3):
        un = torch.empty_like(U[ax])
        F.advect_velocity(ax, un, *U, mask, org, DX, DT)
        want = O.advect_velocity(ax, *u, mat, org, DX, DT)
        assert np.array_equal(bits(host(un)), bits(want)), f"axis {ax}"


@pytest.mark.parametrize("copy_back", [1, 0])
def test_advect_all_bit_exact(cuda, copy_back):
    shape = (14, 12, 20)
    mat, u, T, org = case(5, shape, 0.3)
    w = O.advect_all(*u, T, mat, org, DX, DT)
    mask = F.cell_mask(dev(mat, torch.int32))
    U = [dev(a) for a in u]
    Td = dev(T)
    tmp = [torch.empty_like(a) for a in (*U, Td)]
    ext = torch.empty_like(Td)
    nx, ny, nz = shape
    call("bsp_advect_all", *(ptr(a) for a in (*U, Td, *tmp, ext, mask)), nx, ny, nz, *org, DX,
         DT, copy_back, 0)
    out = (*U, Td) if copy_back else tmp
    for got, want in zip(out, w[:4]):
        assert np.array_equal(bits(host(got)), bits(want))
    assert np.array_equal(bits(host(ext)), bits(w[4]))
    if not copy_back:  # sources untouched
        for got, src in zip((*U, Td), (*u, T)):
            assert np.array_equal(bits(host(got)), bits(src))


@pytest.mark.parametrize("spec,steps", [(S.pot_192(), 3), (S.POT_384, 1)])
def test_pot_scene_bit_exact(cuda, spec, steps):
    """advect_all through the Python mirror on the pot scene (origin as
    compute_grid_dims places it: -nx dx / 2, -ny dx / 2, -4 dx)."""
    mat = S.pot_mat(spec)
    ux, uy, uz = S.velocity_field(mat, seed=7)
    rng = np.random.default_rng(3)
    T = (330.0 + rng.standard_normal(mat.shape)).astype(np.float32)
    dx = 0.0005
    org = (-spec.nx * dx / 2, -spec.ny * dx / 2, -4 * dx)
    want = (ux, uy, uz, T)
    for _ in range(steps):
        want = O.advect_all(*want, mat, org, dx, 0.01)[:4]
    grid = F.Grid.from_numpy(mat, ux, uy, uz, dx)
    grid.T = dev(T)
    grid.origin = org
    ws = F.allocate_fluid_workspace(grid)
    for _ in range(steps):
        F.advect_all(grid, ws, 0.01)
    for got, w in zip((grid.ux, grid.uy, grid.uz, grid.T), want):
        assert np.array_equal(bits(host(got)), bits(w))


def test_argument_checks(cuda):
    m = torch.zeros((4, 4, 4), dtype=torch.uint8, device="cuda")
    a = torch.zeros((4, 4, 4), device="cuda")
    b = torch.zeros((4, 4, 4), device="cuda")
    with pytest.raises(BspError):
        call("bsp_extend_temperature", ptr(a), ptr(a), ptr(m), 4, 4, 4, 0)
    with pytest.raises(BspError):
        call("bsp_advect_velocity", 3, ptr(a), ptr(b), ptr(b), ptr(b), ptr(m), 4, 4, 4, 0.0,
             0.0, 0.0, DX, DT, 0)
    with pytest.raises(BspError):
        call("bsp_advect_temperature", 0, ptr(a), ptr(a), ptr(b), ptr(b), ptr(b), ptr(m), 4, 4,
             4, 0.0, 0.0, 0.0, DX, DT, 0)
    call("bsp_extend_temperature", ptr(a), ptr(b), ptr(m), 0, 4, 4, 0)  # empty: no-op
