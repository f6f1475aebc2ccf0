"""Backward-Euler conduction on the GPU (thermal.py:259-388, 647-658): every
sweep and step is compared bit for bit with the CPU oracle -- random material
grids on both kernel shapes (column: nz % 4 == 0 and aligned; generic:
anything else), int32 and uint8 material ids, air cells left unwritten, the
fused snapshot, odd and even sweep counts, the pot scene at 192x192x128 and
384x384x256, and the argument checks."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

import oracle as O
from boilingsim_b200 import scenes as S
from boilingsim_b200 import thermal as TH
from boilingsim_b200._lib import BspError, call, ptr

pytestmark = pytest.mark.gpu

DX, DT, H, TAMB = 0.002, 0.25, 10.0, 295.15


def dev(a, dt=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dt).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def material_grid(rng, shape):
    """Random materials 0..3 (air = 2) overlaid on blocks of one material, so
    that every face pairing occurs and whole float4 groups are air or solid."""
    mat = rng.integers(0, 4, shape)
    bi = (np.arange(shape[0]) // 2)[:, None, None]
    bj = (np.arange(shape[1]) // 3)[None, :, None]
    bk = (np.arange(shape[2]) // 8)[None, None, :]
    blocks = (7 * bi + 3 * bj + 5 * bk) % 4
    return np.where(rng.random(shape) < 0.7, blocks, mat).astype(np.int32)


def props():
    p = TH.MaterialProps.from_materials("steel_304")
    return p, (p.k, p.rho, p.c_p)


SHAPES = [(9, 10, 128), (7, 9, 36), (6, 5, 7), (1, 1, 4), (3, 17, 260), (2, 1, 1)]


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("u8", [False, True])
def test_sweep_bit_exact(cuda, shape, u8):
    rng = np.random.default_rng(sum(shape) + 7 * u8)
    mat = material_grid(rng, shape)
    T = (280 + 40 * rng.random(shape)).astype(np.float32)
    Told = (280 + 40 * rng.random(shape)).astype(np.float32)
    junk = (1000 * rng.random(shape)).astype(np.float32)
    p, hp = props()
    want = O.conduction_sweep(junk, T, Told, mat, hp, DX, DT, H, TAMB)
    m = dev(mat, torch.int32)
    if u8:
        m = TH.material_ids(m)
    out = dev(junk)
    TH.apply_implicit_conduction_update(out, dev(T), dev(Told), m, p.k_wp, p.rho_wp, p.cp_wp,
                                        DX, DT, H, TAMB)
    assert np.array_equal(bits(host(out)), bits(want))


def test_sweep_unaligned_views_take_the_generic_kernel(cuda):
    rng = np.random.default_rng(4)
    shape = (5, 6, 8)
    n = int(np.prod(shape))
    mat = material_grid(rng, shape)
    T = (280 + 40 * rng.random(shape)).astype(np.float32)
    junk = np.zeros(shape, np.float32)
    p, hp = props()
    want = O.conduction_sweep(junk, T, T, mat, hp, DX, DT, H, TAMB)
    buf = torch.zeros(3 * n + 3, dtype=torch.float32, device="cuda")
    src = buf[1:n + 1].view(shape)
    told = buf[n + 2:2 * n + 2].view(shape)
    src.copy_(dev(T))
    told.copy_(dev(T))
    out = torch.zeros(shape, dtype=torch.float32, device="cuda")
    TH.apply_implicit_conduction_update(out, src, told, dev(mat, torch.int32), p.k_wp, p.rho_wp,
                                        p.cp_wp, DX, DT, H, TAMB)
    assert np.array_equal(bits(host(out)), bits(want))


@pytest.mark.parametrize("n_iter", [0, 1, 2, 5, 16])
@pytest.mark.parametrize("shape", [(8, 12, 128), (6, 7, 9)])
def test_be_step_bit_exact(cuda, shape, n_iter):
    rng = np.random.default_rng(n_iter + shape[2])
    mat = material_grid(rng, shape)
    T = (280 + 40 * rng.random(shape)).astype(np.float32)
    alt = (1000 * rng.random(shape)).astype(np.float32)
    p, hp = props()
    wT, wa, wo = O.conduction_be(T, alt, mat, hp, DX, DT, H, TAMB, n_iter)
    grid = TH.ThermalGrid(*shape, DX, dev(T), dev(mat, torch.int32))
    ws = TH.ThermalWorkspace(torch.full(shape, -3.0, device="cuda"), dev(alt))
    cfg = TH.ThermalConfig()
    cfg.solver.diffusion_max_iter = n_iter
    cfg.heating.ambient_temp_c = TAMB - 273.15
    TH.implicit_conduction_step(grid, p, ws, cfg, DT)
    assert np.array_equal(bits(host(grid.T)), bits(wT))
    assert np.array_equal(bits(host(ws.T_iter_alt)), bits(wa))
    assert np.array_equal(bits(host(ws.T_old_snapshot)), bits(wo))


def pot_temperature(mat, rng):
    T = np.empty(mat.shape, np.float32)
    T[mat == S.MAT_FLUID] = 330.0
    T[mat == S.MAT_POT_WALL] = 380.0
    T[mat == S.MAT_AIR] = 295.15
    T[mat == S.MAT_CARROT] = 300.0
    return (T + rng.standard_normal(mat.shape).astype(np.float32)).astype(np.float32)


@pytest.mark.parametrize("spec,n_iter", [(S.pot_192(), 50), (S.POT_384, 3)])
def test_pot_scene_bit_exact(cuda, spec, n_iter):
    """The production path: cell classes, TMA-fed sweeps."""
    rng = np.random.default_rng(7)
    mat = S.pot_mat(spec)
    T = pot_temperature(mat, rng)
    alt = np.zeros_like(T)
    p, hp = props()
    dx = 0.0005
    wT, wa, wo = O.conduction_be(T, alt, mat, hp, dx, 0.01, H, TAMB, n_iter)
    grid = TH.ThermalGrid(*spec.shape, dx, dev(T), dev(mat, torch.int32))
    ws = TH.allocate_thermal_workspace(grid)
    cfg = TH.ThermalConfig()
    cfg.solver.diffusion_max_iter = n_iter
    cfg.heating.ambient_temp_c = TAMB - 273.15
    TH.implicit_conduction_step(grid, p, ws, cfg, 0.01)
    assert grid.classes, "the pot scene should sweep on cell classes"
    flag = ctypes.c_int(0)
    call("bsp_conduction_error", ctypes.byref(flag))
    assert flag.value == 0
    assert np.array_equal(bits(host(grid.T)), bits(wT))
    assert np.array_equal(bits(host(ws.T_iter_alt)), bits(wa))
    assert np.array_equal(bits(host(ws.T_old_snapshot)), bits(wo))


def block_grid(shape):
    """Nested boxes: an air border, a steel shell (open above mid height), water
    with air above three quarters of the height, and a carrot block -- all
    material pairs, the domain edge, and about a hundred distinct cell
    neighbourhoods."""
    nx, ny, nz = shape
    i = np.arange(nx)[:, None, None]
    j = np.arange(ny)[None, :, None]
    k = np.arange(nz)[None, None, :]

    def inside(m):
        return (i >= m) & (i < nx - m) & (j >= m) & (j < ny - m) & (k >= m) & (k < nz - m)

    mat = np.full(shape, TH.MAT_AIR, np.int32)
    mat[inside(1) | ((k < nz // 2) & inside(0))] = TH.MAT_POT_WALL
    mat[inside(2)] = TH.MAT_FLUID
    mat[inside(2) & (k > (3 * nz) // 4)] = TH.MAT_AIR
    mat[inside(3) & (np.abs(i - nx // 2) <= nx // 5) & (np.abs(j - ny // 2) <= ny // 5)
        & (np.abs(k - nz // 3) <= nz // 6)] = TH.MAT_CARROT
    return mat


BSP_TUNE_COND_TMA = 10


@pytest.fixture
def tma_mode(request):
    call("bsp_set_tuning", BSP_TUNE_COND_TMA, int(request.param))
    yield request.param
    call("bsp_set_tuning", BSP_TUNE_COND_TMA, 1)
    flag = ctypes.c_int(0)
    call("bsp_conduction_error", ctypes.byref(flag))
    assert flag.value == 0, "a TMA-fed sweep gave up waiting"


@pytest.mark.parametrize("tma_mode", [True, False], indirect=True)
@pytest.mark.parametrize("shape", SHAPES + [(8, 12, 144), (5, 9, 16), (17, 3, 384)])
def test_class_sweep_bit_exact(cuda, shape, tma_mode):
    rng = np.random.default_rng(sum(shape) + 100)
    mat = block_grid(shape)
    T = (280 + 40 * rng.random(shape)).astype(np.float32)
    Told = (280 + 40 * rng.random(shape)).astype(np.float32)
    junk = (1000 * rng.random(shape)).astype(np.float32)
    p, hp = props()
    want = O.conduction_sweep(junk, T, Told, mat, hp, DX, DT, H, TAMB)
    c = TH.cell_classes(dev(mat, torch.int32))
    assert c is not None and 1 <= c.n_classes <= 128
    # classes are dense 1..n-1 on non-air cells, 0x80 on air
    cl = host(c.cls)
    air = mat == TH.MAT_AIR
    assert np.all(cl[air] == 0x80)
    if (~air).any():
        assert cl[~air].min() == 1 and cl[~air].max() == c.n_classes - 1
    out, t_iter, t_old = dev(junk), dev(T), dev(Told)  # keep the inputs alive over the call
    call("bsp_conduction_sweep_cls", ptr(out), ptr(t_iter), ptr(t_old), ptr(c.cls),
         ptr(c.patterns), c.n_classes, ptr(c.tiles), *shape, ptr(p.k_wp), ptr(p.rho_wp), ptr(p.cp_wp), 4, DX,
         DT, H, TAMB, TH.MAT_AIR, 0)
    assert np.array_equal(bits(host(out)), bits(want))


@pytest.mark.parametrize("tma_mode", [True, False], indirect=True)
@pytest.mark.parametrize("n_iter", [0, 1, 2, 7])
@pytest.mark.parametrize("shape", [(8, 12, 128), (6, 7, 9), (10, 9, 48)])
def test_class_step_bit_exact(cuda, shape, n_iter, tma_mode):
    rng = np.random.default_rng(n_iter + 31)
    mat = block_grid(shape)
    T = (280 + 40 * rng.random(shape)).astype(np.float32)
    alt = (1000 * rng.random(shape)).astype(np.float32)
    p, hp = props()
    wT, wa, wo = O.conduction_be(T, alt, mat, hp, DX, DT, H, TAMB, n_iter)
    grid = TH.ThermalGrid(*shape, DX, dev(T), dev(mat, torch.int32))
    ws = TH.ThermalWorkspace(torch.full(shape, -3.0, device="cuda"), dev(alt))
    cfg = TH.ThermalConfig()
    cfg.solver.diffusion_max_iter = n_iter
    cfg.heating.ambient_temp_c = TAMB - 273.15
    TH.implicit_conduction_step(grid, p, ws, cfg, DT)
    assert grid.classes
    assert np.array_equal(bits(host(grid.T)), bits(wT))
    assert np.array_equal(bits(host(ws.T_iter_alt)), bits(wa))
    assert np.array_equal(bits(host(ws.T_old_snapshot)), bits(wo))


def test_too_many_classes_falls_back_to_material_ids(cuda):
    rng = np.random.default_rng(9)
    shape = (24, 24, 32)
    mat = rng.integers(0, 4, shape).astype(np.int32)
    assert TH.cell_classes(dev(mat, torch.int32)) is None  # hundreds of neighbourhoods
    T = (280 + 40 * rng.random(shape)).astype(np.float32)
    p, hp = props()
    wT, wa, wo = O.conduction_be(T, np.zeros_like(T), mat, hp, DX, DT, H, TAMB, 4)
    grid = TH.ThermalGrid(*shape, DX, dev(T), dev(mat, torch.int32))
    ws = TH.allocate_thermal_workspace(grid)
    cfg = TH.ThermalConfig()
    cfg.solver.diffusion_max_iter = 4
    cfg.heating.ambient_temp_c = TAMB - 273.15
    TH.implicit_conduction_step(grid, p, ws, cfg, DT)
    assert grid.classes is False and grid.mat_id is not None
    assert np.array_equal(bits(host(grid.T)), bits(wT))


def test_argument_checks(cuda):
    p, _ = props()
    a = torch.zeros((4, 4, 4), device="cuda")
    b = torch.zeros((4, 4, 4), device="cuda")
    m = torch.zeros((4, 4, 4), dtype=torch.int32, device="cuda")
    base = [ptr(a), ptr(b), ptr(b), ptr(m), 4, 4, 4, ptr(p.k_wp), ptr(p.rho_wp), ptr(p.cp_wp)]
    tail = [DX, DT, H, TAMB, 2, 0]
    call("bsp_conduction_sweep", *base, 4, *tail)
    for bad_nmat in (0, 9):
        with pytest.raises(BspError):
            call("bsp_conduction_sweep", *base, bad_nmat, *tail)
    with pytest.raises(BspError):  # in place
        call("bsp_conduction_sweep", ptr(a), ptr(a), *base[2:], 4, *tail)
    with pytest.raises(BspError):
        call("bsp_conduction_sweep", 0, *base[1:], 4, *tail)
    # empty grid: success, no work
    call("bsp_conduction_sweep", *base[:4], 0, 4, 4, *base[7:], 4, *tail)
    with pytest.raises(ValueError):
        TH.material_ids(torch.full((4, 4, 4), 5, dtype=torch.int32, device="cuda"))
    # class preparation rejects ids outside [0, n_mat) instead of aliasing them
    bad = torch.zeros((6, 5, 8), dtype=torch.int32, device="cuda")
    bad[2, 2, 2] = 9
    with pytest.raises(BspError):
        TH.cell_classes(bad)
    bad[2, 2, 2] = -1
    with pytest.raises(BspError):
        TH.cell_classes(bad)
