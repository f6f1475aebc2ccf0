"""Synthetic pot scenes: material masks and seeded MAC velocity fields.

The reference measures the projection on simulated pot scenes, not on a public
dataset, so workloads here are generated from its voxelisation rules:

* material ids ``MAT_FLUID=0, MAT_POT_WALL=1, MAT_AIR=2, MAT_CARROT=3``
  (``python/boilingsim/geometry.py:39-42``);
* pot wall / cavity / free surface classification by cell centre
  (``geometry.py:62-152``): a cell is wall if it lies in the bottom slab or in
  the side-wall annulus, fluid if it is in the cavity below the water line,
  air otherwise (including everything above the water line -- the free
  surface is a Dirichlet p=0 boundary);
* ingredients stamped over FLUID cells only (``geometry.py:155-219``), here a
  horizontal x-axis carrot cylinder at mid water depth;
* velocity seeding as the reference's parity test does
  (``python/tests/test_pressure_parity.py:184-187``): ``rng = default_rng(seed)``
  and ``0.05 * standard_normal`` for ux, uy, uz in that order, float32;
  then three passes of a 3x3x3 box mean (edge-replicated), a Gaussian
  buoyant plume on the pot axis (sigma = 3 cells) added to fluid z-faces,
  and the no-slip rule of ``fluid.py:111-165`` (as ``pipeline.py:606-607``
  applies it before every projection).

``single_carrot_mat(dx)`` restates ``build_pot_geometry`` for the reference's
``configs/scenarios/single_carrot.yaml`` (used by its projection parity test).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

MAT_FLUID, MAT_POT_WALL, MAT_AIR, MAT_CARROT = 0, 1, 2, 3


@dataclass(frozen=True)
class PotSpec:
    """Integer pot geometry in cell units (pot axis at the grid centre)."""

    nx: int
    ny: int
    nz: int
    r_in: float        # cavity radius
    t_w: int           # wall and bottom thickness
    water_line: float  # cavity cells with k + 0.5 < water_line are fluid
    carrot_r: float    # 0 disables the carrot
    carrot_len: float

    @property
    def shape(self):
        return (self.nx, self.ny, self.nz)


# Workloads (sizes and seeds as stated in the benchmark configuration).
POT_64 = PotSpec(64, 64, 48, r_in=28, t_w=2, water_line=40, carrot_r=6, carrot_len=30)
POT_384 = PotSpec(384, 384, 256, r_in=168, t_w=12, water_line=213, carrot_r=36,
                  carrot_len=180)


def pot_192(t_w: int = 2) -> PotSpec:
    """192x192x128 pot; wall thickness 2/3/4 cells (steel/aluminium/copper-like)."""
    return PotSpec(192, 192, 128, r_in=84, t_w=t_w, water_line=107, carrot_r=18,
                   carrot_len=90)


def pot_mat(spec: PotSpec) -> np.ndarray:
    """int32 material ids (nx, ny, nz) for a pot with a horizontal carrot."""
    nx, ny, nz = spec.shape
    ci = (np.arange(nx, dtype=np.float64) + 0.5)[:, None, None]
    cj = (np.arange(ny, dtype=np.float64) + 0.5)[None, :, None]
    ck = (np.arange(nz, dtype=np.float64) + 0.5)[None, None, :]
    ax, ay = nx / 2.0, ny / 2.0
    r = np.sqrt((ci - ax) ** 2 + (cj - ay) ** 2)
    mat = np.full((nx, ny, nz), MAT_AIR, dtype=np.int32)
    in_outer = r < spec.r_in + spec.t_w
    wall = in_outer & ((ck < spec.t_w) | (r >= spec.r_in))
    cavity = (r < spec.r_in) & (ck >= spec.t_w)
    fluid = cavity & (ck < spec.water_line)
    mat[np.broadcast_to(fluid, mat.shape)] = MAT_FLUID
    mat[np.broadcast_to(wall, mat.shape)] = MAT_POT_WALL
    if spec.carrot_r > 0:
        zc = 0.5 * (spec.t_w + spec.water_line)
        rp = np.sqrt((cj - ay) ** 2 + (ck - zc) ** 2)
        along = np.abs(ci - ax)
        carrot = (rp < spec.carrot_r) & (along < 0.5 * spec.carrot_len)
        carrot = np.broadcast_to(carrot, mat.shape) & (mat == MAT_FLUID)
        mat[carrot] = MAT_CARROT
    return mat


def _box3(a: np.ndarray, passes: int = 3) -> np.ndarray:
    """``passes`` x 3x3x3 box mean with edge replication, in float32."""
    from scipy.ndimage import uniform_filter

    out = a
    for _ in range(passes):
        out = uniform_filter(out, size=3, mode="nearest").astype(np.float32, copy=False)
    return out


def no_slip(ux, uy, uz, mat, mat_fluid: int = MAT_FLUID):
    """In-place ``enforce_no_slip`` (fluid.py:111-165) on numpy arrays."""
    f = mat == mat_fluid
    ux[0] = 0.0
    ux[-1] = 0.0
    ux[1:-1][~(f[:-1] & f[1:])] = 0.0
    uy[:, 0] = 0.0
    uy[:, -1] = 0.0
    uy[:, 1:-1][~(f[:, :-1] & f[:, 1:])] = 0.0
    uz[:, :, 0] = 0.0
    uz[:, :, -1] = 0.0
    uz[:, :, 1:-1][~(f[:, :, :-1] & f[:, :, 1:])] = 0.0


def velocity_field(mat: np.ndarray, seed: int = 7, amp: float = 0.05,
                   plume: float = 0.1, sigma: float = 3.0, smooth: bool = True,
                   apply_no_slip: bool = True):
    """Seeded MAC face velocities (ux, uy, uz) float32 for a scene."""
    nx, ny, nz = mat.shape
    rng = np.random.default_rng(seed)
    ux = (rng.standard_normal((nx + 1, ny, nz)).astype(np.float32) * np.float32(amp))
    uy = (rng.standard_normal((nx, ny + 1, nz)).astype(np.float32) * np.float32(amp))
    uz = (rng.standard_normal((nx, ny, nz + 1)).astype(np.float32) * np.float32(amp))
    if smooth:
        ux, uy, uz = _box3(ux), _box3(uy), _box3(uz)
    if plume != 0.0:
        ci = (np.arange(nx) + 0.5)[:, None]
        cj = (np.arange(ny) + 0.5)[None, :]
        r2 = (ci - nx / 2.0) ** 2 + (cj - ny / 2.0) ** 2
        g = (plume * np.exp(-r2 / (2.0 * sigma * sigma))).astype(np.float32)
        f = mat == MAT_FLUID
        face_fluid = np.zeros((nx, ny, nz + 1), dtype=bool)
        face_fluid[:, :, 1:-1] = f[:, :, :-1] & f[:, :, 1:]
        uz += np.where(face_fluid, g[:, :, None], np.float32(0.0)).astype(np.float32)
    if apply_no_slip:
        no_slip(ux, uy, uz, mat)
    return (np.ascontiguousarray(ux, np.float32), np.ascontiguousarray(uy, np.float32),
            np.ascontiguousarray(uz, np.float32))


def random_batch_specs(count: int = 64, seed: int = 7):
    """Uneven pot instances from 48^3 to 128x128x96 cells: radius fills the box
    minus the wall and a 2-cell pad, water level 0.6-0.85 of the height,
    carrot radius 4-10 cells.  Returns a list of (PotSpec, velocity seed)."""
    rng = np.random.default_rng(seed)
    out = []
    for n in range(count):
        nxy = int(rng.integers(12, 33)) * 4          # 48 .. 128
        nz = int(rng.integers(12, 25)) * 4           # 48 .. 96
        t_w = int(rng.integers(2, 5))
        r_in = nxy / 2.0 - t_w - 2
        level = float(rng.uniform(0.6, 0.85))
        cr = float(rng.integers(4, 11))
        water = t_w + level * (nz - t_w)
        cr = min(cr, 0.45 * (water - t_w))
        out.append((PotSpec(nxy, nxy, nz, r_in=r_in, t_w=t_w, water_line=water,
                            carrot_r=cr, carrot_len=min(1.2 * r_in, 5.0 * cr)),
                    seed * 1000 + n))
    return out


# ---------------------------------------------------------------------------
# Restatement of build_pot_geometry for configs/scenarios/single_carrot.yaml
# ---------------------------------------------------------------------------

SINGLE_CARROT = dict(diameter_m=0.20, height_m=0.12, wall_thickness_m=0.003,
                     base_thickness_m=0.005, fill_fraction=0.75,
                     carrot_diameter_m=0.025, carrot_length_m=0.05,
                     carrot_position=(0.0, 0.0, 0.03))


def compute_grid_dims(dx: float, diameter_m: float, height_m: float, pad_cells: int = 4):
    """geometry.py:317-338 (Python float arithmetic, as the reference)."""
    r_outer = diameter_m / 2
    pad = pad_cells * dx
    nx = int(math.ceil((2 * r_outer + 2 * pad) / dx))
    ny = int(math.ceil((2 * r_outer + 2 * pad) / dx))
    nz = int(math.ceil((height_m + 2 * pad) / dx))
    nx += nx % 2
    ny += ny % 2
    origin = (-nx * dx / 2, -ny * dx / 2, -pad)
    return nx, ny, nz, origin


def single_carrot_mat(dx: float = 0.004, spec: dict = SINGLE_CARROT) -> np.ndarray:
    """int32 mat for the single-carrot pot (geometry.py:62-152, 155-219 with the
    vertical (axis z) carrot whose base is at ``carrot_position``), evaluated in
    float32 like the Warp kernels."""
    f32 = np.float32
    nx, ny, nz, origin = compute_grid_dims(dx, spec["diameter_m"], spec["height_m"])
    dxf = f32(dx)
    px = f32(origin[0]) + (np.arange(nx, dtype=f32) + f32(0.5)) * dxf
    py = f32(origin[1]) + (np.arange(ny, dtype=f32) + f32(0.5)) * dxf
    pz = f32(origin[2]) + (np.arange(nz, dtype=f32) + f32(0.5)) * dxf
    X, Y, Z = np.meshgrid(px, py, pz, indexing="ij")
    r_outer = f32(spec["diameter_m"] / 2)
    r_inner = f32(spec["diameter_m"] / 2 - spec["wall_thickness_m"])
    h_outer = f32(spec["height_m"])
    base = f32(spec["base_thickness_m"])
    h_inner = f32(spec["height_m"] - spec["base_thickness_m"])
    water_line = f32(spec["base_thickness_m"] + spec["fill_fraction"] *
                     (spec["height_m"] - spec["base_thickness_m"]))

    def sdf_cyl(x, y, z, r, h):
        d_xy = np.sqrt(x * x + y * y).astype(f32) - r
        d_z = np.abs(z - h * f32(0.5)) - h * f32(0.5)
        out = np.sqrt(np.maximum(d_xy, f32(0)) ** 2 + np.maximum(d_z, f32(0)) ** 2)
        ins = np.minimum(np.maximum(d_xy, d_z), f32(0))
        return (out + ins).astype(f32)

    d_outer = sdf_cyl(X, Y, Z, r_outer, h_outer)
    d_inner = sdf_cyl(X, Y, Z - base, r_inner, h_inner)
    sdf = np.maximum(d_outer, -d_inner)
    r_xy = np.sqrt(X * X + Y * Y).astype(f32)
    water = (r_xy < r_inner) & (Z > base) & (Z < water_line)
    mat = np.where(sdf < 0, MAT_POT_WALL, np.where(water, MAT_FLUID, MAT_AIR)).astype(np.int32)
    # carrot: axis z, centre = base point, range [cz, cz + length]
    cx, cy, cz = (f32(c) for c in spec["carrot_position"])
    rc = f32(spec["carrot_diameter_m"] / 2.0)
    L = f32(spec["carrot_length_m"])
    rx, ry, rz = X - cx, Y - cy, Z - cz
    rp = np.sqrt(rx * rx + ry * ry).astype(f32)
    carrot = (rp < rc) & (rz > f32(0)) & (rz < L) & (mat == MAT_FLUID)
    mat[carrot] = MAT_CARROT
    return mat


def parity_random_grid(rng: np.random.Generator, shape):
    """(mat, p_old, div_u) as python/tests/test_pressure_parity.py:51-67: an
    outer air ring, interior fluid/wall/air/carrot drawn 0.60/0.15/0.20/0.05,
    p_old ~ N(0,1), div ~ 0.1 N(0,1)."""
    nx, ny, nz = shape
    mat = np.full(shape, MAT_AIR, dtype=np.int32)
    choice = rng.choice([0, 1, 2, 3], size=(nx - 2, ny - 2, nz - 2),
                        p=[0.60, 0.15, 0.20, 0.05]).astype(np.int32)
    mat[1:-1, 1:-1, 1:-1] = choice
    p_old = rng.standard_normal(shape).astype(np.float32)
    div_u = rng.standard_normal(shape).astype(np.float32) * 0.1
    return mat, p_old, div_u


PARITY_CASES = [(1, (16, 16, 16)), (2, (24, 12, 20)), (3, (8, 32, 8)), (42, (20, 20, 20)),
                (101, (12, 24, 16)), (202, (16, 12, 24)), (303, (28, 16, 14)),
                (404, (10, 10, 30))]
