"""Backward-Euler thermal conduction -- host-side mirror of the reference API.

Drop-in for the implicit-conduction part of ``python/boilingsim/thermal.py``:

* ``MaterialProps`` (``thermal.py:45-122``): per-material rho, c_p, k arrays
  indexed by material id ``[fluid, pot_wall, air, carrot]``, with device
  copies ``rho_wp`` / ``cp_wp`` / ``k_wp``; the values are those of the
  reference's ``data/materials.json`` (air: dry air at 25 C, 1 atm);
* ``ThermalWorkspace`` / ``allocate_thermal_workspace`` (``thermal.py:564-582``):
  ``T_old_snapshot`` and the Jacobi ping-pong buffer ``T_iter_alt``;
* ``apply_implicit_conduction_update`` -- one Jacobi sweep with the Warp
  kernel's argument list (``thermal.py:259-388``);
* ``implicit_conduction_step`` -- the backward-Euler branch of
  ``conduct_one_step`` (``thermal.py:647-658``): snapshot, ``diffusion_max_iter``
  sweeps ping-ponging ``grid.T`` and ``T_iter_alt``, odd-count copy back.  The
  source terms that ``conduct_one_step`` applies afterwards (stove base flux,
  evaporative cooling) are the caller's.  The first call on a grid numbers its
  cell neighbourhoods (``cell_classes``) and later calls sweep on those class
  bytes; a geometry with more than 127 neighbourhoods uses material ids.

Every call runs the sm_100a kernels of libbsproj.so on the caller's stream;
results are bit-identical to the reference arithmetic.  There is no CPU path.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import torch

from ._lib import call, ptr, stream_handle

MAT_FLUID, MAT_POT_WALL, MAT_AIR, MAT_CARROT = 0, 1, 2, 3

# (rho kg/m^3, c_p J/(kg K), k W/(m K)) of data/materials.json; air as in
# MaterialProps.from_scenario (thermal.py:108-111).
MATERIALS = {
    "water": (997.0, 4186.0, 0.606),
    "steel_304": (8000.0, 500.0, 16.2),
    "cast_iron": (7200.0, 460.0, 55.0),
    "aluminum": (2700.0, 900.0, 237.0),
    "copper": (8960.0, 385.0, 401.0),
    "carrot": (1040.0, 3900.0, 0.605),
    "air": (1.184, 1005.0, 0.0262),
}


@dataclass
class MaterialProps:
    rho: np.ndarray
    c_p: np.ndarray
    k: np.ndarray
    rho_wp: torch.Tensor
    cp_wp: torch.Tensor
    k_wp: torch.Tensor

    @classmethod
    def from_materials(cls, pot_material: str = "steel_304", device: str = "cuda:0"):
        """The four-material table [water, pot, air, carrot] (thermal.py:106-122)."""
        rows = [MATERIALS["water"], MATERIALS[pot_material], MATERIALS["air"],
                MATERIALS["carrot"]]
        rho, cp, k = (np.array([r[i] for r in rows], dtype=np.float32) for i in range(3))
        dev = lambda a: torch.as_tensor(a).to(device)  # noqa: E731
        return cls(rho, cp, k, dev(rho), dev(cp), dev(k))

    @property
    def n_mat(self) -> int:
        return int(self.rho.shape[0])


@dataclass
class ThermalSolverConfig:
    """The conduction knobs of ``config.py:184-215``."""

    diffusion_max_iter: int = 15
    h_conv_outer_w_per_m2_k: float = 10.0
    use_implicit_conduction: bool = True


@dataclass
class HeatingConfig:
    ambient_temp_c: float = 22.0  # config.py:130


@dataclass
class ThermalConfig:
    solver: ThermalSolverConfig = field(default_factory=ThermalSolverConfig)
    heating: HeatingConfig = field(default_factory=HeatingConfig)


@dataclass
class ThermalGrid:
    """The fields of ``Grid`` (geometry.py:253-314) that conduction reads."""

    nx: int
    ny: int
    nz: int
    dx: float
    T: torch.Tensor    # (nx, ny, nz) f32, kelvin
    mat: torch.Tensor  # (nx, ny, nz) int32 material ids
    mat_id: torch.Tensor | None = None  # uint8 copy of mat, derived once
    # conduction cell classes, derived on the first step; False when the geometry
    # has more than 127 neighbourhoods (the material-id kernels serve it then)
    classes: "CellClasses | bool | None" = None

    @property
    def shape(self):
        return (self.nx, self.ny, self.nz)


@dataclass
class ThermalWorkspace:
    T_old_snapshot: torch.Tensor
    T_iter_alt: torch.Tensor


def allocate_thermal_workspace(grid, device: str = "cuda:0") -> ThermalWorkspace:
    shp = grid.shape
    return ThermalWorkspace(torch.zeros(shp, dtype=torch.float32, device=device),
                            torch.zeros(shp, dtype=torch.float32, device=device))


def material_ids(mat: torch.Tensor, n_mat: int = 4, stream=None) -> torch.Tensor:
    """uint8 material ids of an int32 material grid; raises on ids outside
    [0, n_mat) (one device-to-host read of the count)."""
    if mat.dtype != torch.int32 or not mat.is_contiguous():
        raise TypeError("mat must be a contiguous int32 CUDA tensor")
    out = torch.empty(mat.shape, dtype=torch.uint8, device=mat.device)
    bad = torch.zeros(1, dtype=torch.int32, device=mat.device)
    call("bsp_material_ids", ptr(out), ptr(mat), mat.numel(), int(n_mat), ptr(bad),
         stream_handle(stream))
    if int(bad.item()):
        raise ValueError(f"{int(bad.item())} material ids outside [0, {n_mat})")
    return out


@dataclass
class CellClasses:
    """Conduction cell classes of a geometry (bsp_conduction_prepare): one byte
    per cell naming its neighbourhood, and each class's neighbourhood key."""

    cls: torch.Tensor       # (nx, ny, nz) uint8, 0x80 = air
    patterns: torch.Tensor  # (256,) int32 keys
    n_classes: int
    tiles: torch.Tensor | None = None  # tile occupancy for the TMA sweep (nz % 4 == 0)


def cell_classes(mat: torch.Tensor, n_mat: int = 4, mat_air: int = MAT_AIR,
                 stream=None) -> CellClasses | None:
    """Number the distinct cell neighbourhoods of ``mat``; None when there are
    more than 127 (the material-id kernels then serve the geometry)."""
    import ctypes

    from . import _lib

    if mat.dtype != torch.int32 or not mat.is_contiguous():
        raise TypeError("mat must be a contiguous int32 CUDA tensor")
    nx, ny, nz = mat.shape
    cls = torch.empty(mat.shape, dtype=torch.uint8, device=mat.device)
    patterns = torch.zeros(256, dtype=torch.int32, device=mat.device)
    ws = torch.empty(int(_lib.lib().bsp_conduction_prepare_workspace_bytes()), dtype=torch.uint8,
                     device=mat.device)
    n = ctypes.c_int(0)
    code = _lib.lib().bsp_conduction_prepare(ptr(cls), ptr(patterns), ctypes.byref(n), ptr(mat),
                                              nx, ny, nz, int(n_mat), int(mat_air), ptr(ws),
                                              ws.numel(), stream_handle(stream))
    if code == 10010:  # BSP_ERR_CAPACITY
        return None
    _lib.check("bsp_conduction_prepare", code)
    tiles = None
    if nz % 4 == 0:
        tiles = torch.empty(int(_lib.lib().bsp_conduction_tile_flags_bytes(nx, ny, nz)),
                            dtype=torch.uint8, device=mat.device)
        call("bsp_conduction_tile_flags", ptr(tiles), ptr(cls), nx, ny, nz,
             stream_handle(stream))
    return CellClasses(cls, patterns, int(n.value), tiles)


def _check_f32(*ts):
    for t in ts:
        if isinstance(t, torch.Tensor) and (t.dtype != torch.float32 or not t.is_contiguous()):
            raise TypeError("temperature fields must be contiguous float32 CUDA tensors")


def apply_implicit_conduction_update(T_dst, T_iter, T_old, mat, k_arr, rho_arr, cp_arr,
                                     dx: float, dt: float, h_conv_air: float, T_amb_k: float,
                                     mat_air: int = MAT_AIR, mat_fluid: int = MAT_FLUID,
                                     stream=None) -> None:
    """One Jacobi sweep of the backward-Euler system (thermal.py:259-388).

    ``mat`` is the int32 material grid or its uint8 copy (``material_ids``);
    ``mat_fluid`` is accepted for signature parity and unused, as in the
    reference kernel."""
    del mat_fluid
    _check_f32(T_dst, T_iter, T_old)
    nx, ny, nz = T_dst.shape
    fn = "bsp_conduction_sweep_u8" if mat.dtype == torch.uint8 else "bsp_conduction_sweep"
    call(fn, ptr(T_dst), ptr(T_iter), ptr(T_old), ptr(mat), nx, ny, nz, ptr(k_arr),
         ptr(rho_arr), ptr(cp_arr), int(k_arr.shape[0]), float(dx), float(dt),
         float(h_conv_air), float(T_amb_k), int(mat_air), stream_handle(stream))


def implicit_conduction_step(grid, props: MaterialProps, ws: ThermalWorkspace, cfg, dt: float,
                             device: str = "cuda:0", stream=None) -> None:
    """The backward-Euler branch of ``conduct_one_step`` (thermal.py:647-658)."""
    del device
    _check_f32(grid.T, ws.T_iter_alt, ws.T_old_snapshot)
    nx, ny, nz = grid.shape
    T_amb_k = float(cfg.heating.ambient_temp_c + 273.15)
    h = float(cfg.solver.h_conv_outer_w_per_m2_k)
    n_iter = int(cfg.solver.diffusion_max_iter)
    props_args = (ptr(props.k_wp), ptr(props.rho_wp), ptr(props.cp_wp), props.n_mat)
    if getattr(grid, "classes", None) is None and props.n_mat <= 7:
        grid.classes = cell_classes(grid.mat, props.n_mat, MAT_AIR, stream) or False
    if grid.classes:
        c = grid.classes
        call("bsp_conduction_be_cls", ptr(grid.T), ptr(ws.T_iter_alt), ptr(ws.T_old_snapshot),
             ptr(c.cls), ptr(c.patterns), c.n_classes, ptr(c.tiles), nx, ny, nz, *props_args,
             float(grid.dx), float(dt), h, T_amb_k, MAT_AIR, n_iter, stream_handle(stream))
        return
    if getattr(grid, "mat_id", None) is None:
        grid.mat_id = material_ids(grid.mat, props.n_mat, stream)
    call("bsp_conduction_be_u8", ptr(grid.T), ptr(ws.T_iter_alt), ptr(ws.T_old_snapshot),
         ptr(grid.mat_id), nx, ny, nz, *props_args, float(grid.dx), float(dt), h, T_amb_k,
         MAT_AIR, n_iter, stream_handle(stream))
