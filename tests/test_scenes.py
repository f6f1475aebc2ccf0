"""CPU tests of the synthetic scene generators and the host-side solver
selection logic (no GPU calls)."""
from __future__ import annotations

import numpy as np
import pytest

from boilingsim_b200 import scenes as S


@pytest.mark.parametrize("spec", [S.POT_64, S.pot_192(2), S.pot_192(4)], ids=str)
def test_pot_mask_rules(spec):
    mat = S.pot_mat(spec)
    assert mat.shape == spec.shape and mat.dtype == np.int32
    f = mat == S.MAT_FLUID
    # fluid never touches the outer layer (the reference's pad, geometry.py:317-338)
    assert not f[0].any() and not f[-1].any() and not f[:, 0].any() and not f[:, -1].any()
    assert not f[:, :, 0].any() and not f[:, :, -1].any()
    # bottom wall below the cavity, air above the water line
    nx, ny = spec.nx // 2, spec.ny // 2
    assert mat[nx, ny, 0] == S.MAT_POT_WALL
    assert mat[nx, ny, spec.nz - 1] == S.MAT_AIR
    assert (mat == S.MAT_CARROT).sum() > 0
    assert set(np.unique(mat)) <= {0, 1, 2, 3}


def test_single_carrot_grid_dims():
    """compute_grid_dims for single_carrot.yaml at dx = 4 mm is 58x58x38."""
    assert S.compute_grid_dims(0.004, 0.20, 0.12)[:3] == (58, 58, 38)
    mat = S.single_carrot_mat(0.004)
    assert mat.shape == (58, 58, 38)
    assert (mat == S.MAT_CARROT).sum() > 0 and (mat == S.MAT_FLUID).sum() > 10000


def test_velocity_field_seeded_and_no_slip():
    mat = S.pot_mat(S.POT_64)
    a = S.velocity_field(mat, seed=7)
    b = S.velocity_field(mat, seed=7)
    c = S.velocity_field(mat, seed=8)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    assert not np.array_equal(a[0], c[0])
    ux, uy, uz = a
    assert ux.shape == (65, 64, 48) and uy.shape == (64, 65, 48) and uz.shape == (64, 64, 49)
    f = mat == 0
    # no-slip: faces touching a non-fluid cell are zero
    assert np.all(ux[1:-1][~(f[:-1] & f[1:])] == 0)
    assert np.all(uz[:, :, 0] == 0) and np.all(uz[:, :, -1] == 0)
    # plume: upward mean flow near the axis, below the carrot (k 15..27)
    assert uz[30:34, 30:34, 4:13].mean() > 0.05


def test_batch_specs_ranges():
    specs = S.random_batch_specs(64, seed=7)
    assert len(specs) == 64
    for spec, seed in specs:
        assert 48 <= spec.nx <= 128 and 48 <= spec.nz <= 96 and spec.nx == spec.ny
        frac = (spec.water_line - spec.t_w) / (spec.nz - spec.t_w)
        assert 0.6 <= frac <= 0.85


def test_parity_grid_generator_matches_reference_recipe():
    """test_pressure_parity.py:51-67: outer air ring, interior draws."""
    rng = np.random.default_rng(1)
    mat, p, div = S.parity_random_grid(rng, (16, 16, 16))
    assert np.all(mat[0] == 2) and np.all(mat[:, :, -1] == 2)
    frac = np.bincount(mat[1:-1, 1:-1, 1:-1].ravel(), minlength=4) / 14 ** 3
    assert abs(frac[0] - 0.6) < 0.05
    assert p.dtype == np.float32 and div.dtype == np.float32


def test_solver_selection(monkeypatch):
    from boilingsim_b200 import fluid as F

    monkeypatch.delenv("BOILINGSIM_PRESSURE_SOLVER", raising=False)
    monkeypatch.delenv("BOILINGSIM_USE_RUST_PRESSURE", raising=False)
    assert F._select_pressure_solver() == "jacobi"
    monkeypatch.setenv("BOILINGSIM_USE_RUST_PRESSURE", "1")
    assert F._select_pressure_solver() == "rust-jacobi"
    monkeypatch.setenv("BOILINGSIM_PRESSURE_SOLVER", "cg-rust")
    with pytest.raises(ValueError):
        F._select_pressure_solver()
    monkeypatch.delenv("BOILINGSIM_USE_RUST_PRESSURE")
    assert F._select_pressure_solver() == "cg-rust"
    monkeypatch.setenv("BOILINGSIM_PRESSURE_SOLVER", "bogus")
    with pytest.raises(ValueError):
        F._select_pressure_solver()


def test_simcore_size_checks():
    from boilingsim_b200 import sim_core

    with pytest.raises(RuntimeError):
        sim_core._check_i32(2 ** 31)
    sim_core._check_i32(0, 5, 2 ** 31 - 1)
