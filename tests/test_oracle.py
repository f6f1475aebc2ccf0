"""CPU tests of the oracle: known answers from the reference's tests, golden
vectors produced by the reference's own CUDA kernels, and solver sanity."""
from __future__ import annotations

import glob
import os

import numpy as np
import pytest

import oracle as O
from boilingsim_b200 import scenes as S

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_analytic_linear_and_quadratic_fields():
    """python/tests/test_pressure_cg.py:62-69: A(i+j+k) = 0 and A(i^2) = -2 at
    interior all-fluid cells."""
    shape = (10, 9, 12)
    mat = np.zeros(shape, np.int32)
    for fused in (True, False):
        a = O.spmv(O.analytic_linear_field(shape), mat, fused=fused)
        assert np.abs(a[1:-1, 1:-1, 1:-1]).max() == 0.0
        a = O.spmv(O.analytic_quadratic_field(shape), mat, fused=fused)
        assert np.all(a[1:-1, 1:-1, 1:-1] == -2.0)
    a64 = O.apply_A_f64(O.analytic_quadratic_field(shape).astype(np.float64), mat)
    assert np.all(a64[1:-1, 1:-1, 1:-1] == -2.0)


def test_jacobi_fixed_point_is_the_linear_system():
    """laplacian_spmv.cu:12-20: a Jacobi fixed point satisfies A p = b."""
    rng = np.random.default_rng(5)
    mat, _, div = S.parity_random_grid(rng, (12, 10, 14))
    p, it, rel = O.solve_f64(div, mat, 0.002, 0.01, 997.0, tol=1e-13)
    assert rel < 1e-12
    pj = O.jacobi_step(p.astype(np.float32), div, mat, 0.002, 0.01, 997.0)
    f = mat == 0
    assert np.max(np.abs(pj[f] - p[f])) <= 1e-5 * max(1.0, np.abs(p).max())


def test_jacobi_reduces_divergence_walled_box():
    """test_fluid.py:118-144 shape: 16^3 walled box, rng 42, velocities x0.1,
    1500 sweeps; max|div| < 1e-3 and at least a 1000x reduction."""
    n = 16
    mat = np.full((n, n, n), 1, np.int32)  # _make_walled_grid: one-cell wall shell
    mat[1:-1, 1:-1, 1:-1] = 0
    rng = np.random.default_rng(42)
    ux = (rng.standard_normal((n + 1, n, n)) * 0.1).astype(np.float32)
    uy = (rng.standard_normal((n, n + 1, n)) * 0.1).astype(np.float32)
    uz = (rng.standard_normal((n, n, n + 1)) * 0.1).astype(np.float32)
    ux, uy, uz = O.enforce_no_slip(ux, uy, uz, mat)
    d0 = np.abs(O.divergence(ux, uy, uz, mat, 0.002)).max()
    out = O.projection_jacobi(ux, uy, uz, mat, 0.002, 0.01, 997.0, 1500)
    assert d0 > 1.0
    assert out["max_div"] < 1e-3
    assert out["max_div"] < d0 * 1e-3


def test_hydrostatic_box_stays_at_rest():
    """test_fluid.py:218-235: zero velocity stays zero through a projection."""
    mat = S.pot_mat(S.PotSpec(16, 16, 16, r_in=6, t_w=1, water_line=12, carrot_r=0,
                              carrot_len=0))
    z = lambda s: np.zeros(s, np.float32)  # noqa: E731
    out = O.projection_jacobi(z((17, 16, 16)), z((16, 17, 16)), z((16, 16, 17)), mat, 0.001,
                              0.01, 997.0, 50)
    assert out["max_div"] == 0.0
    assert np.abs(out["ux"]).max() < 1e-6


def test_pcg_sign_gate():
    """test_pressure_cg.py:49-156: 8x8x16 all-fluid box with air at k = 0 and
    k = -1 and div = -1e-3 on k in [4, 12) gives p > 0 there."""
    mat = np.zeros((8, 8, 16), np.int32)
    mat[:, :, 0] = 2
    mat[:, :, -1] = 2
    div = np.zeros((8, 8, 16), np.float32)
    div[:, :, 4:12] = -1e-3
    p, it = O.pcg(div, mat, 0.002, 0.001, 997.0, 1e-5, 200)
    assert it > 0
    assert np.all(p[:, :, 4:12] > 0)


def test_pcg_tolerance_contract():
    """test_pressure_cg.py:275-343: tight tolerance gives a smaller residual
    than a loose one (< 0.5x) and < 1e-3 in the inf-norm relative sense."""
    mat = np.zeros((16, 16, 24), np.int32)
    mat[:, :, 0] = 2
    mat[:, :, -1] = 2
    rng = np.random.default_rng(42)
    div = (rng.standard_normal(mat.shape) * 5e-3).astype(np.float32)
    dx, dt, rho = 0.002, 0.001, 997.0

    def res_inf(p):
        b = O.rhs_f64(div, mat, dx, dt, rho)
        ap = O.apply_A_f64(p.astype(np.float64), mat)
        return np.abs(ap - b).max() / np.abs(b).max()

    p_loose, _ = O.pcg(div, mat, dx, dt, rho, 1e-2, 200)
    p_tight, _ = O.pcg(div, mat, dx, dt, rho, 1e-6, 200)
    assert res_inf(p_tight) < 0.5 * res_inf(p_loose)
    assert res_inf(p_tight) < 1e-3


def test_fp64_oracle_solve_and_residual_floor_of_fp32():
    """The FP64 solve reaches 1e-12; rounding it to FP32 already costs a
    residual near 1e-6 on the 64x64x48 pot (why the tolerance solver keeps an
    FP64 iterate)."""
    mat = S.pot_mat(S.POT_64)
    ux, uy, uz = S.velocity_field(mat, seed=7)
    div = O.divergence(ux, uy, uz, mat, 0.002)
    p, it, rel = O.solve_f64(div, mat, 0.002, 0.01, 997.0, tol=1e-12)
    assert rel < 1e-11
    r32 = O.rel_residual(p.astype(np.float32), div, mat, 0.002, 0.01, 997.0)
    assert 1e-8 < r32 < 1e-5


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "sweep_*.npz"))))
def test_golden_one_sweep(path):
    """One Jacobi sweep of the reference's own CUDA kernel (built from
    jacobi_pressure.cu, FMA on and off) vs the oracle: bit-identical."""
    g = np.load(path)
    out = O.jacobi_step(g["p_old"], g["div"], g["mat"], float(g["dx"]), float(g["dt"]),
                        float(g["rho"]))
    for key in ("ref_fma", "ref_nofma"):
        if key in g:
            assert np.array_equal(out.view(np.uint32), g[key].view(np.uint32)), key


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "spmv_*.npz"))))
def test_golden_spmv_and_diag(path):
    """laplacian_spmv / diag_inverse_apply of the reference CUDA vs the oracle."""
    g = np.load(path)
    assert np.array_equal(O.spmv(g["p"], g["mat"], fused=True).view(np.uint32),
                          g["ap_fma"].view(np.uint32))
    assert np.array_equal(O.spmv(g["p"], g["mat"], fused=False).view(np.uint32),
                          g["ap_nofma"].view(np.uint32))
    assert np.array_equal(O.diag_inverse(g["p"], g["mat"]).view(np.uint32),
                          g["z"].view(np.uint32))


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "solve_*.npz"))))
def test_golden_fixed_count_solve(path):
    """pressure_solve_launch (n sweeps, odd-count copy) of the reference CUDA."""
    g = np.load(path)
    p = O.pressure_solve(g["p0"], g["div"], g["mat"], float(g["dx"]), float(g["dt"]),
                         float(g["rho"]), int(g["n_iter"]))
    assert np.array_equal(p.view(np.uint32), g["ref"].view(np.uint32))


def test_golden_vectors_present():
    """The reference-generated fixtures are committed (parity is pinned)."""
    assert glob.glob(os.path.join(GOLDEN, "sweep_*.npz")), "no golden sweep fixtures"


@pytest.mark.parametrize("name", ["pcg_box_0.01", "pcg_box_1e-06"])
def test_oracle_pcg_matches_reference_pcg_goldens(name):
    """The oracle's PCG against the reference's own pressure_solve_pcg_launch
    (pressure_solve_pcg.cu:89-243, run on a B200 from oracle/_ref by
    tests/golden/make_golden.py): the same iteration count (the check
    cadence, every 5 iterations from iteration 8, makes a one-check difference
    5 iterations) and the same pressure to within the FP32 PCG's own rounding
    (the reference sums its dot products in FP32, the oracle in FP64)."""
    d = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    dx, dt, rho, tol = (float(d[k]) for k in ("dx", "dt", "rho", "tol"))
    p, it = O.pcg(d["div"], d["mat"], dx, dt, rho, tol, 200)
    assert abs(it - int(d["iters"])) <= 5, (it, int(d["iters"]))
    fl = d["mat"] == 0
    ref = d["p"].astype(np.float64)
    err = np.linalg.norm(p[fl] - ref[fl]) / np.linalg.norm(ref[fl])
    assert err <= 1e-5, err
    # both stop below the tolerance on the true residual within FP32 rounding
    assert O.rel_residual(p, d["div"], d["mat"], dx, dt, rho) <= 1.5 * tol
    b = O.compute_b(d["div"], d["mat"], dx, dt, rho)
    assert O.dot_f64(b, b) == pytest.approx(float(d["bsq"]), rel=1e-6)


def test_oracle_cg_vector_ops_known_answers():
    """axpy_device.cu:20-99 and scale.cu:11-17 restated: fused multiply-add
    rounding (one rounding, as the reference's FMA build), the negated alpha,
    the den == 0 -> 0 rule of divide_scalars (axpy_device.cu:90)."""
    x = np.array([1.0, 3.0, -2.0, 1e8], np.float32)
    y = np.array([0.5, 1.0, 4.0, 1.0], np.float32)
    a = np.float32(1.0 / 3.0)
    got = O.axpy(y, x, a)
    want = (a.astype(np.float64) * x.astype(np.float64) + y.astype(np.float64)).astype(np.float32)
    assert np.array_equal(got, want)
    assert np.array_equal(O.axpy(y, x, a, negate=True), O.axpy(y, x, -a))
    assert np.array_equal(O.scaled_axpy(y, x, a), O.axpy(y, x, a))
    assert O.divide_scalars(3.0, 0.0) == 0.0
    assert O.divide_scalars(3.0, 2.0) == np.float32(1.5)
    assert np.array_equal(O.scale(x, 2.0), x * np.float32(2.0))
