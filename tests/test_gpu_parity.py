"""GPU parity tests: the CUDA library, called through its C ABI, against the CPU
oracle (bit-exact for the FP32 stencil path) and, where built, against the
reference's own CUDA kernels compiled from source (oracle/_ref)."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

import oracle as O
from boilingsim_b200 import _lib, scenes as S
from boilingsim_b200._lib import call, ptr

pytestmark = pytest.mark.gpu


def dev(a, dt=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dt).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def mask_of(mat_t):
    nx, ny, nz = mat_t.shape
    m = torch.empty(mat_t.shape, dtype=torch.uint8, device="cuda")
    call("bsp_mask_from_mat", ptr(m), ptr(mat_t), nx, ny, nz, 0, 2, 0)
    return m


PARAMS = [(seed, shape) for seed, shape in S.PARITY_CASES] + [
    (7, (16, 16, 32)), (8, (12, 20, 64)), (9, (5, 7, 132))]  # column-kernel shapes


def _case(seed, shape):
    rng = np.random.default_rng(seed)
    mat, p_old, div = S.parity_random_grid(rng, shape)
    dx = float(rng.uniform(0.0005, 0.004))
    dt = float(rng.uniform(0.0001, 0.01))
    rho = float(rng.uniform(900.0, 1100.0))
    return mat, p_old, div, dx, dt, rho


@pytest.mark.parametrize("seed,shape", PARAMS)
def test_one_sweep_bit_exact_int32_and_mask(cuda, seed, shape):
    """Gate 1 of test_pressure_parity.py:112-156, tightened to bit equality:
    reference launcher (int32 mat) and the uint8-mask sweep both match the
    oracle bit for bit."""
    mat, p_old, div, dx, dt, rho = _case(seed, shape)
    want = O.jacobi_step(p_old, div, mat, dx, dt, rho)
    nx, ny, nz = shape
    m, p, d = dev(mat, torch.int32), dev(p_old), dev(div)
    out = torch.full(shape, 7.0, device="cuda")
    call("jacobi_pressure_launch", ptr(out), ptr(p), ptr(d), ptr(m), nx, ny, nz, dx, dt, rho, 0, 2)
    assert np.array_equal(bits(host(out)), bits(want))
    out2 = torch.full(shape, 7.0, device="cuda")
    call("bsp_jacobi_sweep", ptr(out2), ptr(p), ptr(d), ptr(mask_of(m)), nx, ny, nz, dx, dt, rho, 0)
    assert np.array_equal(bits(host(out2)), bits(want))


def test_one_sweep_misaligned_pointers_use_generic_path(cuda):
    """A field that does not start on a 16-byte boundary is still exact."""
    mat, p_old, div, dx, dt, rho = _case(3, (8, 16, 32))
    n = mat.size
    buf_p = torch.zeros(n + 1, device="cuda")
    buf_p[1:] = dev(p_old).ravel()
    buf_o = torch.zeros(n + 1, device="cuda")
    m, d = dev(mat, torch.int32), dev(div)
    call("bsp_jacobi_sweep", ptr(buf_o) + 4, ptr(buf_p) + 4, ptr(d), ptr(mask_of(m)), 8, 16, 32,
         dx, dt, rho, 0)
    got = host(buf_o)[1:].reshape(mat.shape)
    assert np.array_equal(bits(got), bits(O.jacobi_step(p_old, div, mat, dx, dt, rho)))


@pytest.mark.parametrize("n_iter", [200, 7])
def test_fixed_count_solve_single_carrot(cuda, n_iter):
    """Gate 2 of test_pressure_parity.py:159-224 (single-carrot pot at dx = 4 mm,
    rng 7, x0.05, 200 sweeps): the reference asks max_rel < 1e-4; the result
    here is bit-identical to the oracle.  Also the odd-count copy (7)."""
    mat = S.single_carrot_mat(0.004)
    assert mat.shape == (58, 58, 38)
    rng = np.random.default_rng(7)
    nx, ny, nz = mat.shape
    ux = rng.standard_normal((nx + 1, ny, nz)).astype(np.float32) * 0.05
    uy = rng.standard_normal((nx, ny + 1, nz)).astype(np.float32) * 0.05
    uz = rng.standard_normal((nx, ny, nz + 1)).astype(np.float32) * 0.05
    div = O.divergence(ux, uy, uz, mat, 0.004)
    want = O.pressure_solve(np.zeros_like(div), div, mat, 0.004, 0.01, 997.0, n_iter)
    m, d = dev(mat, torch.int32), dev(div)
    p = torch.zeros(mat.shape, device="cuda")
    tmp = torch.zeros_like(p)
    call("pressure_solve_launch", ptr(p), ptr(tmp), ptr(d), ptr(m), nx, ny, nz, 0.004, 0.01,
         997.0, n_iter, 0, 2)
    assert np.array_equal(bits(host(p)), bits(want))
    m8 = mask_of(m)
    for rhs_ws in (None, torch.zeros_like(p)):
        p2 = torch.zeros_like(p)
        tmp2 = torch.zeros_like(p)
        call("bsp_jacobi_solve", ptr(p2), ptr(tmp2), ptr(d), ptr(rhs_ws), ptr(m8), nx, ny, nz,
             0.004, 0.01, 997.0, n_iter, 0, 0)
        assert np.array_equal(bits(host(p2)), bits(want))


@pytest.mark.parametrize("shape,n_iter", [((20, 18, 32), 2), ((24, 50, 48), 5),
                                          ((9, 16, 144), 8), ((16, 16, 16), 3)])
def test_temporally_blocked_sweeps_bit_exact(cuda, shape, n_iter):
    """Pairs of sweeps fused into one pass (tblock 0 / 2) give the same bits as
    one sweep per pass (tblock 1) and as the oracle, from a random start that
    is not zero off fluid (the first sweep then runs alone)."""
    rng = np.random.default_rng(n_iter + shape[2])
    mat, p_old, div = S.parity_random_grid(rng, shape)
    dx, dt, rho = 0.002, 0.01, 997.0
    want = O.pressure_solve(p_old, div, mat, dx, dt, rho, n_iter)
    nx, ny, nz = shape
    m8 = mask_of(dev(mat, torch.int32))
    d = dev(div)
    for tblock in (0, 1, 2):
        p = dev(p_old)
        tmp = torch.zeros_like(p)
        rhs = torch.zeros_like(p)
        call("bsp_jacobi_solve", ptr(p), ptr(tmp), ptr(d), ptr(rhs), ptr(m8), nx, ny, nz, dx,
             dt, rho, n_iter, tblock, 0)
        assert np.array_equal(bits(host(p)), bits(want)), tblock
    flag = ctypes.c_int(-1)
    call("bsp_sweep2_error", ctypes.byref(flag))
    assert flag.value == 0


def _segment_mat(nz):
    """Rows of 128-cell k segments of the three kinds the ZNF sweep tells
    apart: no fluid cell (air, or air and solid), fluid without a solid face
    neighbour, and fluid beside solid."""
    mat = np.full((6, 10, nz), 2, np.int32)   # air
    mat[1:5, 2:5, 130:nz - 6] = 0                # fluid next to air only
    mat[1:5, 6, 3:100] = 0                       # fluid ...
    mat[1:5, 6, 100] = 1                         # ... beside a wall cell
    mat[2, 8, 10:40] = 3                         # solid among air: no fluid
    mat[3, 3, 60:70] = 0                         # a fluid pocket in segment 0
    mat[3, 3, 70] = 3
    return mat


@pytest.mark.parametrize("nz", [256, 200])
def test_znf_sweep_segment_shortcuts_bit_exact(cuda, nz):
    """The ZNF sweep's warp-uniform shortcuts (+0 for segments without fluid,
    raw neighbour sums where no fluid cell touches a solid one) give the bits
    of the oracle's sweeps, full and partial k segments (nz 256 and 200)."""
    mat = _segment_mat(nz)
    rng = np.random.default_rng(nz)
    div = rng.standard_normal(mat.shape).astype(np.float32) * 0.3
    p_old = rng.standard_normal(mat.shape).astype(np.float32)
    dx, dt, rho = 0.002, 0.01, 997.0
    nx, ny, _ = mat.shape
    want = O.pressure_solve(p_old, div, mat, dx, dt, rho, 6)
    m8 = mask_of(dev(mat, torch.int32))
    try:
        for prefetch in (0, 2, 3):  # BSP_TUNE_SWEEP_PREFETCH
            call("bsp_set_tuning", 26, prefetch)
            p = dev(p_old)
            tmp = torch.zeros_like(p)
            rhs = torch.zeros_like(p)
            call("bsp_jacobi_solve", ptr(p), ptr(tmp), ptr(dev(div)), ptr(rhs), ptr(m8), nx, ny,
                 nz, dx, dt, rho, 6, 1, 0)
            assert np.array_equal(bits(host(p)), bits(want)), prefetch
    finally:
        call("bsp_set_tuning", 26, 2)


@pytest.mark.parametrize("spec", [S.POT_64, S.PotSpec(40, 36, 30, 14, 2, 24, 4, 12)],
                         ids=["pot64", "pot40x36x30"])
def test_full_projection_bit_exact(cuda, spec):
    """fluid.py:612-734 end to end (zero p, divergence, 200 sweeps, gradient
    subtract, diagnostic divergence) vs the oracle: p, u and max|div| equal."""
    mat = S.pot_mat(spec)
    ux, uy, uz = S.velocity_field(mat, seed=7)
    want = O.projection_jacobi(ux, uy, uz, mat, 0.002, 0.01, 997.0, 200)
    nx, ny, nz = mat.shape
    m = mask_of(dev(mat, torch.int32))
    U = [dev(a) for a in (ux, uy, uz)]
    p = torch.full(mat.shape, 3.0, device="cuda")
    tmp = torch.full(mat.shape, 3.0, device="cuda")
    div = torch.zeros(mat.shape, device="cuda")
    mx = torch.zeros(1, device="cuda")
    call("bsp_projection_jacobi", ptr(p), ptr(tmp), ptr(div), *[ptr(u) for u in U], ptr(m), nx,
         ny, nz, 0.002, 0.01, 997.0, 200, 0, ptr(mx), 0)
    assert np.array_equal(bits(host(p)), bits(want["p"]))
    for got, key in zip(U, ("ux", "uy", "uz")):
        assert np.array_equal(bits(host(got)), bits(want[key])), key
    assert np.array_equal(bits(host(div)), bits(want["div"]))
    assert float(host(mx)[0]) == want["max_div"]


def test_pressure_projection_python_api(cuda, monkeypatch):
    """The host mirror of pressure_projection (default 'jacobi' back-end)
    returns the oracle's max|div| and pressure."""
    from boilingsim_b200 import fluid as F

    monkeypatch.delenv("BOILINGSIM_PRESSURE_SOLVER", raising=False)
    monkeypatch.delenv("BOILINGSIM_USE_RUST_PRESSURE", raising=False)
    mat = S.pot_mat(S.POT_64)
    ux, uy, uz = S.velocity_field(mat, seed=3)
    want = O.projection_jacobi(ux, uy, uz, mat, 0.002, 0.01, 997.0, 200)
    grid = F.Grid.from_numpy(mat, ux, uy, uz, 0.002)
    ws = F.allocate_fluid_workspace(grid)
    got = F.pressure_projection(grid, ws, F.ScenarioConfig(), dt=0.01, rho=997.0)
    assert got == want["max_div"]
    assert np.array_equal(bits(host(grid.p)), bits(want["p"]))
    monkeypatch.setenv("BOILINGSIM_USE_RUST_PRESSURE", "1")
    grid2 = F.Grid.from_numpy(mat, ux, uy, uz, 0.002)
    got2 = F.pressure_projection(grid2, F.allocate_fluid_workspace(grid2), F.ScenarioConfig(),
                                 dt=0.01, rho=997.0)
    assert got2 == want["max_div"]


@pytest.mark.parametrize("seed,shape", [(11, (14, 12, 18)), (12, (9, 20, 13)), (13, (8, 8, 64))])
def test_spmv_and_diag_bit_exact(cuda, seed, shape):
    rng = np.random.default_rng(seed)
    mat, p, _ = S.parity_random_grid(rng, shape)
    mat[0, 3, 4] = 0
    nx, ny, nz = shape
    m, pp = dev(mat, torch.int32), dev(p)
    out = torch.zeros(shape, device="cuda")
    call("laplacian_spmv_launch", ptr(out), ptr(pp), ptr(m), nx, ny, nz, 0, 2)
    assert np.array_equal(bits(host(out)), bits(O.spmv(p, mat, fused=True)))
    out2 = torch.zeros(shape, device="cuda")
    call("bsp_spmv", ptr(out2), ptr(pp), ptr(mask_of(m)), nx, ny, nz, 0)
    assert np.array_equal(bits(host(out2)), bits(O.spmv(p, mat, fused=True)))
    z = torch.zeros(shape, device="cuda")
    call("diag_inverse_apply_launch", ptr(z), ptr(pp), ptr(m), nx, ny, nz, 0, 2)
    assert np.array_equal(bits(host(z)), bits(O.diag_inverse(p, mat)))


@pytest.mark.parametrize("spec", [S.PotSpec(24, 20, 28, 8, 2, 20, 3, 8),
                                  S.PotSpec(24, 20, 30, 8, 2, 20, 3, 8),
                                  S.PotSpec(16, 40, 132, 6, 2, 100, 3, 6)],
                         ids=["four-cell", "one-cell", "four-cell-partial"])
def test_divergence_gradient_no_slip_bit_exact(cuda, spec):
    """Divergence (with max|div|), gradient subtraction and no-slip against the
    oracle, bit for bit: nz % 4 == 0 takes the four-cell kernels (a partial
    last block of k quads at nz = 132), nz = 30 the one-cell ones."""
    mat = S.pot_mat(spec)
    rng = np.random.default_rng(4)
    nx, ny, nz = mat.shape
    ux = rng.standard_normal((nx + 1, ny, nz)).astype(np.float32)
    uy = rng.standard_normal((nx, ny + 1, nz)).astype(np.float32)
    uz = rng.standard_normal((nx, ny, nz + 1)).astype(np.float32)
    p = rng.standard_normal(mat.shape).astype(np.float32)
    m = mask_of(dev(mat, torch.int32))
    U = [dev(a) for a in (ux, uy, uz)]
    div = torch.zeros(mat.shape, device="cuda")
    mx = torch.zeros(1, device="cuda")
    call("bsp_divergence", ptr(div), *[ptr(u) for u in U], ptr(m), nx, ny, nz, 0.003, ptr(mx), 0)
    want = O.divergence(ux, uy, uz, mat, 0.003)
    assert np.array_equal(bits(host(div)), bits(want))
    assert float(host(mx)[0]) == float(np.abs(want).max())
    p_d = dev(p)  # keep device buffers referenced while the kernel may run
    call("bsp_subtract_gradient", *[ptr(u) for u in U], ptr(p_d), ptr(m), nx, ny, nz, 0.003,
         0.01, 997.0, 0)
    wg = O.subtract_gradient(ux, uy, uz, p, mat, 0.003, 0.01, 997.0)
    for got, w in zip(U, wg):
        assert np.array_equal(bits(host(got)), bits(w))
    call("bsp_enforce_no_slip", *[ptr(u) for u in U], ptr(m), nx, ny, nz, 0)
    wn = O.enforce_no_slip(*wg, mat)
    for got, w in zip(U, wn):
        assert np.array_equal(bits(host(got)), bits(w))


def test_empty_sizes_are_noops(cuda):
    x = torch.ones(4, device="cuda")
    for nx, ny, nz in [(0, 4, 4), (4, 0, 4), (4, 4, 0), (-1, 2, 2)]:
        call("jacobi_pressure_launch", ptr(x), ptr(x), ptr(x), ptr(x), nx, ny, nz, 1.0, 1.0, 1.0,
             0, 2)
        call("pressure_solve_launch", ptr(x), ptr(x), ptr(x), ptr(x), nx, ny, nz, 1.0, 1.0, 1.0,
             5, 0, 2)
    call("pressure_solve_launch", ptr(x), ptr(x), ptr(x), ptr(x), 2, 2, 1, 1.0, 1.0, 1.0, 0, 0, 2)
    call("dot_launch", ptr(x), ptr(x), 0, ptr(x), ptr(x))
    assert host(x)[0] == 0.0  # n = 0 dot writes 0 to the result


def test_native_entry_points_reject_bad_arguments(cuda):
    x = torch.zeros(64, device="cuda")
    with pytest.raises(_lib.BspError) as e:
        call("bsp_jacobi_sweep", 0, ptr(x), ptr(x), ptr(x), 4, 4, 4, 1.0, 1.0, 1.0, 0)
    assert e.value.code == 10002
    with pytest.raises(_lib.BspError) as e:
        call("bsp_jacobi_sweep", ptr(x), ptr(x), ptr(x), ptr(x), 4, 4, 4, 1.0, 1.0, 1.0, 0)
    assert e.value.code == 10003


def test_dot_fp64_deterministic(cuda):
    rng = np.random.default_rng(0)
    n = 1_000_003
    x = rng.standard_normal(n).astype(np.float32)
    y = rng.standard_normal(n).astype(np.float32)
    ws = torch.zeros(1024, device="cuda")
    res = torch.zeros(1, device="cuda")
    xd, yd = dev(x), dev(y)
    call("dot_launch", ptr(xd), ptr(yd), n, ptr(ws), ptr(res))
    want = float(np.dot(x.astype(np.float64), y.astype(np.float64)))
    assert abs(float(host(res)[0]) - want) <= 1e-6 * abs(want) + 1e-3


def test_div6_exhaustive(cuda):
    """The 3-instruction division by 6 equals IEEE division on all 2^32 inputs."""
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    call("bsp_selftest_div6", ptr(cnt), 0)
    assert int(host(cnt)[0]) == 0


def _run_pcg(mat, div, dx, dt, rho, tol, max_iter):
    nx, ny, nz = mat.shape
    z = lambda *s: torch.zeros(s, dtype=torch.float32, device="cuda")  # noqa: E731
    p = z(nx, ny, nz)
    ws = [z(nx, ny, nz) for _ in range(5)] + [z(1024)] + [z(1) for _ in range(7)]
    it = ctypes.c_int(-1)
    div_d, mat_d = dev(div), dev(mat, torch.int32)
    call("pressure_solve_pcg_launch", ptr(p), ptr(div_d), ptr(mat_d), nx, ny,
         nz, dx, dt, rho, 0, 2, tol, max_iter, *[ptr(w) for w in ws], ctypes.byref(it))
    return host(p), it.value, float(host(ws[10])[0])


def test_pcg_matches_oracle_pcg(cuda):
    """Same algorithm and FP64 inner products as the oracle PCG: the iteration
    count agrees within one check period and the solutions agree to the
    tolerance scale."""
    mat = S.pot_mat(S.POT_64)
    ux, uy, uz = S.velocity_field(mat, seed=7)
    div = O.divergence(ux, uy, uz, mat, 0.002)
    p, it, _ = _run_pcg(mat, div, 0.002, 0.01, 997.0, 1e-5, 2000)
    po, ito = O.pcg(div, mat, 0.002, 0.01, 997.0, 1e-5, 2000)
    assert abs(it - ito) <= 5
    p_star, _, _ = O.solve_f64(div, mat, 0.002, 0.01, 997.0, tol=1e-12)
    assert O.rel_error(p, p_star, mat) < 1e-4
    assert O.rel_residual(p, div, mat, 0.002, 0.01, 997.0) < 3e-5


def test_pcg_gates(cuda):
    """test_pressure_cg.py gates: sign (p > 0 under negative div), bsq with
    max_iter = 0 (rel < 1e-4 vs numpy), tolerance contract."""
    mat = np.zeros((8, 8, 16), np.int32)
    mat[:, :, 0] = 2
    mat[:, :, -1] = 2
    div = np.zeros(mat.shape, np.float32)
    div[:, :, 4:12] = -1e-3
    p, it, _ = _run_pcg(mat, div, 0.002, 0.001, 997.0, 1e-5, 200)
    assert it > 0 and np.all(p[:, :, 4:12] > 0)
    rng = np.random.default_rng(3)
    div2 = (rng.standard_normal(mat.shape) * 1e-3).astype(np.float32)
    _, it0, bsq = _run_pcg(mat, div2, 0.002, 0.001, 997.0, 1e-5, 0)
    b = O.rhs_f64(div2, mat, 0.002, 0.001, 997.0)
    assert it0 == 0 and abs(bsq - float((b * b).sum())) <= 1e-4 * float((b * b).sum())
    mat3 = np.zeros((16, 16, 24), np.int32)
    mat3[:, :, 0] = 2
    mat3[:, :, -1] = 2
    div3 = (np.random.default_rng(42).standard_normal(mat3.shape) * 5e-3).astype(np.float32)

    def res_inf(pp):
        bb = O.rhs_f64(div3, mat3, 0.002, 0.001, 997.0)
        return np.abs(O.apply_A_f64(pp.astype(np.float64), mat3) - bb).max() / np.abs(bb).max()

    pl, _, _ = _run_pcg(mat3, div3, 0.002, 0.001, 997.0, 1e-2, 200)
    pt, _, _ = _run_pcg(mat3, div3, 0.002, 0.001, 997.0, 1e-6, 200)
    assert res_inf(pt) < 0.5 * res_inf(pl) and res_inf(pt) < 1e-3
    # zero right-hand side: zero iterations, p = 0
    p0, it0, _ = _run_pcg(mat3, np.zeros_like(div3), 0.002, 0.001, 997.0, 1e-6, 200)
    assert it0 == 0 and not p0.any()


@pytest.mark.skipif(O.ref_library(True) is None, reason="reference CUDA not built (oracle/_ref)")
@pytest.mark.parametrize("seed,shape", PARAMS)
def test_against_reference_cuda_kernel(cuda, seed, shape):
    """The reference's own jacobi_pressure.cu (built from source, FMA on and
    off) and this library give identical bits on the parity grids."""
    mat, p_old, div, dx, dt, rho = _case(seed, shape)
    nx, ny, nz = shape
    m, p, d = dev(mat, torch.int32), dev(p_old), dev(div)
    ours = torch.zeros(shape, device="cuda")
    call("jacobi_pressure_launch", ptr(ours), ptr(p), ptr(d), ptr(m), nx, ny, nz, dx, dt, rho, 0, 2)
    for fma in (True, False):
        L = O.ref_library(fma)
        P_, I_, F_ = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
        L.jacobi_pressure_launch.argtypes = [P_, P_, P_, P_, I_, I_, I_, F_, F_, F_, I_, I_]
        ref = torch.zeros(shape, device="cuda")
        assert L.jacobi_pressure_launch(ptr(ref), ptr(p), ptr(d), ptr(m), nx, ny, nz, dx, dt, rho,
                                        0, 2) == 0
        assert np.array_equal(bits(host(ref)), bits(host(ours)))


def test_autotune_jacobi_choice_stays_bit_exact(cuda):
    """After the sweep autotuner (plane chunk x sweeps per pass) the default
    solve uses its choice and still matches the oracle bit for bit."""
    from boilingsim_b200 import fluid as F

    mat = S.pot_mat(S.POT_64)
    ux, uy, uz = S.velocity_field(mat, seed=5)
    grid = F.Grid.from_numpy(mat, ux, uy, uz, 0.002)
    ws = F.allocate_fluid_workspace(grid)
    try:
        rows = F.autotune_jacobi(grid, ws, 0.01, 997.0, sweeps=10)
        assert len(rows) == 12 and all(r["status"] == 0 for r in rows)
        want = O.projection_jacobi(ux, uy, uz, mat, 0.002, 0.01, 997.0, 20)
        cfg = F.ScenarioConfig(F.SolverConfig(pressure_max_iter=20))
        F.pressure_projection(grid, ws, cfg, 0.01, 997.0)
        assert np.array_equal(bits(host(grid.p)), bits(want["p"]))
    finally:
        call("bsp_set_tuning", 1, 0)
        call("bsp_set_tuning", 8, 1)
