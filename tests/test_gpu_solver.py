"""GPU tests of the to-tolerance solver (bsp_solve_tol) against the FP64 CPU
oracle: the FP64 residual of the returned iterate, the error against the FP64
oracle solve p*, storage variants, warm start, degenerate inputs."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle as O
from boilingsim_b200 import scenes as S
from boilingsim_b200.fluid import cell_mask
from boilingsim_b200.solver import TolSolver, solve_tolerance

pytestmark = pytest.mark.gpu

DX, DT, RHO = 0.002, 0.01, 997.0

COARSE_CLUSTER_DEFAULT = 16  # BSP_TUNE_COARSE_CLUSTER as the library starts


@pytest.fixture(scope="module")
def pot64():
    mat = S.pot_mat(S.POT_64)
    ux, uy, uz = S.velocity_field(mat, seed=7)
    div = O.divergence(ux, uy, uz, mat, DX)
    p_star, _, rel = O.solve_f64(div, mat, DX, DT, RHO, tol=1e-13)
    assert rel < 1e-12
    return mat, div, p_star


@pytest.mark.parametrize("storage,tol", [("fp32", 1e-6), ("fp32", 1e-9), ("fp16", 1e-6),
                                         ("bf16", 1e-6)])
def test_solve_reaches_fp64_residual(cuda, pot64, storage, tol):
    mat, div, p_star = pot64
    res = solve_tolerance(div, mat, DX, DT, RHO, tol=tol, storage=storage)
    assert res.status == 0
    rel = O.rel_residual64(res.p64, div, mat, DX, DT, RHO)
    # the device's FP64 residual agrees with the oracle's evaluation
    assert rel <= tol * 1.0001 and abs(rel - res.rel_residual) <= 1e-3 * rel + 1e-15
    err = O.rel_error(res.p64, p_star, mat)
    assert err < 50 * tol
    # the float output is the FP64 iterate rounded
    p32 = res.p.cpu().numpy()
    assert np.array_equal(p32, np.where(mat == 0, res.p64, 0.0).astype(np.float32))
    assert res.levels >= 3
    assert res.inner_iterations < 120


def test_warm_start_from_solution_needs_no_inner_work(cuda, pot64):
    mat, div, p_star = pot64
    mat_t = torch.as_tensor(mat).cuda()
    solver = TolSolver(cell_mask(mat_t))
    div_t = torch.as_tensor(div).cuda()
    p0 = torch.as_tensor(p_star.astype(np.float32)).cuda()
    res = solver.solve(div_t, DX, DT, RHO, tol=1e-5, p=p0, warm_start=True)
    assert res.status == 0 and res.inner_iterations == 0


def test_zero_rhs_gives_zero_pressure(cuda, pot64):
    mat, div, _ = pot64
    res = solve_tolerance(np.zeros_like(div), mat, DX, DT, RHO, tol=1e-6)
    assert res.status == 0 and res.inner_iterations == 0
    assert not res.p.cpu().numpy().any()


def test_not_converged_is_reported(cuda, pot64):
    mat, div, _ = pot64
    res = solve_tolerance(div, mat, DX, DT, RHO, tol=1e-12, max_outer=1, max_inner=2,
                          raise_on_fail=False)
    assert res.status == 10005 and res.rel_residual > 1e-12


@pytest.mark.parametrize("storage", ["fp32", "fp16"])
def test_column_and_row_level0_kernels_agree(cuda, pot64, storage):
    """The level-0 column kernels and the per-row kernels implement the same
    V-cycle and CG steps (FP32 sums in a different order): same convergence."""
    from boilingsim_b200 import _lib

    mat, div, p_star = pot64
    out = {}
    try:
        for col in (1, 0):
            _lib.call("bsp_set_tuning", 2, col)
            res = solve_tolerance(div, mat, DX, DT, RHO, tol=1e-7, storage=storage)
            assert res.status == 0
            out[col] = res
    finally:
        _lib.call("bsp_set_tuning", 2, 1)
    slack = 2 if storage == "fp32" else max(3, out[0].inner_iterations // 8)
    assert abs(out[1].inner_iterations - out[0].inner_iterations) <= slack
    assert O.rel_error(out[1].p64, out[0].p64, mat) < 1e-5


@pytest.mark.parametrize("storage", ["fp32", "fp16", "bf16"])
@pytest.mark.parametrize("spec", [S.POT_64, S.PotSpec(66, 50, 80, 20, 3, 60, 5, 20)],
                         ids=["pot64", "ny50_nz80"])
def test_tma_and_shared_plane_kernels_bit_identical(cuda, storage, spec):
    """The TMA-fed column kernels and the load-per-thread ones compute the same
    operations in the same order: bit-identical iterates and counts."""
    from boilingsim_b200 import _lib

    mat = S.pot_mat(spec)
    ux, uy, uz = S.velocity_field(mat, seed=5)
    div = O.divergence(ux, uy, uz, mat, DX)
    out = {}
    try:
        for tma in (1, 0):
            _lib.call("bsp_set_tuning", 4, tma)
            res = solve_tolerance(div, mat, DX, DT, RHO, tol=1e-7, storage=storage)
            assert res.status == 0
            out[tma] = (res.inner_iterations, res.outer_iterations, res.p64.copy())
    finally:
        _lib.call("bsp_set_tuning", 4, 1)
    assert out[1][:2] == out[0][:2]
    assert np.array_equal(out[1][2], out[0][2])


@pytest.mark.parametrize("storage", ["fp32", "fp16", "bf16"])
@pytest.mark.parametrize("spec", [S.POT_64, S.PotSpec(66, 50, 80, 20, 3, 60, 5, 20)],
                         ids=["pot64", "ny50_nz80"])
def test_update_fused_into_restriction_matches_separate_update(cuda, storage, spec):
    """The CG update applied inside the next level-0 restriction computes the
    same r and e values as the separate update kernel (only the FP64 sum of
    ||r||^2 runs in another order): same iteration counts and iterate."""
    from boilingsim_b200 import _lib

    mat = S.pot_mat(spec)
    ux, uy, uz = S.velocity_field(mat, seed=4)
    div = O.divergence(ux, uy, uz, mat, DX)
    out = {}
    try:
        for fuse in (1, 0):
            _lib.call("bsp_set_tuning", 6, fuse)
            res = solve_tolerance(div, mat, DX, DT, RHO, tol=1e-7, storage=storage)
            assert res.status == 0
            assert O.rel_residual64(res.p64, div, mat, DX, DT, RHO) <= 1e-7 * 1.0001
            out[fuse] = (res.inner_iterations, res.outer_iterations, res.p64.copy())
    finally:
        _lib.call("bsp_set_tuning", 6, 1)
    assert out[1][:2] == out[0][:2]
    assert np.array_equal(out[1][2], out[0][2])


@pytest.mark.parametrize("storage", ["fp32", "bf16"])
@pytest.mark.parametrize("spec", [S.POT_64, S.pot_192(3)], ids=["pot64", "pot192"])
def test_fused_coarse_cycle_matches_per_level_kernels(cuda, storage, spec):
    """The one-launch coarse V-cycle (cooperative kernel) and the per-level
    kernels apply the same operator (sums in another order): same convergence
    and the same solution to the tolerance."""
    from boilingsim_b200 import _lib

    mat = S.pot_mat(spec)
    ux, uy, uz = S.velocity_field(mat, seed=9)
    div = O.divergence(ux, uy, uz, mat, DX)
    out = {}
    try:
        _lib.call("bsp_set_tuning", 15, 0)  # every coarse level in the one launch
        for fused in (1, 0):
            _lib.call("bsp_set_tuning", 5, fused)
            res = solve_tolerance(div, mat, DX, DT, RHO, tol=1e-7, storage=storage)
            assert res.status == 0
            assert O.rel_residual64(res.p64, div, mat, DX, DT, RHO) <= 1e-7 * 1.0001
            out[fused] = res
    finally:
        _lib.call("bsp_set_tuning", 5, 1)
        _lib.call("bsp_set_tuning", 15, 3)
    slack = 2 if storage == "fp32" else max(3, out[0].inner_iterations // 8)
    assert abs(out[1].inner_iterations - out[0].inner_iterations) <= slack
    assert O.rel_error(out[1].p64, out[0].p64, mat) < 1e-5


@pytest.mark.parametrize("spec", [S.pot_192(2), S.PotSpec(70, 54, 37, 22, 3, 29, 5, 20),
                                  S.PotSpec(66, 50, 44, 20, 3, 33, 5, 20)],
                         ids=["pot192", "odd70x54x37", "odd_ny66x50x44"])
def test_solve_other_shapes(cuda, spec):
    mat = S.pot_mat(spec)
    ux, uy, uz = S.velocity_field(mat, seed=11)
    div = O.divergence(ux, uy, uz, mat, DX)
    res = solve_tolerance(div, mat, DX, DT, RHO, tol=1e-6)
    assert res.status == 0
    assert O.rel_residual64(res.p64, div, mat, DX, DT, RHO) <= 1e-6


def test_autotune_solve_keeps_a_working_choice(cuda):
    """The autotuner times every plane chunk x coarse-cycle candidate on the
    problem, keeps the fastest, and solves afterwards still meet the
    tolerance (the setup is rebuilt for the new tile geometry)."""
    from boilingsim_b200 import _lib

    mat = S.pot_mat(S.pot_192(3))
    ux, uy, uz = S.velocity_field(mat, seed=3)
    div = O.divergence(ux, uy, uz, mat, DX)
    solver = TolSolver(cell_mask(torch.as_tensor(mat).cuda()), "fp16")
    d = torch.as_tensor(div).cuda()
    try:
        rows = solver.autotune(d, DX, DT, RHO, tol=1e-6)
        assert len(rows) == 14 and all(r["status"] == 0 for r in rows)
        assert all(r["ms"] > 0 for r in rows)
        res = solver.solve(d, DX, DT, RHO, tol=1e-6)
        assert res.status == 0
        assert O.rel_residual64(res.p64, div, mat, DX, DT, RHO) <= 1e-6
    finally:
        _lib.call("bsp_set_tuning", 7, 0)
        _lib.call("bsp_set_tuning", 5, 1)


@pytest.mark.parametrize("size", [96, 192])
def test_coarse_cycle_fused_phases_bit_identical(cuda, size):
    """The one-launch coarse V-cycle with t formed where it is read (fused
    phases, fewer grid barriers; BSP_TUNE_COARSE_PHASES = 1) gives the same
    bits as with t stored in phases of its own (= 0, the default)."""
    from boilingsim_b200 import _lib

    spec = S.PotSpec(size, size, size * 2 // 3, r_in=size / 2 - 4, t_w=2,
                     water_line=size * 0.5, carrot_r=4, carrot_len=size // 3)
    mat = S.pot_mat(spec)
    ux, uy, uz = S.velocity_field(mat, seed=5)
    div = O.divergence(ux, uy, uz, mat, DX)
    out = {}
    try:
        for fused in (0, 1):
            _lib.call("bsp_set_tuning", 12, fused)
            res = solve_tolerance(div, mat, DX, DT, RHO, tol=1e-6, storage="fp16")
            out[fused] = (res.p64.copy(), res.inner_iterations, res.rel_residual)
    finally:
        _lib.call("bsp_set_tuning", 12, 0)
    assert out[0][1] == out[1][1]
    assert np.array_equal(out[0][0], out[1][0])
    assert O.rel_residual64(out[1][0], div, mat, DX, DT, RHO) <= 1.0001e-6


@pytest.mark.parametrize("storage,size", [("fp16", 96), ("fp32", 192), ("bf16", 192)])
def test_coarse_cycle_tail_in_shared_memory_bit_identical(cuda, storage, size):
    """The levels CTA 0 runs alone, staged in its shared memory
    (BSP_TUNE_COARSE_TAIL = 1), give the same bits as the same phases on
    global memory (= 0, the default)."""
    from boilingsim_b200 import _lib

    spec = S.PotSpec(size, size, size * 2 // 3, r_in=size / 2 - 4, t_w=3,
                     water_line=size * 0.45, carrot_r=5, carrot_len=size // 3)
    mat = S.pot_mat(spec)
    ux, uy, uz = S.velocity_field(mat, seed=9)
    div = O.divergence(ux, uy, uz, mat, DX)
    out = {}
    try:
        _lib.call("bsp_set_tuning", 24, 0)  # the cooperative kernel, where the option lives
        for tail in (0, 1):
            _lib.call("bsp_set_tuning", 14, tail)
            res = solve_tolerance(div, mat, DX, DT, RHO, tol=1e-6, storage=storage)
            out[tail] = (res.p64.copy(), res.inner_iterations)
    finally:
        _lib.call("bsp_set_tuning", 14, 0)
        _lib.call("bsp_set_tuning", 24, COARSE_CLUSTER_DEFAULT)
    assert out[0][1] == out[1][1]
    assert np.array_equal(out[0][0], out[1][0])
    assert O.rel_residual64(out[1][0], div, mat, DX, DT, RHO) <= 1.0001e-6


@pytest.mark.parametrize("storage,size", [("fp16", 96), ("fp32", 192), ("fp16", 192)])
def test_coarse_cycle_in_one_cluster_bit_identical(cuda, storage, size):
    """The coarse cycle run by one thread-block cluster with hardware cluster
    barriers (BSP_TUNE_COARSE_CLUSTER = 8 or 16 CTAs), its smallest levels in
    CTA 0's shared memory or not (BSP_TUNE_CLUSTER_TAIL), in CTA 0 alone below
    0, 2048 or 16384 cells (BSP_TUNE_CLUSTER_TAIL_CELLS), gives the bits of
    the cooperative kernel over every SM (= 0), host-driven and in the
    device-driven graph: the same phases on the same quads, only spread over
    other CTAs."""
    from boilingsim_b200 import _lib

    spec = S.PotSpec(size, size, size * 2 // 3, r_in=size / 2 - 4, t_w=3,
                     water_line=size * 0.45, carrot_r=5, carrot_len=size // 3)
    mat = S.pot_mat(spec)
    ux, uy, uz = S.velocity_field(mat, seed=11)
    div = O.divergence(ux, uy, uz, mat, DX)
    out = {}
    try:
        for cl, tail, cells in ((0, 0, 2048), (8, 0, 2048), (16, 1, 2048), (16, 0, 2048),
                                (16, 0, 16384), (16, 0, 0)):
            _lib.call("bsp_set_tuning", 24, cl)
            _lib.call("bsp_set_tuning", 25, tail)
            _lib.call("bsp_set_tuning", 27, cells)
            for graph in (False, True):
                res = solve_tolerance(div, mat, DX, DT, RHO, tol=1e-6, storage=storage,
                                      graph=graph)
                assert res.status == 0
                out[cl, tail, cells, graph] = (res.p64.copy(), res.inner_iterations)
    finally:
        _lib.call("bsp_set_tuning", 24, COARSE_CLUSTER_DEFAULT)
        _lib.call("bsp_set_tuning", 25, 0)
        _lib.call("bsp_set_tuning", 27, 16384)
    for key, (p64, its) in out.items():
        assert its == out[0, 0, 2048, key[3]][1], key
        assert np.array_equal(p64, out[0, 0, 2048, key[3]][0]), key
    assert O.rel_residual64(out[16, 0, 2048, True][0], div, mat, DX, DT, RHO) <= 1.0001e-6


def test_coarse_split_level3_on_tile_kernels(cuda):
    """Level 3 on the tile kernels too (BSP_TUNE_COARSE_SPLIT = 3, the
    default; it applies where level 3 keeps 32-cell rows and 32 K cells, here
    a 256^3 pot) against the cluster cycle from level 3 (= 2): the same
    V-cycle with sums in another order -- the same convergence, the same
    solution to the tolerance."""
    from boilingsim_b200 import _lib

    spec = S.PotSpec(256, 256, 256, r_in=118, t_w=4, water_line=190, carrot_r=12,
                     carrot_len=80)
    mat = S.pot_mat(spec)
    ux, uy, uz = S.velocity_field(mat, seed=13)
    div = O.divergence(ux, uy, uz, mat, DX)
    out = {}
    try:
        for split in (3, 2):
            _lib.call("bsp_set_tuning", 15, split)
            res = solve_tolerance(div, mat, DX, DT, RHO, tol=1e-6, storage="fp16", graph=True)
            assert res.status == 0
            assert O.rel_residual64(res.p64, div, mat, DX, DT, RHO) <= 1e-6 * 1.0001
            out[split] = res
    finally:
        _lib.call("bsp_set_tuning", 15, 3)
    assert abs(out[3].inner_iterations - out[2].inner_iterations) <= 2
    assert O.rel_error(out[3].p64, out[2].p64, mat) < 1e-5


@pytest.mark.parametrize("storage", ["fp32", "fp16"])
def test_coarse_split_level1_on_tile_kernels(cuda, storage):
    """Level 1 on the column tile kernels with the one-launch cycle from level 2
    (BSP_TUNE_COARSE_SPLIT = 1; the default 3 also takes levels 2-3) applies the same V-cycle as the
    one launch over every coarse level (one sweep a side on level 1 in both;
    sums in another order): same convergence, the same solution to the
    tolerance, on a pot whose level 1 takes the column layout."""
    from boilingsim_b200 import _lib

    mat = S.pot_mat(S.pot_192(3))
    ux, uy, uz = S.velocity_field(mat, seed=9)
    div = O.divergence(ux, uy, uz, mat, DX)
    out = {}
    try:
        _lib.call("bsp_set_tuning", 17, 1)  # the same V-cycle in both arms
        for split in (1, 0):
            _lib.call("bsp_set_tuning", 15, split)
            res = solve_tolerance(div, mat, DX, DT, RHO, tol=1e-7, storage=storage)
            assert res.status == 0
            assert O.rel_residual64(res.p64, div, mat, DX, DT, RHO) <= 1e-7 * 1.0001
            out[split] = res
    finally:
        _lib.call("bsp_set_tuning", 15, 3)
        _lib.call("bsp_set_tuning", 17, 2)
    slack = 2 if storage == "fp32" else max(3, out[0].inner_iterations // 8)
    assert abs(out[1].inner_iterations - out[0].inner_iterations) <= slack
    assert O.rel_error(out[1].p64, out[0].p64, mat) < 1e-5


@pytest.mark.parametrize("storage", ["fp32", "fp16"])
def test_level1_two_sweeps_converge_faster(cuda, storage):
    """Two smoothing sweeps a side on level 1 (BSP_TUNE_L1_SWEEPS = 2, the
    default, split mode) keep the V-cycle symmetric positive definite: the
    solve meets the tolerance in no more inner iterations than with one
    sweep."""
    from boilingsim_b200 import _lib

    mat = S.pot_mat(S.pot_192(3))
    ux, uy, uz = S.velocity_field(mat, seed=9)
    div = O.divergence(ux, uy, uz, mat, DX)
    out = {}
    try:
        _lib.call("bsp_set_tuning", 15, 1)
        for sweeps in (1, 2):
            _lib.call("bsp_set_tuning", 17, sweeps)
            res = solve_tolerance(div, mat, DX, DT, RHO, tol=1e-7, storage=storage)
            assert res.status == 0
            assert O.rel_residual64(res.p64, div, mat, DX, DT, RHO) <= 1e-7 * 1.0001
            out[sweeps] = res
    finally:
        _lib.call("bsp_set_tuning", 17, 2)
        _lib.call("bsp_set_tuning", 15, 3)
    assert out[2].inner_iterations <= out[1].inner_iterations
    assert O.rel_error(out[2].p64, out[1].p64, mat) < 1e-5


@pytest.mark.parametrize("storage", ["fp32", "fp16"])
@pytest.mark.parametrize("spec", [S.POT_64, S.pot_192(3)], ids=["pot64", "pot192"])
def test_l0_trilinear_transfers_converge_faster(cuda, storage, spec):
    """Trilinear transfers between levels 0 and 1 (BSP_TUNE_L0_TRILINEAR = 1:
    the prolongation renormalised over the fluid parents, the restriction its
    transpose) keep the V-cycle symmetric positive definite: the solve meets
    the FP64 tolerance, in fewer inner iterations than with piecewise-constant
    transfers, and reaches the same pressure to the tolerance."""
    from boilingsim_b200 import _lib

    mat = S.pot_mat(spec)
    ux, uy, uz = S.velocity_field(mat, seed=8)
    div = O.divergence(ux, uy, uz, mat, DX)
    out = {}
    try:
        for tri in (0, 1):
            _lib.call("bsp_set_tuning", 19, tri)
            res = solve_tolerance(div, mat, DX, DT, RHO, tol=1e-7, storage=storage)
            assert res.status == 0
            assert O.rel_residual64(res.p64, div, mat, DX, DT, RHO) <= 1e-7 * 1.0001
            out[tri] = res
    finally:
        _lib.call("bsp_set_tuning", 19, 0)
    assert out[1].inner_iterations < out[0].inner_iterations
    assert O.rel_error(out[1].p64, out[0].p64, mat) < 1e-5


@pytest.mark.parametrize("storage", ["fp32", "fp16"])
def test_scalars_in_last_cta_match_one_block_kernels(cuda, pot64, storage):
    """The inner check, beta and alpha computed by the last CTA of the level-0
    kernel before each (BSP_TUNE_FUSE_SCALARS = 1) and by the one-block
    kernels (= 0, the default) apply the same updates to FP64 sums taken in
    another fixed order: the same iteration counts and the same pressure to
    FP64 rounding of the recurrences."""
    from boilingsim_b200 import _lib

    mat, div, _ = pot64
    out = {}
    try:
        for fuse in (1, 0):
            _lib.call("bsp_set_tuning", 21, fuse)
            for graph in (False, True):
                res = solve_tolerance(div, mat, DX, DT, RHO, tol=1e-7, storage=storage,
                                      graph=graph)
                assert res.status == 0
                out[fuse, graph] = res
    finally:
        _lib.call("bsp_set_tuning", 21, 0)
    for graph in (False, True):
        a, b = out[1, graph], out[0, graph]
        assert (a.inner_iterations, a.outer_iterations) == (b.inner_iterations, b.outer_iterations)
        assert O.rel_error(a.p64, b.p64, mat) < 1e-9


@pytest.mark.parametrize("storage", ["fp32", "fp16"])
def test_programmatic_dependent_launch_bit_identical(cuda, pot64, storage):
    """The tile and scalar kernels launched with programmatic dependent launch
    (BSP_TUNE_PDL = 1: each waits in griddepcontrol.wait for the kernel before
    it) compute exactly what the plainly serialised launches compute, host-
    driven and through the device-driven graph."""
    from boilingsim_b200 import _lib

    mat, div, _ = pot64
    out = {}
    try:
        for pdl in (1, 0):
            _lib.call("bsp_set_tuning", 23, pdl)
            for graph in (False, True):
                res = solve_tolerance(div, mat, DX, DT, RHO, tol=1e-7, storage=storage,
                                      graph=graph)
                assert res.status == 0
                out[pdl, graph] = res
    finally:
        _lib.call("bsp_set_tuning", 23, 1)
    for graph in (False, True):
        a, b = out[1, graph], out[0, graph]
        assert (a.inner_iterations, a.outer_iterations) == (b.inner_iterations, b.outer_iterations)
        assert np.array_equal(a.p64, b.p64)
