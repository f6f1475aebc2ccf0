"""GPU tests of the device-driven solve (one CUDA graph with conditional WHILE
nodes) and of the batched solve of uneven pot scenes (one graph launch)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle as O
from boilingsim_b200 import scenes as S
from boilingsim_b200.fluid import cell_mask
from boilingsim_b200.solver import BatchSolver, TolSolver

pytestmark = pytest.mark.gpu

DX, DT, RHO = 0.002, 0.01, 997.0


def _scene(spec, seed):
    mat = S.pot_mat(spec)
    ux, uy, uz = S.velocity_field(mat, seed=seed)
    return mat, O.divergence(ux, uy, uz, mat, DX)


@pytest.mark.parametrize("storage,spec", [("fp32", S.POT_64), ("fp16", S.POT_64),
                                          ("fp32", S.pot_192(3))],
                         ids=["pot64-fp32", "pot64-fp16", "pot192-fp32"])
def test_graph_solve_matches_host_driven_solve(cuda, storage, spec):
    """Same kernels in the same order: the graph-driven solve reproduces the
    host-driven one bit for bit, and replaying the graph does too.  The 192
    pot (nz % 4 == 0 on every level) runs the coarse levels as one cooperative
    kernel inside the graph's WHILE body."""
    mat, div = _scene(spec, 7)
    solver = TolSolver(cell_mask(torch.as_tensor(mat).cuda()), storage)
    d = torch.as_tensor(div).cuda()
    r1 = solver.solve(d, DX, DT, RHO, tol=1e-6)
    x1 = r1.p64_dev.clone()
    r2 = solver.solve(d, DX, DT, RHO, tol=1e-6, graph=True)
    x2 = r2.p64_dev.clone()
    r3 = solver.solve(d, DX, DT, RHO, tol=1e-6, graph=True)
    assert r1.status == r2.status == r3.status == 0
    assert r1.inner_iterations == r2.inner_iterations == r3.inner_iterations
    assert torch.equal(x1, x2) and torch.equal(x2, r3.p64_dev)
    assert O.rel_residual64(x2.cpu().numpy(), div, mat, DX, DT, RHO) <= 1e-6


def test_graph_solve_not_converged_terminates(cuda):
    """The WHILE loops end on the iteration caps even without convergence."""
    mat, div = _scene(S.POT_64, 8)
    solver = TolSolver(cell_mask(torch.as_tensor(mat).cuda()))
    res = solver.solve(torch.as_tensor(div).cuda(), DX, DT, RHO, tol=1e-14, max_outer=2,
                       max_inner=3, graph=True, raise_on_fail=False)
    assert res.status == 10005
    assert res.inner_iterations <= 2 * 3


def test_batched_uneven_scenes_one_launch(cuda):
    """Six pot scenes of different sizes solved by one graph launch: every
    instance meets the tolerance and equals its individual solve."""
    specs = S.random_batch_specs(6, seed=5)
    mats, divs = [], []
    for spec, seed in specs:
        m, d = _scene(spec, seed)
        mats.append(m)
        divs.append(d)
    masks = [cell_mask(torch.as_tensor(m).cuda()) for m in mats]
    dd = [torch.as_tensor(d).cuda() for d in divs]
    ps = [torch.zeros(m.shape, dtype=torch.float32, device="cuda") for m in mats]
    batch = BatchSolver(masks)
    for _ in range(2):  # build, then replay
        infos = batch.solve(dd, ps, DX, DT, RHO, tol=1e-6)
        assert len(infos) == 6
        for info in infos:
            assert info.rel_residual <= 1e-6 and info.inner_iterations > 0
    for m, d, p, mask in zip(mats, dd, ps, masks):
        single = TolSolver(mask).solve(d, DX, DT, RHO, tol=1e-6)
        assert torch.equal(single.p, p)
        assert O.rel_residual64(single.p64, d.cpu().numpy(), m, DX, DT, RHO) <= 1e-6
