"""fluid.ProjectionPipeline: independent projections with host buffers, two
in flight on their own streams, give the bits of fluid.pressure_projection run
one at a time on the same inputs (p, the corrected velocities and max|div|)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from boilingsim_b200 import fluid as F, scenes as S

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("solver", ["b200-mixed", "b200-mg", "b200-jacobi", "b200-learned"])
def test_pipeline_matches_one_at_a_time(cuda, monkeypatch, solver):
    monkeypatch.setenv("BOILINGSIM_PRESSURE_SOLVER", solver)
    spec = S.PotSpec(48, 48, 32, r_in=20, t_w=2, water_line=24, carrot_r=3, carrot_len=14)
    mat = S.pot_mat(spec)
    dx, dt, rho = 0.002, 0.01, 997.0
    cfg = F.ScenarioConfig(F.SolverConfig(pressure_tol=1e-6, pressure_max_iter=60))
    fields = [S.velocity_field(mat, seed=seed) for seed in (3, 4, 5)]

    # one at a time through the projection API
    want = []
    grid = F.Grid.from_numpy(mat, *fields[0], dx)
    ws = F.allocate_fluid_workspace(grid)
    for u in fields:
        for d, a in zip((grid.ux, grid.uy, grid.uz), u):
            d.copy_(torch.as_tensor(a))
        md = F.pressure_projection(grid, ws, cfg, dt, rho)
        want.append(([t.cpu().numpy().copy() for t in (grid.ux, grid.uy, grid.uz, grid.p)], md))

    # the pipeline: all three submitted before the first result is taken
    pipe = F.ProjectionPipeline(grid.mat, dx, cfg, depth=3)
    hin = [[torch.as_tensor(a).pin_memory() for a in u] for u in fields]
    hout = [[torch.empty(a.shape, dtype=torch.float32).pin_memory() for a in u] +
            [torch.empty(mat.shape, dtype=torch.float32).pin_memory()] for u in fields]
    tickets = [pipe.submit(*hin[q], *hout[q], dt, rho) for q in range(3)]
    for q, t in enumerate(tickets):
        md = pipe.result(t)
        got = [h.numpy() for h in hout[q]]
        for g, w in zip(got, want[q][0]):
            assert np.array_equal(g.view(np.uint32), w.view(np.uint32)), (solver, q)
        assert md == want[q][1]
    # a slot taken again: the earlier ticket's result is gone
    t4 = pipe.submit(*hin[0], *hout[0], dt, rho)
    with pytest.raises(ValueError):
        pipe.result(tickets[0])
    assert pipe.result(t4) == want[0][1]


def test_pipeline_rejects_default_stream_back_ends(cuda, monkeypatch):
    monkeypatch.setenv("BOILINGSIM_PRESSURE_SOLVER", "cg-rust")
    mat = torch.zeros((8, 8, 8), dtype=torch.int32, device="cuda")
    with pytest.raises(ValueError):
        F.ProjectionPipeline(mat, 0.002, F.ScenarioConfig())
