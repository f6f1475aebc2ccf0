"""Mixed-precision solves on the 192x192x128 pot with steel-, aluminium- and
copper-like walls (2/3/4 cells): FP32, FP16 and BF16 storage of the inner
vectors, refinement to FP64 rel-residual 1e-6, error against the FP64 CPU
oracle solve p*.  Prints one summary line per case (pytest -s shows it)."""
from __future__ import annotations

import json

import numpy as np
import pytest
import torch

import oracle as O
from boilingsim_b200 import scenes as S
from boilingsim_b200.fluid import cell_mask
from boilingsim_b200.solver import TolSolver

pytestmark = pytest.mark.gpu

DX, DT, RHO = 0.002, 0.01, 997.0


@pytest.mark.parametrize("wall", [2, 3, 4])
def test_mixed_precision_error_vs_fp64_oracle(cuda, wall):
    mat = S.pot_mat(S.pot_192(wall))
    ux, uy, uz = S.velocity_field(mat, seed=7)
    div = O.divergence(ux, uy, uz, mat, DX)
    p_star, it, rel = O.solve_f64(div, mat, DX, DT, RHO, tol=1e-11, max_iter=20000)
    assert rel <= 1e-11
    mask = cell_mask(torch.as_tensor(mat).cuda())
    d = torch.as_tensor(div).cuda()
    for storage in ("fp32", "fp16", "bf16"):
        res = TolSolver(mask, storage).solve(d, DX, DT, RHO, tol=1e-6)
        assert res.status == 0
        x = res.p64
        r = O.rel_residual64(x, div, mat, DX, DT, RHO)
        err = O.rel_error(x, p_star, mat)
        err32 = O.rel_error(res.p.cpu().numpy(), p_star, mat)
        print(json.dumps({"case": "pot192", "wall": wall, "storage": storage,
                          "inner_iterations": res.inner_iterations,
                          "outer_iterations": res.outer_iterations, "rel_residual_fp64": r,
                          "rel_error_vs_fp64_oracle": err, "rel_error_float_output": err32}))
        assert r <= 1e-6
        assert err <= 1e-4
