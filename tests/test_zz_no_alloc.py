"""GPU test of bsp_dot_noalloc, the dot product for callers that cannot
allocate device memory (a foreign-language host holding only its own arrays,
or a loop stepping under a fixed device-memory budget): its partial sums live
in a file-scope device array instead of a caller workspace.

It is checked through the C ABI against the workspace-taking dot_launch on two
calls in a row -- a large call that fills many partial slots, then a smaller
one, so stale partials left by the first call must not leak into the second.
This file is collected last so that a failure here never hides another test.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from boilingsim_b200 import _lib
from boilingsim_b200._lib import call, ptr

pytestmark = pytest.mark.gpu


def _dot_with_workspace(x, y):
    ws = torch.zeros(1024, dtype=torch.float32, device="cuda")
    res = torch.zeros(1, dtype=torch.float32, device="cuda")
    call("dot_launch", ptr(x), ptr(y), x.numel(), ptr(ws), ptr(res))
    torch.cuda.synchronize()
    return float(res.item())


def _dot_noalloc(x, y):
    res = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
    call("bsp_dot_noalloc", ptr(x), ptr(y), x.numel(), ptr(res), 0)
    torch.cuda.synchronize()
    return float(res.item())


def test_noalloc_dot_matches_workspace_dot_twice(cuda):
    g = torch.Generator(device="cuda").manual_seed(123)
    x1 = torch.randn(5_000_011, generator=g, device="cuda")
    y1 = torch.randn(5_000_011, generator=g, device="cuda")
    x2 = torch.randn(70_001, generator=g, device="cuda") + 0.5
    y2 = torch.randn(70_001, generator=g, device="cuda") + 0.5
    for x, y in ((x1, y1), (x2, y2)):
        got = _dot_noalloc(x, y)
        want = _dot_with_workspace(x, y)  # FP64 sum rounded to float
        exact = float(np.dot(x.cpu().numpy().astype(np.float64), y.cpu().numpy().astype(np.float64)))
        assert abs(got - want) <= 1e-6 * abs(exact) + 1e-3
        assert abs(got - exact) <= 1e-9 * (abs(exact) + x.numel())


def test_noalloc_dot_limits(cuda):
    x = torch.ones(4, device="cuda")
    res = torch.full((1,), 7.0, dtype=torch.float64, device="cuda")
    call("bsp_dot_noalloc", ptr(x), ptr(x), 0, ptr(res), 0)
    torch.cuda.synchronize()
    assert float(res.item()) == 0.0
    with pytest.raises(_lib.BspError) as e:
        call("bsp_dot_noalloc", ptr(x), ptr(x), 67_108_864 + 1, ptr(res), 0)
    assert e.value.code == 10001
