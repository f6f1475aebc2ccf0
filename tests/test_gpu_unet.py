"""GPU tests of the learned warm start: each tensor-core kernel (convolution
forward, data gradient, weight gradient) and the whole network's forward
pass and parameter gradients against the CPU oracle (oracle/unet_oracle.py,
FP64 with BF16 rounding at the points where the GPU stores BF16), and a short
training run that must lower the loss."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import unet_oracle as U
from boilingsim_b200 import _lib, learned as LR, scenes as S
from boilingsim_b200._lib import call, ptr

pytestmark = pytest.mark.gpu


def bf(a):
    return torch.as_tensor(U.bf16_round(np.asarray(a, np.float32))).to(torch.bfloat16).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.float().cpu().numpy()


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("cin,cout,relu", [(16, 16, 1), (16, 32, 0), (32, 64, 1), (64, 128, 1),
                                           (128, 16, 0), (48, 80, 1)])
def test_conv3_forward_matches_oracle(cuda, cin, cout, relu):
    rng = np.random.default_rng(cin * 7 + cout)
    dims = (6, 5, 9)
    x = U.bf16_round(rng.standard_normal(dims + (cin,)).astype(np.float32)).astype(np.float64)
    w = U.bf16_round((rng.standard_normal((27, cout, cin)) * 0.1).astype(np.float32)).astype(
        np.float64)
    b = rng.standard_normal(cout).astype(np.float32)
    want = U.conv3(x, w, b)
    if relu:
        want = np.maximum(want, 0)
    out = torch.empty((np.prod(dims), cout), dtype=torch.bfloat16, device="cuda")
    xd, wd, bd = bf(x), bf(w), torch.as_tensor(b).cuda()
    call("bsp_unet_conv3_fwd", ptr(out), ptr(xd), ptr(wd), ptr(bd), *dims, cin, cout, relu, 0)
    got = host(out).reshape(dims + (cout,))
    # one BF16 rounding of the output: |err| <= 2^-8 |value|
    assert np.all(np.abs(got - want) <= 2 ** -8 * np.abs(want) + 1e-5 * np.abs(want).max())


@pytest.mark.parametrize("cin,cout", [(16, 16), (16, 32), (64, 32), (128, 128), (32, 96)])
def test_conv3_gradients_match_oracle(cuda, cin, cout):
    rng = np.random.default_rng(cin + 3 * cout)
    dims = (8, 6, 10)
    x = U.bf16_round(rng.standard_normal(dims + (cin,)).astype(np.float32)).astype(np.float64)
    w = U.bf16_round((rng.standard_normal((27, cout, cin)) * 0.1).astype(np.float32)).astype(
        np.float64)
    g = U.bf16_round(rng.standard_normal(dims + (cout,)).astype(np.float32)).astype(np.float64)
    dx, dw, db = U.conv3_grad(x, w, g)
    xd, wd, gd = bf(x), bf(w), bf(g)
    nb = int(_lib.lib().bsp_unet_wgrad_workspace_bytes(*dims, cin, cout))
    ws = torch.empty(nb // 4 + 1, dtype=torch.float32, device="cuda")
    gw = torch.empty((27, cout, cin), dtype=torch.float32, device="cuda")
    gb = torch.empty(cout, dtype=torch.float32, device="cuda")
    call("bsp_unet_conv3_wgrad", ptr(gw), ptr(gb), ptr(gd), ptr(xd), *dims, cin, cout, ptr(ws),
         nb, 0)
    # FP32 accumulation of exact BF16 products
    assert rel(host(gw), dw) < 1e-5 and rel(host(gb), db) < 1e-5
    wt = torch.empty((27, cin, cout), dtype=torch.bfloat16, device="cuda")
    call("bsp_unet_flip_weights", ptr(wt), ptr(wd), cin, cout, 0)
    gx = torch.empty((np.prod(dims), cin), dtype=torch.bfloat16, device="cuda")
    call("bsp_unet_conv3_fwd", ptr(gx), ptr(gd), ptr(wt), None, *dims, cout, cin, 0, 0)
    got = host(gx).reshape(dims + (cin,))
    assert np.all(np.abs(got - dx) <= 2 ** -8 * np.abs(dx) + 1e-5 * np.abs(dx).max())


def _small_scene(shape, seed):
    spec = S.PotSpec(shape[0], shape[1], shape[2], r_in=shape[0] // 2 - 3, t_w=2,
                     water_line=int(shape[2] * 0.75), carrot_r=2, carrot_len=shape[0] // 2)
    mat = S.pot_mat(spec)
    ux, uy, uz = S.velocity_field(mat, seed=seed)
    return mat, (ux, uy, uz)


def test_network_forward_and_gradients_match_oracle(cuda):
    """Forward prediction and every parameter gradient of a randomly
    initialised network on a 16x16x16 pot, against the FP64 oracle that
    rounds to BF16 where the GPU stores BF16."""
    from boilingsim_b200 import fluid as F

    dims = (16, 16, 16)
    mat, vel = _small_scene(dims, 3)
    dx, dt, rho = 0.002, 0.01, 997.0
    mat_t = torch.as_tensor(mat).cuda()
    mask = F.cell_mask(mat_t)
    U_ = [torch.as_tensor(a).cuda() for a in vel]
    div = torch.zeros(dims, dtype=torch.float32, device="cuda")
    F.compute_divergence(div, *U_, mask, dx)
    net = LR.UNet(seed=5)
    # non-zero biases and a random target exercise every term
    g = torch.Generator().manual_seed(1)
    for L in net.layers:
        L.b.copy_(torch.randn(L.cout, generator=g) * 0.05)
    net.hb.fill_(0.1)
    target = torch.randn(dims, generator=g).cuda() * 1e-3
    pred, c = net.forward(div, mask, dims, dx, dt, rho)
    c["pred"] = pred
    net.zero_grad()
    loss = float(net.backward(c, target, loss="l2").item())
    s, Sc, nfl = c["scales"]
    fluid = (mat == 0)
    x0 = host(c["x0"]).reshape(dims + (16,)).astype(np.float64)
    P = {f"{L.name}.w": L.w.cpu().numpy().astype(np.float64) for L in net.layers}
    P.update({f"{L.name}.b": L.b.cpu().numpy().astype(np.float64) for L in net.layers})
    P["head.w"] = net.hw.cpu().numpy().astype(np.float64)
    P["head.b"] = net.hb.cpu().numpy().astype(np.float64)
    want_pred, want_loss, G = U.forward_backward(x0, P, fluid, host(target).astype(np.float64),
                                                 Sc, norm=c["norm"])
    assert rel(host(pred), want_pred) < 2e-2
    assert abs(loss - want_loss) <= 2e-2 * abs(want_loss)
    for L in net.layers:
        assert rel(host(L.gw), G[L.name + ".w"]) < 5e-2, L.name
        assert rel(host(L.gb), G[L.name + ".b"]) < 5e-2, L.name
    assert rel(host(net.g_hw), G["head.w"]) < 2e-2
    assert rel(host(net.g_hb), G["head.b"]) < 2e-2


def test_training_lowers_the_loss(cuda):
    """Fifty Adam steps on one scene drive its loss well below the start."""
    from boilingsim_b200 import fluid as F
    from boilingsim_b200.solver import TolSolver

    dims = (32, 32, 24)
    mat, vel = _small_scene(dims, 11)
    dx, dt, rho = 0.002, 0.01, 997.0
    mask = F.cell_mask(torch.as_tensor(mat).cuda())
    div = torch.zeros(dims, dtype=torch.float32, device="cuda")
    F.compute_divergence(div, *[torch.as_tensor(a).cuda() for a in vel], mask, dx)
    p = torch.zeros_like(div)
    TolSolver(mask).solve(div, dx, dt, rho, tol=1e-8, p=p)
    for loss in ("l2", "energy"):
        net = LR.UNet(seed=2)
        first = float(net.train_step(div, mask, p, dx, dt, rho, lr=2e-3, loss=loss).item())
        for _ in range(49):
            last = float(net.train_step(div, mask, p, dx, dt, rho, lr=2e-3, loss=loss).item())
        assert np.isfinite(last) and last < 0.3 * first, loss


def test_trained_network_saves_iterations(cuda):
    """The committed weights (trained on 20k plain-solver triples of the
    batched pot variants) on held-out scenes: the prediction's residual is
    well below ||b|| (the zero start's), and the solve started from it reaches
    the same FP64 tolerance in fewer inner iterations.  A network with
    untrained weights does not come close."""
    net = LR.UNet.load()
    fresh = LR.UNet(seed=123)
    cold_total = warm_total = 0
    for spec in (S.PotSpec(96, 96, 64, r_in=43.0, t_w=3, water_line=50.0, carrot_r=6.0,
                           carrot_len=30.0), S.pot_192(4)):
        rows = LR.evaluate(net, spec, seeds=(7, 8), plume=0.15)
        untrained = LR.evaluate(fresh, spec, seeds=(7,), plume=0.15)
        for r in rows:
            assert r["warm_rel_residual"] <= 1e-6 and r["cold_rel_residual"] <= 1e-6
            assert r["net_rel_residual"] < 0.3, r
            assert r["warm_inner"] <= r["cold_inner"], r
            cold_total += r["cold_inner"]
            warm_total += r["warm_inner"]
        assert untrained[0]["net_rel_residual"] > 3 * rows[0]["net_rel_residual"]
    assert warm_total < cold_total


def test_learned_projection_back_end(cuda, monkeypatch):
    """BOILINGSIM_PRESSURE_SOLVER=b200-learned: the projection starts the FP16
    solve from the network and still meets the tolerance."""
    from boilingsim_b200 import fluid as F
    import oracle as O

    monkeypatch.setenv("BOILINGSIM_PRESSURE_SOLVER", "b200-learned")
    monkeypatch.delenv("BOILINGSIM_USE_RUST_PRESSURE", raising=False)
    mat = S.pot_mat(S.POT_64)
    ux, uy, uz = S.velocity_field(mat, seed=13)
    grid = F.Grid.from_numpy(mat, ux, uy, uz, 0.002)
    ws = F.allocate_fluid_workspace(grid)
    cfg = F.ScenarioConfig(F.SolverConfig(pressure_tol=1e-6))
    div = O.divergence(ux, uy, uz, mat, 0.002)
    F.pressure_projection(grid, ws, cfg, 0.01, 997.0)
    res = F._TOL_SOLVERS[next(iter(F._TOL_SOLVERS))].last
    assert res.status == 0
    torch.cuda.synchronize()
    assert O.rel_residual64(res.p64_dev.cpu().numpy(), div, mat, 0.002, 0.01, 997.0) <= 1e-6


def test_energy_norm_loss_and_head_gradient(cuda):
    """The energy-norm loss (y - t)^T A (y - t) / t^T A t and its head
    gradients against the FP64 operator of the oracle."""
    from boilingsim_b200 import fluid as F
    import oracle as O

    dims = (16, 16, 16)
    mat, vel = _small_scene(dims, 4)
    dx, dt, rho = 0.002, 0.01, 997.0
    mask = F.cell_mask(torch.as_tensor(mat).cuda())
    div = torch.zeros(dims, dtype=torch.float32, device="cuda")
    F.compute_divergence(div, *[torch.as_tensor(a).cuda() for a in vel], mask, dx)
    net = LR.UNet(seed=6)
    target = torch.randn(dims, generator=torch.Generator().manual_seed(3)).cuda() * 1e-3
    pred, c = net.forward(div, mask, dims, dx, dt, rho)
    c["pred"] = pred
    net.zero_grad()
    loss = float(net.backward(c, target, loss="energy").item())
    S = c["scales"][1]
    fl = mat == 0
    d = np.where(fl, (host(pred).astype(np.float64) - host(target)) / S, 0.0)
    t = np.where(fl, host(target).astype(np.float64) / S, 0.0)
    Ad = np.where(fl, O.apply_A_f64(d, mat), 0.0)
    nA = float((t * np.where(fl, O.apply_A_f64(t, mat), 0.0)).sum())
    assert abs(loss - (d * Ad).sum() / nA) <= 1e-3 * abs(loss)
    gy = 2.0 * Ad / nA
    u1 = host(c["u1"]).reshape(dims + (16,)).astype(np.float64)
    assert rel(host(net.g_hw), np.einsum("ijk,ijkc->c", gy, u1)) < 1e-3
    assert rel(host(net.g_hb), np.array([gy.sum()])) < 1e-3
