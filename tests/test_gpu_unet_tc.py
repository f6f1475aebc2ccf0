"""GPU tests of the tensor-core (tcgen05 / TMEM / TMA) inference path of the
warm-start U-Net (csrc/unet_tc.cu) on the padded layout.

* One convolution against the FP64 oracle (oracle/unet_oracle.py) and a plain
  PyTorch FP32 conv3d of the same BF16 operands: within one BF16 rounding of
  the output; halo rows exactly zero.  Shapes cover every layer of the
  network (resident and streamed weights, cout tiles of 16 / 32 / 64, two
  cout tiles for 128), odd grid sizes, bias, ReLU and the fused skip add.
* The padded pack / pool / upsample / head kernels bit for bit against the
  unpadded training kernels.
* The whole forward pass (TcPlan) against the training forward pass
  (mma.sync kernels) and against the oracle network.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

import unet_oracle as U
from boilingsim_b200 import _lib, learned as LR, scenes as S
from boilingsim_b200._lib import call, ptr

pytestmark = pytest.mark.gpu


def rows_of(dims):
    return int(_lib.lib().bsp_unet_tc_rows(*dims))


def pad(x):
    """(nx, ny, nz, c) -> padded rows x c (zero halo), BF16 on the GPU."""
    nx, ny, nz, c = x.shape
    out = torch.zeros((nx + 2, ny + 2, nz + 2, c), dtype=torch.bfloat16, device="cuda")
    out[1:-1, 1:-1, 1:-1] = torch.as_tensor(np.ascontiguousarray(x), dtype=torch.float32).cuda()
    return out.reshape(-1, c)


def unpad(t, dims):
    nx, ny, nz = dims
    torch.cuda.synchronize()
    a = t.float().reshape(nx + 2, ny + 2, nz + 2, -1)
    return a[1:-1, 1:-1, 1:-1].cpu().numpy(), a


def halo_is_zero(a):
    m = torch.ones(a.shape[:3], dtype=torch.bool, device=a.device)
    m[1:-1, 1:-1, 1:-1] = False
    return bool((a[m] == 0).all())


def bf64(a):
    return U.bf16_round(np.asarray(a, np.float32)).astype(np.float64)


CASES = [  # (cin, cout, dims, relu, bias, skip)
    (16, 16, (6, 5, 9), 1, True, False),
    (16, 16, (12, 10, 20), 1, True, True),
    (32, 16, (8, 8, 8), 1, True, True),
    (16, 32, (7, 9, 11), 0, True, False),
    (32, 32, (10, 6, 33), 1, True, False),
    (64, 32, (6, 6, 6), 1, True, True),
    (32, 64, (5, 7, 9), 1, True, False),
    (64, 64, (6, 5, 4), 1, True, False),
    (128, 64, (4, 6, 8), 1, True, True),
    (64, 128, (3, 3, 3), 1, True, False),
    (128, 128, (4, 4, 5), 0, False, False),
    (16, 16, (24, 24, 128), 1, True, False),
]


@pytest.mark.parametrize("cin,cout,dims,relu,bias,skip", CASES)
def test_tc_conv_matches_oracle_and_torch(cuda, cin, cout, dims, relu, bias, skip):
    rng = np.random.default_rng(cin * 131 + cout + dims[2])
    x = bf64(rng.standard_normal(dims + (cin,)))
    w = bf64(rng.standard_normal((27, cout, cin)) * (1.0 / np.sqrt(27 * cin)))
    b = rng.standard_normal(cout).astype(np.float32) * 0.1 if bias else None
    sk = bf64(rng.standard_normal(dims + (cout,))) if skip else None
    want = U.conv3(x, w, b if b is not None else np.zeros(cout))
    if relu:
        want = np.maximum(want, 0)
    pre = np.abs(want)  # the layer's value before the skip add
    if skip:
        want = bf64(want) + sk
    # plain PyTorch FP32 reference of the same operands
    xt = torch.as_tensor(x, dtype=torch.float32).cuda().permute(3, 0, 1, 2)[None]
    wt = torch.as_tensor(w, dtype=torch.float32).cuda().reshape(3, 3, 3, cout, cin)
    wt = wt.permute(3, 4, 0, 1, 2).contiguous()
    ref = torch.nn.functional.conv3d(xt, wt, torch.as_tensor(b).cuda() if bias else None,
                                     padding=1)[0].permute(1, 2, 3, 0)
    if relu:
        ref = torch.relu(ref)
    if skip:
        ref = ref.to(torch.bfloat16).float() + torch.as_tensor(sk, dtype=torch.float32).cuda()
    xin = pad(x)
    wd = torch.as_tensor(w, dtype=torch.float32).to(torch.bfloat16).cuda()
    wimg = torch.empty(27 * cin * cout, dtype=torch.bfloat16, device="cuda")
    call("bsp_unet_tc_weights", ptr(wimg), ptr(wd), cin, cout, 0)
    out = torch.zeros((rows_of(dims), cout), dtype=torch.bfloat16, device="cuda")
    out[:] = 7.0  # every row a tile covers is written (halo rows with zeros)
    out[: (dims[1] + 2) * (dims[2] + 2) + dims[2] + 3] = 0.0
    skp = pad(sk) if skip else None
    bd = torch.as_tensor(b).cuda() if bias else None
    call("bsp_unet_tc_conv3", ptr(out), ptr(xin), ptr(wimg), ptr(bd) if bias else None,
         ptr(skp) if skip else None, *dims, cin, cout, relu, 0)
    got, full = unpad(out, dims)
    flag = np.zeros(1, np.int32)
    call("bsp_unet_tc_error", flag.ctypes.data)
    assert flag[0] == 0
    # one BF16 rounding of the output; with the skip add, one of the layer's
    # value and one of the sum
    bound = 2 ** -8 * (np.abs(want) + (pre if skip else 0.0))
    scale = np.abs(want).max()
    assert np.all(np.abs(got - want) <= bound + 2e-5 * scale)
    assert np.all(np.abs(got - ref.cpu().numpy()) <= bound + 1e-4 * scale)
    # halo rows between the first and the last interior row are written as zeros
    nx, ny, nz = dims
    R, P = nz + 2, (ny + 2) * (nz + 2)
    q = torch.arange(full.numel() // cout, device="cuda")
    k, j, i = q % R, (q // R) % (ny + 2), q // P
    halo = (k == 0) | (k == R - 1) | (j == 0) | (j == ny + 1) | (i == 0) | (i == nx + 1)
    span = (q >= P + R + 1) & (q <= nx * P + ny * R + nz)
    assert bool((full.reshape(-1, cout)[halo & span] == 0).all())


@pytest.mark.parametrize("cin,cout,dims", [(16, 16, (40, 36, 64)), (32, 32, (20, 18, 32)),
                                           (64, 128, (8, 6, 16))])
def test_tc_conv_epilogue_warpgroups_bit_identical(cuda, cin, cout, dims):
    """One epilogue warpgroup with two CTAs per SM, or two, three or four
    warpgroups in one CTA (BSP_TUNE_CONV_EPILOGUE; the work items rotate over
    the TMEM accumulators that fit) give the same bits, and the cycle
    accounting counts every work item once."""
    rng = np.random.default_rng(cin + cout)
    x = bf64(rng.standard_normal(dims + (cin,)))
    w = bf64(rng.standard_normal((27, cout, cin)) * (1.0 / np.sqrt(27 * cin)))
    b = torch.as_tensor(rng.standard_normal(cout).astype(np.float32) * 0.1).cuda()
    sk = pad(bf64(rng.standard_normal(dims + (cout,))))
    xin = pad(x)
    wd = torch.as_tensor(w, dtype=torch.float32).to(torch.bfloat16).cuda()
    wimg = torch.empty(27 * cin * cout, dtype=torch.bfloat16, device="cuda")
    call("bsp_unet_tc_weights", ptr(wimg), ptr(wd), cin, cout, 0)
    nx, ny, nz = dims
    R, P = nz + 2, (ny + 2) * (nz + 2)
    tiles = (nx * P + ny * R + nz - (P + R + 1) + 126) // 126
    ct = 64 if cout % 64 == 0 else (32 if cout % 32 == 0 else 16)
    outs = {}
    try:
        for nepi in (4, 3, 2, 1):
            call("bsp_set_tuning", 16, nepi)
            out = torch.zeros((rows_of(dims), cout), dtype=torch.bfloat16, device="cuda")
            tr = np.zeros(8, np.uint64)
            call("bsp_unet_tc_trace", None, 1)
            call("bsp_unet_tc_conv3", ptr(out), ptr(xin), ptr(wimg), ptr(b), ptr(sk), *dims, cin,
                 cout, 1, 0)
            torch.cuda.synchronize()
            call("bsp_unet_tc_trace", tr.ctypes.data, 0)
            assert int(tr[6]) == tiles * (cout // ct)
            outs[nepi] = out.view(torch.int16).cpu().numpy()
    finally:
        call("bsp_set_tuning", 16, 0)
    flag = np.zeros(1, np.int32)
    call("bsp_unet_tc_error", flag.ctypes.data)
    assert flag[0] == 0
    for nepi in (4, 3, 1):
        assert np.array_equal(outs[2], outs[nepi]), nepi


def test_tc_padded_layout_kernels_bit_exact(cuda):
    """pack / pool / upsample / head on the padded layout give the same bits as
    the unpadded kernels of the training path."""
    from boilingsim_b200 import fluid as F

    dims = (16, 24, 32)
    spec = S.PotSpec(*dims, r_in=6, t_w=2, water_line=24, carrot_r=2, carrot_len=8)
    mat = S.pot_mat(spec)
    ux, uy, uz = S.velocity_field(mat, seed=4)
    mask = F.cell_mask(torch.as_tensor(mat).cuda())
    div = torch.zeros(dims, device="cuda")
    F.compute_divergence(div, *[torch.as_tensor(a).cuda() for a in (ux, uy, uz)], mask, 0.002)
    n = int(np.prod(dims))
    x_ref = torch.empty((n, 16), dtype=torch.bfloat16, device="cuda")
    call("bsp_unet_pack_input", ptr(x_ref), ptr(div), ptr(mask), n, 2.0, 0)
    xp = torch.full((rows_of(dims), 16), 5.0, dtype=torch.bfloat16, device="cuda")
    s_dev = torch.tensor([0.5], device="cuda")  # input divided by 0.5: scaled by 2 exactly
    call("bsp_unet_tc_pack", ptr(xp), ptr(div), ptr(mask), *dims, ptr(s_dev), 0)
    got, full = unpad(xp, dims)
    assert np.array_equal(got.reshape(n, 16), x_ref.float().cpu().numpy())
    assert halo_is_zero(full)
    # pool of a random 32-channel field
    rng = np.random.default_rng(9)
    a = bf64(rng.standard_normal(dims + (32,)))
    ad = torch.as_tensor(a.reshape(n, 32), dtype=torch.float32).to(torch.bfloat16).cuda()
    cd = tuple(d // 2 for d in dims)
    pr = torch.empty((n // 8, 32), dtype=torch.bfloat16, device="cuda")
    call("bsp_unet_pool", ptr(pr), ptr(ad), *dims, 32, 0, 0, 0)
    pp = torch.full((rows_of(cd), 32), 5.0, dtype=torch.bfloat16, device="cuda")
    call("bsp_unet_tc_pool", ptr(pp), ptr(pad(a)), *dims, 32, 0)
    got, full = unpad(pp, cd)
    assert np.array_equal(got.reshape(-1, 32), pr.float().cpu().numpy()) and halo_is_zero(full)
    # upsample the pooled field back
    ur = torch.empty((n, 32), dtype=torch.bfloat16, device="cuda")
    call("bsp_unet_up", ptr(ur), ptr(pr), *dims, 32, 0, 0)
    up = torch.full((rows_of(dims), 32), 5.0, dtype=torch.bfloat16, device="cuda")
    call("bsp_unet_tc_up", ptr(up), ptr(pp), *dims, 32, 0)
    got, full = unpad(up, dims)
    assert np.array_equal(got.reshape(n, 32), ur.float().cpu().numpy()) and halo_is_zero(full)
    # head
    hw = torch.randn(16, device="cuda")
    hb = torch.randn(1, device="cuda")
    p_ref = torch.empty(dims, device="cuda")
    call("bsp_unet_head_fwd", ptr(p_ref), ptr(x_ref), ptr(hw), ptr(hb), ptr(mask), n, 2.5, 0)
    p_tc = torch.empty(dims, device="cuda")
    s_one = torch.ones(1, device="cuda")
    call("bsp_unet_tc_head", ptr(p_tc), ptr(xp), ptr(hw), ptr(hb), ptr(mask), *dims, ptr(s_one),
         2.5, 0)
    assert torch.equal(p_tc, p_ref)
    # the device input scale: RMS of div over the fluid cells
    from boilingsim_b200.learned import scene_scales

    ws = torch.empty(int(_lib.lib().bsp_unet_scale_workspace_bytes()) // 8 + 1,
                     dtype=torch.float64, device="cuda")
    s_d = torch.zeros(1, device="cuda")
    call("bsp_unet_input_scale", ptr(s_d), ptr(div), ptr(mask), *dims, ptr(ws), ws.numel() * 8,
         0)
    s_host = scene_scales(div, mask, 0.002, 0.01, 997.0)[0]
    assert abs(float(s_d.item()) - s_host) <= 1e-6 * s_host


@pytest.mark.parametrize("dims", [(16, 16, 16), (48, 40, 32)])
def test_tc_forward_matches_training_forward_and_oracle(cuda, dims):
    """The whole network: tensor-core inference against the mma.sync forward
    pass and against the FP64 oracle network (BF16 where the GPU stores
    BF16); trained weights, a pot scene."""
    from boilingsim_b200 import fluid as F

    spec = S.PotSpec(*dims, r_in=dims[0] // 2 - 3, t_w=2, water_line=int(dims[2] * 0.75),
                     carrot_r=2, carrot_len=dims[0] // 2)
    mat = S.pot_mat(spec)
    ux, uy, uz = S.velocity_field(mat, seed=11)
    mask = F.cell_mask(torch.as_tensor(mat).cuda())
    div = torch.zeros(dims, device="cuda")
    F.compute_divergence(div, *[torch.as_tensor(a).cuda() for a in (ux, uy, uz)], mask, 0.002)
    net = LR.UNet.load()
    p_tc = net.predict(div, mask, 0.002, 0.01, 997.0, backend="tc")
    p_mma = net.predict(div, mask, 0.002, 0.01, 997.0, backend="mma")
    torch.cuda.synchronize()
    a, b = p_tc.cpu().numpy(), p_mma.cpu().numpy()
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 3e-2
    # the oracle network
    _, c = net.forward(div, mask, dims, 0.002, 0.01, 997.0)
    x0 = c["x0"].float().cpu().numpy().reshape(dims + (16,)).astype(np.float64)
    P = {f"{L.name}.w": L.w.cpu().numpy().astype(np.float64) for L in net.layers}
    P.update({f"{L.name}.b": L.b.cpu().numpy().astype(np.float64) for L in net.layers})
    P["head.w"] = net.hw.cpu().numpy().astype(np.float64)
    P["head.b"] = net.hb.cpu().numpy().astype(np.float64)
    s, Sc, nfl = c["scales"]
    want, _, _ = U.forward_backward(x0, P, mat == 0, np.zeros(dims), Sc)
    assert np.linalg.norm(a - want) / np.linalg.norm(want) < 5e-2
    # repeated runs on the same plan give the same bits (buffers reused)
    p2 = net.predict(div, mask, 0.002, 0.01, 997.0, backend="tc")
    assert torch.equal(p2, p_tc)


def test_energy_scale_of_a_guess(cuda):
    """bsp_unet_energy_scale multiplies a starting pressure by
    gamma = (b . p) / (p . A p), the scale that minimises the A-norm error; the
    scaled guess is then no farther from the solution than zero."""
    import oracle as O
    from boilingsim_b200 import fluid as F

    spec = S.PotSpec(32, 32, 24, r_in=13, t_w=2, water_line=19, carrot_r=3, carrot_len=12)
    mat = S.pot_mat(spec)
    ux, uy, uz = S.velocity_field(mat, seed=2)
    dx, dt, rho = 0.002, 0.01, 997.0
    div = O.divergence(ux, uy, uz, mat, dx)
    rng = np.random.default_rng(3)
    p = np.where(mat == 0, rng.standard_normal(mat.shape), 0.0).astype(np.float32)
    mask = F.cell_mask(torch.as_tensor(mat).cuda())
    pd, dd = torch.as_tensor(p).cuda(), torch.as_tensor(div).cuda()
    Ap = torch.empty_like(pd)
    call("bsp_spmv", ptr(Ap), ptr(pd), ptr(mask), *mat.shape, 0)
    ws = torch.empty(int(_lib.lib().bsp_unet_scale_workspace_bytes()) // 8 + 1,
                     dtype=torch.float64, device="cuda")
    g = torch.zeros(1, device="cuda")
    factor = -(rho * dx * dx / dt)
    call("bsp_unet_energy_scale", ptr(pd), ptr(Ap), ptr(dd), ptr(mask), *mat.shape, factor,
         ptr(ws), ws.numel() * 8, ptr(g), 0)
    got = pd.cpu().numpy()
    fl = mat == 0
    b = np.where(fl, np.float32(factor) * div, 0.0).astype(np.float64)
    Ap64 = Ap.cpu().numpy().astype(np.float64)
    gamma = float((b * p).sum() / (p.astype(np.float64) * Ap64).sum())
    assert abs(float(g.item()) - gamma) <= 1e-5 * abs(gamma)
    assert np.allclose(got, p * np.float32(g.item()), rtol=0, atol=0)
    # A-norm error of the scaled guess against the FP64 solution <= that of zero
    pstar, _, _ = O.solve_f64(div, mat, dx, dt, rho, tol=1e-12)
    e = got.astype(np.float64) - pstar
    anorm = lambda v: float(v @ O.apply_A_f64(v.reshape(mat.shape), mat).ravel())  # noqa: E731
    assert anorm(e.ravel()) <= anorm(pstar.ravel())
    # the keep rule: the relative residual ||b - gamma A p|| / ||b|| of the
    # scaled guess from the same sums; kept below keep_below, else zeroed
    rel = float(np.linalg.norm(b - gamma * Ap64) / np.linalg.norm(b))
    for keep_below, kept in ((rel * 1.5, True), (rel * 0.5, False), (0.0, True)):
        pk = torch.as_tensor(p).cuda()
        gk = torch.zeros(1, device="cuda")
        rk = torch.zeros(1, device="cuda")
        call("bsp_unet_energy_scale_keep", ptr(pk), ptr(Ap), ptr(dd), ptr(mask), *mat.shape,
             factor, keep_below, ptr(ws), ws.numel() * 8, ptr(gk), ptr(rk), 0)
        assert abs(float(rk.item()) - rel) <= 1e-4 * rel
        if kept:
            assert torch.equal(pk, pd) and float(gk.item()) == float(g.item())
        else:
            assert float(gk.item()) == 0.0 and not torch.any(pk != 0)


@pytest.mark.parametrize("mode", ["full", "coarse", "coarse4"])
def test_warm_start_guess_graph_and_solve(cuda, mode):
    """WarmStart.guess: the CUDA-graph replay gives the same bits as the eager
    launches; the guess is zero off fluid, scaled so that it is no farther
    from the solution than zero in the A-norm, and the solve started from it
    meets the FP64 tolerance."""
    import oracle as O
    from boilingsim_b200 import fluid as F
    from boilingsim_b200.solver import TolSolver

    # coarse4 needs every dimension divisible by 32 (the network's grid by 8)
    spec = S.POT_64 if mode != "coarse4" else S.PotSpec(96, 96, 64, r_in=42, t_w=2,
                                                          water_line=50, carrot_r=6,
                                                          carrot_len=30)
    mat = S.pot_mat(spec)
    ux, uy, uz = S.velocity_field(mat, seed=5)
    dx, dt, rho = 0.002, 0.01, 997.0
    div = O.divergence(ux, uy, uz, mat, dx)
    mat_t = torch.as_tensor(mat).cuda()
    mask = F.cell_mask(mat_t)
    dd = torch.as_tensor(div).cuda()
    ws = LR.WarmStart(LR.UNet.load(), mat_t, mask, mode=mode)
    a = torch.empty_like(dd)
    b = torch.empty_like(dd)
    ws.guess(dd, dx, dt, rho, out=a, graph=False)
    ws.guess(dd, dx, dt, rho, out=b, graph=True)
    ws.guess(dd, dx, dt, rho, out=b, graph=True)  # replay
    torch.cuda.synchronize()
    assert torch.equal(a, b)
    g = a.cpu().numpy()
    assert np.isfinite(g).all() and np.all(g[mat != 0] == 0.0)
    pstar, _, _ = O.solve_f64(div, mat, dx, dt, rho, tol=1e-12)
    e = g.astype(np.float64) - pstar
    anorm = lambda v: float((v * O.apply_A_f64(v, mat)).sum())  # noqa: E731
    assert anorm(e) <= anorm(pstar) * (1 + 1e-6)
    solver = TolSolver(mask, "fp16")
    res = solver.solve(dd, dx, dt, rho, tol=1e-6, p=a.clone(), warm_start=True)
    assert res.status == 0
    assert O.rel_residual64(res.p64, div, mat, dx, dt, rho) <= 1.0001e-6


@pytest.mark.parametrize("dims", [(8, 12, 16), (6, 10, 14)], ids=["four-cell", "one-cell"])
def test_prolong_matches_trilinear(cuda, dims):
    """bsp_unet_prolong (the four-cell kernel when nz % 4 == 0, the one-cell one
    otherwise): every fluid fine cell gets the trilinear interpolation of the
    coarse field at fine position / 2 - 1/4 (clamped), non-fluid cells 0."""
    from boilingsim_b200 import fluid as F

    rng = np.random.default_rng(5)
    nx, ny, nz = dims
    mat = np.where(rng.random(dims) < 0.7, 0, 2).astype(np.int32)
    mask = F.cell_mask(torch.as_tensor(mat).cuda())
    pc = rng.standard_normal((nx // 2, ny // 2, nz // 2)).astype(np.float32)
    out = torch.full(dims, 7.0, device="cuda")
    call("bsp_unet_prolong", ptr(out), ptr(torch.as_tensor(pc).cuda()), ptr(mask), *dims, 0)

    def lin(d, nc):
        if d & 1:
            return d >> 1, min((d >> 1) + 1, nc - 1), 0.75
        return max((d >> 1) - 1, 0), d >> 1, 0.25

    want = np.zeros(dims, np.float64)
    for i in range(nx):
        i0, i1, wi = lin(i, nx // 2)
        for j in range(ny):
            j0, j1, wj = lin(j, ny // 2)
            for k in range(nz):
                if mat[i, j, k] != 0:
                    continue
                k0, k1, wk = lin(k, nz // 2)
                c = lambda a, b: wk * pc[a, b, k0] + (1 - wk) * pc[a, b, k1]  # noqa: E731
                want[i, j, k] = wi * (wj * c(i0, j0) + (1 - wj) * c(i0, j1)) + \
                    (1 - wi) * (wj * c(i1, j0) + (1 - wj) * c(i1, j1))
    got = out.cpu().numpy()
    assert np.all(got[mat != 0] == 0.0)
    assert np.allclose(got, want, rtol=1e-5, atol=1e-6)
