"""GPU parity of the reference's CG vector launchers and of its PCG.

The launchers of crates/cuda-kernels/src/axpy_device.cu:20-145 and
scale.cu:11-34 (axpy_device_launch, scaled_axpy_launch, divide_scalars_launch,
compute_b_launch, zero_buffer_launch, scale_inplace_launch), called through
the C ABI with the reference's argument lists, against the oracle's
restatement bit for bit and, where oracle/_ref was built, against the
reference's own kernels.  pressure_solve_pcg_launch is checked against the
reference PCG's golden outputs (tests/golden/pcg_box_*.npz).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np
import pytest
import torch

import oracle as O
from boilingsim_b200 import scenes as S
from boilingsim_b200._lib import call, ptr
from boilingsim_b200.sim_core import SimCore

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def dev(a, dt=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dt).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _ref_lib():
    """The reference's own launchers (oracle/_ref, FMA build) with their
    argument types declared (pointers as c_void_p), or None if not built."""
    path = O.ref_library_path(True)
    if not os.path.exists(path):
        return None
    L = O.ref_library(True)
    P, I = ctypes.c_void_p, ctypes.c_int
    L.axpy_device_launch.argtypes = [P, P, P, I, I]
    L.axpy_device_launch.restype = I
    return L


def _vec(rng, n, scale=1.0):
    return (rng.standard_normal(n) * scale).astype(np.float32)


@pytest.mark.parametrize("n,negate", [(1, 0), (257, 1), (1_000_003, 0), (1_000_003, 1)])
def test_axpy_device_launch_bit_exact(cuda, n, negate):
    """axpy_device.cu:20-45: y = (+/-alpha) x + y with alpha read on the
    device; one rounding per element (the reference's FMA build)."""
    rng = np.random.default_rng(n + negate)
    x, y = _vec(rng, n), _vec(rng, n, 3.0)
    alpha = np.float32(rng.uniform(-2, 2))
    yd, xd, ad = dev(y), dev(x), dev([alpha])
    assert call("axpy_device_launch", ptr(yd), ptr(xd), ptr(ad), n, negate) == 0
    want = O.axpy(y, x, alpha, negate=bool(negate))
    assert np.array_equal(bits(host(yd)), bits(want))
    ref = _ref_lib()
    if ref is not None:
        yr = dev(y)
        assert ref.axpy_device_launch(ptr(yr), ptr(xd), ptr(ad), n, negate) == 0
        assert np.array_equal(bits(host(yr)), bits(want))


@pytest.mark.parametrize("n,in_place", [(5, False), (1_000_003, False), (65_536, True)])
def test_scaled_axpy_launch_bit_exact(cuda, n, in_place):
    """axpy_device.cu:51-77: p_out = z + beta p_old, in place allowed
    (p_out == p_old, the CG direction update)."""
    rng = np.random.default_rng(n)
    z, p_old = _vec(rng, n), _vec(rng, n, 2.0)
    beta = np.float32(rng.uniform(0, 1))
    zd, pd, bd = dev(z), dev(p_old), dev([beta])
    out = pd if in_place else torch.full((n,), 9.0, device="cuda")
    assert call("scaled_axpy_launch", ptr(out), ptr(zd), ptr(pd), ptr(bd), n) == 0
    assert np.array_equal(bits(host(out)), bits(O.scaled_axpy(z, p_old, beta)))


@pytest.mark.parametrize("num,den", [(3.0, 2.0), (1.0, 3.0), (-7.5, 0.0), (0.0, 0.0),
                                     (1e-30, 1e30), (2.5e38, 0.5)])
def test_divide_scalars_launch(cuda, num, den):
    """axpy_device.cu:84-99: result = num / den, and 0 when den == 0
    (axpy_device.cu:90) -- the guard CG relies on when pAp or rz vanishes."""
    nd, dd = dev([num]), dev([den])
    res = torch.full((1,), 123.0, device="cuda")
    assert call("divide_scalars_launch", ptr(nd), ptr(dd), ptr(res)) == 0
    got = host(res)[0]
    want = O.divide_scalars(num, den)
    assert bits(np.float32(got)) == bits(want)


@pytest.mark.parametrize("seed,shape", [(1, (7, 9, 11)), (2, (32, 16, 48)), (3, (3, 3, 3))])
def test_compute_b_launch_bit_exact(cuda, seed, shape):
    """axpy_device.cu:104-137: b = scale div on fluid cells, 0 elsewhere (the
    caller passes scale = -rho dx^2 / dt, pressure_solve_pcg.cu:129-139)."""
    rng = np.random.default_rng(seed)
    mat, _, div = S.parity_random_grid(rng, shape)
    scale = np.float32(-(997.0 * 0.002 * 0.002) / 0.01)
    b = torch.full(shape, 5.0, device="cuda")
    div_d, mat_d = dev(div), dev(mat, torch.int32)
    assert call("compute_b_launch", ptr(b), ptr(div_d), ptr(mat_d), *shape, float(scale), 0) == 0
    want = np.where(mat == 0, scale * div, np.float32(0.0)).astype(np.float32)
    assert np.array_equal(bits(host(b)), bits(want))


def test_zero_buffer_and_scale_inplace(cuda):
    """axpy_device.cu:142-145 (zero n floats, the rest untouched) and the FFI
    probe scale.cu:11-34 (x *= s, synchronous); sizes <= 0 are a no-op."""
    rng = np.random.default_rng(4)
    x = _vec(rng, 1000)
    xd = dev(x)
    assert call("zero_buffer_launch", ptr(xd), 600) == 0
    got = host(xd)
    assert np.all(got[:600] == 0.0) and np.array_equal(got[600:], x[600:])
    assert call("zero_buffer_launch", ptr(xd), 0) == 0
    xd = dev(x)
    assert call("scale_inplace_launch", ptr(xd), 1000, 0.75) == 0
    assert np.array_equal(bits(xd.cpu().numpy()), bits(O.scale(x, 0.75)))  # already synchronous
    assert call("scale_inplace_launch", ptr(xd), -1, 2.0) == 0


@pytest.mark.parametrize("n", [1, 1023, 4_000_037])
def test_dot_launch_fp64_accumulation(cuda, n):
    """dot_reduce.cu:92-115 contract (result to a device float, >= 1024-float
    workspace); here accumulated in FP64, so it equals the FP64 dot rounded to
    float up to the last bit."""
    rng = np.random.default_rng(n)
    x, y = _vec(rng, n), _vec(rng, n)
    ws = torch.zeros(1024, device="cuda")
    res = torch.zeros(1, device="cuda")
    xd, yd = dev(x), dev(y)
    assert call("dot_launch", ptr(xd), ptr(yd), n, ptr(ws), ptr(res)) == 0
    exact = float(np.dot(x.astype(np.float64), y.astype(np.float64)))
    got = float(host(res)[0])
    assert abs(got - exact) <= 2 * abs(float(np.spacing(np.float32(exact)))) + 1e-12


def _pcg_ws(shape):
    z = lambda *s: torch.zeros(s, dtype=torch.float32, device="cuda")  # noqa: E731
    bufs = [z(*shape) for _ in range(5)] + [z(1024)] + [z(1) for _ in range(7)]
    return bufs


@pytest.mark.parametrize("name", ["pcg_box_0.01", "pcg_box_1e-06"])
def test_pcg_launch_matches_reference_pcg_goldens(cuda, name):
    """pressure_solve_pcg_launch against the reference kernel's own outputs
    (pressure_solve_pcg.cu:89-243, tests/golden): the same iteration count
    within one check (5 iterations) and the same pressure within the FP32
    PCG's rounding (the reference sums its dots in FP32, this library in
    FP64)."""
    d = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    dx, dt, rho, tol = (float(d[k]) for k in ("dx", "dt", "rho", "tol"))
    shape = d["mat"].shape
    p = torch.full(shape, 3.0, device="cuda")
    ws = _pcg_ws(shape)
    div_d, mat_d = dev(d["div"]), dev(d["mat"], torch.int32)
    it = SimCore(0).pressure_solve_pcg(ptr(p), ptr(div_d), ptr(mat_d), *shape, dx, dt, rho, tol,
                                       200, *[ptr(w) for w in ws])
    assert abs(it - int(d["iters"])) <= 5, (it, int(d["iters"]))
    fl = d["mat"] == 0
    got = host(p)
    ref = d["p"].astype(np.float64)
    assert np.linalg.norm(got[fl] - ref[fl]) / np.linalg.norm(ref[fl]) <= 1e-5
    assert np.all(got[~fl] == 0.0)
    # the same algorithm as the oracle's (FP64 dots in another reduction order)
    po, ito = O.pcg(d["div"], d["mat"], dx, dt, rho, tol, 200)
    assert abs(it - ito) <= 5
    assert np.linalg.norm(got[fl] - po[fl]) / np.linalg.norm(po[fl]) <= 1e-5
    assert float(host(ws[10])[0]) == pytest.approx(float(d["bsq"]), rel=1e-6)  # dev_bsq


@pytest.mark.parametrize("shape", [(40, 36, 64), (33, 20, 200), (24, 24, 12)])
def test_pcg_quad_form_matches_one_cell_form(cuda, shape):
    """The four-cell form of the PCG phases (BSP_TUNE_PCG_QUAD = 1, nz % 4 ==
    0: vector loads, k neighbours by shuffles, units of 128 cells including a
    partial one when nz % 128 != 0) performs the one-cell form's per-cell
    operations; only the FP64 partial sums run in another order, so the
    iteration counts agree within one check and the pressures to FP32
    rounding of the recurrences."""
    rng = np.random.default_rng(sum(shape))
    mat, _, div = S.parity_random_grid(rng, shape)
    out = {}
    try:
        for quad in (1, 0):
            call("bsp_set_tuning", 18, quad)
            p = torch.full(shape, 3.0, device="cuda")
            ws = _pcg_ws(shape)
            div_d, mat_d = dev(div), dev(mat, torch.int32)
            it = SimCore(0).pressure_solve_pcg(ptr(p), ptr(div_d), ptr(mat_d), *shape, 0.002, 0.01,
                                               997.0, 1e-6, 400, *[ptr(w) for w in ws])
            out[quad] = (it, host(p).astype(np.float64))
    finally:
        call("bsp_set_tuning", 18, 1)
    assert abs(out[1][0] - out[0][0]) <= 5
    fl = mat == 0
    a, b = out[1][1], out[0][1]
    assert np.all(a[~fl] == 0.0)
    assert np.linalg.norm(a[fl] - b[fl]) <= 1e-4 * np.linalg.norm(b[fl])
