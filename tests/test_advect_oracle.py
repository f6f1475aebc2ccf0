"""CPU checks of the semi-Lagrangian advection restatement (oracle):
fluid.py:39-104 (trilinear sampling, velocity at a point), :338-498
(extension of T into solids, T and face-velocity advection), :737-776
(advect_all).

The reference's Warp kernels cannot run here and its tests hold no vectors
for them, so the restatement is pinned by its own test of the path,
python/tests/test_fluid.py:147-187 (sum of T over fluid cells drifts < 2 %
over 20 steps of a projected random flow in a walled 12^3 box), and by
closed-form answers: a uniform field stays uniform, zero velocity leaves
every field unchanged, a uniform flow translates a linear profile exactly
(trilinear interpolation reproduces linear functions), the extension rule
takes the first fluid neighbour in the order -x, +x, -y, +y, -z, +z, and
the face rules (boundary faces zero, faces between two non-fluid cells
kept)."""
from __future__ import annotations

import math

import numpy as np

import oracle as O

F, W, A = O.MAT_FLUID, O.MAT_POT_WALL, O.MAT_AIR


def walled(n):
    mat = np.full((n, n, n), W, np.int32)
    mat[1:-1, 1:-1, 1:-1] = F
    return mat


def faces(shape):
    nx, ny, nz = shape
    return (nx + 1, ny, nz), (nx, ny + 1, nz), (nx, ny, nz + 1)


def test_reference_drift_test_restated():
    """test_fluid.py:147-187 on the oracle: walled 12^3, cosine T in x,
    N(0, 0.05) velocities, no-slip, 1500-sweep projection, 20 advect_all steps
    at dt 0.01: relative drift of sum T over fluid cells < 0.02."""
    n, dx = 12, 0.002
    mat = walled(n)
    T = np.full((n, n, n), 293.15, np.float32)
    for i in range(1, n - 1):
        T[i] = 293.15 + 30.0 * math.cos(math.pi * (i - n / 2) / n)
    rng = np.random.default_rng(0)
    u = [(rng.standard_normal(s).astype(np.float32) * 0.05) for s in faces(mat.shape)]
    u = list(O.enforce_no_slip(*u, mat))
    proj = O.projection_jacobi(*u, mat, dx, 0.01, 997.0, 1500)
    ux, uy, uz = proj["ux"], proj["uy"], proj["uz"]
    assert proj["max_div"] < 1e-2
    fluid = mat == F
    s0 = float(T[fluid].astype(np.float64).sum())
    org = (0.0, 0.0, 0.0)
    for _ in range(20):
        ux, uy, uz, T, _ = O.advect_all(ux, uy, uz, T, mat, org, dx, 0.01)
    s1 = float(T[fluid].astype(np.float64).sum())
    assert abs(s1 - s0) / abs(s0) < 0.02


def test_uniform_fields_stay_uniform_and_zero_flow_is_identity():
    rng = np.random.default_rng(2)
    mat = walled(10)
    org = (-0.01, -0.01, -0.004)
    T = np.full(mat.shape, 300.0, np.float32)
    u = [(rng.standard_normal(s).astype(np.float32) * 0.05) for s in faces(mat.shape)]
    ux, uy, uz, T1, _ = O.advect_all(*u, T, mat, org, 0.001, 0.01)
    assert np.all(T1 == 300.0)
    z = [np.zeros(s, np.float32) for s in faces(mat.shape)]
    Tr = (280 + 40 * rng.random(mat.shape)).astype(np.float32)
    ux, uy, uz, T2, _ = O.advect_all(*z, Tr, mat, (0.0, 0.0, 0.0), 0.002, 0.01)
    assert np.allclose(T2, Tr, rtol=0, atol=1e-4)
    assert np.all(ux == 0) and np.all(uy == 0) and np.all(uz == 0)


def test_uniform_flow_translates_a_linear_profile():
    """ux = U everywhere, T linear in x: the backtrace lands U dt upstream and
    trilinear interpolation is exact on linear data, so T_new = T - a U dt."""
    n, dx, dt, U, a = 16, 0.002, 0.01, 0.05, 100.0
    mat = np.full((n, n, n), F, np.int32)
    x = (np.arange(n) + 0.5) * dx
    T = np.broadcast_to((300.0 + a * x)[:, None, None], mat.shape).astype(np.float32).copy()
    ext = O.extend_temperature(T, mat)
    ux = np.full((n + 1, n, n), U, np.float32)
    uy = np.zeros((n, n + 1, n), np.float32)
    uz = np.zeros((n, n, n + 1), np.float32)
    Tn = O.advect_temperature(T, ext, ux, uy, uz, mat, (0.0, 0.0, 0.0), dx, dt)
    inner = slice(2, n - 2)
    want = T - a * U * dt
    np.testing.assert_allclose(Tn[inner, inner, inner], want[inner, inner, inner], atol=2e-4)


def test_extension_takes_first_fluid_neighbour_in_face_order():
    mat = np.full((3, 3, 3), W, np.int32)
    T = np.arange(27, dtype=np.float32).reshape(3, 3, 3)
    c = (1, 1, 1)
    # fluid at +x and -y of the centre: -x is not fluid, +x is -> +x wins over -y
    mat[2, 1, 1] = F
    mat[1, 0, 1] = F
    ext = O.extend_temperature(T, mat)
    assert ext[c] == T[2, 1, 1]
    assert ext[2, 1, 1] == T[2, 1, 1]  # fluid keeps its own value
    # isolated solid keeps its own value
    assert ext[0, 2, 2] == T[0, 2, 2]


def test_face_rules():
    rng = np.random.default_rng(4)
    mat = np.full((6, 5, 4), A, np.int32)
    mat[2:4, 1:4, 1:3] = F
    u = [(rng.standard_normal(s).astype(np.float32)) for s in faces(mat.shape)]
    for ax in range(3):
        un = O.advect_velocity(ax, *u, mat, (0.0, 0.0, 0.0), 0.002, 0.001)
        src = u[ax]
        idx = [slice(None)] * 3
        idx[ax] = 0
        assert np.all(un[tuple(idx)] == 0)
        idx[ax] = -1
        assert np.all(un[tuple(idx)] == 0)
        # interior faces between two non-fluid cells keep their value
        nf = mat != F
        lo = [slice(None)] * 3
        hi = [slice(None)] * 3
        lo[ax] = slice(0, -1)
        hi[ax] = slice(1, None)
        both = nf[tuple(lo)] & nf[tuple(hi)]
        inner = [slice(None)] * 3
        inner[ax] = slice(1, -1)
        assert np.array_equal(un[tuple(inner)][both], src[tuple(inner)][both])


def test_uniform_flow_translates_a_linear_face_profile():
    """advect_ux with ux = U + b y on all-fluid cells and uy = uz = 0: the
    backtrace moves (U + b y) dt along x only, and ux is constant along x,
    so interior faces keep their value (up to rounding)."""
    n, dx, dt, U, b = 12, 0.002, 0.01, 0.05, 2.0
    mat = np.full((n, n, n), F, np.int32)
    y = (np.arange(n) + 0.5) * dx
    ux = np.broadcast_to((U + b * y)[None, :, None], (n + 1, n, n)).astype(np.float32).copy()
    uy = np.zeros((n, n + 1, n), np.float32)
    uz = np.zeros((n, n, n + 1), np.float32)
    un = O.advect_velocity(0, ux, uy, uz, mat, (0.0, 0.0, 0.0), dx, dt)
    inner = (slice(2, n - 1), slice(1, n - 1), slice(1, n - 1))
    np.testing.assert_allclose(un[inner], ux[inner], rtol=0, atol=1e-6)
    assert np.all(un[0] == 0) and np.all(un[-1] == 0)
