"""CPU checks of the backward-Euler conduction restatement (oracle) against
closed-form answers of the discrete system of thermal.py:259-388.

The reference holds no stored vectors for this kernel and its Warp code cannot
run here, so the restatement is pinned by known answers of the equations it
states: the cell-centred cosine mode's backward-Euler decay factor, Newton
cooling of an isolated solid cell, the harmonic-mean face conductivity at a
water/steel face, energy conservation in a closed box, and the ping-pong /
snapshot contract of conduct_one_step (thermal.py:647-658)."""
from __future__ import annotations

import math

import numpy as np

import oracle as O

WATER = (997.0, 4186.0, 0.606)
STEEL = (8000.0, 500.0, 16.2)
AIR = (1.184, 1005.0, 0.0262)
CARROT = (1040.0, 3900.0, 0.605)


def props(rows=(WATER, STEEL, AIR, CARROT)):
    rho, cp, k = (np.array([r[i] for r in rows], np.float32) for i in range(3))
    return k, rho, cp


def test_cosine_mode_decays_by_the_backward_euler_factor():
    nx, dx = 40, 0.0005
    k, rho, cp = props()
    alpha = float(k[1]) / (float(rho[1]) * float(cp[1]))
    dt = 0.5 * dx * dx / alpha  # gamma = 0.5
    x = np.arange(nx) + 0.5
    amp = 50.0
    T = (300.0 + amp * np.cos(math.pi * x / nx)).astype(np.float32)[:, None, None]
    mat = np.full((nx, 1, 1), 1, np.int32)
    Tn, _, Told = O.conduction_be(T, np.zeros_like(T), mat, (k, rho, cp), dx, dt, 10.0, 295.0,
                                  n_iter=120)
    assert np.array_equal(Told, T)
    gamma = dt * alpha / (dx * dx)
    lam = 2.0 - 2.0 * math.cos(math.pi / nx)
    want = 300.0 + amp / (1.0 + gamma * lam) * np.cos(math.pi * x / nx)
    np.testing.assert_allclose(Tn[:, 0, 0], want, rtol=0, atol=2e-4)


def test_newton_cooling_of_an_isolated_cell():
    k, rho, cp = props()
    mat = np.full((3, 3, 3), 2, np.int32)
    mat[1, 1, 1] = 1
    T = np.full((3, 3, 3), 123.0, np.float32)
    T[1, 1, 1] = 400.0
    dx, dt, h, tamb = 0.002, 0.05, 10.0, 295.15
    out = O.conduction_sweep(np.full_like(T, -1.0), T, T, mat, (k, rho, cp), dx, dt, h, tamb)
    g = dt * h / (float(rho[1]) * float(cp[1]) * dx)
    want = (400.0 + 6 * g * tamb) / (1 + 6 * g)
    assert abs(out[1, 1, 1] - want) < 1e-4
    # air cells are not written
    assert np.all(np.delete(out.ravel(), 13) == -1.0)


def test_harmonic_mean_face_conductivity():
    k, rho, cp = props()
    mat = np.array([0, 1], np.int32)[:, None, None]
    T = np.array([300.0, 340.0], np.float32)[:, None, None]
    dx, dt = 0.001, 0.01
    out = O.conduction_sweep(np.zeros_like(T), T, T, mat, (k, rho, cp), dx, dt, 10.0, 295.0)
    kw, ks = float(k[0]), float(k[1])
    kf = 2 * kw * ks / (kw + ks)
    gw = dt * kf / (float(rho[0]) * float(cp[0]) * dx * dx)
    gs = dt * kf / (float(rho[1]) * float(cp[1]) * dx * dx)
    assert abs(out[0, 0, 0] - (300.0 + gw * 340.0) / (1 + gw)) < 1e-4
    assert abs(out[1, 0, 0] - (340.0 + gs * 300.0) / (1 + gs)) < 1e-4


def test_closed_steel_box_conserves_energy():
    shape = (10, 9, 8)
    k, rho, cp = props()
    mat = np.full(shape, 1, np.int32)
    T = np.full(shape, 293.15, np.float32)
    T[:4, :4, :4] = 400.0
    dt = 2.0
    Tn, _, _ = O.conduction_be(T, np.zeros_like(T), mat, (k, rho, cp), 0.002, dt, 10.0,
                               295.0, n_iter=400)
    e0, e1 = T.astype(np.float64).sum(), Tn.astype(np.float64).sum()
    assert abs(e1 - e0) / e0 < 1e-6
    assert Tn.max() < 400.0 and Tn.min() > 293.15


def test_odd_count_copies_the_ping_pong_buffer_back():
    rng = np.random.default_rng(5)
    shape = (6, 5, 7)
    k, rho, cp = props()
    mat = rng.integers(0, 4, shape).astype(np.int32)
    T = (280 + 40 * rng.random(shape)).astype(np.float32)
    alt = (rng.random(shape) * 1000).astype(np.float32)
    args = ((k, rho, cp), 0.002, 0.5, 10.0, 295.15)
    Te, ae, oe = O.conduction_be(T, alt, mat, *args, n_iter=4)
    To, ao, oo = O.conduction_be(T, alt, mat, *args, n_iter=5)
    assert np.array_equal(oe, T) and np.array_equal(oo, T)
    # odd: T == T_alt everywhere, air cells included (the whole-array copy)
    assert np.array_equal(To, ao)
    air = mat == 2
    assert np.array_equal(ao[air], alt[air])   # never written
    assert np.array_equal(Te[air], T[air])     # even: T's air cells untouched
    # the step equals the sweeps done one by one
    a = alt.copy()
    cur = T.copy()
    for it in range(5):
        if it % 2 == 0:
            a = O.conduction_sweep(a, cur, T, mat, *args)
        else:
            cur = O.conduction_sweep(cur, a, T, mat, *args)
    assert np.array_equal(a, ao)


def test_newton_cooling_pulls_a_uniform_block_toward_ambient():
    """A steel block in air, uniform and above T_amb: every step lowers every
    block cell and none falls below T_amb; the corners (three air faces) cool
    fastest, the centre slowest."""
    k, rho, cp = props()
    mat = np.full((8, 8, 8), 2, np.int32)
    mat[1:-1, 1:-1, 1:-1] = 1
    T = np.full(mat.shape, 400.0, np.float32)
    solid = mat == 1
    prev = T
    for _ in range(3):
        Tn, _, _ = O.conduction_be(prev, np.zeros_like(prev), mat, (k, rho, cp), 0.002, 50.0,
                                   10.0, 295.0, n_iter=30)
        assert np.all(Tn[solid] < prev[solid]) and np.all(Tn[solid] > 295.0)
        prev = Tn
    assert prev[1, 1, 1] < prev[4, 4, 4]
