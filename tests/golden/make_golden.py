"""Generate golden vectors from the reference's own CUDA kernels.

The reference's hot-path sources (crates/cuda-kernels/src/{jacobi_pressure,
laplacian_spmv,diag_inverse_apply,dot_reduce,axpy_device,pressure_solve_pcg}.cu)
are compiled from source by ``oracle/Makefile`` into
``oracle/_ref/libref_fma.so`` (the reference's default nvcc flags) and
``oracle/_ref/libref_nofma.so`` (its ``--fmad=false`` bit-exact build).  This
script runs them on a GPU through ctypes on the inputs the reference's own
tests use and stores inputs and outputs as small .npz fixtures:

* ``sweep_<seed>.npz`` -- one ``jacobi_pressure_launch`` on the 8 (seed, shape)
  cases of python/tests/test_pressure_parity.py:112-121 with the grid generator
  of :51-67 and dx, dt, rho drawn as :138-140;
* ``spmv_<seed>.npz``  -- ``laplacian_spmv_launch`` (both builds) and
  ``diag_inverse_apply_launch`` on random grids;
* ``solve_<name>.npz`` -- ``pressure_solve_launch`` (200 and 7 sweeps) on the
  single-carrot pot at dx = 4 mm seeded as test_pressure_parity.py:176-187;
* ``pcg_<name>.npz``  -- ``pressure_solve_pcg_launch`` results and iteration
  counts on the tolerance-contract grid of test_pressure_cg.py:275-343.

Usage (needs a GPU):  python tests/golden/make_golden.py --out tests/golden
"""
from __future__ import annotations

import argparse
import ctypes
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "boiling-sim_b200"))

import oracle as O  # noqa: E402
from boilingsim_b200 import scenes as S  # noqa: E402

P = ctypes.c_void_p
I = ctypes.c_int
F = ctypes.c_float


def _bind(lib):
    lib.jacobi_pressure_launch.argtypes = [P, P, P, P, I, I, I, F, F, F, I, I]
    lib.pressure_solve_launch.argtypes = [P, P, P, P, I, I, I, F, F, F, I, I, I]
    lib.laplacian_spmv_launch.argtypes = [P, P, P, I, I, I, I, I]
    lib.diag_inverse_apply_launch.argtypes = [P, P, P, I, I, I, I, I]
    lib.pressure_solve_pcg_launch.argtypes = ([P, P, P, I, I, I, F, F, F, I, I, F, I] + [P] * 13
                                              + [ctypes.POINTER(ctypes.c_int)])
    for fn in ("jacobi_pressure_launch", "pressure_solve_launch", "laplacian_spmv_launch",
               "diag_inverse_apply_launch", "pressure_solve_pcg_launch"):
        getattr(lib, fn).restype = I
    return lib


def dev(a, dt):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dt).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def one_sweep(lib, mat, p_old, div, dx, dt, rho):
    nx, ny, nz = mat.shape
    out = torch.zeros(mat.shape, dtype=torch.float32, device="cuda")
    m, p, d = dev(mat, torch.int32), dev(p_old, torch.float32), dev(div, torch.float32)
    assert lib.jacobi_pressure_launch(out.data_ptr(), p.data_ptr(), d.data_ptr(), m.data_ptr(),
                                      nx, ny, nz, dx, dt, rho, 0, 2) == 0
    return host(out)


def spmv(lib, mat, p):
    nx, ny, nz = mat.shape
    out = torch.zeros(mat.shape, dtype=torch.float32, device="cuda")
    m, pp = dev(mat, torch.int32), dev(p, torch.float32)
    assert lib.laplacian_spmv_launch(out.data_ptr(), pp.data_ptr(), m.data_ptr(), nx, ny, nz,
                                     0, 2) == 0
    return host(out)


def diag(lib, mat, r):
    nx, ny, nz = mat.shape
    out = torch.zeros(mat.shape, dtype=torch.float32, device="cuda")
    m, rr = dev(mat, torch.int32), dev(r, torch.float32)
    assert lib.diag_inverse_apply_launch(out.data_ptr(), rr.data_ptr(), m.data_ptr(), nx, ny, nz,
                                         0, 2) == 0
    return host(out)


def solve(lib, mat, p0, div, dx, dt, rho, n_iter):
    nx, ny, nz = mat.shape
    p = dev(p0, torch.float32)
    tmp = torch.zeros_like(p)
    m, d = dev(mat, torch.int32), dev(div, torch.float32)
    assert lib.pressure_solve_launch(p.data_ptr(), tmp.data_ptr(), d.data_ptr(), m.data_ptr(),
                                     nx, ny, nz, dx, dt, rho, n_iter, 0, 2) == 0
    return host(p)


def pcg(lib, mat, div, dx, dt, rho, tol, max_iter):
    nx, ny, nz = mat.shape
    z = lambda *s: torch.zeros(s, dtype=torch.float32, device="cuda")  # noqa: E731
    p = z(nx, ny, nz)
    ws = [z(nx, ny, nz) for _ in range(5)] + [z(1024)] + [z(1) for _ in range(7)]
    m, d = dev(mat, torch.int32), dev(div, torch.float32)
    it = ctypes.c_int(0)
    assert lib.pressure_solve_pcg_launch(p.data_ptr(), d.data_ptr(), m.data_ptr(), nx, ny, nz,
                                         dx, dt, rho, 0, 2, tol, max_iter,
                                         *[w.data_ptr() for w in ws], ctypes.byref(it)) == 0
    return host(p), int(it.value), float(host(ws[10])[0])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    fma = _bind(O.ref_library(True))
    nofma = _bind(O.ref_library(False))

    for seed, shape in S.PARITY_CASES:
        rng = np.random.default_rng(seed)
        mat, p_old, div = S.parity_random_grid(rng, shape)
        dx = float(rng.uniform(0.0005, 0.004))
        dt = float(rng.uniform(0.0001, 0.01))
        rho = float(rng.uniform(900.0, 1100.0))
        np.savez_compressed(os.path.join(args.out, f"sweep_{seed}.npz"), mat=mat, p_old=p_old,
                            div=div, dx=np.float32(dx), dt=np.float32(dt), rho=np.float32(rho),
                            ref_fma=one_sweep(fma, mat, p_old, div, dx, dt, rho),
                            ref_nofma=one_sweep(nofma, mat, p_old, div, dx, dt, rho))

    for seed, shape in [(11, (14, 12, 18)), (12, (9, 20, 13))]:
        rng = np.random.default_rng(seed)
        mat, p, _ = S.parity_random_grid(rng, shape)
        mat[0, 3, 4] = 0  # fluid on the outer layer: out-of-range neighbours are air
        np.savez_compressed(os.path.join(args.out, f"spmv_{seed}.npz"), mat=mat, p=p,
                            ap_fma=spmv(fma, mat, p), ap_nofma=spmv(nofma, mat, p),
                            z=diag(fma, mat, p))

    mat = S.single_carrot_mat(0.004)
    rng = np.random.default_rng(7)
    ux = rng.standard_normal((mat.shape[0] + 1,) + mat.shape[1:]).astype(np.float32) * 0.05
    uy = rng.standard_normal((mat.shape[0], mat.shape[1] + 1, mat.shape[2])).astype(np.float32) * 0.05
    uz = rng.standard_normal(mat.shape[:2] + (mat.shape[2] + 1,)).astype(np.float32) * 0.05
    div = O.divergence(ux, uy, uz, mat, 0.004)
    p0 = np.zeros(mat.shape, np.float32)
    for n in (200, 7):
        np.savez_compressed(os.path.join(args.out, f"solve_carrot_{n}.npz"), mat=mat, p0=p0,
                            div=div, dx=np.float32(0.004), dt=np.float32(0.01),
                            rho=np.float32(997.0), n_iter=np.int32(n),
                            ref=solve(fma, mat, p0, div, 0.004, 0.01, 997.0, n))

    mat = np.zeros((16, 16, 24), np.int32)
    mat[:, :, 0] = 2
    mat[:, :, -1] = 2
    div = (np.random.default_rng(42).standard_normal(mat.shape) * 5e-3).astype(np.float32)
    for tol in (1e-2, 1e-6):
        p, it, bsq = pcg(fma, mat, div, 0.002, 0.001, 997.0, tol, 200)
        np.savez_compressed(os.path.join(args.out, f"pcg_box_{tol:g}.npz"), mat=mat, div=div,
                            p=p, iters=np.int32(it), bsq=np.float32(bsq), tol=np.float32(tol),
                            dx=np.float32(0.002), dt=np.float32(0.001), rho=np.float32(997.0))
    print("golden vectors written to", args.out)


if __name__ == "__main__":
    main()
