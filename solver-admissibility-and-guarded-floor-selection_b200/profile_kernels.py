"""Standalone launches of single kernels of the library, for timing and for ncu.

    python profile_kernels.py smoother-step NX NY NZ [REPS] [--stack plain|canonical] [--precision fp32|fp64]
    python profile_kernels.py dense N [REPS] [--band BW]
    python profile_kernels.py policy NX NY NZ [--restart R] [--precision mixed|fp64]

smoother-step: builds the 4-level hierarchy on an NX x NY x NZ cantilever
(random E in [1e-3, 1.001)), then times REPS fused fine smoothing steps with
simpfem_gmg_time_smoother_step (each launch after an L2-evicting write, on
pseudo-random vectors) and prints the average launch time and the algorithmic
bandwidth.  dense: factors and inverts a random SPD N x N matrix (banded with
lower bandwidth BW when --band is given, as the coarsest level is) with
simpfem_dense_cholesky_inverse REPS times and prints the best time.
policy: one guarded solve of the plain-stack policy on the NX x NY x NZ cantilever
(seeded void p = 0.35 state, cone filter r = 1.5, SIMP p = 3) after three warm-up
states, bracketed by cudaProfilerStart/Stop so that `ncu --profile-from-start off`
sees exactly that solve; --restart bounds the FGMRES basis (device memory) of
the capture.  All exit 0 on success, so the same command line can run under ncu
afterwards.
"""

from __future__ import annotations

import argparse
import ctypes
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)


def smoother_step(a) -> None:
    import numpy as np
    import torch

    from gpu_fem import _lib
    from gpu_fem.paper4 import CANONICAL_STACK, PLAIN_JACOBI_STACK, _build_components
    from gpu_fem.presets import cantilever_spec

    nx, ny, nz = a.nx, a.ny, a.nz
    st = dict(CANONICAL_STACK if a.stack == "canonical" else PLAIN_JACOBI_STACK)
    st["fine_smoother"] = a.precision
    cyc = "fp32" if a.precision == "fp32" else "fp64"
    spec, bc, free, fg, ed, F, mf, gmg = _build_components(cantilever_spec(nx, ny, nz), cycle_precision=cyc, **st)
    E = torch.as_tensor(1e-3 + np.random.default_rng(0).random(nx * ny * nz), device="cuda")
    gmg.setup(E)
    avg = ctypes.c_float()
    _lib.call("simpfem_gmg_time_smoother_step", gmg._h, 0, a.reps, ctypes.byref(avg), _lib.stream_ptr())
    torch.cuda.synchronize()
    ndof = 3 * (nx + 1) * (ny + 1) * (nz + 1)
    ne = nx * ny * nz
    s = 4 if a.precision == "fp32" else 8
    nvec = 4 if a.stack == "plain" else 6  # u, rhs, dinv (+ d) read, x (+ d) written
    alg = nvec * s * ndof + s * ne + ndof
    print(f"smoother-step {a.stack} {a.precision} {nx}x{ny}x{nz}: avg {avg.value * 1e3:.2f} us, "
          f"algorithmic {alg / 1e6:.1f} MB, {alg / (avg.value * 1e-3) / 1e9:.1f} GB/s")


def dense(a) -> None:
    import torch

    from gpu_fem import _lib

    n = a.n
    g = torch.Generator(device="cuda")
    g.manual_seed(0)
    if a.band is None:
        Q = torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g)
        A0 = Q @ Q.T / n + torch.eye(n, dtype=torch.float64, device="cuda")
    else:
        # symmetric, band of random entries, diagonally dominant
        R = torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g)
        i = torch.arange(n, device="cuda")
        inband = (i[:, None] - i[None, :]).abs() <= a.band
        A0 = torch.where(inband, R, torch.zeros_like(R))
        A0 = torch.tril(A0, -1) + torch.tril(A0, -1).T + torch.diag(torch.full((n,), 2.0 * a.band + 2.0,
                                                                             dtype=torch.float64, device="cuda"))
    A = torch.empty_like(A0)
    Li = torch.empty_like(A0)
    info = ctypes.c_int()
    best = float("inf")
    for _ in range(a.reps):
        A.copy_(A0)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        _lib.call("simpfem_dense_cholesky_inverse", n, _lib.ptr(A), _lib.ptr(Li), ctypes.byref(info),
                  _lib.stream_ptr())
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    if info.value != 0:
        raise SystemExit(f"factorisation failed: info {info.value}")
    if a.band is None:
        gflop = 2.0 * n ** 3 / 3.0 / 1e9
        print(f"dense n={n}: best {best:.3f} ms over {a.reps}, {gflop:.1f} GFLOP, {gflop / best:.2f} TFLOP/s")
    else:
        print(f"dense n={n} band={a.band}: best {best:.3f} ms over {a.reps}")


def policy(a) -> None:
    import numpy as np
    import torch

    from gpu_fem.paper4 import PLAIN_JACOBI_STACK
    from gpu_fem.policy import GuardedFloorPolicy
    from gpu_fem.presets import cantilever_spec
    from gpu_fem.pub_simp_solver import _build_density_filter

    nx, ny, nz = a.nx, a.ny, a.nz
    H = _build_density_filter(nx, ny, 1.5, nz)
    mixed = a.precision == "mixed"
    stack = dict(PLAIN_JACOBI_STACK, fine_smoother="fp32" if mixed else "fp64")
    pol = GuardedFloorPolicy(cantilever_spec(nx, ny, nz), penal=3.0, tol=1e-6, restart=a.restart,
                             maxiter=a.restart, probe_iters=100, probe_r50=50, raised_rho_mins=(1e-3, 1e-2),
                             stack=stack, cycle_precision="fp32" if mixed else "fp64")

    def state(seed):
        solid = (np.random.default_rng(seed).random(nx * ny * nz) >= 0.35).astype(np.float64)
        return torch.as_tensor(np.asarray(H @ solid), device="cuda")

    for seed in range(3):
        pol.run(state(seed))
    d = state(3)
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    r = pol.run(d)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    print(f"policy {a.precision} {nx}x{ny}x{nz}: {r['total_iters']} iterations, floor {r['recommended_rho_min']:.0e}, "
          f"setup {r['probe_setup_time_s'] * 1e3:.2f} ms, solve {r['probe_solve_time_s'] * 1e3:.2f} ms, "
          f"guarded {r['solve_converged']}")


def main() -> None:
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    p = sub.add_parser("smoother-step")
    p.add_argument("nx", type=int)
    p.add_argument("ny", type=int)
    p.add_argument("nz", type=int)
    p.add_argument("reps", type=int, nargs="?", default=20)
    p.add_argument("--stack", default="plain", choices=["plain", "canonical"])
    p.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    d = sub.add_parser("dense")
    d.add_argument("n", type=int)
    d.add_argument("reps", type=int, nargs="?", default=5)
    d.add_argument("--band", type=int, default=None)
    q = sub.add_parser("policy")
    q.add_argument("nx", type=int)
    q.add_argument("ny", type=int)
    q.add_argument("nz", type=int)
    q.add_argument("--restart", type=int, default=300)
    q.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    a = ap.parse_args()
    {"smoother-step": smoother_step, "dense": dense, "policy": policy}[a.cmd](a)


if __name__ == "__main__":
    main()
