"""Reference runs of the guarded floor policy on the benchmark workload's own states.

    SIMPFEM_REFERENCE_ROOT=<reference checkout> python tests/golden/make_baseline_golden.py [--xlarge]

The workload's states are not Bernoulli solid masks (the reference drivers'
generator) but filtered void-probability fields: element e is void with
probability p = (0.2, 0.35, 0.5)[seed % 3] (numpy default_rng(seed)), otherwise
solid, and the mask is smoothed by the reference's own cone filter
``_build_density_filter(nelx, nely, 1.5, nelz)`` (pub_simp_solver.py:215-243);
E = rho_min + (1 - rho_min) rho^3.  The hierarchy is the damped-Jacobi 4-level
V-cycle (``_build_components(..., fine_smoother="fp64", smoother_type="jacobi")``,
run_experiments_e1_e10.py:128-179), and every state of a run goes through one
hierarchy in seed order, as the drivers reuse theirs.

For each state the reference's own MatrixFreeKff, GalerkinMatFreeGMG and
_cupy_fgmres (run unmodified on the host through ``_refshim``) carry out the
policy of run_gmg_floor_detector_prospective.py:220-354: a 100-iteration probe
at 1e-12, the driver's own ``_classify`` on r50 / r100, the ladder
{1e-3, 1e-2} on a raise (else a full solve at 1e-12), each attempt judged by
the recomputed FP64 residual, the post-solve fallback after a failed keep.

Written per state: the decision fields, the probe history, the selected
solve's iterations, residuals and compliance F.x, ||x|| and every STRIDE-th
entry of x.  A second replay with E multiplied by (1 + 1e-14 N(0, 1)) records
the reference's own round-off envelope of compliance and x.

Outputs: baseline_policy_80x40x20.npz (seeds 0-5, the plain FP64 workload on
80 x 40 x 20) and, with --xlarge, baseline_policy_160x80x40.npz (seeds 0-1 on
160 x 80 x 40, the measured workload's size).
"""

from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import _refshim  # noqa: E402

PROBS = (0.2, 0.35, 0.5)
CASES = {
    "80x40x20": dict(preset="cantilever_gpu_medium", seeds=list(range(6)), stride=31),
    "160x80x40": dict(preset="cantilever_gpu_xlarge", seeds=[0, 1], stride=211),
}


def state(H, n: int, seed: int) -> np.ndarray:
    p = PROBS[seed % len(PROBS)]
    solid = (np.random.default_rng(seed).random(n) >= p).astype(np.float64)
    return np.asarray(H @ solid)


def run_case(name: str, pert_seed: int = 0) -> dict:
    case = CASES[name]
    paper4 = _refshim.load_paper4_runner()
    drv = _refshim.load_driver_module(os.path.join("experiments", "phase5", "run_gmg_floor_detector_prospective.py"))
    mg = _refshim.load("multigrid_v4")
    pss = _refshim.load("pub_simp_solver")
    spec, bc, free, _, _, F, mf_op, gmg = paper4._build_components(
        case["preset"], n_levels=4, fine_smoother="fp64", smoother_type="jacobi")
    n = spec.nelx * spec.nely * spec.nelz
    H = pss._build_density_filter(spec.nelx, spec.nely, 1.5, spec.nelz)
    b_norm = float(np.linalg.norm(F))
    pert = 1.0 if pert_seed == 0 else 1.0 + 1e-14 * np.random.default_rng(pert_seed).standard_normal(n)
    tol, penal = 1e-6, 3.0
    rows = []
    for seed in case["seeds"]:
        rho = state(H, n, seed)

        def solve_at_floor(rho_min, maxiter, history):
            E = (rho_min + (1.0 - rho_min) * rho ** penal) * pert
            gmg.setup(E)
            x, iters, reported = mg._cupy_fgmres(lambda v: mf_op.matvec(v, E), F, gmg.apply, tol=tol,
                                                 maxiter=maxiter, restart=300, history=history)
            final = float(np.linalg.norm(F - mf_op.matvec(x, E)) / b_norm)
            return dict(rho_min=rho_min, iters=int(iters), reported=bool(reported), converged=final <= tol,
                        final=final, x=x)

        t0 = time.perf_counter()
        probe_history: list = []
        probe = solve_at_floor(1e-12, 100, probe_history)
        r50 = probe_history[min(50, len(probe_history) - 1)]
        r100 = probe_history[min(100, len(probe_history) - 1)]
        raise_floor, trigger = drv._classify(r50, r100, high_residual_threshold=1e-2,
                                             plateau_residual_threshold=1e-4, plateau_ratio_threshold=0.6)
        ladder = [1e-3, 1e-2] if raise_floor else [1e-12]
        attempted: list = []
        sel = None

        def sequence(floors):
            nonlocal sel
            for f in floors:
                if f in attempted:
                    continue
                attempted.append(f)
                sel = solve_at_floor(f, 300, [])
                if sel["converged"]:
                    break

        sequence(ladder)
        fallback = False
        if not sel["converged"] and not raise_floor:
            fallback = True
            sequence([1e-3, 1e-2])
        x = sel["x"]
        rows.append(dict(
            seed=seed, p=PROBS[seed % len(PROBS)], r50=float(r50), r100=float(r100), trigger=trigger,
            raise_floor=bool(raise_floor), fallback=fallback, attempted=";".join(f"{v:.0e}" for v in attempted),
            rho_min=sel["rho_min"], iters=sel["iters"], reported=sel["reported"], converged=bool(sel["converged"]),
            final=sel["final"], probe_iters=probe["iters"], compliance=float(np.dot(F, x)),
            x_norm=float(np.linalg.norm(x)), x_sample=np.asarray(x[:: case["stride"]]),
            probe_history=list(map(float, probe_history)), seconds=time.perf_counter() - t0))
        print(name, pert_seed, {k: v for k, v in rows[-1].items() if k not in ("x_sample", "probe_history")},
              flush=True)
    return dict(rows=rows, stride=case["stride"], preset=case["preset"])


def write(name: str) -> None:
    ref = run_case(name)
    alt = run_case(name, pert_seed=99)
    rows, prow = ref["rows"], alt["rows"]
    out = dict(
        meta=json.dumps(dict(preset=ref["preset"], stride=ref["stride"], probs=PROBS, rmin=1.5, penal=3.0,
                             tol=1e-6, restart=300, maxiter=300, probe_iters=100, probe_r50=50,
                             ladder=[1e-3, 1e-2], stack="damped Jacobi, 4 levels, fp64",
                             pert="E * (1 + 1e-14 N(0,1)), default_rng(99)")),
        rows=json.dumps([{k: v for k, v in r.items() if k not in ("x_sample", "probe_history")} for r in rows]),
        pert_rows=json.dumps([{k: v for k, v in r.items() if k not in ("x_sample", "probe_history")}
                              for r in prow]),
        x_sample=np.stack([r["x_sample"] for r in rows]),
        pert_x_sample=np.stack([r["x_sample"] for r in prow]),
        probe_history=json.dumps([r["probe_history"] for r in rows]),
    )
    path = os.path.join(HERE, f"baseline_policy_{name}.npz")
    np.savez_compressed(path, **out)
    print("wrote", path)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--xlarge", action="store_true", help="also the 160x80x40 states (slow on a CPU)")
    ap.add_argument("--only-xlarge", action="store_true")
    a = ap.parse_args()
    if not a.only_xlarge:
        write("80x40x20")
    if a.xlarge or a.only_xlarge:
        write("160x80x40")
