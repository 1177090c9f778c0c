"""The prospective floor-detector driver with the reference's output schema.

Same command-line flags, state generator, policy and CSV files as the
reference's experiments/phase5/run_gmg_floor_detector_prospective.py
(:90-513): for every seed and solid probability, the binary state
``random(seed) < p`` is solved by the probe / r50-r100 rule / floor ladder /
FP64 guard policy (gpu_fem.policy.GuardedFloorPolicy, the canonical stack by
default) and one row goes to ``prospective_summary.csv`` with the reference's
columns in the reference's order, plus the probe's and every attempted solve's
residual histories to ``prospective_history.csv``.  The reference's summary and
figure scripts read these files unchanged.

Differences, by construction of this build: memory columns come from the CUDA
device and the torch allocator (``*_cupy_pool_*`` hold the allocator's
allocated / reserved MB) after the policy's last solve; a probe that converged
at the baseline floor is reused as the answer (the identical deterministic
computation the reference repeats), and its history is written again as the
``recommended_solve`` phase.

    python prospective_driver.py --preset cantilever_gpu_medium --probabilities 0.10,0.15 --seeds 23 \\
        --out-dir results/
"""

from __future__ import annotations

import argparse
import csv
import os
import sys
from pathlib import Path

import numpy as np

if __package__ in (None, ""):
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    __package__ = "gpu_fem"  # noqa: A001

from . import _lib  # noqa: E402

SUMMARY_FIELDS = [
    "preset", "seed", "solid_probability", "baseline_rho_min", "raised_rho_min", "raised_rho_mins",
    "recommended_rho_min", "attempted_rho_mins", "n_floor_attempts", "penal", "probe_iters", "restart", "maxiter",
    "tol", "stack_variant", "n_levels", "fine_smoother", "smoother_type", "cycle_type", "coarse_correction_policy",
    "root_local_correction_mode", "root_local_correction_inner_steps", "root_local_correction_inner_restart",
    "inner_krylov_steps", "inner_krylov_restart", "solid_count", "solid_fraction", "n_components",
    "largest_component", "largest_fraction_of_solid", "support_to_load_patch_components", "probe_r50", "probe_r100",
    "probe_r100_over_r50", "probe_setup_time_s", "probe_solve_time_s", "probe_gpu_used_mb_after_solve",
    "probe_cupy_pool_used_mb_after_solve", "trigger", "predicted_raise_floor", "severity_jump_triggered",
    "severity_jump_r50_threshold", "severity_jump_rho_min", "post_solve_fallback_triggered", "detector_false_keep",
    "solve_converged", "solver_reported_converged", "solve_iters", "solve_final_rel_residual",
    "selected_setup_time_s", "selected_solve_time_s", "selected_gpu_used_mb_after_solve",
    "selected_cupy_pool_used_mb_after_solve", "selected_cupy_pool_total_mb_after_solve",
    "failed_ladder_setup_time_s", "failed_ladder_solve_time_s", "recorded_policy_time_s",
]
HISTORY_FIELDS = ["seed", "solid_probability", "phase", "rho_min", "iter", "rel_residual"]


def connectivity(mask: np.ndarray) -> dict:
    """6-connected solid components of an (nelx, nely, nelz) mask: how many, the
    largest, and how many touch both the x = 0 support face and the load patch
    (x = nelx - 1, |y - nely//2| <= 1, |z - nelz//2| <= 1), as the reference's
    _connectivity (:35-76) counts them."""
    from scipy import ndimage

    mask = np.asarray(mask, dtype=bool)
    nelx, nely, nelz = mask.shape
    labels, n = ndimage.label(mask, structure=ndimage.generate_binary_structure(3, 1))
    sizes = np.bincount(labels.ravel(), minlength=n + 1)[1:]
    support = set(np.unique(labels[0][labels[0] > 0]).tolist())
    cy, cz = nely // 2, nelz // 2
    patch = labels[nelx - 1, max(0, cy - 1):cy + 2, max(0, cz - 1):cz + 2]
    load = set(np.unique(patch[patch > 0]).tolist())
    solid = int(mask.sum())
    largest = int(sizes.max()) if n else 0
    return {
        "solid_count": solid,
        "solid_fraction": solid / mask.size,
        "n_components": int(n),
        "largest_component": largest,
        "largest_fraction_of_solid": largest / max(solid, 1),
        "support_to_load_patch_components": len(support & load),
    }


def write_csv(path: Path, rows: list, fields: list) -> None:
    path.parent.mkdir(parents=True, exist_ok=True)
    with path.open("w", newline="", encoding="utf-8") as f:
        writer = csv.DictWriter(f, fieldnames=fields)
        writer.writeheader()
        writer.writerows(rows)


def _memory():
    torch = _lib.require_cuda()
    free_b, total_b = torch.cuda.mem_get_info()
    return (total_b - free_b) / 1e6, torch.cuda.memory_allocated() / 1e6, torch.cuda.memory_reserved() / 1e6


def _parse_floats(v: str) -> list:
    return [float(x.strip()) for x in v.split(",") if x.strip()]


def _parse_ints(v: str) -> list:
    return [int(x.strip()) for x in v.split(",") if x.strip()]


def build_parser() -> argparse.ArgumentParser:
    p = argparse.ArgumentParser()
    p.add_argument("--preset", default="cantilever_gpu_medium")
    p.add_argument("--probabilities", default="0.10,0.15,0.18,0.20")
    p.add_argument("--seeds", default="23")
    p.add_argument("--baseline-rho-min", type=float, default=1e-12)
    p.add_argument("--raised-rho-min", type=float, default=1e-3)
    p.add_argument("--raised-rho-mins", default="")
    p.add_argument("--penal", default=4.5, type=float)
    p.add_argument("--probe-iters", default=100, type=int)
    p.add_argument("--probe-r50", default=50, type=int)
    p.add_argument("--restart", default=300, type=int)
    p.add_argument("--maxiter", default=300, type=int)
    p.add_argument("--tol", default=1e-6, type=float)
    p.add_argument("--stack-variant", default="canonical")
    p.add_argument("--n-levels", default=4, type=int)
    p.add_argument("--fine-smoother", default="fp64")
    p.add_argument("--smoother-type", default="chebyshev", choices=["chebyshev", "jacobi"])
    p.add_argument("--cycle-type", default="v", choices=["v", "w"])
    p.add_argument("--coarse-correction-policy", default="residual_line_search",
                   choices=["none", "residual_line_search"])
    p.add_argument("--root-local-correction-mode", default="node_block_inner_fgmres",
                   choices=["none", "node_block_line_search", "node_block_inner_fgmres"])
    p.add_argument("--root-local-correction-inner-steps", default=20, type=int)
    p.add_argument("--root-local-correction-inner-restart", default=20, type=int)
    p.add_argument("--inner-krylov-steps", default=10, type=int)
    p.add_argument("--inner-krylov-restart", default=10, type=int)
    p.add_argument("--high-residual-threshold", type=float, default=1e-2)
    p.add_argument("--plateau-residual-threshold", type=float, default=1e-4)
    p.add_argument("--plateau-ratio-threshold", type=float, default=0.6)
    p.add_argument("--severity-jump-r50-threshold", type=float, default=0.0)
    p.add_argument("--severity-jump-rho-min", type=float, default=1e-2)
    p.add_argument("--cycle-precision", default="fp64", choices=["fp64", "fp32"],
                   help="fp32: this build's mixed-precision cycle (no reference counterpart)")
    p.add_argument("--out-dir", default="results/gmg_solver_floor_detector_prospective")
    return p


def run(args) -> tuple:
    """Returns (summary rows, history rows) and writes the two CSV files."""
    from .policy import GuardedFloorPolicy
    from .presets import get_preset

    spec = get_preset(args.preset)
    raised = _parse_floats(args.raised_rho_mins) if args.raised_rho_mins.strip() else [args.raised_rho_min]
    stack = dict(fine_smoother=args.fine_smoother, smoother_type=args.smoother_type, cycle_type=args.cycle_type,
                 coarse_correction_policy=args.coarse_correction_policy,
                 root_local_correction_mode=args.root_local_correction_mode,
                 root_local_correction_inner_steps=args.root_local_correction_inner_steps,
                 root_local_correction_inner_restart=args.root_local_correction_inner_restart,
                 inner_krylov_steps=args.inner_krylov_steps, inner_krylov_restart=args.inner_krylov_restart)
    pol = GuardedFloorPolicy(
        spec, penal=args.penal, tol=args.tol, restart=args.restart, maxiter=args.maxiter,
        probe_iters=args.probe_iters, probe_r50=args.probe_r50, baseline_rho_min=args.baseline_rho_min,
        raised_rho_mins=raised, high_residual_threshold=args.high_residual_threshold,
        plateau_residual_threshold=args.plateau_residual_threshold,
        plateau_ratio_threshold=args.plateau_ratio_threshold,
        severity_jump_r50_threshold=args.severity_jump_r50_threshold,
        severity_jump_rho_min=args.severity_jump_rho_min, stack=stack, n_levels=args.n_levels,
        cycle_precision=args.cycle_precision)
    torch = _lib.require_cuda()
    summary, history = [], []
    print("seed,p,r50,r100,trigger,recommended_rho_min,solve_converged,solver_reported_converged,"
          "solve_iters,solve_final_rel_residual,attempted_rho_mins", flush=True)
    for seed in _parse_ints(args.seeds):
        field = np.random.default_rng(seed).random(spec.nelx * spec.nely * spec.nelz)
        field = field.reshape(spec.nelx, spec.nely, spec.nelz)
        for p in _parse_floats(args.probabilities):
            solid = field < p
            conn = connectivity(solid)
            r = pol.run(torch.as_tensor(solid.reshape(-1).astype(np.float64), device="cuda"), binary=True)
            torch.cuda.synchronize()
            used, alloc, reserved = _memory()
            row = {
                "preset": args.preset, "seed": seed, "solid_probability": p,
                "baseline_rho_min": args.baseline_rho_min, "raised_rho_min": args.raised_rho_min,
                "raised_rho_mins": ";".join(f"{v:.0e}" for v in raised),
                "recommended_rho_min": r["recommended_rho_min"], "attempted_rho_mins": r["attempted_rho_mins"],
                "n_floor_attempts": r["n_floor_attempts"], "penal": args.penal, "probe_iters": args.probe_iters,
                "restart": args.restart, "maxiter": args.maxiter, "tol": args.tol,
                "stack_variant": args.stack_variant, "n_levels": args.n_levels, "fine_smoother": args.fine_smoother,
                "smoother_type": args.smoother_type, "cycle_type": args.cycle_type,
                "coarse_correction_policy": args.coarse_correction_policy,
                "root_local_correction_mode": args.root_local_correction_mode,
                "root_local_correction_inner_steps": args.root_local_correction_inner_steps,
                "root_local_correction_inner_restart": args.root_local_correction_inner_restart,
                "inner_krylov_steps": args.inner_krylov_steps, "inner_krylov_restart": args.inner_krylov_restart,
                **conn,
                "probe_r50": r["probe_r50"], "probe_r100": r["probe_r100"],
                "probe_r100_over_r50": r["probe_r100_over_r50"],
                "probe_setup_time_s": r["probe_setup_time_s"], "probe_solve_time_s": r["probe_solve_time_s"],
                "probe_gpu_used_mb_after_solve": used, "probe_cupy_pool_used_mb_after_solve": alloc,
                "trigger": r["trigger"], "predicted_raise_floor": r["predicted_raise_floor"],
                "severity_jump_triggered": r["severity_jump_triggered"],
                "severity_jump_r50_threshold": args.severity_jump_r50_threshold,
                "severity_jump_rho_min": args.severity_jump_rho_min,
                "post_solve_fallback_triggered": r["post_solve_fallback_triggered"],
                "detector_false_keep": r["detector_false_keep"], "solve_converged": r["solve_converged"],
                "solver_reported_converged": r["solver_reported_converged"], "solve_iters": r["solve_iters"],
                "solve_final_rel_residual": r["solve_final_rel_residual"],
                "selected_setup_time_s": r["selected_setup_time_s"],
                "selected_solve_time_s": r["selected_solve_time_s"],
                "selected_gpu_used_mb_after_solve": used, "selected_cupy_pool_used_mb_after_solve": alloc,
                "selected_cupy_pool_total_mb_after_solve": reserved,
                "failed_ladder_setup_time_s": r["failed_ladder_setup_time_s"],
                "failed_ladder_solve_time_s": r["failed_ladder_solve_time_s"],
                "recorded_policy_time_s": r["recorded_policy_time_s"],
            }
            summary.append(row)
            for i, v in enumerate(r["probe_history"]):
                history.append({"seed": seed, "solid_probability": p, "phase": "probe",
                                "rho_min": args.baseline_rho_min, "iter": i, "rel_residual": float(v)})
            for a in r["attempts"]:
                for i, v in enumerate(a.history):
                    history.append({"seed": seed, "solid_probability": p, "phase": "recommended_solve",
                                    "rho_min": a.rho_min, "iter": i, "rel_residual": float(v)})
            print(f"{seed},{p:.4g},{r['probe_r50']:.12g},{r['probe_r100']:.12g},{r['trigger']},"
                  f"{r['recommended_rho_min']:.0e},{r['solve_converged']},{r['solver_reported_converged']},"
                  f"{r['solve_iters']},{r['solve_final_rel_residual']:.12g},{r['attempted_rho_mins']}", flush=True)
    out = Path(args.out_dir)
    write_csv(out / "prospective_summary.csv", summary, SUMMARY_FIELDS)
    write_csv(out / "prospective_history.csv", history, HISTORY_FIELDS)
    return summary, history


def main(argv=None) -> None:
    run(build_parser().parse_args(argv))


if __name__ == "__main__":
    main()
