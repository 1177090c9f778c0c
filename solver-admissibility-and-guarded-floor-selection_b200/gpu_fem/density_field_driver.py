"""The density-field floor-detector driver with the reference's output schema.

Same command-line flags, policy and CSV files as the reference's
experiments/phase5/run_gmg_floor_detector_density_field.py (:104-440): every
``.npy`` density field (one value per element, clipped to [0, 1]) is solved by
the probe / r50-r100 rule / floor ladder / FP64 guard policy with
E = rho_min + (1 - rho_min) rho^penal on the canonical stack (line search,
node-block inner-FGMRES root-local correction, inner Krylov 10; 4 levels,
V-cycle, Chebyshev), and one row goes to ``density_detector_summary.csv`` with
the reference's columns in its order; the probe's and every attempted solve's
residual histories go to ``density_detector_history.csv``.  The connectivity
columns count the 6-connected components of ``rho >= solid_threshold``.

Differences, by construction of this build, as in prospective_driver.py:
memory columns come from the CUDA device and the torch allocator after the
policy's last solve, and a probe that converged at the baseline floor is
reused as the answer (its history is written again as the
``recommended_solve`` phase, as the reference's repeated solve writes it).

    python density_field_driver.py --preset cantilever_gpu_xlarge \\
        --density-paths runs/C512_MF/rho_best.npy --out-dir results/
"""

from __future__ import annotations

import argparse
import os
import sys
from pathlib import Path

import numpy as np

if __package__ in (None, ""):
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    __package__ = "gpu_fem"  # noqa: A001

from . import _lib  # noqa: E402
from .prospective_driver import _memory, _parse_floats, connectivity, write_csv  # noqa: E402

# run_gmg_floor_detector_density_field.py:381-429, in this order
SUMMARY_FIELDS = [
    "preset", "density_path", "density_name", "n_elem", "density_min", "density_max", "density_mean",
    "density_grayness", "baseline_rho_min", "raised_rho_mins", "recommended_rho_min", "attempted_rho_mins",
    "n_floor_attempts", "penal", "fine_smoother", "probe_iters", "restart", "maxiter", "tol", "solid_count",
    "solid_fraction", "n_components", "largest_component", "largest_fraction_of_solid", "probe_r50", "probe_r100",
    "probe_r100_over_r50", "probe_setup_time_s", "probe_solve_time_s", "probe_gpu_used_mb_after_solve",
    "probe_cupy_pool_used_mb_after_solve", "trigger", "predicted_raise_floor", "post_solve_fallback_triggered",
    "detector_false_keep", "solve_converged", "solver_reported_converged", "solve_iters",
    "solve_final_rel_residual", "selected_setup_time_s", "selected_solve_time_s",
    "selected_gpu_used_mb_after_solve", "selected_cupy_pool_used_mb_after_solve",
    "selected_cupy_pool_total_mb_after_solve", "failed_ladder_setup_time_s", "failed_ladder_solve_time_s",
    "recorded_policy_time_s",
]
HISTORY_FIELDS = ["density_name", "density_path", "phase", "rho_min", "iter", "rel_residual"]
CONNECTIVITY_FIELDS = ("solid_count", "solid_fraction", "n_components", "largest_component",
                       "largest_fraction_of_solid")
# the canonical stack the reference driver builds (:147-159)
CANONICAL = dict(smoother_type="chebyshev", cycle_type="v", coarse_correction_policy="residual_line_search",
                 root_local_correction_mode="node_block_inner_fgmres", root_local_correction_inner_steps=20,
                 root_local_correction_inner_restart=20, inner_krylov_steps=10, inner_krylov_restart=10)


def density_stats(density: np.ndarray) -> dict:
    d = np.asarray(density, dtype=np.float64)
    return {"density_min": float(np.min(d)), "density_max": float(np.max(d)), "density_mean": float(np.mean(d)),
            "density_grayness": float(np.mean(4.0 * d * (1.0 - d)))}


def load_density(path: Path, n_elem: int, preset: str) -> np.ndarray:
    d = np.asarray(np.load(path), dtype=np.float64).reshape(-1)
    if d.size != n_elem:
        raise ValueError(f"{path} has {d.size} entries, expected {n_elem} for preset {preset}")
    return np.clip(d, 0.0, 1.0)


def build_parser() -> argparse.ArgumentParser:
    p = argparse.ArgumentParser()
    p.add_argument("--preset", default="cantilever_gpu_medium")
    p.add_argument("--density-paths", required=True,
                   help="Comma-separated .npy density fields with one value per element.")
    p.add_argument("--baseline-rho-min", type=float, default=1e-12)
    p.add_argument("--raised-rho-mins", default="1e-3,1e-2")
    p.add_argument("--penal", default=4.5, type=float)
    p.add_argument("--solid-threshold", default=0.5, type=float)
    p.add_argument("--fine-smoother", default="fp64", choices=["fp64", "fp32", "bf16"])
    p.add_argument("--probe-iters", default=100, type=int)
    p.add_argument("--probe-r50", default=50, type=int)
    p.add_argument("--restart", default=300, type=int)
    p.add_argument("--maxiter", default=300, type=int)
    p.add_argument("--tol", default=1e-6, type=float)
    p.add_argument("--high-residual-threshold", type=float, default=1e-2)
    p.add_argument("--plateau-residual-threshold", type=float, default=1e-4)
    p.add_argument("--plateau-ratio-threshold", type=float, default=0.6)
    p.add_argument("--cycle-precision", default="fp64", choices=["fp64", "fp32"],
                   help="fp32: this build's mixed-precision cycle (no reference counterpart)")
    p.add_argument("--out-dir", default="results/gmg_solver_floor_detector_density")
    return p


def run(args) -> tuple:
    """Returns (summary rows, history rows) and writes the two CSV files."""
    from .policy import GuardedFloorPolicy
    from .presets import get_preset

    spec = get_preset(args.preset)
    n_elem = spec.nelx * spec.nely * spec.nelz
    raised = _parse_floats(args.raised_rho_mins)
    pol = GuardedFloorPolicy(
        spec, penal=args.penal, tol=args.tol, restart=args.restart, maxiter=args.maxiter,
        probe_iters=args.probe_iters, probe_r50=args.probe_r50, baseline_rho_min=args.baseline_rho_min,
        raised_rho_mins=raised, high_residual_threshold=args.high_residual_threshold,
        plateau_residual_threshold=args.plateau_residual_threshold,
        plateau_ratio_threshold=args.plateau_ratio_threshold,
        stack=dict(CANONICAL, fine_smoother=args.fine_smoother), n_levels=4, cycle_precision=args.cycle_precision)
    torch = _lib.require_cuda()
    summary, history = [], []
    print("density,r50,r100,trigger,recommended_rho_min,solve_converged,solver_reported_converged,"
          "solve_iters,solve_final_rel_residual", flush=True)
    for path in (Path(x.strip()) for x in args.density_paths.split(",") if x.strip()):
        density = load_density(path, n_elem, args.preset)
        mask = density.reshape(spec.nelx, spec.nely, spec.nelz) >= args.solid_threshold
        conn = connectivity(mask)
        r = pol.run(torch.as_tensor(density, device="cuda"))
        torch.cuda.synchronize()
        used, alloc, reserved = _memory()
        row = {
            "preset": args.preset, "density_path": str(path), "density_name": path.parent.name, "n_elem": n_elem,
            **density_stats(density),
            "baseline_rho_min": args.baseline_rho_min, "raised_rho_mins": ";".join(f"{v:.0e}" for v in raised),
            "recommended_rho_min": r["recommended_rho_min"], "attempted_rho_mins": r["attempted_rho_mins"],
            "n_floor_attempts": r["n_floor_attempts"], "penal": args.penal, "fine_smoother": args.fine_smoother,
            "probe_iters": args.probe_iters, "restart": args.restart, "maxiter": args.maxiter, "tol": args.tol,
            **{k: conn[k] for k in CONNECTIVITY_FIELDS},
            "probe_r50": r["probe_r50"], "probe_r100": r["probe_r100"],
            "probe_r100_over_r50": r["probe_r100_over_r50"],
            "probe_setup_time_s": r["probe_setup_time_s"], "probe_solve_time_s": r["probe_solve_time_s"],
            "probe_gpu_used_mb_after_solve": used, "probe_cupy_pool_used_mb_after_solve": alloc,
            "trigger": r["trigger"], "predicted_raise_floor": r["predicted_raise_floor"],
            "post_solve_fallback_triggered": r["post_solve_fallback_triggered"],
            "detector_false_keep": r["detector_false_keep"], "solve_converged": r["solve_converged"],
            "solver_reported_converged": r["solver_reported_converged"], "solve_iters": r["solve_iters"],
            "solve_final_rel_residual": r["solve_final_rel_residual"],
            "selected_setup_time_s": r["selected_setup_time_s"], "selected_solve_time_s": r["selected_solve_time_s"],
            "selected_gpu_used_mb_after_solve": used, "selected_cupy_pool_used_mb_after_solve": alloc,
            "selected_cupy_pool_total_mb_after_solve": reserved,
            "failed_ladder_setup_time_s": r["failed_ladder_setup_time_s"],
            "failed_ladder_solve_time_s": r["failed_ladder_solve_time_s"],
            "recorded_policy_time_s": r["recorded_policy_time_s"],
        }
        summary.append(row)
        for i, v in enumerate(r["probe_history"]):
            history.append({"density_name": row["density_name"], "density_path": str(path), "phase": "probe",
                            "rho_min": args.baseline_rho_min, "iter": i, "rel_residual": float(v)})
        for a in r["attempts"]:
            for i, v in enumerate(a.history):
                history.append({"density_name": row["density_name"], "density_path": str(path),
                                "phase": "recommended_solve", "rho_min": a.rho_min, "iter": i,
                                "rel_residual": float(v)})
        print(f"{path},{r['probe_r50']:.12g},{r['probe_r100']:.12g},{r['trigger']},"
              f"{r['recommended_rho_min']:.0e},{r['solve_converged']},{r['solver_reported_converged']},"
              f"{r['solve_iters']},{r['solve_final_rel_residual']:.12g}", flush=True)
    out = Path(args.out_dir)
    write_csv(out / "density_detector_summary.csv", summary, SUMMARY_FIELDS)
    write_csv(out / "density_detector_history.csv", history, HISTORY_FIELDS)
    print(f"Wrote {out / 'density_detector_summary.csv'}", flush=True)
    print(f"Wrote {out / 'density_detector_history.csv'}", flush=True)
    return summary, history


def main(argv=None) -> None:
    run(build_parser().parse_args(argv))


if __name__ == "__main__":
    main()
