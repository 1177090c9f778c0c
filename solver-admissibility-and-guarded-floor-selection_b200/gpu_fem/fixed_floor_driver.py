"""The fixed-floor control driver with the reference's output schema.

Same flags, manifest format and CSV files as the reference's
experiments/phase5/run_gmg_fixed_floor_controls.py (:26-203): every manifest
row (``case_id, case_type, preset, seed, solid_probability, density_path,
floors, penal``) names a state -- ``random``: ``random(seed) < p`` as 0/1
densities; ``density``: a stored ``.npy`` field, clipped to [0, 1] -- solved at
each listed floor with E = floor + (1 - floor) rho^penal by FGMRES(restart)
on the canonical stack (one hierarchy per preset, reused across rows and
floors as the reference reuses it, so the lambda_max cache carries over), with
the FP64 true residual recomputed after each solve.  One row per (case, floor)
goes to ``fixed_floor_control_summary.csv`` and the residual history to
``fixed_floor_control_history.csv``, in the reference's column order.

    python fixed_floor_driver.py --manifest fixed_floor_control_manifest.csv --density-root <dir> --out-dir results/
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
from .density_field_driver import CANONICAL  # noqa: E402
from .prospective_driver import write_csv  # noqa: E402

# run_gmg_fixed_floor_controls.py:173-196, in this order
SUMMARY_FIELDS = [
    "case_id", "case_type", "preset", "seed", "solid_probability", "density_path", "n_elem", "rho_min", "penal",
    "density_mean", "density_grayness", "restart", "maxiter", "tol", "setup_time_s", "solve_time_s",
    "solve_converged", "solver_reported_converged", "solve_iters", "solve_final_rel_residual", "compliance",
    "history_len",
]
HISTORY_FIELDS = ["case_id", "preset", "rho_min", "iter", "rel_residual"]


def read_manifest(path: Path) -> list:
    with Path(path).open(newline="", encoding="utf-8") as f:
        return list(csv.DictReader(f))


def parse_floors(text: str) -> list:
    """Floors separated by ';' or ','."""
    return [float(x.strip()) for x in text.replace(",", ";").split(";") if x.strip()]


def density_for_case(row: dict, n_elem: int, root: Path) -> np.ndarray:
    if row["case_type"] == "density":
        d = np.asarray(np.load(Path(root) / row["density_path"]), dtype=np.float64).reshape(-1)
        if d.size != n_elem:
            raise ValueError(f"{row['case_id']} has {d.size} entries, expected {n_elem}")
        return np.clip(d, 0.0, 1.0)
    if row["case_type"] == "random":
        field = np.random.default_rng(int(row["seed"])).random(n_elem)
        return (field < float(row["solid_probability"])).astype(np.float64)
    raise ValueError(f"unknown case_type {row['case_type']!r}")


def build_parser() -> argparse.ArgumentParser:
    p = argparse.ArgumentParser()
    p.add_argument("--manifest", default="fixed_floor_control_manifest.csv")
    p.add_argument("--density-root", default=".",
                   help="folder the manifest's density paths are relative to (the reference's repository root)")
    p.add_argument("--out-dir", default="results/gmg_fixed_floor_controls")
    p.add_argument("--restart", type=int, default=300)
    p.add_argument("--maxiter", type=int, default=300)
    p.add_argument("--tol", type=float, default=1e-6)
    p.add_argument("--cycle-precision", default="fp64", choices=["fp64", "fp32"],
                   help="fp32: this build's mixed-precision cycle (no reference counterpart)")
    return p


def run(args) -> tuple:
    """Returns (summary rows, history rows) and writes the two CSV files."""
    from .policy import GuardedFloorPolicy
    from .presets import get_preset

    torch = _lib.require_cuda()
    rows = read_manifest(Path(args.manifest))
    by_preset: dict = {}
    for r in rows:
        by_preset.setdefault(r["preset"], []).append(r)
    summary, history = [], []
    for preset, preset_rows in by_preset.items():
        spec = get_preset(preset)
        n_elem = spec.nelx * spec.nely * spec.nelz
        pol = GuardedFloorPolicy(spec, tol=args.tol, restart=args.restart, maxiter=args.maxiter,
                                 stack=dict(CANONICAL, fine_smoother="fp64"), n_levels=4,
                                 cycle_precision=args.cycle_precision)
        for r in preset_rows:
            density = density_for_case(r, n_elem, Path(args.density_root))
            d_gpu = torch.as_tensor(density, device="cuda")
            penal = float(r["penal"])
            pol.penal = penal
            for floor in parse_floors(r["floors"]):
                hist: list = []
                a = pol.solve_at_floor(d_gpu, floor, maxiter=args.maxiter, history=hist)
                compliance = float(torch.dot(pol.F_free_gpu, pol.last_x))
                summary.append({
                    "case_id": r["case_id"], "case_type": r["case_type"], "preset": preset, "seed": r["seed"],
                    "solid_probability": r["solid_probability"], "density_path": r["density_path"],
                    "n_elem": density.size, "rho_min": floor, "penal": penal,
                    "density_mean": float(np.mean(density)),
                    "density_grayness": float(np.mean(4.0 * density * (1.0 - density))),
                    "restart": args.restart, "maxiter": args.maxiter, "tol": args.tol,
                    "setup_time_s": a.setup_time_s, "solve_time_s": a.solve_time_s,
                    "solve_converged": int(a.true_converged),
                    "solver_reported_converged": int(a.solver_reported_converged), "solve_iters": a.iters,
                    "solve_final_rel_residual": a.final_rel_residual, "compliance": compliance,
                    "history_len": len(hist),
                })
                for i, v in enumerate(hist):
                    history.append({"case_id": r["case_id"], "preset": preset, "rho_min": floor, "iter": i,
                                    "rel_residual": float(v)})
                print(f"{r['case_id']},{preset},rho={floor:.0e},conv={int(a.true_converged)},iters={a.iters},"
                      f"res={a.final_rel_residual:.3e},solve_s={a.solve_time_s:.2f}", flush=True)
    out = Path(args.out_dir)
    write_csv(out / "fixed_floor_control_summary.csv", summary, SUMMARY_FIELDS)
    write_csv(out / "fixed_floor_control_history.csv", history, HISTORY_FIELDS)
    print(f"Wrote {out / 'fixed_floor_control_summary.csv'}")
    print(f"Wrote {out / 'fixed_floor_control_history.csv'}")
    return summary, history


def main(argv=None) -> None:
    run(build_parser().parse_args(argv))


if __name__ == "__main__":
    main()
