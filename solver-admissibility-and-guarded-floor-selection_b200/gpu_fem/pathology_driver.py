"""Targeted multigrid pathology diagnostics with the reference's output files.

Same cases, flags and outputs as the reference's
experiments/phase5/run_pathology_diagnostics.py (:102-434): for each selected
hard or control case the hierarchy is built with the requested stack, one
cycle is traced on the load vector (GalerkinMatFreeGMG.cycle_trace, measured
on the device), per-level aggregates are formed from the visits, and unless
``--skip-solve`` the matching FGMRES solve runs.  Written:
``pathology_summary.csv`` (one row per case), ``pathology_visits.csv`` (one row
per level visit), ``pathology_solve_history.csv`` and ``pathology_traces.json``,
with the reference's column order (the first row's keys, then any new key).

    python pathology_driver.py --preset cantilever_gpu_medium --cases hardset --out-dir results/
"""

from __future__ import annotations

import argparse
import csv
import json
import os
import sys
from pathlib import Path

import numpy as np

if __package__ in (None, ""):
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    __package__ = "gpu_fem"  # noqa: A001

from . import _lib  # noqa: E402


def write_csv(path: Path, rows: list) -> None:
    """Header = the first row's keys, then keys first seen in later rows (:84-95)."""
    if not rows:
        return
    fields = list(rows[0].keys())
    for r in rows[1:]:
        for k in r:
            if k not in fields:
                fields.append(k)
    with open(path, "w", newline="") as f:
        w = csv.DictWriter(f, fieldnames=fields)
        w.writeheader()
        w.writerows(rows)


def make_cases() -> dict:
    """The seven cases of the reference driver (:102-178): builders of the
    element moduli on the device for a ProblemSpec."""
    from .paper4 import _E_e, _E_e_heterogeneous

    def dev(a):
        return _lib.require_cuda().as_tensor(a, device="cuda")

    def checkerboard(spec):
        n = spec.nelx * spec.nely * spec.nelz
        return 1e-9 + (1.0 - 1e-9) * dev((np.arange(n) % 2).astype(np.float64)) ** 3.0

    def layered_band(spec):
        rho = np.repeat((np.arange(spec.nelx) < spec.nelx // 2).astype(np.float64), spec.nely * spec.nelz)
        return 1e-9 + (1.0 - 1e-9) * dev(rho) ** 3.0

    def mixed_very_low(spec):
        n = spec.nelx * spec.nely * spec.nelz
        rho = np.where(np.random.default_rng(19).random(n) < 0.1, 1.0, 1e-12)
        return 1e-12 + (1.0 - 1e-12) * dev(rho) ** 4.5

    return {
        "uniform-vf0.5": dict(family="control", volfrac=0.5, rho_min=0.5, penal=3.0, seed="deterministic",
                              build=lambda spec: _E_e(spec, rho_scalar=0.5, penal=3.0)),
        "layered-band": dict(family="control", volfrac=0.5, rho_min=1e-9, penal=3.0, seed="deterministic",
                             build=layered_band),
        "binary-vf0.2-p1.5": dict(family="hardset", volfrac=0.2, rho_min=1e-9, penal=1.5, seed=7,
                                  build=lambda spec: _E_e_heterogeneous(spec, volfrac=0.2, penal=1.5, rho_min=1e-9,
                                                                        seed=7)),
        "binary-vf0.8-p4.5": dict(family="hardset", volfrac=0.8, rho_min=1e-9, penal=4.5, seed=13,
                                  build=lambda spec: _E_e_heterogeneous(spec, volfrac=0.8, penal=4.5, rho_min=1e-9,
                                                                        seed=13)),
        "checkerboard": dict(family="hardset", volfrac=0.5, rho_min=1e-9, penal=3.0, seed="deterministic",
                             build=checkerboard),
        "rho-min-1e-12": dict(family="hardset", volfrac=0.5, rho_min=1e-12, penal=3.0, seed=17,
                              build=lambda spec: _E_e_heterogeneous(spec, volfrac=0.5, penal=3.0, rho_min=1e-12,
                                                                    seed=17)),
        "mixed-very-low": dict(family="hardset", volfrac=0.1, rho_min=1e-12, penal=4.5, seed=19,
                               build=mixed_very_low),
    }


def select_cases(case_map: dict, selector: str) -> list:
    if selector == "all":
        return list(case_map)
    if selector in ("hardset", "controls"):
        family = "hardset" if selector == "hardset" else "control"
        return [k for k, v in case_map.items() if v["family"] == family]
    names = [c.strip() for c in selector.split(",") if c.strip()]
    unknown = [n for n in names if n not in case_map]
    if unknown:
        raise ValueError(f"Unknown case names: {unknown}")
    return names


def trace_aggregates(trace) -> dict:
    """Per-cycle aggregates of the visits (:181-206)."""
    visits = sorted(trace.visits, key=lambda v: v.visit_id)
    inner = [v for v in visits if not v.is_coarsest]
    root = next((v for v in visits if v.level == 0), None)
    nan = float("nan")
    second = [v.second_corrected_residual_vs_corrected for v in visits
              if v.second_corrected_residual_vs_corrected is not None]
    return {
        "root_presmooth_residual_ratio": root.presmooth_residual_ratio if root else nan,
        "root_corrected_residual_vs_presmooth": root.corrected_residual_vs_presmooth if root else nan,
        "root_postsmooth_residual_ratio": root.postsmooth_residual_ratio if root else nan,
        "root_correction_scale_applied": root.correction_scale_applied if root else nan,
        "max_coarse_space_gap_ratio": max((v.coarse_space_gap_ratio for v in inner), default=0.0),
        "worst_first_correction_ratio": max((v.corrected_residual_vs_presmooth for v in inner), default=0.0),
        "worst_second_correction_ratio": max(second, default=0.0),
        "min_correction_alignment": min((v.correction_alignment for v in inner), default=0.0),
        "min_correction_scale_applied": min((v.correction_scale_applied for v in inner), default=1.0),
        "rejected_corrections": sum(1 for v in inner if v.correction_scale_applied <= 1e-12),
    }


def build_parser() -> argparse.ArgumentParser:
    p = argparse.ArgumentParser()
    p.add_argument("--preset", default="cantilever_gpu_medium")
    p.add_argument("--cases", default="hardset",
                   help="hardset, controls, all, or comma-separated explicit case names")
    p.add_argument("--n-levels", default=4, type=int)
    p.add_argument("--fine-smoother", default="fp64")
    p.add_argument("--smoother-type", default="chebyshev")
    p.add_argument("--cycle-type", default="v", choices=["v", "w"])
    p.add_argument("--coarse-policy", default="none", choices=["none", "residual_line_search"])
    p.add_argument("--coarse-acceptance-ratio", default=1.0, type=float)
    p.add_argument("--coarse-max-scale", default=1.0, type=float)
    p.add_argument("--root-enrichment-mode", default="none",
                   choices=["none", "weighted_residual_second", "weighted_gap_second", "void_residual_second",
                            "void_gap_second"])
    p.add_argument("--root-enrichment-weight-floor", default=1e-6, type=float)
    p.add_argument("--root-enrichment-weight-power", default=0.5, type=float)
    p.add_argument("--root-local-correction-mode", default="none",
                   choices=["none", "node_block_line_search", "node_block_inner_fgmres"])
    p.add_argument("--root-local-correction-max-scale", default=1.0, type=float)
    p.add_argument("--root-local-correction-inner-steps", default=10, type=int)
    p.add_argument("--root-local-correction-inner-restart", default=None, type=int)
    p.add_argument("--inner-fgmres-steps", default=0, type=int)
    p.add_argument("--inner-fgmres-restart", default=None, type=int)
    p.add_argument("--restart", default=50, type=int)
    p.add_argument("--maxiter", default=500, type=int)
    p.add_argument("--tol", default=1e-6, type=float)
    p.add_argument("--skip-solve", action="store_true")
    p.add_argument("--cycle-precision", default="fp64", choices=["fp64", "fp32"],
                   help="fp32: this build's mixed-precision cycle (no reference counterpart)")
    p.add_argument("--out-dir", default="results")
    return p


def run(args) -> tuple:
    """Returns (summary rows, visit rows, history rows, traces) and writes the four files."""
    from .paper4 import _build_components, _fgmres

    out = Path(args.out_dir)
    out.mkdir(parents=True, exist_ok=True)
    case_map = make_cases()
    names = select_cases(case_map, args.cases)
    summary, visits_out, history_out, traces = [], [], [], []
    print(f"Phase 5 pathology diagnostics: preset={args.preset} cases={names}")
    for name in names:
        meta = case_map[name]
        spec, _, _, _, _, F, mf_op, gmg = _build_components(
            args.preset, n_levels=args.n_levels, fine_smoother=args.fine_smoother, smoother_type=args.smoother_type,
            cycle_type=args.cycle_type, coarse_correction_policy=args.coarse_policy,
            coarse_correction_acceptance_ratio=args.coarse_acceptance_ratio,
            coarse_correction_max_scale=args.coarse_max_scale, root_enrichment_mode=args.root_enrichment_mode,
            root_enrichment_weight_floor=args.root_enrichment_weight_floor,
            root_enrichment_weight_power=args.root_enrichment_weight_power,
            root_local_correction_mode=args.root_local_correction_mode,
            root_local_correction_max_scale=args.root_local_correction_max_scale,
            root_local_correction_inner_steps=args.root_local_correction_inner_steps,
            root_local_correction_inner_restart=args.root_local_correction_inner_restart,
            inner_krylov_steps=args.inner_fgmres_steps, inner_krylov_restart=args.inner_fgmres_restart,
            cycle_precision=args.cycle_precision)
        E = meta["build"](spec)
        gmg.setup(E)
        trace = gmg.cycle_trace(F, cycle_type=args.cycle_type)
        agg = trace_aggregates(trace)
        conv, iters, err, hist, final = None, None, "", [], float("nan")
        if not args.skip_solve:
            try:
                _, iters, conv = _fgmres(lambda v: mf_op.matvec(v, E), F, gmg.apply, tol=args.tol,
                                         maxiter=args.maxiter, restart=args.restart, history=hist)
                if hist:
                    final = float(hist[-1])
            except Exception as exc:  # recorded in the row, as the reference does
                conv, iters, err = 0, -1, str(exc)
        row = {
            "case": name, "family": meta["family"], "preset": args.preset, "cycle_type": trace.cycle_type,
            "n_levels": args.n_levels, "fine_smoother": args.fine_smoother, "smoother_type": args.smoother_type,
            "coarse_correction_policy": trace.coarse_correction_policy,
            "coarse_correction_acceptance_ratio": trace.coarse_correction_acceptance_ratio,
            "coarse_correction_max_scale": trace.coarse_correction_max_scale,
            "root_enrichment_mode": trace.root_enrichment_mode,
            "root_enrichment_weight_floor": trace.root_enrichment_weight_floor,
            "root_enrichment_weight_power": trace.root_enrichment_weight_power,
            "root_local_correction_mode": trace.root_local_correction_mode,
            "root_local_correction_inner_steps": trace.root_local_correction_inner_steps,
            "root_local_correction_inner_restart": trace.root_local_correction_inner_restart,
            "root_local_correction_raw_scale": trace.root_local_correction_raw_scale,
            "root_local_correction_applied_scale": trace.root_local_correction_applied_scale,
            "root_local_correction_residual_ratio": trace.root_local_correction_residual_ratio,
            "inner_krylov_steps": trace.inner_krylov_steps, "inner_krylov_restart": trace.inner_krylov_restart,
            "contrast_ratio": trace.contrast_ratio, "is_high_contrast": trace.is_high_contrast,
            "fine_degree_adapt": trace.fine_degree_adapt, "coarse_iters_adapt": trace.coarse_iters_adapt,
            "rhs_norm": trace.rhs_norm, "jacobi_action_norm": trace.jacobi_action_norm,
            "output_norm": trace.output_norm, "z_over_jacobi": trace.z_over_jacobi, "rz": trace.rz,
            "pd": int(trace.pd), "output_residual_norm": trace.output_residual_norm,
            "output_residual_ratio": trace.output_residual_ratio, "volfrac": meta["volfrac"],
            "rho_min": meta["rho_min"], "penal": meta["penal"], "seed": meta["seed"], "solve_converged": conv,
            "solve_iters": iters, "solve_final_rel_residual": final, "solve_history_len": len(hist),
            "solve_error": err,
        }
        row.update(agg)
        summary.append(row)
        for v in sorted(trace.visits, key=lambda v: v.visit_id):
            vr = {"case": name, "family": meta["family"], "preset": args.preset, "solve_converged": conv,
                  "solve_iters": iters}
            vr.update(v.to_dict())
            visits_out.append(vr)
        for i, r in enumerate(hist):
            history_out.append({
                "case": name, "family": meta["family"], "preset": args.preset, "cycle_type": trace.cycle_type,
                "coarse_correction_policy": trace.coarse_correction_policy,
                "root_enrichment_mode": trace.root_enrichment_mode,
                "root_local_correction_mode": trace.root_local_correction_mode,
                "inner_krylov_steps": trace.inner_krylov_steps, "iter": i, "rel_residual": float(r)})
        traces.append({"case": name, "family": meta["family"], "summary": row, "trace": trace.to_dict()})
        print(f"  {name:<20} conv={conv} iters={iters} z/jac={trace.z_over_jacobi:.3g} "
              f"root_post={agg['root_postsmooth_residual_ratio']:.3g} gap_max={agg['max_coarse_space_gap_ratio']:.3g} "
              f"align_min={agg['min_correction_alignment']:.3g} scale_min={agg['min_correction_scale_applied']:.3g}")
    write_csv(out / "pathology_summary.csv", summary)
    write_csv(out / "pathology_visits.csv", visits_out)
    write_csv(out / "pathology_solve_history.csv", history_out)
    with open(out / "pathology_traces.json", "w") as f:
        json.dump(traces, f, indent=2, default=str)
    print(f"\nWrote {out / 'pathology_summary.csv'}")
    print(f"Wrote {out / 'pathology_visits.csv'}")
    if history_out:
        print(f"Wrote {out / 'pathology_solve_history.csv'}")
    print(f"Wrote {out / 'pathology_traces.json'}")
    return summary, visits_out, history_out, traces


def main(argv=None) -> None:
    run(build_parser().parse_args(argv))


if __name__ == "__main__":
    main()
