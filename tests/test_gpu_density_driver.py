"""The density-field driver run with the arguments of the reference driver's
golden run (cantilever_3d; fields gray, binary35, binary60; probe 30 / r50 at
15, maxiter 60; canonical stack, FP64 smoothing): the same rows in the same
order with identical trigger, selected floor, attempted floors, convergence
flags and connectivity; iteration counts within one; the probe's residual
history entry by entry inside the reference's own round-off envelope (1000
times the running maximum of its deviation under a 1e-14 perturbation of the
densities, density_detector_cantilever_3d_pert_history.csv, floored at 1e-9:
the canonical stack's line-search and root-local decisions follow residual
norms, so round-off grows along a stalled probe); the final true residual at
or below the tolerance; both CSV files with the reference's headers."""

import csv
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_driver_reproduces_reference_rows(cuda, tmp_path):
    from gpu_fem.density_field_driver import build_parser, run

    fields = np.load(os.path.join(GOLDEN, "density_driver_fields.npz"))
    paths = []
    for name in fields.files:
        os.makedirs(tmp_path / name)
        np.save(tmp_path / name / "rho.npy", fields[name])
        paths.append(str(tmp_path / name / "rho.npy"))
    args = build_parser().parse_args([
        "--preset", "cantilever_3d", "--density-paths", ",".join(paths), "--probe-iters", "30",
        "--probe-r50", "15", "--maxiter", "60", "--out-dir", str(tmp_path / "out")])
    summary, history = run(args)
    with open(os.path.join(GOLDEN, "density_detector_cantilever_3d_summary.csv"), newline="") as f:
        ref = list(csv.DictReader(f))
    with open(tmp_path / "out" / "density_detector_summary.csv", newline="") as f:
        got = list(csv.DictReader(f))
    assert len(got) == len(ref) == len(summary) == 3
    for g, r in zip(got, ref):
        for k in ("preset", "density_name", "n_elem", "trigger", "recommended_rho_min", "attempted_rho_mins",
                  "n_floor_attempts", "solve_converged", "solver_reported_converged", "predicted_raise_floor",
                  "post_solve_fallback_triggered", "detector_false_keep", "solid_count", "n_components",
                  "largest_component", "raised_rho_mins", "fine_smoother"):
            assert g[k] == r[k], (k, r["density_name"], g[k], r[k])
        assert abs(int(g["solve_iters"]) - int(r["solve_iters"])) <= 1, r["density_name"]
        assert float(g["solve_final_rel_residual"]) <= 1e-6
    with open(tmp_path / "out" / "density_detector_history.csv", newline="") as f:
        h = list(csv.DictReader(f))
    with open(os.path.join(GOLDEN, "density_detector_cantilever_3d_history.csv"), newline="") as f:
        href = list(csv.DictReader(f))
    assert len(h) == len(history) > 0
    assert {row["phase"] for row in h} == {row["phase"] for row in href}
    with open(os.path.join(GOLDEN, "density_detector_cantilever_3d_pert_history.csv"), newline="") as f:
        hpert = list(csv.DictReader(f))

    def probe(rows, name):
        return np.array([float(x["rel_residual"]) for x in rows if x["density_name"] == name and x["phase"] == "probe"])

    for name in fields.files:
        a, b, c = probe(h, name), probe(href, name), probe(hpert, name)
        assert len(a) == len(b) == len(c), name
        env = np.maximum(1e-9, 1000.0 * np.maximum.accumulate(np.abs(c - b) / b))
        dev = np.abs(a - b) / b
        assert np.all(dev <= env), (name, dev, env)
