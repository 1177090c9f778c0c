"""The prospective driver run with the arguments of the reference driver's
golden run (cantilever_3d, seeds 3 and 5, solid probabilities 0.2 / 0.35 / 0.6,
ladder 1e-3, 1e-2, probe 30 / r50 at 15, maxiter 60, canonical stack): the same
rows in the same order with identical trigger, selected floor, attempted floors
and convergence flags, connectivity columns equal, and both CSV files written
with the reference's headers."""

import csv
import os

import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_driver_reproduces_reference_decisions(cuda, tmp_path):
    from gpu_fem.prospective_driver import build_parser, run

    args = build_parser().parse_args([
        "--preset", "cantilever_3d", "--probabilities", "0.2,0.35,0.6", "--seeds", "3,5",
        "--raised-rho-mins", "1e-3,1e-2", "--probe-iters", "30", "--probe-r50", "15",
        "--maxiter", "60", "--out-dir", str(tmp_path)])
    summary, history = run(args)
    with open(os.path.join(GOLDEN, "policy_cantilever_3d_summary.csv"), newline="") as f:
        ref = list(csv.DictReader(f))
    with open(tmp_path / "prospective_summary.csv", newline="") as f:
        got = list(csv.DictReader(f))
    assert len(got) == len(ref) == len(summary)
    for g, r in zip(got, ref):
        for k in ("preset", "seed", "solid_probability", "trigger", "recommended_rho_min", "attempted_rho_mins",
                  "n_floor_attempts", "solve_converged", "solver_reported_converged", "predicted_raise_floor",
                  "solid_count", "n_components", "largest_component", "support_to_load_patch_components"):
            assert g[k] == r[k], (k, r["seed"], r["solid_probability"], g[k], r[k])
    with open(tmp_path / "prospective_history.csv", newline="") as f:
        h = list(csv.DictReader(f))
    assert len(h) == len(history) > 0
    assert {row["phase"] for row in h} <= {"probe", "recommended_solve"}
