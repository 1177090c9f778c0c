"""The fixed-floor control driver on the reference driver's golden manifest
(cantilever_3d: two Bernoulli states and a stored gray field, floors down to
1e-12, canonical stack, FGMRES restart 300, maxiter 80): the same rows in the
same order, identical convergence flags, every solve at true relative
residual <= 1e-6, compliance to 1e-6 relative, iteration counts within one;
the first four residual-history entries of every solve to 1e-7 and the first
ten to 1e-4 (the canonical stack's line-search and root-local choices follow
residual norms: the reference's own history moves by 7e-5 within 15
iterations under a 1e-14 perturbation of a binary cantilever_3d state,
density_detector_cantilever_3d_pert_history.csv)."""

import csv
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_driver_reproduces_reference_rows(cuda, tmp_path):
    from gpu_fem.fixed_floor_driver import build_parser, run

    os.makedirs(tmp_path / "fields" / "gray")
    np.save(tmp_path / "fields" / "gray" / "rho.npy",
            np.load(os.path.join(GOLDEN, "density_driver_fields.npz"))["gray"])
    args = build_parser().parse_args([
        "--manifest", os.path.join(GOLDEN, "fixed_floor_manifest_cantilever_3d.csv"),
        "--density-root", str(tmp_path), "--out-dir", str(tmp_path / "out"), "--maxiter", "80"])
    summary, history = run(args)
    with open(os.path.join(GOLDEN, "fixed_floor_cantilever_3d_summary.csv"), newline="") as f:
        ref = list(csv.DictReader(f))
    with open(tmp_path / "out" / "fixed_floor_control_summary.csv", newline="") as f:
        got = list(csv.DictReader(f))
    assert len(got) == len(ref) == len(summary)
    for g, r in zip(got, ref):
        for k in ("case_id", "case_type", "preset", "seed", "solid_probability", "density_path", "n_elem",
                  "rho_min", "penal", "solve_converged", "solver_reported_converged"):
            assert g[k] == r[k], (k, r["case_id"], g[k], r[k])
        assert float(g["solve_final_rel_residual"]) <= 1e-6
        assert float(g["compliance"]) == pytest.approx(float(r["compliance"]), rel=1e-6), r["case_id"]
        assert abs(int(g["solve_iters"]) - int(r["solve_iters"])) <= 1, (r["case_id"], r["rho_min"])
    with open(os.path.join(GOLDEN, "fixed_floor_cantilever_3d_history.csv"), newline="") as f:
        href = list(csv.DictReader(f))
    for r in ref:
        key = (r["case_id"], r["rho_min"])
        a = [float(x["rel_residual"]) for x in history if (x["case_id"], str(x["rho_min"])) == key]
        b = [float(x["rel_residual"]) for x in href if (x["case_id"], x["rho_min"]) == key]
        assert len(a) > 0 and len(b) > 0
        np.testing.assert_allclose(a[:4], b[:4], rtol=1e-7, atol=0, err_msg=str(key))
        np.testing.assert_allclose(a[:10], b[:10], rtol=1e-4, atol=0, err_msg=str(key))
