"""The fixed-floor control driver's schema and manifest handling against the
reference driver's own run (fixed_floor_cantilever_3d_*.csv, made by
tests/golden/make_fixed_floor_golden.py from the unchanged reference)."""

import csv
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _rows(name):
    with open(os.path.join(GOLDEN, name), newline="") as f:
        r = csv.DictReader(f)
        return r.fieldnames, list(r)


def test_csv_headers_match_reference_driver():
    from gpu_fem.fixed_floor_driver import HISTORY_FIELDS, SUMMARY_FIELDS

    assert SUMMARY_FIELDS == _rows("fixed_floor_cantilever_3d_summary.csv")[0]
    assert HISTORY_FIELDS == _rows("fixed_floor_cantilever_3d_history.csv")[0]


def test_manifest_cases_and_density_statistics(tmp_path):
    from gpu_fem.fixed_floor_driver import density_for_case, parse_floors, read_manifest

    manifest = read_manifest(os.path.join(GOLDEN, "fixed_floor_manifest_cantilever_3d.csv"))
    os.makedirs(tmp_path / "fields" / "gray")
    np.save(tmp_path / "fields" / "gray" / "rho.npy", np.load(os.path.join(GOLDEN, "density_driver_fields.npz"))["gray"])
    _, ref = _rows("fixed_floor_cantilever_3d_summary.csv")
    expected = [(m["case_id"], f) for m in manifest for f in parse_floors(m["floors"])]
    assert [(r["case_id"], float(r["rho_min"])) for r in ref] == expected
    for m in manifest:
        d = density_for_case(m, 24 * 12 * 6, tmp_path)
        for r in (r for r in ref if r["case_id"] == m["case_id"]):
            assert float(np.mean(d)) == pytest.approx(float(r["density_mean"]), rel=1e-15)
            assert float(np.mean(4.0 * d * (1.0 - d))) == pytest.approx(float(r["density_grayness"]), rel=1e-14,
                                                                        abs=1e-300)


def test_parse_floors_and_unknown_case():
    from gpu_fem.fixed_floor_driver import density_for_case, parse_floors

    assert parse_floors("1e-12;1e-3,1e-2") == [1e-12, 1e-3, 1e-2]
    with pytest.raises(ValueError, match="case_type"):
        density_for_case({"case_type": "other"}, 4, ".")


def test_parser_defaults_follow_reference():
    """run_gmg_fixed_floor_controls.py:61-66 defaults (paths are relative here)."""
    from gpu_fem.fixed_floor_driver import build_parser

    a = build_parser().parse_args([])
    assert (a.restart, a.maxiter, a.tol) == (300, 300, 1e-6)
    assert a.manifest.endswith("fixed_floor_control_manifest.csv") and a.density_root == "."
