"""The prospective driver's output schema and connectivity statistics against
the reference driver's own output on cantilever_3d (policy_cantilever_3d_*.csv,
made by running the unchanged reference driver; tests/golden/make_golden.py)."""

import csv
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _rows(name):
    with open(os.path.join(GOLDEN, name), newline="") as f:
        r = csv.DictReader(f)
        return r.fieldnames, list(r)


def test_csv_headers_match_reference_driver():
    from gpu_fem.prospective_driver import HISTORY_FIELDS, SUMMARY_FIELDS

    assert SUMMARY_FIELDS == _rows("policy_cantilever_3d_summary.csv")[0]
    assert HISTORY_FIELDS == _rows("policy_cantilever_3d_history.csv")[0]


def test_connectivity_matches_reference_driver():
    from gpu_fem.prospective_driver import connectivity

    _, rows = _rows("policy_cantilever_3d_summary.csv")
    for r in rows:
        field = np.random.default_rng(int(r["seed"])).random(24 * 12 * 6).reshape(24, 12, 6)
        c = connectivity(field < float(r["solid_probability"]))
        for k in ("solid_count", "n_components", "largest_component", "support_to_load_patch_components"):
            assert c[k] == int(r[k]), (k, r["seed"], r["solid_probability"])
        for k in ("solid_fraction", "largest_fraction_of_solid"):
            assert abs(c[k] - float(r[k])) <= 1e-15, k


def test_write_csv_round_trip(tmp_path):
    from gpu_fem.prospective_driver import HISTORY_FIELDS, write_csv

    rows = [{"seed": 3, "solid_probability": 0.2, "phase": "probe", "rho_min": 1e-12, "iter": 0, "rel_residual": 1.0}]
    write_csv(tmp_path / "h.csv", rows, HISTORY_FIELDS)
    with open(tmp_path / "h.csv", newline="") as f:
        assert f.read().splitlines() == [",".join(HISTORY_FIELDS), "3,0.2,probe,1e-12,0,1.0"]
