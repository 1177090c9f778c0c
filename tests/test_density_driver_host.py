"""The density-field driver's output schema, density statistics and
connectivity against the reference driver's own output on three cantilever_3d
fields (density_detector_cantilever_3d_*.csv, made by running the unchanged
reference driver: tests/golden/make_density_driver_golden.py)."""

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
    from gpu_fem.density_field_driver import HISTORY_FIELDS, SUMMARY_FIELDS

    assert SUMMARY_FIELDS == _rows("density_detector_cantilever_3d_summary.csv")[0]
    assert HISTORY_FIELDS == _rows("density_detector_cantilever_3d_history.csv")[0]


def test_density_stats_and_connectivity_match_reference_driver():
    from gpu_fem.density_field_driver import CONNECTIVITY_FIELDS, density_stats
    from gpu_fem.prospective_driver import connectivity

    fields = np.load(os.path.join(GOLDEN, "density_driver_fields.npz"))
    _, rows = _rows("density_detector_cantilever_3d_summary.csv")
    assert [r["density_name"] for r in rows] == list(fields.files)
    for r in rows:
        d = np.clip(fields[r["density_name"]], 0.0, 1.0)
        st = density_stats(d)
        for k, v in st.items():
            assert v == pytest.approx(float(r[k]), rel=1e-15, abs=1e-300), k
        c = connectivity(d.reshape(24, 12, 6) >= 0.5)
        for k in CONNECTIVITY_FIELDS:
            assert float(c[k]) == pytest.approx(float(r[k]), rel=1e-15), (k, r["density_name"])


def test_load_density_checks_size(tmp_path):
    from gpu_fem.density_field_driver import load_density

    np.save(tmp_path / "rho.npy", np.linspace(-0.5, 1.5, 12))
    d = load_density(tmp_path / "rho.npy", 12, "x")
    assert d.min() == 0.0 and d.max() == 1.0
    with pytest.raises(ValueError, match="expected 13"):
        load_density(tmp_path / "rho.npy", 13, "x")


def test_parser_defaults_follow_reference():
    from gpu_fem.density_field_driver import build_parser

    a = build_parser().parse_args(["--density-paths", "a.npy"])
    assert (a.preset, a.baseline_rho_min, a.raised_rho_mins, a.penal, a.solid_threshold, a.fine_smoother) == (
        "cantilever_gpu_medium", 1e-12, "1e-3,1e-2", 4.5, 0.5, "fp64")
    assert (a.probe_iters, a.probe_r50, a.restart, a.maxiter, a.tol) == (100, 50, 300, 300, 1e-6)
