"""The pathology driver's host logic against the reference driver's own run
(pathology_{v,w}_*.csv, made by tests/golden/make_pathology_golden.py from the
unchanged reference): the per-cycle aggregates recomputed from the reference's
visit rows equal its summary columns, case selection, and the CSV header rule."""

import csv
import dataclasses
import os

import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
AGGREGATES = ("root_presmooth_residual_ratio", "root_corrected_residual_vs_presmooth",
              "root_postsmooth_residual_ratio", "root_correction_scale_applied", "max_coarse_space_gap_ratio",
              "worst_first_correction_ratio", "worst_second_correction_ratio", "min_correction_alignment",
              "min_correction_scale_applied", "rejected_corrections")


def _rows(name):
    with open(os.path.join(GOLDEN, name), newline="") as f:
        return list(csv.DictReader(f))


def _visit(row):
    from gpu_fem.multigrid_v4 import MultigridCycleVisit

    kw = {}
    for f in dataclasses.fields(MultigridCycleVisit):
        s = row[f.name]
        if f.name in ("cycle_type", "coarsest_mode", "notes"):
            kw[f.name] = s
        elif f.name == "is_coarsest":
            kw[f.name] = s == "True"
        elif f.name in ("visit_id", "level", "n_coarse_corrections"):
            kw[f.name] = int(s)
        else:
            kw[f.name] = None if s == "" else float(s)
    return MultigridCycleVisit(**kw)


@pytest.mark.parametrize("run", ["v", "w"])
def test_aggregates_from_reference_visits(run):
    from types import SimpleNamespace

    from gpu_fem.pathology_driver import trace_aggregates

    summary = _rows(f"pathology_{run}_summary.csv")
    visits = _rows(f"pathology_{run}_visits.csv")
    for s in summary:
        agg = trace_aggregates(SimpleNamespace(visits=[_visit(v) for v in visits if v["case"] == s["case"]]))
        for k in AGGREGATES:
            assert float(agg[k]) == pytest.approx(float(s[k]), rel=1e-15), (run, s["case"], k)


def test_case_selection():
    from gpu_fem.pathology_driver import select_cases

    cases = {"a": {"family": "control"}, "b": {"family": "hardset"}, "c": {"family": "hardset"}}
    assert select_cases(cases, "all") == ["a", "b", "c"]
    assert select_cases(cases, "hardset") == ["b", "c"]
    assert select_cases(cases, "controls") == ["a"]
    assert select_cases(cases, "c, a") == ["c", "a"]
    with pytest.raises(ValueError, match="Unknown"):
        select_cases(cases, "a,zz")


def test_write_csv_header_is_first_row_then_new_keys(tmp_path):
    from gpu_fem.pathology_driver import write_csv

    write_csv(tmp_path / "x.csv", [{"a": 1, "b": 2}, {"b": 3, "c": 4}])
    with open(tmp_path / "x.csv", newline="") as f:
        assert f.read().splitlines() == ["a,b,c", "1,2,", ",3,4"]
    write_csv(tmp_path / "none.csv", [])
    assert not (tmp_path / "none.csv").exists()


def test_case_table_matches_reference_run():
    from gpu_fem.pathology_driver import make_cases

    cases = make_cases()
    summary = _rows("pathology_v_summary.csv")
    assert [s["case"] for s in summary] == list(cases)
    for s in summary:
        c = cases[s["case"]]
        assert s["family"] == c["family"] and s["seed"] == str(c["seed"])
        for k in ("volfrac", "rho_min", "penal"):
            assert float(s[k]) == c[k], (s["case"], k)


def test_parser_defaults_follow_reference():
    """run_pathology_diagnostics.py:209-246 defaults."""
    from gpu_fem.pathology_driver import build_parser

    a = build_parser().parse_args([])
    assert (a.preset, a.cases, a.n_levels, a.fine_smoother, a.smoother_type, a.cycle_type) == (
        "cantilever_gpu_medium", "hardset", 4, "fp64", "chebyshev", "v")
    assert (a.coarse_policy, a.coarse_acceptance_ratio, a.coarse_max_scale) == ("none", 1.0, 1.0)
    assert (a.root_enrichment_mode, a.root_enrichment_weight_floor, a.root_enrichment_weight_power) == (
        "none", 1e-6, 0.5)
    assert (a.root_local_correction_mode, a.root_local_correction_inner_steps,
            a.root_local_correction_inner_restart) == ("none", 10, None)
    assert (a.inner_fgmres_steps, a.inner_fgmres_restart, a.restart, a.maxiter, a.tol, a.skip_solve) == (
        0, None, 50, 500, 1e-6, False)
