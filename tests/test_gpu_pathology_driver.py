"""The pathology driver on the reference driver's two golden runs
(cantilever_3d, all seven cases; ``v``: default stack with the FGMRES solve,
``w``: W-cycle, line search, void-gap enrichment, node-block line search,
trace only): the same rows and columns in the same order; names, flags,
adaptive parameters, notes and counts identical; every traced norm, ratio,
cosine and scale to 1e-6 relative (these cases reach moduli contrasts of
1e12); solve convergence identical and iteration counts within one.  A
W-cycle line-search scale that is zero to round-off may carry the
'nonpositive_correction_scale' note on one side only.

A case whose reference trace holds a line-search scale above 1e6 or a
"cosine" outside [-1, 1] is compared in structure only (visit ids, levels,
coarse-correction counts, coarsest modes, the stack, the right-hand side's
norms): there a coarse correction lies in a near-null direction of the coarse
operator (moduli 1e-9 / 1e-12 in a W-cycle), so the scale is a ratio of
round-off (the reference records 4.7e13 and a cosine of 2.88 for the
checkerboard, visit 9) and the accept / clip decision, with every norm after
it, follows the summation order.  In the golden runs that is the W-cycle
trace of 'checkerboard' and 'rho-min-1e-12'; the other twelve case traces
are compared in full."""

import csv
import os

import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
EXACT = {"case", "family", "preset", "cycle_type", "n_levels", "fine_smoother", "smoother_type",
         "coarse_correction_policy", "root_enrichment_mode", "root_local_correction_mode", "is_high_contrast",
         "fine_degree_adapt", "coarse_iters_adapt", "pd", "seed", "solve_converged", "rejected_corrections",
         "solve_error", "visit_id", "level", "is_coarsest", "n_coarse_corrections", "coarsest_mode", "notes",
         "inner_krylov_steps", "inner_krylov_restart", "root_local_correction_inner_steps",
         "root_local_correction_inner_restart"}
COUNTS = {"solve_iters", "solve_history_len"}
STRUCTURE = {"case", "family", "preset", "cycle_type", "n_levels", "fine_smoother", "smoother_type",
             "coarse_correction_policy", "root_enrichment_mode", "root_local_correction_mode", "is_high_contrast",
             "fine_degree_adapt", "coarse_iters_adapt", "contrast_ratio", "rhs_norm", "jacobi_action_norm",
             "visit_id", "level", "is_coarsest", "n_coarse_corrections", "coarsest_mode"}


def _round_off_cases(run):
    """Cases whose reference trace is dominated by round-off (see the module docstring)."""
    _, rows = _read(os.path.join(GOLDEN, f"pathology_{run}_visits.csv"))
    bad = set()
    for r in rows:
        for k in ("correction_scale_raw", "second_correction_scale_raw"):
            if r[k] not in ("", "None") and abs(float(r[k])) > 1e6:
                bad.add(r["case"])
        for k in ("correction_alignment", "second_correction_alignment"):
            if r[k] not in ("", "None") and abs(float(r[k])) > 1.0 + 1e-9:
                bad.add(r["case"])
    return bad
RUNS = {"v": ["--maxiter", "150"],
        "w": ["--cycle-type", "w", "--coarse-policy", "residual_line_search", "--root-enrichment-mode",
              "void_gap_second", "--root-local-correction-mode", "node_block_line_search", "--skip-solve"]}


def _read(path):
    with open(path, newline="") as f:
        r = csv.DictReader(f)
        return r.fieldnames, list(r)


def _round_off_note(row):
    """A W-cycle line-search scale that is zero to round-off (|raw| <= 1e-12)
    has a sign, and so a 'nonpositive_correction_scale' note, that depends on
    the summation order."""
    raws = (row.get("correction_scale_raw"), row.get("second_correction_scale_raw"))
    return any(r not in (None, "") and abs(float(r)) <= 1e-12 for r in raws)


def _close(k, a, b, where, row):
    if k == "notes" and a != b and _round_off_note(row):
        assert set(a.split("|")) ^ set(b.split("|")) <= {"nonpositive_correction_scale", ""}, (where, a, b)
    elif k in EXACT or b in ("", "None", "True", "False") or a in ("", "None"):
        assert a == b, (where, k, a, b)
    elif k in COUNTS:
        assert abs(int(a) - int(b)) <= 1, (where, k, a, b)
    elif k == "solve_final_rel_residual":
        assert float(a) == pytest.approx(float(b), rel=0.05, nan_ok=True), (where, k, a, b)
    else:
        try:
            fb = float(b)
        except ValueError:
            assert a == b, (where, k, a, b)
            return
        assert float(a) == pytest.approx(fb, rel=1e-6, abs=1e-12, nan_ok=True), (where, k, a, b)


@pytest.mark.parametrize("run", sorted(RUNS))
def test_driver_reproduces_reference_run(cuda, tmp_path, run):
    from gpu_fem.pathology_driver import build_parser, run as drive

    drive(build_parser().parse_args(["--preset", "cantilever_3d", "--cases", "all", "--out-dir", str(tmp_path)]
                                    + RUNS[run]))
    names = ["summary", "visits"] + (["solve_history"] if run == "v" else [])
    structure_only = _round_off_cases(run)
    assert len(structure_only) <= 2
    for name in names:
        fa, got = _read(tmp_path / f"pathology_{name}.csv")
        fb, ref = _read(os.path.join(GOLDEN, f"pathology_{run}_{name}.csv"))
        assert fa == fb, name
        if name == "solve_history":
            # iteration counts may differ by one: compare the first entries of each case
            for case in {r["case"] for r in ref}:
                a = [float(r["rel_residual"]) for r in got if r["case"] == case][:5]
                b = [float(r["rel_residual"]) for r in ref if r["case"] == case][:5]
                assert a == pytest.approx(b, rel=1e-6), case
            continue
        assert len(got) == len(ref), name
        for g, r in zip(got, ref):
            keys = STRUCTURE & set(fb) if r["case"] in structure_only else fb
            for k in keys:
                _close(k, g[k], r[k], (run, name, r["case"], r.get("visit_id")), r)
    assert (tmp_path / "pathology_traces.json").exists()
