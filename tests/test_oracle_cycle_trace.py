"""The oracle's cycle trace (oracle/gmg.py GMG.cycle_trace) pinned to the
reference's own ``GalerkinMatFreeGMG.cycle_trace`` output
(tests/golden/cycle_trace_cant24.json, made by make_cycle_trace_golden.py):
every visit, every field, for V and W cycles, line search, both enrichment
families, both root-local corrections and FP32 coarse levels."""

import json
import math
import os

import numpy as np
import pytest

from oracle import solver as S
from oracle.gmg import GMG, VISIT_FIELDS

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "cycle_trace_cant24.json")


def _load():
    with open(GOLDEN) as fh:
        return json.load(fh)


def _round_off_sign_note(visit: dict) -> bool:
    """A line-search scale that is zero to round-off (|raw| <= 1e-12: the second
    coarse correction of a W-cycle just above an exact coarsest solve) has a
    sign, and so a 'nonpositive_correction_scale' note, that depends on the
    summation order."""
    raws = (visit.get("correction_scale_raw"), visit.get("second_correction_scale_raw"))
    return any(r is not None and abs(r) <= 1e-12 for r in raws)


def assert_trace_close(got: dict, want: dict, rtol: float, path: str = "") -> None:
    """Same keys; strings, booleans, None and infinities exact; finite numbers
    within rtol relative (plus rtol absolute, for cosines and scales near zero)."""
    assert set(got) == set(want), (path, sorted(set(got) ^ set(want)))
    for k, b in want.items():
        a = got[k]
        where = f"{path}.{k}"
        if k == "notes" and a != b and _round_off_sign_note(want):
            diff = set(a.split("|")) ^ set(b.split("|"))
            assert diff <= {"nonpositive_correction_scale", ""}, (where, a, b)
        elif k == "visits":
            assert len(a) == len(b), where
            for i, (va, vb) in enumerate(zip(a, b)):
                assert list(va) == list(VISIT_FIELDS), where
                assert_trace_close(va, vb, rtol, f"{where}[{i}]")
        elif b is None or isinstance(b, (str, bool)):
            assert a == b, (where, a, b)
        elif isinstance(b, float) and math.isinf(b):
            assert a == b, (where, a, b)
        else:
            assert a is not None and abs(float(a) - float(b)) <= rtol * (abs(float(b)) + 1.0), (where, a, b)


def _oracle_trace(ref, stack, tag, n_levels=3):
    op = S.Operator(24, 12, 6, ref["cant24/free"])
    g = GMG(op, n_levels=n_levels, **dict(dict(fine_smoother="fp64"), **stack))
    g.setup(ref[f"cant24/E_{tag}"])
    return g.cycle_trace(ref["cant24/rhs"])


@pytest.mark.parametrize("key", sorted(_load()["traces"]))
def test_oracle_trace_matches_reference(ref, key):
    case = _load()["traces"][key]
    got = _oracle_trace(ref, case["stack"], key.split("/")[1], case.get("n_levels", 3))
    rtol = 1e-6 if key.startswith("level_fp32") else 1e-9
    assert_trace_close(got, case["trace"], rtol, key)


def test_trace_output_is_the_preconditioner_without_inner_krylov(ref):
    """The traced cycle plus the root-local correction is apply() when no
    inner Krylov wrapper is configured."""
    op = S.Operator(24, 12, 6, ref["cant24/free"])
    stack = dict(fine_smoother="fp64", coarse_correction_policy="residual_line_search",
                 root_local_correction_mode="node_block_line_search")
    g = GMG(op, n_levels=3, **stack)
    g.setup(ref["cant24/E_mid"])
    rhs = ref["cant24/rhs"]
    z = g.apply(rhs)
    tr = g.cycle_trace(rhs)
    assert tr["output_norm"] == pytest.approx(float(np.linalg.norm(z)), rel=1e-12)
    assert tr["rz"] == pytest.approx(float(rhs @ z), rel=1e-12)


def test_trace_rejects_unknown_cycle_and_missing_setup(ref):
    op = S.Operator(24, 12, 6, ref["cant24/free"])
    g = GMG(op, n_levels=3, fine_smoother="fp64")
    with pytest.raises(RuntimeError, match="setup"):
        g.cycle_trace(ref["cant24/rhs"])
    g.setup(ref["cant24/E_mid"])
    with pytest.raises(ValueError, match="cycle_type"):
        g.cycle_trace(ref["cant24/rhs"], cycle_type="f")


def _diagnostics():
    return sorted(_load()["diagnostics"])


@pytest.mark.parametrize("key", _diagnostics())
def test_oracle_probe_quality_and_kappa_match_reference(ref, key):
    case = _load()["diagnostics"][key]
    op = S.Operator(24, 12, 6, ref["cant24/free"])
    g = GMG(op, n_levels=3, **dict(dict(fine_smoother="fp64"), **case["stack"]))
    g.setup(ref[f"cant24/E_{key.split('/')[1]}"])
    pq = g.probe_quality(ref["cant24/rhs"])
    want = case["probe_quality"]
    assert pq["finite"] == want["finite"] and pq["pd"] == want["pd"]
    for k in ("z_norm", "jacobi_norm", "z_over_jacobi"):
        assert pq[k] == pytest.approx(want[k], rel=1e-9), k
    assert g.estimate_kappa_eff(30) == pytest.approx(case["kappa_eff_30"], rel=1e-8)
