"""Host logic of GalerkinMatFreeGMG.cycle_trace, without a GPU: the library's
record layout (include/simpfem.h, simpfem_gmg_cycle_trace) encoded from the
oracle's traces of the reference-pinned cases, decoded by
gpu_fem.multigrid_v4.trace_from_records, must give back the same dictionary
field for field (ratios, None fields, notes, the root-local note on the root
visit)."""

import json
import math
import os

import numpy as np
import pytest

from oracle import solver as S
from oracle.gmg import GMG

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "cycle_trace_cant24.json")
CC_NOTES = ["", "degenerate_correction", "rejected_correction", "nonpositive_correction_scale",
            "clipped_correction_scale"]
RL_NOTES = ["", "degenerate_root_local_correction", "rejected_root_local_inner_fgmres", "root_local_inner_fgmres",
            "nonpositive_root_local_scale", "clipped_root_local_scale"]


def _nan(v):
    return math.nan if v is None else float(v)


def encode(tr: dict, enrich_mode: str):
    """The oracle's trace in the library's record layout."""
    rows = []
    local_note = ""
    for v in tr["visits"]:
        r = np.full(32, np.nan)
        notes = [n for n in v["notes"].split("|") if n]
        if v["level"] == 0 and not v["is_coarsest"] and notes and notes[-1] in RL_NOTES:
            local_note = notes.pop()
        cc = [n for n in notes if n in CC_NOTES]
        second = v["n_coarse_corrections"] == 2
        r[0], r[1], r[2], r[3] = v["visit_id"], v["level"], float(v["is_coarsest"]), v["n_coarse_corrections"]
        r[4], r[5], r[6], r[7] = v["rhs_norm"], v["jacobi_action_norm"], v["presmooth_solution_norm"], \
            v["presmooth_residual_norm"]
        r[8], r[9], r[10] = v["restricted_rhs_norm"], v["projector_norm"], v["coarse_space_gap_norm"]
        r[11], r[12], r[13] = v["coarse_correction_norm"], v["prolongated_correction_norm"], v["correction_alignment"]
        r[14], r[15], r[16] = _nan(v["correction_scale_raw"]), v["correction_scale_applied"], \
            v["corrected_residual_norm"]
        if second:
            r[17] = v["second_corrected_residual_norm"] / v["second_corrected_residual_vs_corrected"]
            r[18], r[19], r[20] = v["second_restricted_rhs_norm"], v["second_coarse_correction_norm"], \
                v["second_prolongated_correction_norm"]
            r[21], r[22], r[23] = v["second_correction_alignment"], _nan(v["second_correction_scale_raw"]), \
                v["second_correction_scale_applied"]
            r[24] = v["second_corrected_residual_norm"]
        else:
            r[17] = v["corrected_residual_norm"]
        r[25], r[26] = v["postsmooth_solution_norm"], v["postsmooth_residual_norm"]
        # notes of the first and second correction; empty notes are dropped
        # when they are joined, so one note of two corrections decodes the
        # same from either slot
        n1 = cc[0] if cc else ""
        n2 = cc[1] if len(cc) > 1 else ""
        r[27] = CC_NOTES.index(n1)
        r[28] = CC_NOTES.index(n2) if second else -1
        r[29] = float(f"root_enrichment:{enrich_mode}" in notes)
        r[30] = float("extra_fine_postsmooth" in notes)
        r[31] = ["none", "dense", "iterative"].index(v["coarsest_mode"]) if v["is_coarsest"] else -1
        rows.append(r)
    s = np.full(16, np.nan)
    pre = tr["output_residual_norm"] / tr["root_local_correction_residual_ratio"]
    s[:9] = [tr["rhs_norm"], tr["jacobi_action_norm"], tr["output_norm"], tr["rz"], tr["output_residual_norm"],
             pre, _nan(tr["root_local_correction_raw_scale"]), tr["root_local_correction_applied_scale"],
             RL_NOTES.index(local_note)]
    s[9:13] = [tr["contrast_ratio"], float(tr["is_high_contrast"]), tr["fine_degree_adapt"], tr["coarse_iters_adapt"]]
    return np.array(rows), s


def _options(tr):
    keys = ("coarse_correction_policy", "coarse_correction_acceptance_ratio", "coarse_correction_max_scale",
            "root_enrichment_mode", "root_enrichment_weight_floor", "root_enrichment_weight_power",
            "root_local_correction_mode", "root_local_correction_inner_steps", "root_local_correction_inner_restart",
            "inner_krylov_steps", "inner_krylov_restart")
    return {k: tr[k] for k in keys}


with open(GOLDEN) as _fh:
    _KEYS = sorted(json.load(_fh)["traces"])


@pytest.mark.parametrize("key", _KEYS)
def test_records_decode_to_the_oracle_trace(ref, key):
    from gpu_fem.multigrid_v4 import trace_from_records
    from test_oracle_cycle_trace import assert_trace_close

    with open(GOLDEN) as fh:
        case = json.load(fh)["traces"][key]
    op = S.Operator(24, 12, 6, ref["cant24/free"])
    g = GMG(op, n_levels=case.get("n_levels", 3), **dict(dict(fine_smoother="fp64"), **case["stack"]))
    g.setup(ref[f"cant24/E_{key.split('/')[1]}"])
    tr = g.cycle_trace(ref["cant24/rhs"])
    visits, summary = encode(tr, tr["root_enrichment_mode"])
    got = trace_from_records(visits, summary, tr["cycle_type"], _options(tr)).to_dict()
    assert_trace_close(got, tr, 1e-12, key)


def test_safe_ratio_and_empty_notes():
    from gpu_fem.multigrid_v4 import _safe_ratio

    assert _safe_ratio(0.0, 0.0) == 0.0
    assert _safe_ratio(1.0, 0.0) == math.inf
    assert _safe_ratio(3.0, 2.0) == 1.5
