"""Golden traces of one multigrid cycle from the reference's own ``cycle_trace``.

Run from the repository root where the reference source tree is readable
(its root given by SIMPFEM_REFERENCE_ROOT):

    python tests/golden/make_cycle_trace_golden.py

``GalerkinMatFreeGMG.cycle_trace`` (gpu_fem/multigrid_v4.py:1362-1728) runs
unmodified on the host through the numpy-backed ``cupy`` stand-in in
``_refshim.py``, on the inputs already committed in ``reference_small.npz``
(the cant24 moduli ``E_hi`` / ``E_mid`` and right-hand side ``rhs``).  Each
trace is written with the reference's own ``to_dict()`` into
``cycle_trace_cant24.json``; the oracle's restatement (oracle/gmg.py) is
pinned to it, and through the oracle the device trace.  The same file holds
the two other diagnostics of the hierarchy, ``probe_quality`` (:1348-1360) and
``estimate_kappa_eff`` (:1057-1117), for the linear stacks; the Lanczos start
vector is the stand-in's ``RandomState(0).standard_normal`` (numpy's generator).
"""

from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import _refshim  # noqa: E402
from make_golden import STACKS, _build  # noqa: E402

TRACE_STACKS = {
    "plain_cheb": STACKS["plain_cheb"],
    "plain_jacobi": STACKS["plain_jacobi"],
    "wcycle": STACKS["wcycle"],
    "line_search": STACKS["line_search"],
    "enrich": STACKS["enrich"],
    "enrich_void": STACKS["enrich_void"],
    "nb_line_search": STACKS["nb_line_search"],
    "canonical": STACKS["canonical"],
    "level_fp32": STACKS["level_fp32"],
    "wcycle_enrich": dict(cycle_type="w", coarse_correction_policy="residual_line_search",
                          root_enrichment_mode="void_gap_second"),
}


def main() -> None:
    presets = _refshim.load("presets")
    spec = presets.get_preset("cantilever_3d")
    fx = np.load(os.path.join(HERE, "reference_small.npz"))
    rhs = fx["cant24/rhs"]
    out = {"case": "cant24", "n_levels": 3, "traces": {}}
    for sname, stack in TRACE_STACKS.items():
        for tag in ("hi", "mid"):
            _, _, _, _, gmg = _build(spec, 3, stack)
            gmg.setup(fx[f"cant24/E_{tag}"])
            tr = gmg.cycle_trace(rhs).to_dict()
            out["traces"][f"{sname}/{tag}"] = {"stack": stack, "trace": tr}
    # one level: the trace is a single coarsest visit whose solve is the fine smoother
    _, _, _, _, gmg = _build(spec, 1, {})
    gmg.setup(fx["cant24/E_mid"])
    out["traces"]["single_level/mid"] = {"stack": {}, "n_levels": 1, "trace": gmg.cycle_trace(rhs).to_dict()}
    out["diagnostics"] = {}
    for sname in ("plain_cheb", "plain_jacobi", "wcycle", "level_fp32"):
        for tag in ("hi", "mid"):
            _, _, _, _, gmg = _build(spec, 3, TRACE_STACKS[sname])
            gmg.setup(fx[f"cant24/E_{tag}"])
            pq = gmg.probe_quality(rhs)
            kappa = gmg.estimate_kappa_eff(30)
            out["diagnostics"][f"{sname}/{tag}"] = {"stack": TRACE_STACKS[sname], "probe_quality": pq,
                                                    "kappa_eff_30": kappa}
    path = os.path.join(HERE, "cycle_trace_cant24.json")
    with open(path, "w") as fh:
        json.dump(out, fh, indent=0, sort_keys=True)
    print(f"wrote {path}: {len(out['traces'])} traces")


if __name__ == "__main__":
    main()
