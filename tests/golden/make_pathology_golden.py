"""Golden output of the reference's pathology diagnostics driver.

Run from the repository root where the reference source tree is readable
(its root given by SIMPFEM_REFERENCE_ROOT):

    python tests/golden/make_pathology_golden.py

Runs the unchanged experiments/phase5/run_pathology_diagnostics.py through the
numpy-backed ``cupy`` stand-in (``_refshim.py``) on the cantilever_3d preset,
all seven cases, twice:

* ``v``: the driver's default stack (V-cycle, no safeguards), with the FGMRES
  solve (restart 50, at most 150 iterations);
* ``w``: W-cycle, residual line search, void-gap root enrichment and the
  node-block line-search root-local correction, trace only.

Keeps ``pathology_<run>_summary.csv``, ``pathology_<run>_visits.csv`` and, for
the solved run, ``pathology_v_solve_history.csv``, as the driver wrote them.
"""

from __future__ import annotations

import os
import shutil
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import _refshim  # noqa: E402

RUNS = {
    "v": ["--maxiter", "150"],
    "w": ["--cycle-type", "w", "--coarse-policy", "residual_line_search", "--root-enrichment-mode",
          "void_gap_second", "--root-local-correction-mode", "node_block_line_search", "--skip-solve"],
}


def main() -> None:
    for tag, extra in RUNS.items():
        out = tempfile.mkdtemp(prefix="pathology_")
        try:
            _refshim.run_driver(os.path.join("experiments", "phase5", "run_pathology_diagnostics.py"),
                                ["--preset", "cantilever_3d", "--cases", "all", "--out-dir", out] + extra)
            names = ["summary", "visits"] + (["solve_history"] if tag == "v" else [])
            for name in names:
                shutil.copyfile(os.path.join(out, f"pathology_{name}.csv"),
                                os.path.join(HERE, f"pathology_{tag}_{name}.csv"))
        finally:
            shutil.rmtree(out, ignore_errors=True)
    print("wrote pathology_{v,w}_*.csv")


if __name__ == "__main__":
    main()
