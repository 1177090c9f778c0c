"""Golden output of the reference's floor-rule check driver.

Run from the repository root where the reference source tree is readable
(its root given by SIMPFEM_REFERENCE_ROOT):

    python tests/golden/make_rule_check_golden.py

Writes ``rule_check_thresholds.csv``, a rule table in the format the driver
reads (safety factor, solid probability, median and conservative seed
thresholds; the values are chosen here, the reference's table comes from a
validation run it does not ship), runs the unchanged
experiments/phase5/run_gmg_floor_rule_check.py through the numpy-backed
``cupy`` stand-in (``_refshim.py``) on the cantilever_3d preset, seed 3,
solid probabilities 0.2 and 0.35, maxiter 150 (canonical stack: FP64 Chebyshev
V-cycle, residual line search, node-block root-local FGMRES), and keeps its two
CSV files as ``rule_check_cantilever_3d_summary.csv`` / ``..._history.csv``.
"""

from __future__ import annotations

import csv
import os
import shutil
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import _refshim  # noqa: E402

THRESHOLDS = [
    dict(safety_factor="10", solid_probability="0.2", median_seed_threshold="0.001",
         conservative_seed_threshold="0.01"),
    dict(safety_factor="10", solid_probability="0.35", median_seed_threshold="1e-12",
         conservative_seed_threshold="0.001"),
]
ARGS = ["--preset", "cantilever_3d", "--probabilities", "0.2,0.35", "--seeds", "3", "--maxiter", "150"]


def main() -> None:
    table = os.path.join(HERE, "rule_check_thresholds.csv")
    with open(table, "w", newline="", encoding="utf-8") as f:
        w = csv.DictWriter(f, fieldnames=list(THRESHOLDS[0]))
        w.writeheader()
        w.writerows(THRESHOLDS)
    out = tempfile.mkdtemp(prefix="rule_check_")
    try:
        _refshim.run_driver(os.path.join("experiments", "phase5", "run_gmg_floor_rule_check.py"),
                            ARGS + ["--rule-table", table, "--out-dir", out])
        for name in ("summary", "history"):
            shutil.copyfile(os.path.join(out, f"gmg_floor_rule_{name}.csv"),
                            os.path.join(HERE, f"rule_check_cantilever_3d_{name}.csv"))
    finally:
        shutil.rmtree(out, ignore_errors=True)
    print("wrote rule_check_cantilever_3d_{summary,history}.csv")


if __name__ == "__main__":
    main()
