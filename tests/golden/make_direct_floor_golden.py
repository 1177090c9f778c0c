"""Golden output of the reference's direct-solve floor drivers.

Run from the repository root where the reference source tree is readable
(its root given by SIMPFEM_REFERENCE_ROOT):

    python tests/golden/make_direct_floor_golden.py

Runs the unchanged experiments/phase5/run_direct_floor_atlas.py,
run_direct_floor_conditioning.py and compare_reduced_floor_perturbation.py over
the reference's own package (a copy,
through the numpy ``cupy`` stand-in of ``_refshim.py``) on the cantilever_3d
preset, seed 3, solid probabilities 0.2 and 0.35, floors 1e-12, 1e-6 and 1e-3
(SIMP penal 4.5): sparse assembly from the paper-4 runner's KE_UNIT_3D,
_edof_table_3d and _build_sparse_indices, direct solves (and for the
conditioning driver, the extreme eigenvalues; for the comparison, each raised
floor's solution against the 1e-12 one).  Keeps the drivers' CSV files as
direct_floor_atlas_cantilever_3d.csv, direct_floor_critical_cantilever_3d.csv,
direct_floor_conditioning_cantilever_3d.csv and
reduced_floor_perturbation_cantilever_3d.csv.
"""

from __future__ import annotations

import os
import shutil
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import _refshim  # noqa: E402

ARGS = ["--preset", "cantilever_3d", "--probabilities", "0.2,0.35", "--rho-min-values", "1e-12,1e-6,1e-3",
        "--seeds", "3"]
RUNS = {
    "run_direct_floor_atlas.py": {"direct_floor_atlas.csv": "direct_floor_atlas_cantilever_3d.csv",
                                  "direct_floor_critical.csv": "direct_floor_critical_cantilever_3d.csv"},
    "run_direct_floor_conditioning.py": {"direct_floor_conditioning.csv":
                                         "direct_floor_conditioning_cantilever_3d.csv"},
    "compare_reduced_floor_perturbation.py": {"reduced_floor_perturbation_summary.csv":
                                              "reduced_floor_perturbation_cantilever_3d.csv"},
}


def main() -> None:
    for driver, files in RUNS.items():
        out = tempfile.mkdtemp(prefix="direct_floor_")
        try:
            _refshim.run_driver(os.path.join("experiments", "phase5", driver), ARGS + ["--out-dir", out])
            for src, dst in files.items():
                shutil.copyfile(os.path.join(out, src), os.path.join(HERE, dst))
        finally:
            shutil.rmtree(out, ignore_errors=True)
    print("wrote", [d for files in RUNS.values() for d in files.values()])


if __name__ == "__main__":
    main()
