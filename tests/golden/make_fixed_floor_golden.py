"""Golden output of the reference's fixed-floor control driver.

Run from the repository root where the reference source tree is readable
(its root given by SIMPFEM_REFERENCE_ROOT):

    python tests/golden/make_fixed_floor_golden.py

Writes ``fixed_floor_manifest_cantilever_3d.csv`` (random Bernoulli states and
one stored field, ``gray`` of density_driver_fields.npz, on the cantilever_3d
preset), places the field where the reference driver looks for it (its own
repository root, here the stand-in's copy of the tree), runs the unchanged
experiments/phase5/run_gmg_fixed_floor_controls.py through the numpy-backed
``cupy`` stand-in (``_refshim.py``) and keeps its two CSV files as
``fixed_floor_cantilever_3d_summary.csv`` / ``..._history.csv``.
"""

from __future__ import annotations

import csv
import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import _refshim  # noqa: E402

MANIFEST = [
    dict(case_id="cant3d_s3_p035", case_type="random", preset="cantilever_3d", seed="3", solid_probability="0.35",
         density_path="", floors="1e-12;1e-3;1e-2", penal="4.5"),
    dict(case_id="cant3d_s5_p060", case_type="random", preset="cantilever_3d", seed="5", solid_probability="0.6",
         density_path="", floors="1e-2", penal="4.5"),
    dict(case_id="cant3d_gray", case_type="density", preset="cantilever_3d", seed="", solid_probability="",
         density_path="fields/gray/rho.npy", floors="1e-12;1e-3", penal="3.0"),
]


def main() -> None:
    manifest = os.path.join(HERE, "fixed_floor_manifest_cantilever_3d.csv")
    with open(manifest, "w", newline="", encoding="utf-8") as f:
        w = csv.DictWriter(f, fieldnames=list(MANIFEST[0]))
        w.writeheader()
        w.writerows(MANIFEST)
    _refshim.install()
    dst = os.path.join(_refshim._copy_root(), "fields", "gray")
    os.makedirs(dst, exist_ok=True)
    np.save(os.path.join(dst, "rho.npy"), np.load(os.path.join(HERE, "density_driver_fields.npz"))["gray"])
    out = tempfile.mkdtemp(prefix="fixed_floor_")
    try:
        _refshim.run_driver(os.path.join("experiments", "phase5", "run_gmg_fixed_floor_controls.py"),
                            ["--manifest", manifest, "--out-dir", out, "--maxiter", "80"])
        shutil.copyfile(os.path.join(out, "fixed_floor_control_summary.csv"),
                        os.path.join(HERE, "fixed_floor_cantilever_3d_summary.csv"))
        shutil.copyfile(os.path.join(out, "fixed_floor_control_history.csv"),
                        os.path.join(HERE, "fixed_floor_cantilever_3d_history.csv"))
    finally:
        shutil.rmtree(out, ignore_errors=True)
    print("wrote fixed_floor_cantilever_3d_{summary,history}.csv")


if __name__ == "__main__":
    main()
