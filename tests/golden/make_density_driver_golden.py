"""Golden output of the reference's density-field floor-detector driver.

Run from the repository root where the reference source tree is readable
(its root given by SIMPFEM_REFERENCE_ROOT):

    python tests/golden/make_density_driver_golden.py

Writes three density fields of the cantilever_3d preset (24 x 12 x 6) as
``<name>/rho.npy`` under a scratch folder, runs the unchanged
experiments/phase5/run_gmg_floor_detector_density_field.py on them through the
numpy-backed ``cupy`` stand-in (``_refshim.py``), from inside that folder so
the ``density_path`` column holds the relative paths, and keeps:

* ``density_driver_fields.npz`` -- the three fields, by name;
* ``density_detector_cantilever_3d_summary.csv`` / ``..._history.csv`` -- the
  driver's two CSV files as it wrote them;
* ``density_detector_cantilever_3d_pert_history.csv`` -- the history of a
  second run on the fields times (1 + 1e-14 N(0, 1)): the reference's own
  round-off sensitivity, from which the parity tests take their envelope.

The fields: ``gray`` (a cone-filtered Bernoulli field, intermediate densities),
``binary35`` (solid with probability 0.65, void 1e-9) and ``binary60`` (solid
with probability 0.4: the probe stalls and the ladder is taken).
"""

from __future__ import annotations

import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import _refshim  # noqa: E402

DIMS = (24, 12, 6)


def fields() -> dict:
    pss = _refshim.load("pub_simp_solver")
    n = int(np.prod(DIMS))
    H = pss._build_density_filter(DIMS[0], DIMS[1], 1.5, DIMS[2])
    rng = np.random.default_rng(17)
    gray = np.asarray(H @ (rng.random(n) >= 0.35).astype(np.float64))
    out = {"gray": gray}
    for name, p in (("binary35", 0.35), ("binary60", 0.60)):
        solid = np.random.default_rng(int(100 * p)).random(n) >= p
        out[name] = np.where(solid, 1.0, 1e-9)
    return out


def _run(fs: dict, out: str) -> None:
    paths = []
    for name, rho in fs.items():
        os.makedirs(name, exist_ok=True)
        np.save(os.path.join(name, "rho.npy"), rho)
        paths.append(os.path.join(name, "rho.npy"))
    _refshim.run_driver(
        os.path.join("experiments", "phase5", "run_gmg_floor_detector_density_field.py"),
        ["--preset", "cantilever_3d", "--density-paths", ",".join(paths), "--probe-iters", "30",
         "--probe-r50", "15", "--maxiter", "60", "--out-dir", out],
    )


def main() -> None:
    fs = fields()
    work = tempfile.mkdtemp(prefix="density_driver_")
    old = os.getcwd()
    try:
        os.chdir(work)
        _run(fs, "out")
        shutil.copyfile(os.path.join("out", "density_detector_summary.csv"),
                        os.path.join(HERE, "density_detector_cantilever_3d_summary.csv"))
        shutil.copyfile(os.path.join("out", "density_detector_history.csv"),
                        os.path.join(HERE, "density_detector_cantilever_3d_history.csv"))
        rng = np.random.default_rng(5)
        pert = {k: np.clip(v * (1.0 + 1e-14 * rng.standard_normal(v.size)), 0.0, 1.0) for k, v in fs.items()}
        _run(pert, "out_pert")
        shutil.copyfile(os.path.join("out_pert", "density_detector_history.csv"),
                        os.path.join(HERE, "density_detector_cantilever_3d_pert_history.csv"))
    finally:
        os.chdir(old)
        shutil.rmtree(work, ignore_errors=True)
    np.savez_compressed(os.path.join(HERE, "density_driver_fields.npz"), **fs)
    print("wrote density_detector_cantilever_3d_{summary,history}.csv and density_driver_fields.npz")


if __name__ == "__main__":
    main()
