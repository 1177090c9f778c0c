"""Golden data for the SIMP loop entry (run_simp_surrogate_gpu) as the
reference's trajectory driver calls it.

Run from the repository root where the reference source tree is readable
(its root given by SIMPFEM_REFERENCE_ROOT):

    python tests/golden/make_trajectory_driver_golden.py

Runs experiments/phase5/run_simp_floor_trajectory.py unchanged (a copy, through
the numpy ``cupy`` stand-in of ``_refshim.py``) on the cantilever_3d preset
(24x12x6) with a three-level hierarchy, FP64 smoothing, FGMRES restart 300,
maxiter 150 and the schedule-only parameter controller the driver installs:

* ``guarded``: ``--policy guarded_adaptive`` (floors 1e-12 | 1e-3, 1e-2; probe
  30 iterations, r50 read at 15), 45 SIMP iterations;
* ``guarded_pert``: the same with the load vector scaled entry by entry by
  (1 + 1e-12 xi), xi standard normal from numpy's default_rng(0) -- the
  reference's own sensitivity to round-off along the trajectory;
* ``fixed``: ``--policy fixed_floor --rho-mins 1e-3``, 20 SIMP iterations,
  and ``fixed_pert``, the same under the perturbed load vector.

Writes, per run, the driver's own trajectory_iters.csv and
trajectory_summary.csv as trajectory_<run>_iters.csv / _summary.csv, and
trajectory_driver_cantilever_3d.npz with each run's rho_final and rho_best.
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

DRIVER = os.path.join("experiments", "phase5", "run_simp_floor_trajectory.py")
COMMON = ["--presets", "cantilever_3d", "--n-levels", "3", "--maxiter", "150", "--restart", "300",
          "--fine-smoother", "fp64", "--probe-iters", "30", "--probe-r50", "15"]
RUNS = {
    "guarded": COMMON + ["--policy", "guarded_adaptive", "--iters", "45"],
    "guarded_pert": COMMON + ["--policy", "guarded_adaptive", "--iters", "45"],
    "fixed": COMMON + ["--policy", "fixed_floor", "--rho-mins", "1e-3", "--iters", "20"],
    "fixed_pert": COMMON + ["--policy", "fixed_floor", "--rho-mins", "1e-3", "--iters", "20"],
}
PERT = 1e-12


def _loads(perturbed: bool) -> None:
    """The reference generator's load vector, scaled by (1 + PERT xi) when perturbed."""
    bcg = _refshim.load("bc_generator")
    original = getattr(bcg, "_unperturbed", bcg.generate_bc)
    bcg._unperturbed = original
    if not perturbed:
        bcg.generate_bc = original
        return

    def generate_bc(spec, *a, **k):
        bc = original(spec, *a, **k)
        xi = np.random.default_rng(0).standard_normal(bc.F.shape)
        bc.F = bc.F * (1.0 + PERT * xi)
        return bc

    bcg.generate_bc = generate_bc


def main() -> None:
    _refshim.install()
    arrays = {}
    for run, argv in RUNS.items():
        _loads(run.endswith("_pert"))
        out = tempfile.mkdtemp(prefix=f"traj_{run}_")
        _refshim.run_driver(DRIVER, argv + ["--out-dir", out])
        for name in ("iters", "summary"):
            shutil.copyfile(os.path.join(out, f"trajectory_{name}.csv"),
                            os.path.join(HERE, f"trajectory_{run}_{name}.csv"))
        case = next(d for d in sorted(os.listdir(out)) if os.path.isdir(os.path.join(out, d)))
        for name in ("rho_final", "rho_best"):
            arrays[f"{run}_{name}"] = np.load(os.path.join(out, case, f"{name}.npy"))
        shutil.rmtree(out)
    np.savez_compressed(os.path.join(HERE, "trajectory_driver_cantilever_3d.npz"), **arrays)
    print("wrote", sorted(arrays))


if __name__ == "__main__":
    main()
