"""Iteration-count envelope of the reference's own fixed-floor controls under round-off.

Run from the repository root where the reference source tree is readable
(its root given by SIMPFEM_REFERENCE_ROOT):

    python tests/golden/make_perturbation_envelope.py [pert_seed ...]

For the 64k cantilever rows of the fixed-floor control manifest
(experiments/phase5/fixed_floor_control_manifest.csv: cant_s23_p035,
cant_s31_p035, C64_MF; floors 1e-12, 1e-3, 1e-2 in manifest order through one
hierarchy, as experiments/phase5/run_gmg_fixed_floor_controls.py:81-135 runs
them) this runs the reference's unmodified canonical stack through the
numpy-backed ``cupy`` stand-in in ``_refshim.py`` with E multiplied by
(1 + 1e-14 * N(0, 1)) for each perturbation seed (seed 0 = no perturbation),
and appends one row per solve to ``perturbation_envelope_64k.csv``:
case, floor, pert_seed, iterations, compliance, true relative residual.

The canonical stack's preconditioner makes discrete choices (the line-search
step, root-local adaptivity) from residual norms, so the reference's own
iteration count on a state can move by many iterations under a 1e-14 change of
E; the CUDA path's counts are judged against this envelope, not against a
single published count.
"""

from __future__ import annotations

import csv
import fcntl
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import _refshim  # noqa: E402

OUT = os.path.join(HERE, "perturbation_envelope_64k.csv")
CASES = ("cant_s23_p035", "cant_s31_p035", "C64_MF")
FLOORS = (1e-12, 1e-3, 1e-2)


def _density(case, n_elem):
    if case.startswith("cant_s"):
        seed = int(case.split("_")[1][1:])
        return (np.random.default_rng(seed).random(n_elem) < 0.35).astype(np.float64)
    rho = np.load(os.path.join(HERE, f"density_{case}.npz"))["rho"].reshape(-1)
    return np.clip(np.asarray(rho, dtype=np.float64), 0.0, 1.0)


def run(pert_seed: int) -> None:
    p4 = _refshim.load_paper4_runner()
    mg = _refshim.load("multigrid_v4")
    spec, bc, free, free_gpu, edof_gpu, F, mf, gmg = p4._build_components(
        "cantilever_gpu_medium", n_levels=4, fine_smoother="fp64", smoother_type="chebyshev", cycle_type="v",
        coarse_correction_policy="residual_line_search", root_local_correction_mode="node_block_inner_fgmres",
        root_local_correction_inner_steps=20, root_local_correction_inner_restart=20, inner_krylov_steps=10,
        inner_krylov_restart=10)
    n = spec.nelx * spec.nely * spec.nelz
    pert = 1.0 if pert_seed == 0 else 1.0 + 1e-14 * np.random.default_rng(pert_seed).standard_normal(n)
    bnorm = float(np.linalg.norm(F))
    for case in CASES:
        dens = _density(case, n)
        for floor in FLOORS:
            E = (floor + (1.0 - floor) * dens ** 4.5) * pert
            gmg.setup(E)
            t0 = time.time()
            x, it, _ = mg._cupy_fgmres(lambda v: mf.matvec(v, E), F, gmg.apply, tol=1e-6, maxiter=300,
                                       restart=300)
            res = float(np.linalg.norm(F - mf.matvec(x, E))) / bnorm
            row = dict(case_id=case, rho_min=floor, pert_seed=pert_seed, solve_iters=int(it),
                       compliance=float(F @ x), final_rel_residual=res)
            with open(OUT, "a", newline="") as f:
                fcntl.flock(f, fcntl.LOCK_EX)  # seeds may run as parallel processes
                w = csv.DictWriter(f, fieldnames=list(row))
                if f.tell() == 0:
                    w.writeheader()
                w.writerow(row)
                f.flush()
                fcntl.flock(f, fcntl.LOCK_UN)
            print(case, floor, pert_seed, it, f"{time.time() - t0:.0f}s", flush=True)


if __name__ == "__main__":
    for s in (sys.argv[1:] or ["0", "99", "100"]):
        run(int(s))
