"""Round-off envelope of the prospective driver's states on cantilever_3d.

    python tests/golden/make_policy_envelope.py

policy_cantilever_3d_summary.csv holds the reference driver's own run
(run_gmg_floor_detector_prospective.py, made by make_golden.py) on six
Bernoulli states of the 24 x 12 x 6 cantilever through one canonical-stack
hierarchy.  This script replays the same states in the same order through the
oracle (oracle/, pinned to the reference by tests/test_oracle.py) with the
element densities multiplied by (1 + 1e-14 * N(0, 1)) for a few perturbation
seeds (seed 0 = no perturbation), and writes the trigger, selected floor and
iteration count of each run to policy_envelope_cantilever_3d.csv.  The
canonical stack's line search and root-local correction make discrete choices
from residual norms, so a count that moves inside this envelope is
round-off, not a defect.
"""

from __future__ import annotations

import csv
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.gmg import GMG  # noqa: E402
from oracle.policy import run_state  # noqa: E402
from oracle.solver import Operator, cantilever_bc  # noqa: E402

NX, NY, NZ = 24, 12, 6
CANONICAL = dict(fine_smoother="fp64", smoother_type="chebyshev", cycle_type="v",
                 coarse_correction_policy="residual_line_search",
                 root_local_correction_mode="node_block_inner_fgmres", root_local_correction_inner_steps=20,
                 root_local_correction_inner_restart=20, inner_krylov_steps=10, inner_krylov_restart=10)


def main(pert_seeds=(0, 99, 100, 101)) -> None:
    with open(os.path.join(HERE, "policy_cantilever_3d_summary.csv"), newline="") as f:
        states = [(int(r["seed"]), float(r["solid_probability"])) for r in csv.DictReader(f)]
    free, F = cantilever_bc(NX, NY, NZ)
    op = Operator(NX, NY, NZ, free)
    Ff = F[free]
    n = NX * NY * NZ
    out = []
    for ps in pert_seeds:
        g = GMG(op, n_levels=4, **CANONICAL)  # one hierarchy per replay, as the driver uses one
        pert = 1.0 if ps == 0 else 1.0 + 1e-14 * np.random.default_rng(ps).standard_normal(n)
        for seed, p in states:
            solid = np.random.default_rng(seed).random(n) < p
            res = run_state(op, g, Ff, lambda rm, s=solid: np.where(s, 1.0, rm) * pert, penal=4.5,
                            raised=(1e-3, 1e-2), probe_iters=30, probe_r50=15, maxiter=60, restart=300)
            sel = res["selected"]
            out.append(dict(seed=seed, solid_probability=p, pert_seed=ps, trigger=res["trigger"],
                            recommended_rho_min=sel["rho_min"], solve_iters=sel["iters"],
                            solve_converged=int(sel["converged"])))
            print(out[-1], flush=True)
    with open(os.path.join(HERE, "policy_envelope_cantilever_3d.csv"), "w", newline="") as f:
        w = csv.DictWriter(f, fieldnames=list(out[0]))
        w.writeheader()
        w.writerows(out)


if __name__ == "__main__":
    main()
