"""The floor-rule check's solves on the GPU against the reference driver's run.

tests/golden/rule_check_cantilever_3d_{summary,history}.csv come from the
unchanged experiments/phase5/run_gmg_floor_rule_check.py (make_rule_check_golden.py):
cantilever_3d, the Bernoulli field of seed 3 at solid probabilities 0.2 and
0.35, the baseline floor 1e-12 and the rule table's floor where it differs.
Here the driver's own steps (:145-214) run through this package:
``paper4._build_components`` with the driver's stack (FP64 Chebyshev V-cycle,
residual line search, node-block root-local FGMRES), E = rho_min + (1 - rho_min)
rho^4.5, ``gmg.setup(E)``, ``_cupy_fgmres`` (restart 300, maxiter 150, tol 1e-6)
and the recomputed true residual.  Per row: the same convergence flag, the true
residual at or below 1e-6, outer iterations within 1 (within 3% on the
133-iteration baseline at p = 0.2, a slowly converging 1e-12 floor), and the
residual history's first 4 entries within 1e-7 relative, first 10 within 1e-4.
"""

import csv
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _rows(name):
    with open(os.path.join(GOLDEN, f"rule_check_cantilever_3d_{name}.csv"), newline="") as f:
        return list(csv.DictReader(f))


def run_rule_check_solves():
    import torch
    from gpu_fem import paper4
    from gpu_fem.multigrid_v4 import _cupy_fgmres

    spec, bc, free, free_gpu, edof_gpu, F, mf_op, gmg = paper4._build_components(
        "cantilever_3d", n_levels=4, fine_smoother="fp64", smoother_type="chebyshev", cycle_type="v",
        coarse_correction_policy="residual_line_search", root_local_correction_mode="node_block_inner_fgmres",
        root_local_correction_inner_steps=20, root_local_correction_inner_restart=20, inner_krylov_steps=10,
        inner_krylov_restart=10)
    b_norm = float(torch.linalg.norm(F))
    field = np.random.default_rng(3).random(spec.nelx * spec.nely * spec.nelz)
    out = []
    for row in _rows("summary"):
        solid = field < float(row["solid_probability"])
        rho_min = float(row["rho_min"])
        rho = torch.as_tensor(np.where(solid, 1.0, rho_min), dtype=torch.float64, device="cuda")
        E = rho_min + (1.0 - rho_min) * rho ** 4.5
        gmg.setup(E)
        history = []
        x, iters, converged = _cupy_fgmres(lambda v: mf_op.matvec(v, E), F, gmg.apply, tol=1e-6, maxiter=150,
                                           restart=300, history=history)
        final = float(torch.linalg.norm(F - mf_op.matvec(x, E))) / b_norm
        out.append(dict(iters=int(iters), converged=int(converged), final=final, history=list(history)))
    return out


def test_rule_check_solves_match_reference(cuda):
    ref = _rows("summary")
    href = _rows("history")
    got = run_rule_check_solves()
    assert len(got) == len(ref) == 3
    for g, r in zip(got, ref):
        key = (r["solid_probability"], r["case_kind"])
        assert g["converged"] == int(r["solve_converged"]), key
        assert g["final"] <= 1e-6, key
        n = int(r["solve_iters"])
        assert abs(g["iters"] - n) <= max(1, int(0.03 * n)), (key, g["iters"], n)
        b = [float(h["rel_residual"]) for h in href
             if (h["solid_probability"], h["case_kind"]) == key]
        assert len(b) == int(r["solve_history_len"])
        np.testing.assert_allclose(g["history"][:4], b[:4], rtol=1e-7, atol=0, err_msg=str(key))
        np.testing.assert_allclose(g["history"][:10], b[:10], rtol=1e-4, atol=0, err_msg=str(key))
