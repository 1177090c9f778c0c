"""The oracle on the benchmark workload's own states, against the reference.

tests/golden/baseline_policy_80x40x20.npz (make_baseline_golden.py) holds the
reference's own guarded policy run (its MatrixFreeKff, GalerkinMatFreeGMG and
_cupy_fgmres, unmodified, on the host) on filtered void-probability states of
the 80 x 40 x 20 cantilever: void probability (0.2, 0.35, 0.5)[seed % 3],
cone filter r = 1.5, E = rho_min + (1 - rho_min) rho^3, the damped-Jacobi
4-level V-cycle, FGMRES restart 300, tol 1e-6, seeds 0-5 through one hierarchy.
The oracle replays the first three states in the same order: trigger, floors,
flags and iteration counts identical; probe history, compliance and the
displacement sample within 1e-9 relative (the reference's own deviation under a
1e-14 perturbation of E is recorded beside them and is far below that).
"""

import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "baseline_policy_80x40x20.npz")


def test_oracle_matches_reference_on_workload_states():
    from oracle.gmg import GMG
    from oracle.policy import run_state
    from oracle.solver import Operator, cantilever_bc, density_filter

    g = np.load(GOLDEN)
    meta = json.loads(str(g["meta"]))
    rows = json.loads(str(g["rows"]))
    pert = json.loads(str(g["pert_rows"]))
    hist = json.loads(str(g["probe_history"]))
    nx, ny, nz = 80, 40, 20
    n = nx * ny * nz
    free, F = cantilever_bc(nx, ny, nz)
    op = Operator(nx, ny, nz, free)
    Ff = F[free]
    H = density_filter(nx, ny, nz, meta["rmin"])
    gmg = GMG(op, n_levels=4, fine_smoother="fp64", smoother_type="jacobi")
    stride = meta["stride"]
    for k, ref in enumerate(rows[:3]):
        seed = ref["seed"]
        p = meta["probs"][seed % len(meta["probs"])]
        rho = H @ (np.random.default_rng(seed).random(n) >= p).astype(np.float64)
        res = run_state(op, gmg, Ff, lambda rm, rho=rho: rho, penal=meta["penal"], raised=tuple(meta["ladder"]),
                        tol=meta["tol"], restart=meta["restart"], maxiter=meta["maxiter"])
        sel = res["selected"]
        assert res["trigger"] == ref["trigger"] and res["attempted"] == ref["attempted"], k
        assert sel["rho_min"] == ref["rho_min"] and sel["converged"] == ref["converged"], k
        assert sel["iters"] == ref["iters"] and bool(res["fallback"]) == ref["fallback"], k
        np.testing.assert_allclose(res["probe_history"], hist[k], rtol=1e-9, atol=1e-15)
        c = float(np.dot(Ff, sel["x"]))
        assert abs(c - ref["compliance"]) <= 1e-9 * ref["compliance"], (k, c, ref["compliance"])
        xs = sel["x"][::stride]
        assert np.linalg.norm(xs - g["x_sample"][k]) <= 1e-9 * np.linalg.norm(g["x_sample"][k]), k
        # the reference's own round-off envelope is far inside these bounds
        assert abs(pert[k]["compliance"] - ref["compliance"]) <= 1e-11 * ref["compliance"]
