"""The oracle's iterative coarsest solve against the reference.

tests/golden/coarse_pcg_reference.npz (make_coarse_pcg_golden.py): the
reference's GalerkinMatFreeGMG with dense_chol_max=0, so the coarsest level is
solved by _fixed_pcg_coarse (solver_v2.py:781-810; 200 iterations on a
high-contrast field, 80 otherwise), on 24 x 12 x 6 and 40 x 20 x 10 cantilevers
with three levels.  The oracle reproduces one apply of each stack and field to
max(1e-10, 100 x the reference's own deviation under a 1e-14 perturbation of
E) -- 80 unconverged PCG iterations on the smooth field amplify round-off, the
reference's own apply moving by up to 1e-6 there -- and the FGMRES solve's
iteration count and history (1e-8).
"""

import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "coarse_pcg_reference.npz")
STACKS = {"jacobi": dict(smoother_type="jacobi"), "cheb": dict()}


def _setup(g, name, stack):
    from oracle.gmg import GMG
    from oracle.solver import Operator, cantilever_bc

    nx, ny, nz = (int(v) for v in g[f"{name}/dims"])
    free, F = cantilever_bc(nx, ny, nz)
    op = Operator(nx, ny, nz, free)
    return op, F[free], GMG(op, n_levels=3, fine_smoother="fp64", dense_chol_max=0, **stack)


@pytest.mark.parametrize("name", ["cant24", "cant40"])
def test_oracle_iterative_coarse_apply_and_solve(name):
    from oracle.solver import fgmres

    g = np.load(GOLDEN)
    for sname, stack in STACKS.items():
        for tag in ("hi", "lo"):
            op, F, gm = _setup(g, name, stack)
            gm.setup(g[f"{name}/E_{tag}"])
            assert gm.coarse_mode == "iterative" and gm.high == bool(g[f"{name}/high_{sname}_{tag}"][0])
            ref = g[f"{name}/apply_{sname}_{tag}"]
            dev = np.linalg.norm(g[f"{name}/apply_pert_{sname}_{tag}"] - ref) / np.linalg.norm(ref)
            z = gm.apply(g[f"{name}/rhs"])
            err = np.linalg.norm(z - ref) / np.linalg.norm(ref)
            assert err <= max(1e-10, 100 * dev), (sname, tag, err, dev)
    op, F, gm = _setup(g, name, STACKS["jacobi"])
    E = g[f"{name}/E_hi"]
    gm.setup(E)
    hist = []
    x, it, conv = fgmres(lambda v: op.matvec(v, E), F, gm.apply, tol=1e-6, maxiter=300, restart=300, history=hist)
    info = g[f"{name}/solve_info"]
    assert (it, int(conv)) == (int(info[0]), int(info[1]))
    np.testing.assert_allclose(hist, g[f"{name}/solve_hist"], rtol=1e-8, atol=1e-15)
