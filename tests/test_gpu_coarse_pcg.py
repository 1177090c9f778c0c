"""The iterative coarsest solve on the GPU against the reference.

tests/golden/coarse_pcg_reference.npz (make_coarse_pcg_golden.py): the
reference's GalerkinMatFreeGMG with dense_chol_max=0, so the coarsest level is
solved by the fixed-count Jacobi PCG _fixed_pcg_coarse (solver_v2.py:781-810;
200 iterations on a high-contrast field, 80 otherwise), as the 1M-element
workload's coarsest level (6,825 free DOFs, above the 5,000 dense limit) is.
Cantilevers 24 x 12 x 6 and 40 x 20 x 10, three levels:

* the hierarchy reports the iterative coarse mode;
* one preconditioner apply per stack (damped Jacobi, Chebyshev) and field
  (high-contrast, smooth) within max(1e-8, 100 x the reference's own
  deviation under a 1e-14 perturbation of E);
* one FGMRES solve (restart 300, tol 1e-6): iteration count and convergence
  identical, history within 1e-6 relative, compliance within max(1e-7, 100 x
  the reference's own deviation), the FP64 guard met.
"""

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "coarse_pcg_reference.npz")
STACKS = {"jacobi": dict(smoother_type="jacobi"), "cheb": dict()}


def _components(dims, stack):
    import torch

    from gpu_fem.bc_generator import generate_bc
    from gpu_fem.multigrid_v4 import GalerkinMatFreeGMG
    from gpu_fem.presets import cantilever_spec
    from gpu_fem.pub_simp_solver import KE_UNIT_3D, _edof_table_3d
    from gpu_fem.solver_v2 import MatrixFreeKff

    spec = cantilever_spec(*dims)
    bc = generate_bc(spec)
    free = bc.free_dofs.astype(np.int32)
    edof = torch.as_tensor(_edof_table_3d(*dims), device="cuda")
    mf = MatrixFreeKff(edof, torch.as_tensor(KE_UNIT_3D, device="cuda"), torch.as_tensor(free, device="cuda"),
                       len(free), bc.ndof)
    gmg = GalerkinMatFreeGMG(mf_op=mf, free=free, free_gpu=free, nelx=dims[0], nely=dims[1], nelz=dims[2],
                             KE_UNIT=KE_UNIT_3D, n_levels=3, fine_smoother="fp64", dense_chol_max=0, **stack)
    return mf, gmg, torch.as_tensor(bc.F[free], device="cuda")


@pytest.mark.parametrize("name", ["cant24", "cant40"])
def test_iterative_coarse_apply(cuda, name):
    torch = cuda
    g = np.load(GOLDEN)
    dims = tuple(int(v) for v in g[f"{name}/dims"])
    for sname, stack in STACKS.items():
        for tag in ("hi", "lo"):
            mf, gmg, _ = _components(dims, stack)
            gmg.setup(torch.as_tensor(g[f"{name}/E_{tag}"], device="cuda"))
            assert gmg.coarse_mode == "iterative"
            assert gmg.is_high_contrast == bool(g[f"{name}/high_{sname}_{tag}"][0])
            ref = g[f"{name}/apply_{sname}_{tag}"]
            dev = np.linalg.norm(g[f"{name}/apply_pert_{sname}_{tag}"] - ref) / np.linalg.norm(ref)
            z = gmg.apply(torch.as_tensor(g[f"{name}/rhs"], device="cuda")).cpu().numpy()
            err = np.linalg.norm(z - ref) / np.linalg.norm(ref)
            assert err <= max(1e-8, 100 * dev), (name, sname, tag, err, dev)


@pytest.mark.parametrize("name", ["cant24", "cant40"])
def test_iterative_coarse_solve(cuda, name):
    torch = cuda
    from gpu_fem.multigrid_v4 import _cupy_fgmres

    g = np.load(GOLDEN)
    dims = tuple(int(v) for v in g[f"{name}/dims"])
    mf, gmg, F = _components(dims, STACKS["jacobi"])
    E = torch.as_tensor(g[f"{name}/E_hi"], device="cuda")
    gmg.setup(E)
    hist = []
    x, it, conv = _cupy_fgmres(lambda v: mf.matvec(v, E), F, gmg.apply, tol=1e-6, maxiter=300, restart=300,
                               history=hist)
    info, pinfo = g[f"{name}/solve_info"], g[f"{name}/solve_pert_info"]
    assert (it, int(conv)) == (int(info[0]), int(info[1]))
    np.testing.assert_allclose(hist, g[f"{name}/solve_hist"], rtol=1e-6, atol=1e-15)
    c = float(torch.dot(F, x))
    dev = abs(pinfo[2] - info[2]) / abs(info[2])
    assert abs(c - info[2]) <= max(1e-7, 100 * dev) * abs(info[2]), (c, info[2], dev)
    res = float(torch.linalg.norm(F - mf.matvec(x, E)) / torch.linalg.norm(F))
    assert res <= 1e-6
