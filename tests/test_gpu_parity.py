"""CUDA path vs the reference's own outputs (fixtures made by tests/golden/make_golden.py)
on small meshes: cantilever 24x12x6, an odd-dimension cantilever 13x7x5 and the
bridge 30x10x5 (point supports, roller BCs)."""

import numpy as np
import pytest

from gpu_fem import presets
from gpu_fem.bc_generator import generate_bc
from gpu_fem.pub_simp_solver import KE_UNIT_3D, _edof_table_3d

pytestmark = pytest.mark.gpu

CASES = {"cant24": "cantilever_3d", "odd13": None, "bridge30": "bridge_3d"}
STACKS = {
    "plain_jacobi": dict(smoother_type="jacobi"),
    "plain_cheb": dict(),
    "line_search": dict(coarse_correction_policy="residual_line_search"),
    "canonical": dict(coarse_correction_policy="residual_line_search",
                      root_local_correction_mode="node_block_inner_fgmres",
                      root_local_correction_inner_steps=20, root_local_correction_inner_restart=20,
                      inner_krylov_steps=10, inner_krylov_restart=10),
    "wcycle": dict(cycle_type="w"),
    "nb_line_search": dict(root_local_correction_mode="node_block_line_search"),
    "enrich": dict(coarse_correction_policy="residual_line_search", root_enrichment_mode="weighted_gap_second"),
    "enrich_void": dict(root_enrichment_mode="void_residual_second"),
    "level_fp32": dict(level_precisions=["fp64", "fp32", "fp32"]),
    "fine_fp32": dict(fine_smoother="fp32"),
}
LOW_PREC = {"level_fp32", "fine_fp32"}


def _spec(name):
    return presets.get_preset(CASES[name]) if CASES[name] else presets.cantilever_spec(13, 7, 5)


def _components(name, stack, n_levels=3):
    import torch

    from gpu_fem.multigrid_v4 import GalerkinMatFreeGMG
    from gpu_fem.solver_v2 import MatrixFreeKff

    spec = _spec(name)
    bc = generate_bc(spec)
    free = bc.free_dofs.astype(np.int32)
    edof = torch.as_tensor(_edof_table_3d(spec.nelx, spec.nely, spec.nelz), device="cuda")
    mf = MatrixFreeKff(edof, torch.as_tensor(KE_UNIT_3D, device="cuda"), torch.as_tensor(free, device="cuda"),
                       len(free), bc.ndof)
    kw = dict(fine_smoother="fp64")
    kw.update(stack)
    gmg = GalerkinMatFreeGMG(mf_op=mf, free=free, free_gpu=free, nelx=spec.nelx, nely=spec.nely, nelz=spec.nelz,
                             KE_UNIT=KE_UNIT_3D, n_levels=n_levels, **kw)
    F = torch.as_tensor(bc.F[free], device="cuda")
    return mf, gmg, F


def _rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("tag", ["hi", "mid", "lo"])
def test_matvec_fp64_fp32_diag(cuda, ref, name, tag):
    mf, _, _ = _components(name, {})
    E = ref[f"{name}/E_{tag}"]
    u = ref[f"{name}/u"]
    y = mf.matvec(cuda.as_tensor(u, device="cuda"), cuda.as_tensor(E, device="cuda")).cpu().numpy()
    assert _rel(y, ref[f"{name}/Ku_{tag}"]) <= 1e-13
    y32 = mf.matvec(cuda.as_tensor(u.astype(np.float32), device="cuda"),
                    cuda.as_tensor(E.astype(np.float32), device="cuda")).cpu().numpy()
    assert y32.dtype == np.float32
    assert _rel(y32, ref[f"{name}/Ku32_{tag}"]) <= 1e-5
    d = mf.extract_diagonal(cuda.as_tensor(E, device="cuda")).cpu().numpy()
    assert _rel(d, ref[f"{name}/diag_{tag}"]) <= 1e-14


@pytest.mark.parametrize("name", list(CASES))
def test_lambda_cache_and_adaptive_params(cuda, ref, name):
    _, gmg, _ = _components(name, {})
    for tag in ("hi", "mid", "lo"):
        gmg.setup(cuda.as_tensor(ref[f"{name}/E_{tag}"], device="cuda"))
        lam = np.array(gmg.lambda_max_per_level)
        np.testing.assert_allclose(lam, ref[f"{name}/lam_{tag}"], rtol=1e-10)
        assert abs(gmg.omega_used - ref[f"{name}/omega_{tag}"][0]) <= 1e-12 * abs(gmg.omega_used)
        ap = gmg.adaptive_params
        exp = ref[f"{name}/adapt_{tag}"]
        assert abs(ap["contrast_ratio"] - exp[0]) <= 1e-12 * exp[0]
        assert int(ap["is_high_contrast"]) == int(exp[1])
        assert ap["fine_degree_adapt"] == int(exp[2]) and ap["coarse_iters_adapt"] == int(exp[3])


@pytest.mark.parametrize("name", list(CASES))
def test_node_block_jacobi(cuda, ref, name):
    from gpu_fem.solver_v2 import NodeBlockJacobiMF

    mf, _, _ = _components(name, {})
    E = cuda.as_tensor(ref[f"{name}/E_hi"], device="cuda")
    spec = _spec(name)
    nb = NodeBlockJacobiMF(mf._edof_gpu, KE_UNIT_3D, mf._free_np, mf._n_free, mf._ndof)
    nb.update(E, scalar_diag=mf.extract_diagonal(E))
    z = nb.apply(cuda.as_tensor(ref[f"{name}/rhs"], device="cuda")).cpu().numpy()
    assert _rel(z, ref[f"{name}/nbj_hi"]) <= 1e-11


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("stack", list(STACKS))
@pytest.mark.parametrize("tag", ["hi", "mid"])
def test_gmg_apply(cuda, ref, name, stack, tag):
    _, gmg, _ = _components(name, STACKS[stack])
    gmg.setup(cuda.as_tensor(ref[f"{name}/E_{tag}"], device="cuda"))
    np.testing.assert_allclose(gmg.lambda_max_per_level, ref[f"{name}/lam_{stack}_{tag}"], rtol=1e-10)
    z = gmg.apply(cuda.as_tensor(ref[f"{name}/rhs"], device="cuda")).cpu().numpy()
    tol = 1e-4 if stack in LOW_PREC else 1e-8
    assert _rel(z, ref[f"{name}/apply_{stack}_{tag}"]) <= tol


def _envelope(h_ref, h_pert, k):
    """Per-iteration tolerance from the reference's own sensitivity: the running
    maximum of its history deviation under a 1e-14 perturbation of E, times 1000,
    floored at 1e-9."""
    k = min(k, len(h_ref), len(h_pert))
    dev = np.abs(h_ref[:k] - h_pert[:k]) / np.abs(h_ref[:k])
    return k, np.maximum(1e-9, 1000.0 * np.maximum.accumulate(dev))


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("stack", ["plain_cheb", "canonical", "plain_jacobi"])
def test_fgmres_full_solve(cuda, ref, name, stack):
    from gpu_fem.multigrid_v4 import _cupy_fgmres

    mf, gmg, F = _components(name, STACKS[stack])
    E = cuda.as_tensor(ref[f"{name}/E_hi"], device="cuda")
    gmg.setup(E)
    hist = []
    x, it, conv = _cupy_fgmres(lambda v: mf.matvec(v, E), F, gmg.apply, tol=1e-6, maxiter=300, restart=300,
                               history=hist)
    info = ref[f"{name}/fgmres_{stack}_info"]
    pinfo = ref[f"{name}/fgmres_{stack}_pert_info"]
    if int(info[0]) == int(pinfo[0]):
        assert (it, int(conv)) == (int(info[0]), int(info[1]))
    h_ref = ref[f"{name}/fgmres_{stack}_hist"]
    k, env = _envelope(h_ref, ref[f"{name}/fgmres_{stack}_pert_hist"], 20)
    dev = np.abs(np.asarray(hist[:k]) - h_ref[:k]) / h_ref[:k]
    assert np.all(dev <= env), (dev, env)
    compl = float(cuda.dot(F, x))
    self_dev = abs(info[2] - pinfo[2]) / abs(info[2])
    assert abs(compl - info[2]) / abs(info[2]) <= max(1e-7, 100 * self_dev)
    if conv:
        res = float(cuda.linalg.norm(F - mf.matvec(x, E)) / cuda.linalg.norm(F))
        assert res <= 1e-6


@pytest.mark.parametrize("name", list(CASES))
def test_pcg_and_restart_rule(cuda, ref, name):
    from gpu_fem.multigrid_v4 import _cupy_fgmres
    from gpu_fem.solver_v2 import _cupy_pcg

    mf, gmg, F = _components(name, {})
    E = cuda.as_tensor(ref[f"{name}/E_mid"], device="cuda")
    gmg.setup(E)
    hist = []
    x, it, conv = _cupy_pcg(lambda v: mf.matvec(v, E), F, gmg.apply, tol=1e-6, maxiter=200, history=hist)
    h_ref = ref[f"{name}/pcg_plain_hist"]
    k, env = _envelope(h_ref, ref[f"{name}/pcg_plain_pert_hist"], 20)
    dev = np.abs(np.asarray(hist[:k]) - h_ref[:k]) / h_ref[:k]
    assert np.all(dev <= env), (dev, env)
    hist = []
    x, it, conv = _cupy_fgmres(lambda v: mf.matvec(v, E), F, gmg.apply, tol=1e-9, maxiter=12, restart=5,
                               history=hist)
    info = ref[f"{name}/fgmres_restart5_info"]
    assert (it, int(conv)) == (int(info[0]), int(info[1]))
    assert len(hist) == len(ref[f"{name}/fgmres_restart5_hist"])
    np.testing.assert_allclose(hist, ref[f"{name}/fgmres_restart5_hist"], rtol=1e-6)
    assert _rel(x.cpu().numpy(), ref[f"{name}/fgmres_restart5_x"]) <= 1e-8
