"""``_build_components`` of the reference's paper-4 runner
(experiments/paper4/run_experiments_e1_e10.py:128-179), the factory every
phase-5 driver calls, returning the same 8-tuple over torch CUDA tensors."""

from __future__ import annotations

import numpy as np

from . import _lib
from .bc_generator import generate_bc
from .multigrid_v4 import GalerkinMatFreeGMG
from .presets import get_preset
from .pub_simp_solver import KE_UNIT_3D, _edof_table_3d
from .solver_v2 import MatrixFreeKff


def _build_components(preset_name, *, n_levels: int = 4, fine_smoother: str = "fp32",
                      smoother_type: str = "chebyshev", level_precisions=None, cycle_type: str = "v",
                      coarse_correction_policy: str = "none", coarse_correction_acceptance_ratio: float = 1.0,
                      coarse_correction_max_scale: float = 1.0, root_enrichment_mode: str = "none",
                      root_enrichment_weight_floor: float = 1e-6, root_enrichment_weight_power: float = 0.5,
                      root_local_correction_mode: str = "none", root_local_correction_max_scale: float = 1.0,
                      root_local_correction_inner_steps: int = 10, root_local_correction_inner_restart=None,
                      inner_krylov_steps: int = 0, inner_krylov_restart=None, fused_op=None,
                      cycle_precision: str = "fp64"):
    """``preset_name`` may also be a ProblemSpec."""
    torch = _lib.require_cuda()
    spec = get_preset(preset_name) if isinstance(preset_name, str) else preset_name
    bc = generate_bc(spec)
    free = bc.free_dofs.astype(np.int32)
    edof = _edof_table_3d(spec.nelx, spec.nely, spec.nelz)
    edof_gpu = torch.as_tensor(edof, device="cuda")
    free_gpu = torch.as_tensor(free.astype(np.int64), device="cuda")
    F_free_gpu = torch.as_tensor(bc.F[free].astype(np.float64), device="cuda")
    mf_op = MatrixFreeKff(edof_gpu=edof_gpu, KE_unit_gpu=torch.as_tensor(KE_UNIT_3D, device="cuda"),
                          free_gpu=free_gpu, n_free=len(free), ndof=bc.ndof,
                          grid_dims=(spec.nelx, spec.nely, spec.nelz))
    gmg = GalerkinMatFreeGMG(
        mf_op=mf_op, free=free, free_gpu=free_gpu, nelx=spec.nelx, nely=spec.nely, nelz=spec.nelz,
        KE_UNIT=KE_UNIT_3D, n_levels=n_levels, fine_smoother=fine_smoother, smoother_type=smoother_type,
        level_precisions=level_precisions, cycle_type=cycle_type,
        coarse_correction_policy=coarse_correction_policy,
        coarse_correction_acceptance_ratio=coarse_correction_acceptance_ratio,
        coarse_correction_max_scale=coarse_correction_max_scale,
        root_enrichment_mode=root_enrichment_mode, root_enrichment_weight_floor=root_enrichment_weight_floor,
        root_enrichment_weight_power=root_enrichment_weight_power,
        root_local_correction_mode=root_local_correction_mode,
        root_local_correction_max_scale=root_local_correction_max_scale,
        root_local_correction_inner_steps=root_local_correction_inner_steps,
        root_local_correction_inner_restart=root_local_correction_inner_restart,
        inner_krylov_steps=inner_krylov_steps, inner_krylov_restart=inner_krylov_restart,
        fused_op=fused_op, cycle_precision=cycle_precision,
    )
    return spec, bc, free, free_gpu, edof_gpu, F_free_gpu, mf_op, gmg


# The two stacks named by the phase-5 drivers (run_gmg_floor_detector_prospective.py:135-152).
CANONICAL_STACK = dict(
    fine_smoother="fp64", smoother_type="chebyshev", cycle_type="v",
    coarse_correction_policy="residual_line_search",
    root_local_correction_mode="node_block_inner_fgmres",
    root_local_correction_inner_steps=20, root_local_correction_inner_restart=20,
    inner_krylov_steps=10, inner_krylov_restart=10,
)
PLAIN_JACOBI_STACK = dict(
    fine_smoother="fp64", smoother_type="jacobi", cycle_type="v",
    coarse_correction_policy="none", root_local_correction_mode="none", inner_krylov_steps=0,
)


# ---------------------------------------------------------------------------
# Moduli fields and Krylov entry points of the same runner (run_experiments_e1_e10.py:182-219),
# used by the phase-5 pathology driver.
def _E_e(spec, rho_scalar: float = 0.5, penal: float = 3.0, E0=1.0, Emin=1e-9):
    """Uniform-density SIMP moduli Emin + (E0 - Emin) rho^penal on the device."""
    torch = _lib.require_cuda()
    n = spec.nelx * spec.nely * spec.nelz
    rho = torch.full((n,), float(rho_scalar), dtype=torch.float64, device="cuda")
    return Emin + (E0 - Emin) * rho ** penal


def _E_e_heterogeneous(spec, volfrac: float = 0.5, penal: float = 3.0, rho_min: float = 0.01,
                       rho_max: float = 1.0, seed: int = 0, E0: float = 1.0, Emin: float = 1e-9):
    """Binary-contrast field: each element rho_max with probability volfrac
    (numpy default_rng(seed)), rho_min otherwise; moduli Emin + (E0 - Emin) rho^penal."""
    torch = _lib.require_cuda()
    n = spec.nelx * spec.nely * spec.nelz
    rng = np.random.default_rng(seed)
    rho = torch.as_tensor(np.where(rng.random(n) < volfrac, rho_max, rho_min).astype(np.float64), device="cuda")
    return Emin + (E0 - Emin) * rho ** penal


def _pcg(A_op, b, M_op, tol=1e-6, maxiter=200, history=None):
    from .solver_v2 import _cupy_pcg

    return _cupy_pcg(A_op, b, M_op, tol=tol, maxiter=maxiter, history=history)


def _fgmres(A_op, b, M_op, tol=1e-6, maxiter=200, restart=32, history=None):
    from .multigrid_v4 import _cupy_fgmres

    return _cupy_fgmres(A_op, b, M_op, tol=tol, maxiter=maxiter, restart=restart, history=history)
