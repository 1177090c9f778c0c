"""Golden data for the in-loop guarded floor policy (GuardedAdaptiveFloorSolverV4).

Run from the repository root where the reference source tree is readable
(its root given by SIMPFEM_REFERENCE_ROOT):

    python tests/golden/make_floor_trajectory_golden.py

Loads ``GuardedAdaptiveFloorSolverV4`` from the reference's
experiments/phase5/run_simp_floor_trajectory.py (a copy, through the numpy
``cupy`` stand-in of ``_refshim.py``) with the solver keywords its driver uses
(``_solver_kwargs``, :244-275) on the cantilever_3d preset, and calls
``solve(rho_phys, penal)`` on a short sequence of density fields through one
solver object, so warm starts and the lambda cache carry over as they do inside
a SIMP loop.  Writes floor_trajectory_cantilever_3d.npz: the fields, and per
call the compliance, the sensitivity dc_phys, the accepted iteration count and
true residual, and the policy event (trigger, selected floor, attempted floors).
"""

from __future__ import annotations

import importlib.util
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import _refshim  # noqa: E402

PENAL = 3.0
KW = dict(enable_warm_start=True, enable_matrix_free=True, enable_fused_cuda=False, enable_matfree_gmg=True,
          matfree_gmg_levels=3, gmg_fine_smoother="fp64", gmg_fine_degree=2, gmg_outer_solver="fgmres",
          gmg_restart=300, gmg_smoother_type="chebyshev", gmg_cycle_type="v", cg_tol=1e-6, cg_maxiter=150,
          enable_profiling=False, guarded_base_rho_min=1e-12, guarded_ladder=(1e-3, 1e-2), guarded_probe_iters=30,
          guarded_probe_r50=15, guarded_high_residual_threshold=1e-2, guarded_plateau_residual_threshold=1e-4,
          guarded_plateau_ratio_threshold=0.6)


def fields(n: int) -> list:
    """Grey and Bernoulli solid/void fields that take the policy through its branches."""
    out = [np.clip(0.3 + 0.02 * np.random.default_rng(0).standard_normal(n), 1e-3, 1.0)]
    for seed, void in ((1, 0.35), (2, 0.5), (3, 0.45)):
        out.append((np.random.default_rng(seed).random(n) >= void).astype(np.float64))
    out.append(np.clip(0.12 + 0.1 * np.random.default_rng(4).standard_normal(n), 1e-3, 1.0))
    return out


def main() -> None:
    _refshim.install()
    path = _refshim._copied_script(os.path.join("experiments", "phase5", "run_simp_floor_trajectory.py"))
    spec = importlib.util.spec_from_file_location("floor_trajectory_driver", path)
    drv = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(drv)
    presets = _refshim.load("presets")
    bcg = _refshim.load("bc_generator")
    pss = _refshim.load("pub_simp_solver")
    spec_ = presets.get_preset("cantilever_3d")
    bc = bcg.generate_bc(spec_)
    nx, ny, nz = spec_.nelx, spec_.nely, spec_.nelz
    solver = drv.GuardedAdaptiveFloorSolverV4(
        edof=pss._edof_table_3d(nx, ny, nz), row_idx=np.empty(0, np.int32), col_idx=np.empty(0, np.int32),
        KE_UNIT=pss.KE_UNIT_3D, free=bc.free_dofs, F=bc.F, ndof=bc.ndof, E0=1.0, Emin=1e-12, backend="cupy",
        amg_ndof_threshold=3000, amg_rebuild_tol=0.15, grid_dims=(nx, ny, nz), **KW)
    rho = fields(nx * ny * nz)
    out = {"rho": np.stack(rho), "penal": np.array(PENAL), "kwargs": np.array(json.dumps(KW))}
    comp, dcs, iters, true, events = [], [], [], [], []
    for r in rho:
        c, dc = solver.solve(r, PENAL)
        comp.append(c)
        dcs.append(dc)
        iters.append(solver.last_cg_iters)
        true.append(solver.last_true_rel_residual)
        ev = solver.policy_events[-1]
        events.append({k: ev[k] for k in ("trigger", "selected_rho_min", "attempted_rho_mins", "fallback_used")})
        print(c, solver.last_cg_iters, solver.last_true_rel_residual, events[-1], flush=True)
    out.update(compliance=np.array(comp), dc=np.stack(dcs), iters=np.array(iters), true_rel_residual=np.array(true),
               events=np.array(json.dumps(events)))
    np.savez_compressed(os.path.join(HERE, "floor_trajectory_cantilever_3d.npz"), **out)


if __name__ == "__main__":
    main()
