"""In-loop guarded floor policy on the GPU vs the reference's own run.

tests/golden/floor_trajectory_cantilever_3d.npz (make_floor_trajectory_golden.py)
holds the reference's GuardedAdaptiveFloorSolverV4 (run_simp_floor_trajectory.py)
on five density fields of the cantilever_3d preset, called in sequence through
one solver object as a SIMP loop does.  The CUDA path must take the same policy
decisions (trigger, selected floor, attempted floors, fallback flag), reach
the guard (true relative residual <= cg_tol) on every call, and give the same
compliance within 1e-6 relative and the same sensitivity field within 1e-4
relative (two solves stopped at a 1e-6 residual, so u agrees to about that).
Iteration counts must lie within 2 of the reference's (round-off in the
canonical FGMRES path moves the last iteration).
"""

import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "floor_trajectory_cantilever_3d.npz")


def test_in_loop_policy_matches_reference(cuda):
    from gpu_fem.bc_generator import generate_bc
    from gpu_fem.floor_trajectory import GuardedAdaptiveFloorSolverV4
    from gpu_fem.presets import get_preset
    from gpu_fem.pub_simp_solver import KE_UNIT_3D, _edof_table_3d

    g = np.load(GOLDEN)
    kw = json.loads(str(g["kwargs"]))
    kw["guarded_ladder"] = tuple(kw["guarded_ladder"])
    events = json.loads(str(g["events"]))
    spec = get_preset("cantilever_3d")
    bc = generate_bc(spec)
    nx, ny, nz = spec.nelx, spec.nely, spec.nelz
    solver = GuardedAdaptiveFloorSolverV4(
        edof=_edof_table_3d(nx, ny, nz), row_idx=np.empty(0, np.int32), col_idx=np.empty(0, np.int32),
        KE_UNIT=KE_UNIT_3D, free=bc.free_dofs, F=bc.F, ndof=bc.ndof, E0=1.0, Emin=1e-12, backend="cupy",
        amg_ndof_threshold=3000, amg_rebuild_tol=0.15, grid_dims=(nx, ny, nz), **kw)
    penal = float(g["penal"])
    for k, rho in enumerate(g["rho"]):
        c, dc = solver.solve(rho, penal)
        ev = solver.policy_events[-1]
        ref = events[k]
        for key in ("trigger", "selected_rho_min", "attempted_rho_mins", "fallback_used"):
            assert ev[key] == ref[key], (k, key, ev[key], ref[key])
        assert solver.last_true_rel_residual <= kw["cg_tol"]
        assert abs(c - g["compliance"][k]) <= 1e-6 * abs(g["compliance"][k]), (k, c, g["compliance"][k])
        assert np.linalg.norm(dc - g["dc"][k]) <= 1e-4 * np.linalg.norm(g["dc"][k]), k
        assert abs(solver.last_cg_iters - int(g["iters"][k])) <= 2, (k, solver.last_cg_iters, g["iters"][k])
