"""Host side of the SIMP loop entry (gpu_fem.simp_gpu) without a GPU.

* ``ScheduleOnlyController`` replayed on the reference trajectory driver's own
  runs (tests/golden/trajectory_{guarded,fixed}_iters.csv, made by
  make_trajectory_driver_golden.py) gives the penal, beta, move and filter
  radius the reference loop recorded after every iteration, with the loop's
  clipping;
* ``TO3DParams`` has the reference's fields and defaults, ``StepState`` its
  fields, ``run_simp_surrogate_gpu`` its parameters in order, and
  ``PureFEMRouter`` always routes to the solve;
* the loop's grayness and checkerboard statistics (torch, any device) equal
  the reference's numpy definitions (pub_simp_solver.py:255-270) on odd and
  even meshes.
"""

import csv
import dataclasses
import inspect
import os

import numpy as np
import torch

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _rows(run):
    with open(os.path.join(GOLDEN, f"trajectory_{run}_iters.csv"), newline="") as f:
        return list(csv.DictReader(f))


def test_schedule_controller_replays_reference_runs():
    from gpu_fem.pub_baseline_controller import ScheduleOnlyController
    from gpu_fem.pub_simp_solver import StepState

    ctl = ScheduleOnlyController()
    for run in ("guarded", "fixed"):
        rows = _rows(run)
        assert len(rows) >= 20
        rmin = 1.5
        for row in rows:
            state = StepState(iteration=int(row["iteration"]), compliance=1.0, best_compliance=1.0, best_iteration=0,
                              volume_fraction=0.3, grayness=0.5, best_grayness=0.5, checkerboard=0.0, obj_slope=0.0,
                              rel_change_1=0.0, rel_change_5=0.0, stagnation_counter=0, penal=0.0, rmin=rmin,
                              move=0.0, beta=0.0, converged=False, best_is_valid=False)
            act = ctl(state, None)
            rmin = float(np.clip(act.get("rmin", rmin), 1.1, 4.0))
            assert float(np.clip(act["penal"], 1.0, 5.0)) == float(row["penal"]), row["iteration"]
            assert float(np.clip(act["beta"], 1.0, 64.0)) == float(row["beta"]), row["iteration"]
            assert float(np.clip(act["move"], 0.03, 0.4)) == float(row["move"]), row["iteration"]
            assert rmin == float(row["rmin"]), row["iteration"]


def test_schedule_controller_replays_published_runs():
    """The reference's published trajectories on cantilever_gpu_medium and
    bridge_gpu_medium, 40 iterations each -- guarded (published_guarded_trajectories_iters.csv)
    and at fixed floors 1e-12, 1e-3, 1e-2 (published_fixed_floor_trajectories_*_iters.csv)
    -- recorded the same continuation parameters after every iteration."""
    from gpu_fem.pub_baseline_controller import ScheduleOnlyController
    from gpu_fem.pub_simp_solver import StepState

    runs = {}
    for name in ("guarded_trajectories", "fixed_floor_trajectories_cantilever", "fixed_floor_trajectories_bridge"):
        with open(os.path.join(GOLDEN, f"published_{name}_iters.csv"), newline="") as f:
            for row in csv.DictReader(f):
                runs.setdefault(row["run_id"], []).append(row)
    assert len(runs) == 8 and all(len(r) == 40 for r in runs.values())
    ctl = ScheduleOnlyController()
    for run in runs.values():
        rmin = 1.5
        for row in run:
            state = StepState(iteration=int(row["iteration"]), compliance=1.0, best_compliance=1.0, best_iteration=0,
                              volume_fraction=0.3, grayness=0.5, best_grayness=0.5, checkerboard=0.0, obj_slope=0.0,
                              rel_change_1=0.0, rel_change_5=0.0, stagnation_counter=0, penal=0.0, rmin=rmin,
                              move=0.0, beta=0.0, converged=False, best_is_valid=False)
            act = ctl(state, None)
            rmin = float(np.clip(act.get("rmin", rmin), 1.1, 4.0))
            assert (float(np.clip(act["penal"], 1.0, 5.0)), float(np.clip(act["beta"], 1.0, 64.0)),
                    float(np.clip(act["move"], 0.03, 0.4)), rmin) == \
                (float(row["penal"]), float(row["beta"]), float(row["move"]), float(row["rmin"])), \
                (row["run_id"], row["iteration"])


def test_schedule_controller_phases_and_restart():
    from gpu_fem.pub_baseline_controller import ScheduleOnlyController
    from gpu_fem.pub_simp_solver import StepState

    def state(it, rmin, c=1.0, best=1.0, valid=False):
        return StepState(iteration=it, compliance=c, best_compliance=best, best_iteration=1, volume_fraction=0.3,
                         grayness=0.1, best_grayness=0.1, checkerboard=0.0, obj_slope=0.0, rel_change_1=0.0,
                         rel_change_5=0.0, stagnation_counter=0, penal=3.0, rmin=rmin, move=0.1, beta=1.0,
                         converged=False, best_is_valid=valid)

    ctl = ScheduleOnlyController()
    assert ctl(state(15, 1.5), None) == {"penal": 1.5, "beta": 1.0, "move": 0.20}
    assert ctl(state(16, 1.5), None) == {"penal": 3.5, "beta": 4.0, "move": 0.15, "rmin": 1.4}
    assert ctl(state(41, 1.3), None)["rmin"] == 1.25
    assert ctl(state(70, 1.22), None) == {"penal": 4.5, "beta": 32.0, "move": 0.05, "rmin": 1.2}
    assert "rmin" not in ctl(state(70, 1.2), None)
    assert ctl(state(30, 1.35, c=1.13, best=1.0, valid=True), None)["restart"] is True
    assert "restart" not in ctl(state(30, 1.35, c=1.13, best=1.0, valid=False), None)
    assert ctl.initial_action(None) == {"penal": 1.0, "beta": 1.0}
    assert ctl.finalize_tail(None)["tail_iters"] == 20


def test_reference_surface():
    from gpu_fem.local_agents import PureFEMRouter
    from gpu_fem.pub_simp_solver import StepState
    from gpu_fem.simp_gpu import TO3DParams, run_simp_surrogate_gpu

    p = TO3DParams()
    assert (p.nelx, p.nely, p.nelz, p.volfrac, p.penal, p.emin, p.rmin, p.move, p.max_iter) == \
        (24, 12, 12, 0.3, 3.0, 1e-9, 1.5, 0.2, 100)
    assert (p.tol, p.compliance_tol, p.compliance_window, p.min_iter, p.use_heaviside) == (0.01, 5e-4, 5, 30, True)
    assert (p.beta_init, p.beta_max, p.eta, p.min_penal_for_best, p.max_gray_for_best) == (1.0, 32.0, 0.5, 3.0, 0.25)
    assert (p.amg_ndof_threshold, p.amg_rebuild_tol) == (3000, 0.15)
    assert [f.name for f in dataclasses.fields(StepState)] == [
        "iteration", "compliance", "best_compliance", "best_iteration", "volume_fraction", "grayness",
        "best_grayness", "checkerboard", "obj_slope", "rel_change_1", "rel_change_5", "stagnation_counter",
        "penal", "rmin", "move", "beta", "converged", "best_is_valid", "compliance_history"]
    assert list(inspect.signature(run_simp_surrogate_gpu).parameters) == [
        "params", "fixed", "free", "F", "ndof", "surrogate", "router", "device", "param_controller",
        "passive_mask", "verbose", "progress_callback", "solver_class", "solver_kwargs"]
    assert PureFEMRouter()(1, 0.5, False, 1.0, rho=None, compliance=1.0) is True


def test_grayness_and_checkerboard_match_reference_definitions():
    from gpu_fem.simp_gpu import _checkerboard, _grayness

    rng = np.random.default_rng(3)
    for dims in ((5, 4, 3), (6, 6, 2), (7, 3, 5), (1, 4, 4)):
        x = rng.random(int(np.prod(dims)))
        assert abs(_grayness(torch.as_tensor(x)) - 4.0 * np.mean(x * (1.0 - x))) <= 1e-15
        R = x.reshape(dims)
        if min(dims) < 2:
            ref = 0.0
        else:
            b = (R[:-1:2, :-1:2, :-1:2] + R[1::2, :-1:2, :-1:2] + R[:-1:2, 1::2, :-1:2] + R[1::2, 1::2, :-1:2]
                 + R[:-1:2, :-1:2, 1::2] + R[1::2, :-1:2, 1::2] + R[:-1:2, 1::2, 1::2] + R[1::2, 1::2, 1::2]) / 8
            ref = float(np.std(b))
        assert abs(_checkerboard(torch.as_tensor(x), *dims) - ref) <= 1e-14, dims


def test_entry_refuses_what_it_does_not_provide():
    """2D meshes, the CPU backend and the reference's default assembled-CSR solver
    are refused by name, before the device is touched."""
    import pytest

    from gpu_fem.simp_gpu import TO3DParams, run_simp_surrogate_gpu
    from gpu_fem.solver_v4 import SolverV4

    with pytest.raises(NotImplementedError, match="3D"):
        run_simp_surrogate_gpu(TO3DParams(nelz=0), None, None, None, 0, None, None, solver_class=SolverV4)
    with pytest.raises(NotImplementedError, match="CUDA device"):
        run_simp_surrogate_gpu(TO3DParams(), None, None, None, 0, None, None, device="cpu", solver_class=SolverV4)
    with pytest.raises(NotImplementedError, match="GPUFEMSolver"):
        run_simp_surrogate_gpu(TO3DParams(), None, None, None, 0, None, None)
