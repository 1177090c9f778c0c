"""Host logic of the in-loop guarded floor policy (GuardedAdaptiveFloorSolverV4).

The decision sequence of run_simp_floor_trajectory.py:129-224 is exercised on
CPU with the underlying SolverV4.solve replaced by a scripted stand-in that
returns chosen iteration counts / true residuals per floor, so every branch is
covered: probe converged, keep -> full solve accepted, keep -> guard failed ->
ladder, raise -> ladder, ladder exhausted.
"""

import numpy as np
import pytest

from gpu_fem import floor_trajectory as ft


def _solver(script, **kw):
    """A GuardedAdaptiveFloorSolverV4 without a GPU: ``script[(phase_index)]`` gives
    (true_rel_residual, history) for each successive SolverV4.solve call."""
    s = object.__new__(ft.GuardedAdaptiveFloorSolverV4)
    s.Emin, s.cg_maxiter, s.cg_tol = 1e-9, 100, 1e-6
    s.guarded_base_rho_min = kw.get("base", 1e-12)
    s.guarded_ladder = kw.get("ladder", (1e-3, 1e-2))
    s.guarded_probe_iters, s.guarded_probe_r50 = 30, 15
    s.guarded_high_residual_threshold, s.guarded_plateau_residual_threshold = 1e-2, 1e-4
    s.guarded_plateau_ratio_threshold = 0.6
    s.policy_events = []
    calls = []

    def fake_solve(self, rho, penal):
        true, hist = script[len(calls)]
        calls.append((self.Emin, self.cg_maxiter))
        self.last_cg_iters = len(hist) - 1
        self.last_cg_history = list(hist)
        self.last_true_rel_residual = true
        return float(len(calls)), np.full(3, float(len(calls)))

    return s, calls, fake_solve


def _hist(r50, r100=None, n=31):
    h = np.geomspace(1.0, r50, 16).tolist()
    h += np.geomspace(r50, r100 if r100 is not None else r50 / 10, n - 16).tolist()
    return h


@pytest.mark.parametrize("case", ["probe_converged", "keep_full", "keep_guard_failed", "raise_ladder", "exhausted"])
def test_policy_branches(monkeypatch, case):
    if case == "probe_converged":
        script = [(5e-7, _hist(1e-3))]
    elif case == "keep_full":
        script = [(1e-4, _hist(1e-3)), (8e-7, _hist(1e-3, n=60))]
    elif case == "keep_guard_failed":
        script = [(1e-4, _hist(1e-3)), (1e-5, _hist(1e-3, n=100)), (9e-7, _hist(1e-3, n=40))]
    elif case == "raise_ladder":
        script = [(1e-2, _hist(5e-2)), (2e-6, _hist(1e-3, n=100)), (7e-7, _hist(1e-3, n=40))]
    else:
        script = [(1e-2, _hist(5e-2)), (2e-6, _hist(1e-3, n=100)), (3e-6, _hist(1e-3, n=100))]
    s, calls, fake = _solver(script)
    monkeypatch.setattr(ft.SolverV4, "solve", fake)
    if case == "exhausted":
        with pytest.raises(RuntimeError, match="exhausted the ladder"):
            s.solve(np.zeros(3), 3.0)
        assert s.policy_events[-1]["fallback_used"] == 1
        assert s.policy_events[-1]["attempted_rho_mins"] == "1e-12;1e-03;1e-02"
        return
    c, dc = s.solve(np.zeros(3), 3.0)
    ev = s.policy_events[-1]
    # the returned answer is the last solve run, which is the accepted one
    assert c == float(len(calls)) and dc[0] == c
    assert s.Emin == 1e-9 and s.cg_maxiter == 100  # restored after each attempt
    assert calls[0] == (1e-12, 30)  # probe: base floor, probe cap
    if case == "probe_converged":
        assert ev["trigger"] == "probe_converged_keep" and ev["selected_rho_min"] == 1e-12
        assert ev["attempted_rho_mins"] == "1e-12" and len(calls) == 1
    elif case == "keep_full":
        assert ev["trigger"] == "keep" and ev["selected_rho_min"] == 1e-12
        assert calls[1] == (1e-12, 100) and ev["attempt_count"] == 2
    elif case == "keep_guard_failed":
        assert ev["trigger"] == "keep_guard_failed" and ev["fallback_used"] == 1
        assert ev["selected_rho_min"] == 1e-3 and ev["attempted_rho_mins"] == "1e-12;1e-12;1e-03"
    else:
        assert ev["trigger"] == "high_r50" and ev["selected_rho_min"] == 1e-2
        assert ev["attempted_rho_mins"] == "1e-12;1e-03;1e-02"
    assert ev["accepted_true_rel_residual"] <= 1e-6 and s.last_selected_rho_min == ev["selected_rho_min"]


def test_history_and_classify():
    t = ft.TrialSolve("probe", 1e-12, 30, 1.0, np.zeros(1), 2, 1e-3, 0.0, [])
    assert t.residual_at(5) == float("inf")
    t.history = [1.0, 0.5, 0.25]
    assert t.residual_at(50) == 0.25 and t.residual_at(1) == 0.5 and t.residual_at(-3) == 1.0
    thr = dict(high_residual_threshold=1e-2, plateau_residual_threshold=1e-4, plateau_ratio_threshold=0.6)
    assert ft._classify(2e-2, 1e-3, **thr) == (True, "high_r50")
    assert ft._classify(1e-3, 7e-4, **thr) == (True, "plateau")
    assert ft._classify(1e-3, 1e-5, **thr) == (False, "keep")


def test_solver_v4_refuses_other_paths():
    from gpu_fem.solver_v4 import SolverV4

    base = dict(edof=None, KE_UNIT=np.eye(24), free=np.arange(3), F=np.zeros(3), ndof=3)
    with pytest.raises(NotImplementedError):
        SolverV4(**base)
    with pytest.raises(ValueError, match="enable_matrix_free=True"):
        SolverV4(**base, enable_matfree_gmg=True, grid_dims=(1, 1, 1))
    with pytest.raises(ValueError, match="grid_dims"):
        SolverV4(**base, enable_matfree_gmg=True, enable_matrix_free=True)
    with pytest.raises(ValueError, match="gmg_outer_solver"):
        SolverV4(**base, enable_matfree_gmg=True, enable_matrix_free=True, grid_dims=(1, 1, 1),
                 gmg_outer_solver="bicg")
