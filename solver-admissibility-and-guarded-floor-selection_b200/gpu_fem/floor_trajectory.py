"""The guarded floor policy inside the SIMP loop (GuardedAdaptiveFloorSolverV4).

Behaviour of experiments/phase5/run_simp_floor_trajectory.py:42-224 (the class
the trajectory driver builds around SolverV4), built here on the decision core
of ``gpu_fem.policy``: each ``solve`` call is a sequence of trial solves at
fixed floors, and the first one whose recomputed FP64 residual
||F - K u|| / ||F|| meets ``cg_tol`` is the answer.

* The probe runs at the base floor with the probe's iteration cap.  If it
  already passes the guard it is the answer ("probe_converged_keep").
* Otherwise the r50 / r100 rule (``policy._classify``) reads the probe history
  and gives the plan: "keep" plans a full solve at the base floor followed by
  the ladder (a failed full solve appends "_guard_failed" to the trigger and
  sets the fallback flag); a raise plans the ladder alone.
* A plan that ends without an accepted trial raises ``RuntimeError``.

Each call appends one event row (the reference's keys) to ``policy_events``.
"""

from __future__ import annotations

import contextlib
import time
from dataclasses import dataclass, field

import numpy as np

from .policy import _classify
from .solver_v4 import SolverV4


@dataclass
class TrialSolve:
    """One SolverV4 solve at a fixed floor and outer-iteration cap."""

    phase: str
    rho_min: float
    maxiter: int
    compliance: float
    dc_phys: np.ndarray
    iters: int
    true_rel_residual: float
    wall_time_s: float
    history: list = field(default_factory=list)

    def residual_at(self, iteration: int) -> float:
        """Relative-residual history entry after ``iteration`` iterations (the last
        entry when the solve stopped earlier; +inf without a history)."""
        if not self.history:
            return float("inf")
        return float(self.history[int(np.clip(iteration, 0, len(self.history) - 1))])

    def passes(self, tol: float) -> bool:
        return self.true_rel_residual <= tol


class GuardedAdaptiveFloorSolverV4(SolverV4):
    def __init__(self, *args, guarded_base_rho_min: float = 1e-12, guarded_ladder=(1e-3, 1e-2),
                 guarded_probe_iters: int = 100, guarded_probe_r50: int = 50,
                 guarded_high_residual_threshold: float = 1e-2, guarded_plateau_residual_threshold: float = 1e-4,
                 guarded_plateau_ratio_threshold: float = 0.6, **kwargs):
        super().__init__(*args, **kwargs)
        self.guarded_base_rho_min = float(guarded_base_rho_min)
        self.guarded_ladder = tuple(float(v) for v in guarded_ladder)
        self.guarded_probe_iters = int(guarded_probe_iters)
        self.guarded_probe_r50 = int(guarded_probe_r50)
        self.guarded_high_residual_threshold = float(guarded_high_residual_threshold)
        self.guarded_plateau_residual_threshold = float(guarded_plateau_residual_threshold)
        self.guarded_plateau_ratio_threshold = float(guarded_plateau_ratio_threshold)
        self.policy_events: list = []
        self.last_selected_rho_min = self.guarded_base_rho_min
        self.last_policy_trigger = ""
        self.last_policy_fallback_used = 0
        self.last_policy_attempted_rho_mins = ""
        self.last_policy_probe_r50 = float("nan")
        self.last_policy_probe_r100 = float("nan")
        self.last_policy_probe_true_rel_residual = float("nan")

    # ------------------------------------------------------------ trial solves
    @contextlib.contextmanager
    def _at_floor(self, rho_min: float, maxiter: int):
        saved = (self.Emin, self.cg_maxiter)
        self.Emin, self.cg_maxiter = float(rho_min), int(maxiter)
        try:
            yield
        finally:
            self.Emin, self.cg_maxiter = saved

    def _trial(self, rho_phys, penal: float, phase: str, rho_min: float, maxiter: int) -> TrialSolve:
        with self._at_floor(rho_min, maxiter):
            t0 = time.perf_counter()
            compliance, dc_phys = SolverV4.solve(self, rho_phys, penal)
            wall = time.perf_counter() - t0
            return TrialSolve(phase, float(rho_min), int(maxiter), float(compliance), dc_phys,
                              int(self.last_cg_iters), float(self.last_true_rel_residual), wall,
                              list(self.last_cg_history))

    def _plan(self, raise_floor: bool) -> list:
        """(phase, floor) of the solves after a probe that missed the guard."""
        keep = [] if raise_floor else [("guarded_keep_full", self.guarded_base_rho_min)]
        return keep + [("ladder", floor) for floor in self.guarded_ladder]

    # ------------------------------------------------------------------ policy
    def solve(self, rho_phys, penal: float):
        probe = self._trial(rho_phys, penal, "probe", self.guarded_base_rho_min, self.guarded_probe_iters)
        r50 = probe.residual_at(self.guarded_probe_r50)
        r100 = probe.residual_at(self.guarded_probe_iters)
        self.last_policy_probe_r50, self.last_policy_probe_r100 = r50, r100
        self.last_policy_probe_true_rel_residual = probe.true_rel_residual
        trials = [probe]
        fallback = 0
        if probe.passes(self.cg_tol):
            trigger, chosen = "probe_converged_keep", probe
        else:
            raise_floor, trigger = _classify(
                r50, r100, high_residual_threshold=self.guarded_high_residual_threshold,
                plateau_residual_threshold=self.guarded_plateau_residual_threshold,
                plateau_ratio_threshold=self.guarded_plateau_ratio_threshold)
            chosen = None
            for phase, floor in self._plan(raise_floor):
                trial = self._trial(rho_phys, penal, phase, floor, self.cg_maxiter)
                trials.append(trial)
                if trial.passes(self.cg_tol):
                    chosen = trial
                    break
                if phase == "guarded_keep_full":
                    fallback, trigger = 1, trigger + "_guard_failed"
        attempted = ";".join(f"{t.rho_min:.0e}" for t in trials)
        event = {"trigger": trigger, "probe_r50": r50, "probe_r100": r100}
        if chosen is None:
            event.update(selected_rho_min=float("nan"), fallback_used=1, attempted_rho_mins=attempted,
                         accepted_true_rel_residual=float("nan"))
            self.policy_events.append(event)
            raise RuntimeError("guarded adaptive floor policy exhausted the ladder")
        self.last_selected_rho_min = chosen.rho_min
        self.last_true_rel_residual = chosen.true_rel_residual
        self.last_cg_iters = chosen.iters
        self.last_cg_history = list(chosen.history)
        self.last_policy_trigger = trigger
        self.last_policy_fallback_used = fallback
        self.last_policy_attempted_rho_mins = attempted
        event.update(selected_rho_min=chosen.rho_min, fallback_used=fallback, attempted_rho_mins=attempted,
                     probe_true_rel_residual=probe.true_rel_residual,
                     accepted_true_rel_residual=chosen.true_rel_residual, accepted_iters=chosen.iters,
                     attempt_count=len(trials), policy_time_s=sum(t.wall_time_s for t in trials))
        self.policy_events.append(event)
        return chosen.compliance, chosen.dc_phys
