"""The guarded floor policy inside the SIMP loop (GuardedAdaptiveFloorSolverV4).

Follows experiments/phase5/run_simp_floor_trajectory.py: ``_history_at``
(:42-46), ``_classify_probe`` (:49-63) and ``GuardedAdaptiveFloorSolverV4``
(:66-224), a SolverV4 whose ``solve`` runs, per SIMP iteration:

1. a probe at the base floor capped at ``guarded_probe_iters`` outer
   iterations; if its recomputed FP64 residual already meets ``cg_tol`` it is
   accepted ("probe_converged_keep");
2. otherwise the r50 / r100 rule on the probe history; "keep" runs the full
   solve at the base floor and accepts it if the guard passes (else the trigger
   gets "_guard_failed" and the ladder follows);
3. the ladder floors in order, accepting the first guarded solve;
4. ``RuntimeError`` when the ladder is exhausted.

Every accepted answer passes ||F - K u|| / ||F|| <= cg_tol recomputed in FP64.
Each SIMP iteration appends one row to ``policy_events``.
"""

from __future__ import annotations

import time

from .solver_v4 import SolverV4


def _history_at(history, iteration: int) -> float:
    if not history:
        return float("inf")
    index = min(max(iteration, 0), len(history) - 1)
    return float(history[index])


def _classify_probe(r50: float, r100: float, *, high_residual_threshold: float, plateau_residual_threshold: float,
                    plateau_ratio_threshold: float) -> tuple[bool, str]:
    if r50 >= high_residual_threshold:
        return True, "high_r50"
    ratio = r100 / max(r50, 1e-300)
    if r100 >= plateau_residual_threshold and ratio >= plateau_ratio_threshold:
        return True, "plateau"
    return False, "keep"


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

    def _solve_with_floor(self, rho_phys, penal: float, *, rho_min: float, maxiter: int, phase: str):
        old_emin, old_maxiter = self.Emin, self.cg_maxiter
        self.Emin, self.cg_maxiter = float(rho_min), int(maxiter)
        try:
            start = time.perf_counter()
            compliance, dc_phys = SolverV4.solve(self, rho_phys, penal)
            elapsed = time.perf_counter() - start
            metrics = {"phase": phase, "rho_min": float(rho_min), "maxiter": int(maxiter),
                       "compliance": float(compliance), "iters": int(self.last_cg_iters),
                       "true_rel_residual": float(self.last_true_rel_residual),
                       "history": list(self.last_cg_history), "wall_time_s": elapsed}
            return compliance, dc_phys, metrics
        finally:
            self.Emin, self.cg_maxiter = old_emin, old_maxiter

    def solve(self, rho_phys, penal: float):
        attempted: list = []
        compliance, dc_phys, probe = self._solve_with_floor(rho_phys, penal, rho_min=self.guarded_base_rho_min,
                                                            maxiter=self.guarded_probe_iters, phase="probe")
        attempted.append(probe)
        r50 = _history_at(probe["history"], self.guarded_probe_r50)
        r100 = _history_at(probe["history"], self.guarded_probe_iters)
        self.last_policy_probe_r50 = r50
        self.last_policy_probe_r100 = r100
        self.last_policy_probe_true_rel_residual = float(probe["true_rel_residual"])
        if probe["true_rel_residual"] <= self.cg_tol:
            selected, trigger, fallback_used = probe, "probe_converged_keep", 0
        else:
            predicted_raise, trigger = _classify_probe(
                r50, r100, high_residual_threshold=self.guarded_high_residual_threshold,
                plateau_residual_threshold=self.guarded_plateau_residual_threshold,
                plateau_ratio_threshold=self.guarded_plateau_ratio_threshold)
            selected, fallback_used = None, 0
            if not predicted_raise:
                compliance, dc_phys, full = self._solve_with_floor(rho_phys, penal, rho_min=self.guarded_base_rho_min,
                                                                   maxiter=self.cg_maxiter, phase="guarded_keep_full")
                attempted.append(full)
                if full["true_rel_residual"] <= self.cg_tol:
                    selected = full
                else:
                    fallback_used = 1
                    trigger = f"{trigger}_guard_failed"
            if selected is None:
                for floor in self.guarded_ladder:
                    compliance, dc_phys, ladder = self._solve_with_floor(rho_phys, penal, rho_min=floor,
                                                                         maxiter=self.cg_maxiter, phase="ladder")
                    attempted.append(ladder)
                    if ladder["true_rel_residual"] <= self.cg_tol:
                        selected = ladder
                        break
            if selected is None:
                self.policy_events.append({
                    "trigger": trigger, "selected_rho_min": float("nan"), "fallback_used": 1,
                    "attempted_rho_mins": ";".join(f"{row['rho_min']:.0e}" for row in attempted),
                    "probe_r50": r50, "probe_r100": r100, "accepted_true_rel_residual": float("nan")})
                raise RuntimeError("guarded adaptive floor policy exhausted the ladder")
        self.last_selected_rho_min = float(selected["rho_min"])
        self.last_true_rel_residual = float(selected["true_rel_residual"])
        self.last_cg_iters = int(selected["iters"])
        self.last_cg_history = list(selected["history"])
        self.last_policy_trigger = trigger
        self.last_policy_fallback_used = int(fallback_used)
        self.last_policy_attempted_rho_mins = ";".join(f"{row['rho_min']:.0e}" for row in attempted)
        self.policy_events.append({
            "trigger": trigger, "selected_rho_min": self.last_selected_rho_min,
            "fallback_used": self.last_policy_fallback_used,
            "attempted_rho_mins": self.last_policy_attempted_rho_mins, "probe_r50": r50, "probe_r100": r100,
            "probe_true_rel_residual": self.last_policy_probe_true_rel_residual,
            "accepted_true_rel_residual": self.last_true_rel_residual, "accepted_iters": self.last_cg_iters,
            "attempt_count": len(attempted), "policy_time_s": sum(float(row["wall_time_s"]) for row in attempted)})
        return compliance, dc_phys
