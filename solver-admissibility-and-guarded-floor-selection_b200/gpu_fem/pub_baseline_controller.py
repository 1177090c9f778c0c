"""The schedule-only SIMP parameter controller (gpu_fem/pub_baseline_controller.py:21-59).

The trajectory driver (experiments/phase5/run_simp_floor_trajectory.py:337-339)
hands ``ScheduleOnlyController()`` to the SIMP loop, which calls it after every
iteration with a ``StepState`` and applies the returned action.  The schedule
is a fixed table of continuation phases keyed by the iteration number:

==============  =====  =====  =====  ==========================
iterations      penal  beta   move   filter radius
==============  =====  =====  =====  ==========================
1 - 15          1.5    1      0.20   unchanged
16 - 40         3.5    4      0.15   down 0.10 a step to 1.35
41 - 65         4.5    16     0.08   down 0.10 a step to 1.25
66 -            4.5    32     0.05   down 0.05 a step to 1.20
==============  =====  =====  =====  ==========================

(the new radius rounded to two decimals), and a restart from the best design
when one is valid and the compliance has risen above 1.12 times its own.  The
other controllers of that module steer studies outside the guarded solve and
are not provided.
"""

from __future__ import annotations

# (last iteration of the phase or None, penal, beta, move, radius floor or None, radius step)
_PHASES = (
    (15, 1.5, 1.0, 0.20, None, 0.0),
    (40, 3.5, 4.0, 0.15, 1.35, 0.10),
    (65, 4.5, 16.0, 0.08, 1.25, 0.10),
    (None, 4.5, 32.0, 0.05, 1.20, 0.05),
)
_RESTART_RATIO = 1.12


class ScheduleOnlyController:
    name = "schedule_only"

    def initial_action(self, params):
        """The continuation's starting point: penal 1, no projection sharpening."""
        return {"penal": 1.0, "beta": 1.0}

    def finalize_tail(self, params):
        """The settings of a tail run from the best design after the main loop."""
        return {"enabled": True, "tail_iters": 20, "restart_from_best": True,
                "penal": 4.5, "rmin": 1.20, "move": 0.05, "beta": 32.0}

    def __call__(self, state, rho):
        phase = next(p for p in _PHASES if p[0] is None or state.iteration <= p[0])
        _, penal, beta, move, radius_floor, radius_step = phase
        action = {"penal": penal, "beta": beta, "move": move}
        if radius_floor is not None and state.rmin > radius_floor:
            action["rmin"] = max(radius_floor, round(state.rmin - radius_step, 2))
        if state.best_is_valid and state.compliance > _RESTART_RATIO * state.best_compliance:
            action["restart"] = True
        return action
