"""The FEM-only router of the SIMP loop (gpu_fem/local_agents.py:62-66).

The SIMP loop asks its router, when a sensitivity surrogate is attached,
whether an iteration takes a finite-element solve (True) or the surrogate's
prediction.  ``PureFEMRouter`` always answers True; the trajectory driver
(experiments/phase5/run_simp_floor_trajectory.py:337) passes it with no
surrogate, so every iteration is a guarded solve.  The module's surrogate
routers and agents steer studies outside the guarded solve and are not
provided.
"""

from __future__ import annotations


class PureFEMRouter:
    name = "pure_fem"

    def __call__(self, iteration: int, uncertainty: float, surrogate_ready: bool, beta: float = 1.0,
                 **kwargs) -> bool:
        return True
