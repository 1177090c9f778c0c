"""Problem description dataclasses (the reference's ``gpu_fem/problem_spec.py:32-313``).

Only the fields the solve path reads are modelled: domain size, mesh counts,
material, volume fraction, supports and loads.  Coordinates follow the
reference: node (i, j, k) sits at (i Lx/nelx, j Ly/nely, k Lz/nelz).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Optional

_CONSTRAINT_DOFS_3D = {
    "fixed": [0, 1, 2],
    "pin_x": [0],
    "pin_y": [1],
    "pin_z": [2],
    "roller_x": [1, 2],
    "roller_y": [0, 2],
    "roller_z": [0, 1],
}
_CONSTRAINT_DOFS_2D = {
    "fixed": [0, 1], "pin_x": [0], "pin_y": [1], "pin_z": [],
    "roller_x": [1], "roller_y": [0], "roller_z": [0, 1],
}


def _dofs_for(constraint: str, ndim: int) -> list[int]:
    table = _CONSTRAINT_DOFS_3D if ndim == 3 else _CONSTRAINT_DOFS_2D
    return list(table.get(constraint, range(ndim)))


@dataclass
class PointSupport:
    x: float
    y: float
    z: float = 0.0
    constraint: str = "fixed"

    def dof_mask(self, ndim: int) -> list[int]:
        return _dofs_for(self.constraint, ndim)


@dataclass
class EdgeSupport:
    edge: str
    constraint: str = "fixed"

    def dof_mask(self, ndim: int) -> list[int]:
        return _dofs_for(self.constraint, ndim)


@dataclass
class PointLoad:
    x: float
    y: float
    z: float = 0.0
    fx: float = 0.0
    fy: float = 0.0
    fz: float = 0.0

    @property
    def magnitude(self) -> float:
        return math.sqrt(self.fx**2 + self.fy**2 + self.fz**2)


@dataclass
class DistributedLoad:
    edge: str
    magnitude: float = -1.0


@dataclass
class ProblemSpec:
    Lx: float = 2.0
    Ly: float = 1.0
    Lz: float = 0.0
    nelx: int = 60
    nely: int = 30
    nelz: int = 0
    E: float = 1.0
    nu: float = 0.3
    volfrac: float = 0.5
    supports: list = field(default_factory=list)
    loads: list = field(default_factory=list)
    passive_regions: list = field(default_factory=list)
    max_iter: Optional[int] = None
    rmin: Optional[float] = None

    @property
    def is_3d(self) -> bool:
        return self.nelz > 0 and self.Lz > 0

    @property
    def ndim(self) -> int:
        return 3 if self.is_3d else 2

    def validate(self) -> list[str]:
        errors = []
        if self.nelx < 1 or self.nely < 1:
            errors.append("nelx and nely must be positive")
        if self.is_3d and self.nelz < 1:
            errors.append("nelz must be positive for 3D problems")
        if not (0.0 < self.volfrac <= 1.0):
            errors.append("volfrac must lie in (0, 1]")
        if not self.supports:
            errors.append("at least one support is required")
        if not self.loads:
            errors.append("at least one load is required")
        return errors
