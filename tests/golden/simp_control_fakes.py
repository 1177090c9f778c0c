"""Deterministic stand-ins shared by make_simp_control_golden.py (around the
reference's run_simp_surrogate_gpu) and tests/test_simp_control_host.py
(around this package's): test infrastructure only.

The numeric steps of both loops are replaced by the same host code -- the
oracle's cone filter, Heaviside projection and OC updates, and a closed-form
stand-in for the solve (compliance sum(w / E), E = Emin + (1 - Emin) rho^p,
with its exact sensitivity) -- so both loops see bit-identical numbers and any
difference between their logs is the loops' own control flow: the router and
surrogate, the passive mask, the best-design gate, the convergence test, the
beta schedule, the parameter controller's actions, radius changes and restarts.
"""

from __future__ import annotations

import os
import sys

import numpy as np

_ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
if _ROOT not in sys.path:
    sys.path.insert(0, _ROOT)

from oracle.simp import heaviside, oc_update, oc_update_projected  # noqa: E402
from oracle.solver import density_filter  # noqa: E402

DIMS = (16, 8, 6)
# "controlled": projection, schedule-only controller, passive mask, surrogate every fourth iteration;
# "plain": the unprojected OC step alone, run until the convergence test stops it
SCENARIOS = {
    "controlled": dict(params=dict(nelx=16, nely=8, nelz=6, volfrac=0.3, penal=3.0, emin=1e-3, rmin=1.5,
                                   max_iter=72, min_iter=30, tol=0.01, use_heaviside=True),
                       controller=True, surrogate=True, passive=True),
    "plain": dict(params=dict(nelx=16, nely=8, nelz=6, volfrac=0.3, penal=3.0, emin=1e-3, rmin=1.5, max_iter=150,
                              min_iter=10, tol=0.01, use_heaviside=False),
                  controller=False, surrogate=False, passive=False),
}
SOLVER_KWARGS = dict(enable_matrix_free=True)
EVENTS: list = []
_FILTERS: dict = {}


def filter_matrix(nx: int, ny: int, nz: int, rmin: float):
    key = (nx, ny, nz, float(rmin))
    if key not in _FILTERS:
        _FILTERS[key] = density_filter(nx, ny, nz, rmin)
    return _FILTERS[key]


def build_density_filter(nelx: int, nely: int, rmin: float, nelz: int = 0):
    """The reference's _build_density_filter signature over the oracle's filter."""
    return filter_matrix(nelx, nely, nelz, rmin)


def project(rho_f, beta: float, eta: float):
    return heaviside(np.asarray(rho_f, dtype=np.float64), beta, eta)


def oc_step(rho, rho_f, dc, beta: float, eta: float, volfrac: float, move: float, H, projected: bool):
    """(rho_new, change) of the oracle's OC update with or without the projection."""
    rho, rho_f, dc = (np.asarray(a, dtype=np.float64) for a in (rho, rho_f, dc))
    if projected:
        rn, change, _, _ = oc_update_projected(rho, rho_f, dc, H, volfrac, move, beta, eta)
    else:
        rn, change, _, _ = oc_update(rho, dc, H, volfrac, move)
    return rn, change


def passive_mask() -> np.ndarray:
    m = np.zeros(DIMS, dtype=np.int32)
    m[13:16, 3:5, :] = 2
    m[4:7, 0:2, 0:2] = 1
    return m.ravel()


def problem():
    """(fixed, free, F, ndof) handed to the loop; only the stand-in solver sees them."""
    nx, ny, nz = DIMS
    ndof = 3 * (nx + 1) * (ny + 1) * (nz + 1)
    return np.arange(0, 3, dtype=np.int32), np.arange(3, ndof, dtype=np.int32), np.ones(ndof), ndof


def _host(x):
    return x.numpy() if hasattr(x, "numpy") else np.asarray(x, dtype=np.float64)


class FakeSolver:
    """compliance = sum(w / E), dc = -w (E0 - Emin) p rho^(p-1) / E^2 with fixed
    positive weights w; records every solve and invalidation in EVENTS."""

    def __init__(self, *, edof, E0: float = 1.0, Emin: float = 1e-9, cg_tol: float = 1e-6, **kwargs):
        n = int(np.asarray(edof).shape[0])
        self.E0, self.Emin, self.cg_tol = float(E0), float(Emin), float(cg_tol)
        self._backend = "cupy"
        self._w = 1.0 + 0.5 * np.sin(0.37 * np.arange(n)) + np.linspace(0.0, 1.0, n)
        self.last_cg_iters = -1
        self.last_true_rel_residual = float("nan")

    def invalidate(self):
        EVENTS.append("invalidate")

    def solve(self, rho_phys, penal: float):
        r = _host(rho_phys)
        E = self.Emin + (self.E0 - self.Emin) * r ** penal
        c = float(np.sum(self._w / E))
        dc = -self._w * (self.E0 - self.Emin) * penal * r ** (penal - 1.0) / E ** 2
        self.last_cg_iters = 10 + int(round(5.0 * penal))
        self.last_true_rel_residual = 1e-7
        EVENTS.append(("solve", float(penal)))
        return c, dc


class EchoSurrogate:
    """Predicts the sensitivity of the last solve; ready after the first one."""

    uncertainty = 0.0

    def __init__(self):
        self._dc = None

    @property
    def is_ready(self) -> bool:
        return self._dc is not None

    def update(self, rho_phys, rho_f, penal, iter_ratio, dc_phys):
        self._dc = np.array(_host(dc_phys), copy=True)

    def predict(self, rho_phys, rho_f, penal, iter_ratio):
        return self._dc, 0.0


def router(iteration, uncertainty, surrogate_ready, beta=1.0, **kwargs):
    """A solve unless the iteration is a multiple of four."""
    return iteration % 4 != 0
