"""Supports and loads -> constrained/free DOFs and force vector.

Restates ``gpu_fem/bc_generator.py:173-251, :381-447`` (``generate_bc``) for 3D
problems: supports and point loads snap to the nearest mesh node (first node on
ties), face supports constrain every node of the named face, distributed loads
use trapezoidal tributary areas, loads on constrained DOFs are zeroed.
"""

from __future__ import annotations

import numpy as np

from .problem_spec import DistributedLoad, EdgeSupport, PointLoad, PointSupport, ProblemSpec


def _node_coords_3d(spec: ProblemSpec) -> np.ndarray:
    i, j, k = np.meshgrid(np.arange(spec.nelx + 1), np.arange(spec.nely + 1),
                          np.arange(spec.nelz + 1), indexing="ij")
    return np.column_stack([i.ravel() * (spec.Lx / spec.nelx), j.ravel() * (spec.Ly / spec.nely),
                            k.ravel() * (spec.Lz / spec.nelz)])


def _face_nodes(face: str, spec: ProblemSpec) -> np.ndarray:
    nx, ny, nz = spec.nelx, spec.nely, spec.nelz
    I, J, K = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    node = (I * (ny + 1) + J) * (nz + 1) + K
    sel = {
        "left": node[0, :, :], "right": node[nx, :, :],
        "bottom": node[:, 0, :], "top": node[:, ny, :],
        "front": node[:, :, 0], "back": node[:, :, nz],
    }
    if face not in sel:
        raise ValueError(f"Unknown 3D face: {face}")
    return sel[face].ravel()


def _nearest_node(coords: np.ndarray, point) -> int:
    d = np.linalg.norm(coords - np.asarray(point, dtype=np.float64)[None, :], axis=1)
    return int(np.argmin(d))


def _tributary_weights(cnodes: np.ndarray, spec: ProblemSpec, face: str) -> np.ndarray:
    if face in ("left", "right"):
        h1, h2, c1, c2 = spec.Ly / spec.nely, spec.Lz / spec.nelz, cnodes[:, 1], cnodes[:, 2]
    elif face in ("bottom", "top"):
        h1, h2, c1, c2 = spec.Lx / spec.nelx, spec.Lz / spec.nelz, cnodes[:, 0], cnodes[:, 2]
    else:
        h1, h2, c1, c2 = spec.Lx / spec.nelx, spec.Ly / spec.nely, cnodes[:, 0], cnodes[:, 1]
    w1 = np.full(len(cnodes), h1)
    w1[(np.abs(c1 - c1.min()) < 0.01 * h1) | (np.abs(c1 - c1.max()) < 0.01 * h1)] = h1 / 2
    w2 = np.full(len(cnodes), h2)
    w2[(np.abs(c2 - c2.min()) < 0.01 * h2) | (np.abs(c2 - c2.max()) < 0.01 * h2)] = h2 / 2
    return w1 * w2


class BCResult:
    __slots__ = ("bc_override", "passive_mask", "fixed_dofs", "free_dofs", "F", "ndof", "node_coords")

    def __init__(self, bc_override, passive_mask, fixed_dofs, free_dofs, F, ndof, node_coords):
        self.bc_override = bc_override
        self.passive_mask = passive_mask
        self.fixed_dofs = fixed_dofs
        self.free_dofs = free_dofs
        self.F = F
        self.ndof = ndof
        self.node_coords = node_coords


def generate_bc(spec: ProblemSpec) -> BCResult:
    errors = spec.validate()
    if errors:
        raise ValueError("ProblemSpec validation failed:\n" + "\n".join(f"  - {e}" for e in errors))
    if not spec.is_3d:
        raise ValueError("only 3D problems are supported by this solver")
    coords = _node_coords_3d(spec)
    ndof = 3 * len(coords)
    fixed = set()
    for sup in spec.supports:
        if isinstance(sup, EdgeSupport):
            nodes = _face_nodes(sup.edge, spec)
        else:
            nodes = [_nearest_node(coords, (sup.x, sup.y, sup.z))]
        for n in nodes:
            for off in sup.dof_mask(3):
                fixed.add(3 * int(n) + off)
    fixed = np.sort(np.array(sorted(fixed), dtype=np.int64))
    free = np.setdiff1d(np.arange(ndof), fixed)
    F = np.zeros(ndof)
    for ld in spec.loads:
        if isinstance(ld, PointLoad):
            n = _nearest_node(coords, (ld.x, ld.y, ld.z))
            F[3 * n] += ld.fx
            F[3 * n + 1] += ld.fy
            F[3 * n + 2] += ld.fz
        elif isinstance(ld, DistributedLoad):
            nodes = _face_nodes(ld.edge, spec)
            w = _tributary_weights(coords[nodes], spec, ld.edge)
            off, sign = {"left": (0, -1.0), "right": (0, 1.0), "bottom": (1, -1.0),
                         "top": (1, 1.0), "front": (2, -1.0), "back": (2, 1.0)}[ld.edge]
            for i, n in enumerate(nodes):
                F[3 * n + off] += ld.magnitude * sign * w[i]
    F[fixed] = 0.0
    if np.max(np.abs(F[free])) < 1e-30:
        raise ValueError("Force vector is zero on all free DOFs. "
                         "Check that loads are not placed on fully-fixed supports.")
    _f, _fr, _F = fixed, free, F

    def bc_override(nelx_arg, nely_arg, nelz_arg):
        return _f, _fr, _F

    return BCResult(bc_override, None, fixed, free, F, ndof, coords)
