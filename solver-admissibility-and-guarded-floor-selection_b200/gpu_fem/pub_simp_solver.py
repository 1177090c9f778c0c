"""Element data of the structured SIMP mesh (boundary inputs of the solve).

Names and semantics follow the reference's ``gpu_fem/pub_simp_solver.py``:

* ``_build_ke_unit_3d`` / ``KE_UNIT_3D`` (pub_simp_solver.py:157-186): 24x24
  stiffness of the trilinear hex8 element in natural coordinates [-1, 1]^3,
  2x2x2 Gauss quadrature, isotropic material (E, nu), Voigt shear order
  (xy, yz, xz), local node order n0..n7 = (0,0,0) (1,0,0) (1,1,0) (0,1,0)
  (0,0,1) (1,0,1) (1,1,1) (0,1,1).
* ``_edof_table_3d`` (:196-207): element -> 24 global DOFs,
  node(i, j, k) = i (ny+1)(nz+1) + j (nz+1) + k, dof = 3 node + c.
* ``_build_density_filter`` (:215-243): cone filter, weights rmin - dist for
  element centroids closer than rmin, rows normalised to sum to one.
* ``_heaviside`` (:245-253).
* ``StepState`` (:116-135): the per-iteration state a SIMP parameter
  controller reads.

The CUDA operator does not use the edof table (node indices are computed from
the grid position); it is provided for callers of the reference API.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sp

# (x, y, z) natural-coordinate signs of the local nodes, reference order
_NODE_SIGNS = np.array(
    [[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
     [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]],
    dtype=np.float64,
)
_NODE_OFFSETS = ((_NODE_SIGNS + 1) // 2).astype(np.int64)


def _elasticity_matrix(nu: float, E: float) -> np.ndarray:
    lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    mu = E / (2.0 * (1.0 + nu))
    D = np.zeros((6, 6))
    D[:3, :3] = lam
    D[np.arange(3), np.arange(3)] = lam + 2.0 * mu
    D[np.arange(3, 6), np.arange(3, 6)] = mu
    return D


def _build_ke_unit_3d(nu: float = 0.3, E: float = 1.0) -> np.ndarray:
    D = _elasticity_matrix(nu, E)
    g = 1.0 / np.sqrt(3.0)
    KE = np.zeros((24, 24))
    for gx, gy, gz in _NODE_SIGNS * g:
        # shape-function gradients of N_a = (1 + x x_a)(1 + y y_a)(1 + z z_a) / 8;
        # the natural coordinates are the physical ones (J = I, det J = 1)
        sx, sy, sz = _NODE_SIGNS[:, 0], _NODE_SIGNS[:, 1], _NODE_SIGNS[:, 2]
        dx = 0.125 * sx * (1 + gy * sy) * (1 + gz * sz)
        dy = 0.125 * sy * (1 + gx * sx) * (1 + gz * sz)
        dz = 0.125 * sz * (1 + gx * sx) * (1 + gy * sy)
        B = np.zeros((6, 24))
        B[0, 0::3] = dx
        B[1, 1::3] = dy
        B[2, 2::3] = dz
        B[3, 0::3] = dy
        B[3, 1::3] = dx
        B[4, 1::3] = dz
        B[4, 2::3] = dy
        B[5, 0::3] = dz
        B[5, 2::3] = dx
        KE += B.T @ D @ B
    return KE


KE_UNIT_3D = _build_ke_unit_3d()


def _edof_table_3d(nelx: int, nely: int, nelz: int) -> np.ndarray:
    i, j, k = np.meshgrid(np.arange(nelx), np.arange(nely), np.arange(nelz), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    ny1, nz1 = nely + 1, nelz + 1
    nodes = np.empty((i.size, 8), dtype=np.int64)
    for a, (ox, oy, oz) in enumerate(_NODE_OFFSETS):
        nodes[:, a] = ((i + ox) * ny1 + (j + oy)) * nz1 + (k + oz)
    edof = 3 * nodes[:, :, None] + np.arange(3)[None, None, :]
    return edof.reshape(i.size, 24).astype(np.int32)


def _build_sparse_indices(edof: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    n = edof.shape[1]
    rows = np.repeat(edof, n, axis=1)
    cols = np.tile(edof, (1, n))
    return rows.ravel().astype(np.int32), cols.ravel().astype(np.int32)


def _build_density_filter(nelx: int, nely: int, rmin: float, nelz: int = 0) -> sp.csr_matrix:
    """Cone filter on element centroids (3D when nelz > 0)."""
    dims = (nelx, nely, nelz) if nelz > 0 else (nelx, nely)
    nd = len(dims)
    n = int(np.prod(dims))
    r = int(np.floor(rmin))
    idx = np.arange(n).reshape(dims)
    coords = np.stack(np.meshgrid(*[np.arange(d) for d in dims], indexing="ij"), axis=-1)
    rows, cols, vals = [np.arange(n)], [np.arange(n)], [np.full(n, float(rmin))]
    rng = range(-r, r + 1)
    offsets = np.array(np.meshgrid(*([rng] * nd), indexing="ij")).reshape(nd, -1).T
    for off in offsets:
        if not off.any():
            continue
        dist = float(np.sqrt(np.sum(off.astype(np.float64) ** 2)))
        if dist > rmin - 1e-10:
            continue
        src = [slice(max(0, -o), d - max(0, o)) for o, d in zip(off, dims)]
        dst = [slice(max(0, o), d - max(0, -o)) for o, d in zip(off, dims)]
        rows.append(idx[tuple(src)].ravel())
        cols.append(idx[tuple(dst)].ravel())
        vals.append(np.full(rows[-1].size, rmin - dist))
    rows = np.concatenate(rows)
    cols = np.concatenate(cols)
    vals = np.concatenate(vals)
    Hs = np.bincount(rows, weights=vals, minlength=n)
    del coords
    return sp.csr_matrix((vals / Hs[rows], (rows, cols)), shape=(n, n))


def _heaviside(rho_f, beta, eta):
    if beta < 1e-6:
        return rho_f.copy()
    return (np.tanh(beta * eta) + np.tanh(beta * (rho_f - eta))) / (
        np.tanh(beta * eta) + np.tanh(beta * (1.0 - eta))
    )


@dataclass
class StepState:
    """What a parameter controller sees after each SIMP iteration: the iteration's
    compliance and the best valid design so far, the physical design's volume
    fraction, grayness 4 mean(rho (1 - rho)) and checkerboard measure, the
    compliance's relative changes, the continuation parameters after the beta
    schedule, and the convergence flags."""
    iteration: int
    compliance: float
    best_compliance: float
    best_iteration: int
    volume_fraction: float
    grayness: float
    best_grayness: float
    checkerboard: float
    obj_slope: float
    rel_change_1: float
    rel_change_5: float
    stagnation_counter: int
    penal: float
    rmin: float
    move: float
    beta: float
    converged: bool
    best_is_valid: bool
    compliance_history: list = field(default_factory=list)
