"""CPU restatement of the SIMP loop steps around the guarded solve (test
infrastructure only).

* ``oc_update_projected``, ``heaviside``, ``heaviside_deriv``: the same step with the
  Heaviside projection (simp_gpu.py:245-290; pub_simp_solver.py:245-253).
* ``oc_update`` follows the reference's GPU OC step (gpu_fem/simp_gpu.py:212-294,
  ``_oc_step_cupy`` without the Heaviside projection): design sensitivities
  H^T dc, volume sensitivities 1 (:262-263), bisection on the multiplier over
  [0, 1e9] for at most 100 steps until the bracket is below 1e-9, the volume of
  every candidate evaluated as sum(H rn) with the sparse filter matrix.
* ``compliance_and_sensitivity`` solves K(E) u = F directly (scipy sparse LU on
  the assembled FP64 stiffness) and returns c = F.u and
  dc = -p (1 - rho_min) rho^(p-1) u_e^T KE u_e, the SIMP sensitivity the
  reference's SolverV4 returns (gpu_fem/solver_v4.py:257-264).
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from .solver import edof_table, ke_unit_3d


def oc_update(rho, dc_phys, H: sp.csr_matrix, volfrac: float, move: float):
    """Returns (rho_new, change, multiplier, bisection steps)."""
    rho = np.asarray(rho, dtype=np.float64)
    n = rho.size
    dc_design = H.T @ np.asarray(dc_phys, dtype=np.float64)
    dv_design = np.ones(n)
    dc_s = np.minimum(dc_design, -1e-12)
    dv_s = np.maximum(dv_design, 1e-12)
    l1, l2 = 0.0, 1e9
    rn = rho
    lm = 0.5 * (l1 + l2)
    steps = 0
    for _ in range(100):
        lm = 0.5 * (l1 + l2)
        rn = np.clip(np.clip(rho * np.sqrt(-dc_s / (lm * dv_s)), rho - move, rho + move), 1e-3, 1.0)
        vol = float((H @ rn).sum())
        steps += 1
        if vol > volfrac * n:
            l1 = lm
        else:
            l2 = lm
        if l2 - l1 < 1e-9:
            break
    return rn, float(np.max(np.abs(rn - rho))), lm, steps


def heaviside(rho_f, beta: float, eta: float):
    """Projection (tanh(b eta) + tanh(b (x - eta))) / (tanh(b eta) + tanh(b (1 - eta)))
    (pub_simp_solver.py:245-248); the identity for beta < 1e-6."""
    rho_f = np.asarray(rho_f, dtype=np.float64)
    if beta < 1e-6:
        return rho_f.copy()
    den = np.tanh(beta * eta) + np.tanh(beta * (1.0 - eta))
    return (np.tanh(beta * eta) + np.tanh(beta * (rho_f - eta))) / den


def heaviside_deriv(rho_f, beta: float, eta: float):
    """d projection / d x = b (1 - tanh(b (x - eta))^2) / denominator (pub_simp_solver.py:250-253)."""
    rho_f = np.asarray(rho_f, dtype=np.float64)
    if beta < 1e-6:
        return np.ones_like(rho_f)
    den = np.tanh(beta * eta) + np.tanh(beta * (1.0 - eta))
    return beta * (1.0 - np.tanh(beta * (rho_f - eta)) ** 2) / den


def oc_update_projected(rho, rho_f, dc_phys, H: sp.csr_matrix, volfrac: float, move: float, beta: float,
                        eta: float):
    """The OC step with the Heaviside projection (simp_gpu.py:245-290, use_heaviside
    with beta > 1e-6): design sensitivities H^T (dc dh) and H^T dh with dh the
    projection's derivative at rho_f; every bisection candidate's volume is the
    projected filtered field's sum.  Returns (rho_new, change, multiplier, steps)."""
    import math

    rho = np.asarray(rho, dtype=np.float64)
    n = rho.size
    den = math.tanh(beta * eta) + math.tanh(beta * (1.0 - eta))
    dh = beta * (1.0 - np.tanh(beta * (np.asarray(rho_f, dtype=np.float64) - eta)) ** 2) / den
    dc_s = np.minimum(H.T @ (np.asarray(dc_phys, dtype=np.float64) * dh), -1e-12)
    dv_s = np.maximum(H.T @ dh, 1e-12)
    l1, l2 = 0.0, 1e9
    rn, lm, steps = rho, 0.5e9, 0
    for _ in range(100):
        lm = 0.5 * (l1 + l2)
        rn = np.clip(np.clip(rho * np.sqrt(-dc_s / (lm * dv_s)), rho - move, rho + move), 1e-3, 1.0)
        vol = float((np.tanh(beta * eta) + np.tanh(beta * (H @ rn - eta))).sum()) / den
        steps += 1
        if vol > volfrac * n:
            l1 = lm
        else:
            l2 = lm
        if l2 - l1 < 1e-9:
            break
    return rn, float(np.max(np.abs(rn - rho))), lm, steps


def stiffness(nx: int, ny: int, nz: int, E: np.ndarray) -> sp.csr_matrix:
    edof = edof_table(nx, ny, nz)
    ke = ke_unit_3d()
    ndof = 3 * (nx + 1) * (ny + 1) * (nz + 1)
    rows = np.repeat(edof, 24, axis=1).ravel()
    cols = np.tile(edof, (1, 24)).ravel()
    vals = (np.asarray(E, dtype=np.float64)[:, None] * ke.ravel()[None, :]).ravel()
    return sp.coo_matrix((vals, (rows, cols)), shape=(ndof, ndof)).tocsr()


def compliance_and_sensitivity(nx, ny, nz, rho_phys, free, F, penal: float, rho_min: float):
    """Direct FP64 solve at E = rho_min + (1 - rho_min) rho^p."""
    rho_phys = np.asarray(rho_phys, dtype=np.float64)
    E = rho_min + (1.0 - rho_min) * rho_phys ** penal
    K = stiffness(nx, ny, nz, E)
    Kff = K[free][:, free]
    u = np.zeros(K.shape[0])
    u[free] = spla.spsolve(Kff.tocsc(), F[free])
    c = float(F @ u)
    edof = edof_table(nx, ny, nz)
    ue = u[edof]
    ce = np.einsum("ei,ij,ej->e", ue, ke_unit_3d(), ue)
    dc = -penal * (1.0 - rho_min) * rho_phys ** (penal - 1.0) * ce
    return c, dc, u
