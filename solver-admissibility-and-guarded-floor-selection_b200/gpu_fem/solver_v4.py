"""SolverV4: the SIMP solver's matrix-free Galerkin-GMG path (gpu_fem/solver_v4.py).

``SolverV4(edof=, row_idx=, col_idx=, KE_UNIT=, free=, F=, ndof=, E0=, Emin=,
backend=, ..., enable_matrix_free=True, enable_matfree_gmg=True, grid_dims=,
...).solve(rho_phys, penal) -> (compliance, dc_phys)`` as the reference's
``SolverV4._solve_cupy_matfree`` (solver_v4.py:149-282) computes it:

* E = Emin + (E0 - Emin) rho^penal on the device; diag(K_ff) through the
  matrix-free operator; ``GalerkinMatFreeGMG.setup(E, fine_diag=diag)``;
* the outer solver (``gmg_outer_solver``: "auto" selects FGMRES when the fine
  smoother is BF16 and PCG otherwise, :183-186) warm-started from the previous
  displacement when ``enable_warm_start`` (reset when penal jumps by more than
  0.5, :166-169), restarted from zero if the warm start does not converge;
* ``last_cg_iters``, ``last_cg_history``, ``last_true_rel_residual`` (the FP64
  recomputed residual ||F - K u|| / ||F||) and ``last_multigrid_quality``;
* compliance = F . u and the sensitivity dc = -penal (E0 - Emin) rho^(penal-1)
  u_e^T KE u_e (:262-268), the element energies from one library kernel
  (``simpfem_element_energy``).

Only this path is on the accelerated solve; the reference's assembled-CSR,
AMG, Torch and CPU backends of SolverV2 are not provided and their options are
refused.
"""

from __future__ import annotations

import time
from typing import Optional

import numpy as np

from . import _lib
from .multigrid_v4 import GalerkinMatFreeGMG, _cupy_fgmres
from .pub_simp_solver import KE_UNIT_3D
from .solver_v2 import MatrixFreeKff, _cupy_pcg


class SolverV4:
    def __init__(self, *, edof, row_idx=None, col_idx=None, KE_UNIT, free, F, ndof: int, E0: float = 1.0,
                 Emin: float = 1e-9, backend: str = "auto", cg_tol: float = 1e-5, cg_maxiter: int = 1000,
                 amg_ndof_threshold: int = 3000, amg_rebuild_tol: float = 0.15, grid_dims=None,
                 enable_warm_start: bool = True, enable_matrix_free: bool = False, enable_matfree_gmg: bool = False,
                 matfree_gmg_levels: int = 4, gmg_fine_smoother: str = "fp32", gmg_fine_degree: int = 2,
                 gmg_outer_solver: str = "auto", gmg_restart: int = 32, gmg_smoother_type: str = "chebyshev",
                 gmg_cheb_lower_frac: float = 1.0 / 30.0, gmg_level_precisions=None, gmg_cycle_type: str = "v",
                 gmg_smooth_iters: int = 2, enable_fused_cuda: bool = False, enable_mixed_precision: bool = False,
                 enable_profiling: bool = False, **unsupported):
        # validation as SolverV4.__init__ (solver_v4.py:67-93)
        if enable_matfree_gmg:
            if not enable_matrix_free:
                raise ValueError("SolverV4 requires enable_matrix_free=True when enable_matfree_gmg=True.")
            if grid_dims is None:
                raise ValueError("SolverV4 requires grid_dims=(nelx, nely, nelz) for the GMG path.")
            if gmg_fine_smoother not in {"fp64", "fp32", "bf16"}:
                raise ValueError(
                    f"gmg_fine_smoother must be one of 'fp64', 'fp32', or 'bf16'; got {gmg_fine_smoother!r}.")
            if gmg_outer_solver not in {"auto", "pcg", "fgmres"}:
                raise ValueError(f"gmg_outer_solver must be 'auto', 'pcg', or 'fgmres'; got {gmg_outer_solver!r}.")
            if gmg_fine_smoother == "bf16" and not enable_fused_cuda:
                raise ValueError(
                    "SolverV4 BF16 fine smoothing requires enable_fused_cuda=True so the WMMA path is available.")
        else:
            raise NotImplementedError("only the matrix-free Galerkin-GMG path of SolverV4 is provided "
                                      "(enable_matrix_free=True, enable_matfree_gmg=True)")
        if unsupported:
            raise NotImplementedError(f"SolverV4 options outside the matrix-free GMG path: {sorted(unsupported)}")
        torch = _lib.require_cuda()
        self.ndof = int(ndof)
        self.E0 = float(E0)
        self.Emin = float(Emin)
        self.cg_tol = float(cg_tol)
        self.cg_maxiter = int(cg_maxiter)
        self._backend = "cupy"  # the reference's name for its CUDA backend; drivers read it
        self._grid_dims = tuple(int(d) for d in grid_dims)
        self._enable_warm_start = bool(enable_warm_start)
        self._enable_profiling = bool(enable_profiling)
        self._free = np.asarray(free, dtype=np.int64)
        self._n_free = int(self._free.size)
        self._n_elem = int(np.prod(self._grid_dims))
        self._free_gpu = torch.as_tensor(self._free, device="cuda")
        self._F_free_gpu = torch.as_tensor(np.asarray(F, dtype=np.float64)[self._free], device="cuda")
        self._KE_unit_np = np.asarray(KE_UNIT, dtype=np.float64)
        self._edof = edof
        self._gmg_kw = dict(n_levels=int(matfree_gmg_levels), coarse_smooth_iters=int(gmg_smooth_iters),
                            fine_smoother=gmg_fine_smoother, fine_smoother_degree=int(gmg_fine_degree),
                            smoother_type=gmg_smoother_type, cheb_lower_frac=float(gmg_cheb_lower_frac),
                            level_precisions=gmg_level_precisions, cycle_type=gmg_cycle_type)
        self._gmg_outer_solver = gmg_outer_solver
        self._gmg_restart = int(gmg_restart)
        self._matfree_op: Optional[MatrixFreeKff] = None
        self._matfree_gmg: Optional[GalerkinMatFreeGMG] = None
        self._u_prev = None
        self._prev_penal = None
        self.last_cg_iters = 0
        self.last_cg_history: list = []
        self.last_true_rel_residual = float("nan")
        self.last_outer_solver = ""
        self.last_multigrid_quality: dict = {}
        self.last_timing: dict = {}

    def _ensure_matfree_components(self) -> None:
        if self._matfree_op is None:
            self._matfree_op = MatrixFreeKff(self._edof, self._KE_unit_np, self._free_gpu, self._n_free, self.ndof,
                                             grid_dims=self._grid_dims)
        if self._matfree_gmg is None:
            nelx, nely, nelz = self._grid_dims
            self._matfree_gmg = GalerkinMatFreeGMG(mf_op=self._matfree_op, free=self._free, free_gpu=self._free_gpu,
                                                   nelx=nelx, nely=nely, nelz=nelz, KE_UNIT=KE_UNIT_3D,
                                                   **self._gmg_kw)

    def invalidate(self) -> None:
        """Drop the warm start (SolverV2.invalidate, solver_v2.py:2397-2404); the
        hierarchy is set up again by every solve anyway."""
        self._u_prev = None

    def solve(self, rho_phys, penal: float):
        torch = _lib.require_cuda()
        stream = torch.cuda.current_stream()
        self._ensure_matfree_components()
        if self._prev_penal is not None and abs(penal - self._prev_penal) > 0.5:
            self._u_prev = None
        self._prev_penal = penal
        t0 = time.perf_counter()
        rho = _lib.as_cuda(rho_phys, torch.float64)
        E_e = self.Emin + (self.E0 - self.Emin) * rho ** penal
        fine_diag = self._matfree_op.extract_diagonal(E_e)
        stream.synchronize()
        t1 = time.perf_counter()
        self._matfree_gmg.setup(E_e, fine_diag=fine_diag)
        stream.synchronize()
        t2 = time.perf_counter()

        def _Kop(v):
            return self._matfree_op.matvec(v, E_e)

        x0 = self._u_prev if self._enable_warm_start else None
        F = self._F_free_gpu
        outer = self._gmg_outer_solver
        if outer == "auto":
            outer = "fgmres" if self._matfree_gmg.uses_bf16_smoother() else "pcg"
        self.last_outer_solver = outer
        history: list = []
        if outer == "pcg":
            U, n_outer, converged = _cupy_pcg(_Kop, F, self._matfree_gmg.apply, x0=x0, tol=self.cg_tol,
                                              maxiter=self.cg_maxiter, history=history)
            if not converged and x0 is not None:
                history = []
                U, n_outer, converged = _cupy_pcg(_Kop, F, self._matfree_gmg.apply, x0=None, tol=self.cg_tol,
                                                  maxiter=self.cg_maxiter, history=history)
        else:
            U, n_outer, converged = _cupy_fgmres(_Kop, F, self._matfree_gmg.apply, x0=x0, tol=self.cg_tol,
                                                 maxiter=self.cg_maxiter, restart=self._gmg_restart, history=history)
            if not converged and x0 is not None:
                history = []
                U, n_outer, converged = _cupy_fgmres(_Kop, F, self._matfree_gmg.apply, x0=None, tol=self.cg_tol,
                                                     maxiter=self.cg_maxiter, restart=self._gmg_restart,
                                                     history=history)
        self.last_cg_iters = int(n_outer)
        self.last_cg_history = list(history)
        b_norm = float(torch.linalg.norm(F))
        self.last_true_rel_residual = float(torch.linalg.norm(F - _Kop(U))) / max(b_norm, 1e-300)
        self.last_multigrid_quality = self._matfree_gmg.probe_quality(F)
        stream.synchronize()
        t3 = time.perf_counter()
        if self._enable_warm_start:
            self._u_prev = U.clone()
        compliance = float(torch.dot(F, U))
        ce = torch.empty(self._n_elem, dtype=torch.float64, device="cuda")
        _lib.call("simpfem_element_energy", self._matfree_op.mesh.handle, _lib.ptr(U.contiguous()), _lib.ptr(ce),
                  _lib.stream_ptr())
        dc = -penal * (self.E0 - self.Emin) * rho ** (penal - 1.0) * ce
        dc_host = dc.cpu().numpy()
        t4 = time.perf_counter()
        if self._enable_profiling:
            self.last_timing = {"assemble_ms": 0.0, "diag_ms": (t1 - t0) * 1e3, "gmg_setup_ms": (t2 - t1) * 1e3,
                                "cg_ms": (t3 - t2) * 1e3, "sensitivity_ms": (t4 - t3) * 1e3,
                                "total_ms": (t4 - t0) * 1e3, "used_gmg": True, "matrix_free": True,
                                "outer_solver": outer, "cg_iters": int(n_outer)}
        return compliance, dc_host


def element_energy(mf_op: MatrixFreeKff, u_free):
    """u_e^T KE u_e per element for a free-DOF displacement (device tensor)."""
    torch = _lib.require_cuda()
    u = _lib.as_cuda(u_free, torch.float64)
    n_elem = int(np.prod(mf_op._dims))
    ce = torch.empty(n_elem, dtype=torch.float64, device="cuda")
    _lib.call("simpfem_element_energy", mf_op.mesh.handle, _lib.ptr(u), _lib.ptr(ce), _lib.stream_ptr())
    return ce
