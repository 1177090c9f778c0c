"""Matrix-free operator, node-block Jacobi and PCG with the reference's signatures.

* ``MatrixFreeKff`` -- gpu_fem/solver_v2.py:1121-1261 (``matvec`` :1182-1222,
  ``extract_diagonal`` :1228-1251).  One sm_100a sweep kernel
  (``simpfem_matvec``) replaces the expand / gather / DGEMM / bincount / restrict
  passes.
* ``NodeBlockJacobiMF`` -- :1268-1451 (``update`` / ``apply``).
* ``_cupy_pcg`` -- :551-623: the library's device-resident PCG when the
  preconditioner is a ``GalerkinMatFreeGMG`` and the operator its fine operator,
  the library's PCG core with callback operators otherwise.
* ``_coarse_free_dofs_injection`` -- :716-763.

Arrays are torch CUDA tensors (numpy inputs are moved to the device).
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._native import get_mesh, grid_from_edof, to_numpy


class MatrixFreeKff:
    def __init__(self, edof_gpu, KE_unit_gpu, free_gpu, n_free: int, ndof: int, grid_dims=None):
        dims = tuple(grid_dims) if grid_dims is not None else grid_from_edof(edof_gpu)
        self._dims = dims
        self._free_np = np.asarray(to_numpy(free_gpu), dtype=np.int32)
        self._KE_unit_np = np.asarray(to_numpy(KE_unit_gpu), dtype=np.float64)
        self._n_free = int(n_free)
        self._ndof = int(ndof)
        self._n_elem = dims[0] * dims[1] * dims[2]
        self._ke_size = 24
        if self._free_np.size != self._n_free:
            raise ValueError("n_free does not match free_gpu")
        self._mesh = get_mesh(dims, self._free_np, self._KE_unit_np)
        if self._mesh.ndof != self._ndof:
            raise ValueError("ndof does not match the mesh")
        self._edof_gpu = edof_gpu
        self._KE_unit = KE_unit_gpu
        self._free_gpu = free_gpu

    @property
    def mesh(self):
        return self._mesh

    def matvec(self, u_free, E_e):
        torch = _lib.require_cuda()
        if isinstance(u_free, torch.Tensor) and u_free.dtype == torch.float32:
            dt, tdt = _lib.F32, torch.float32
        elif not isinstance(u_free, torch.Tensor) and np.asarray(u_free).dtype == np.float32:
            dt, tdt = _lib.F32, torch.float32
        else:
            dt, tdt = _lib.F64, torch.float64
        u = _lib.as_cuda(u_free, tdt)
        E = _lib.as_cuda(E_e, tdt)
        y = torch.empty(self._n_free, dtype=tdt, device="cuda")
        _lib.call("simpfem_matvec", self._mesh.handle, dt, _lib.ptr(E), _lib.ptr(u), _lib.ptr(y),
                  _lib.stream_ptr())
        return y

    def extract_diagonal(self, E_e):
        torch = _lib.require_cuda()
        E = _lib.as_cuda(E_e, torch.float64)
        d = torch.empty(self._n_free, dtype=torch.float64, device="cuda")
        _lib.call("simpfem_extract_diagonal", self._mesh.handle, _lib.ptr(E), _lib.ptr(d), _lib.stream_ptr())
        return d


class NodeBlockJacobiMF:
    def __init__(self, edof_gpu, KE_unit_gpu, free_gpu, n_free: int, ndof: int, grid_dims=None):
        dims = tuple(grid_dims) if grid_dims is not None else grid_from_edof(edof_gpu)
        self._n_free = int(n_free)
        self._ndof = int(ndof)
        self._n_nodes = ndof // 3
        self._mesh = get_mesh(dims, to_numpy(free_gpu), to_numpy(KE_unit_gpu))
        self._blocks = None

    def update(self, E_e, scalar_diag=None) -> None:
        torch = _lib.require_cuda()
        E = _lib.as_cuda(E_e, torch.float64)
        if self._blocks is None:
            self._blocks = torch.empty(self._n_nodes * 9, dtype=torch.float64, device="cuda")
        d = _lib.as_cuda(scalar_diag, torch.float64) if scalar_diag is not None else None
        _lib.call("simpfem_node_blocks", self._mesh.handle, _lib.ptr(E), _lib.ptr(d) if d is not None else None,
                  _lib.ptr(self._blocks), _lib.stream_ptr())

    def apply(self, r):
        torch = _lib.require_cuda()
        if self._blocks is None:
            raise RuntimeError("NodeBlockJacobiMF.update() must be called before apply()")
        in_dtype = r.dtype if isinstance(r, torch.Tensor) else torch.float64
        rr = _lib.as_cuda(r, torch.float64)
        z = torch.empty(self._n_free, dtype=torch.float64, device="cuda")
        _lib.call("simpfem_node_block_apply", self._mesh.handle, _lib.ptr(self._blocks), _lib.ptr(rr), _lib.ptr(z),
                  _lib.stream_ptr())
        return z.to(in_dtype)


def _coarse_free_dofs_injection(nelx_f, nely_f, nelz_f, nelx_c, nely_c, nelz_c, free_f) -> np.ndarray:
    """Coarse free DOFs by injection of coarse node (I, J, K) into fine node
    (2I, 2J, 2K), with the reference's linear-index arithmetic."""
    ndof_c = 3 * (nelx_c + 1) * (nely_c + 1) * (nelz_c + 1)
    ndof_f = 3 * (nelx_f + 1) * (nely_f + 1) * (nelz_f + 1)
    I, J, K = np.meshgrid(np.arange(nelx_c + 1), np.arange(nely_c + 1), np.arange(nelz_c + 1), indexing="ij")
    fine_node = (2 * I * (nely_f + 1) * (nelz_f + 1) + 2 * J * (nelz_f + 1) + 2 * K).ravel()
    mask_f = np.zeros(ndof_f, dtype=bool)
    mask_f[np.asarray(free_f)] = True
    is_free = np.zeros(ndof_c, dtype=bool)
    cn = np.arange(fine_node.size)
    for d in range(3):
        fd = 3 * fine_node + d
        ok = fd < ndof_f
        is_free[(3 * cn + d)[ok]] = mask_f[fd[ok]]
    return np.where(is_free)[0].astype(np.int32)


def _native_gmg(A, M_op):
    """The GalerkinMatFreeGMG behind ``M_op`` when ``A`` is exactly its fine operator."""
    from .multigrid_v4 import GalerkinMatFreeGMG

    gmg = getattr(M_op, "__self__", None)
    if not isinstance(gmg, GalerkinMatFreeGMG) or getattr(M_op, "__func__", None) is not GalerkinMatFreeGMG.apply:
        return None
    if not gmg._is_setup or not callable(A):
        return None
    torch = _lib.require_cuda()
    gen = torch.Generator(device="cuda")
    gen.manual_seed(1234)
    v = torch.randn(gmg._mf_op._n_free, dtype=torch.float64, device="cuda", generator=gen)
    a = A(v)
    if not isinstance(a, torch.Tensor) or a.shape != v.shape:
        return None
    ref = gmg.apply_fine_operator(v)
    den = float(torch.linalg.norm(ref))
    if den == 0.0 or float(torch.linalg.norm(a.to(torch.float64) - ref)) > 1e-12 * den:
        return None
    return gmg


def _cupy_pcg(A, b, M_op, x0=None, tol=1e-5, maxiter=1000, history=None):
    """Preconditioned CG with the up-front convergence check (solver_v2.py:551-623).

    A hierarchy's own fine operator and ``apply`` run the library's PCG; any other
    operator (a callable or a matrix) and preconditioner run on the library's
    device PCG core with the two applied through callbacks."""
    _Aop = A if callable(A) else (lambda v, _A=A: _A @ v)
    gmg = _native_gmg(_Aop, M_op)
    if gmg is not None:
        return gmg._native_pcg(b, x0, tol, maxiter, history)
    from . import _krylov

    return _krylov.pcg(_Aop, b, M_op, x0=x0, tol=tol, maxiter=maxiter, history=history)
