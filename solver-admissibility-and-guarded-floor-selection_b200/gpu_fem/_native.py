"""Native mesh handles shared by the operator, preconditioner and Krylov wrappers.

A mesh handle is keyed by the grid dimensions and the free-DOF list; the
reference's explicit edof table is checked once against the structured
numbering and then dropped (the CUDA operator computes node indices).
"""

from __future__ import annotations

import contextlib
import contextvars
import ctypes
import hashlib

import numpy as np

from . import _lib
from .pub_simp_solver import KE_UNIT_3D, _edof_table_3d

_MESHES: dict = {}


def to_numpy(x) -> np.ndarray:
    try:
        import torch

        if isinstance(x, torch.Tensor):
            return x.detach().cpu().numpy()
    except ImportError:  # pragma: no cover
        pass
    if hasattr(x, "get"):
        return np.asarray(x.get())
    return np.asarray(x)


def grid_from_edof(edof) -> tuple[int, int, int]:
    """(nelx, nely, nelz) of a structured edof table in the reference's numbering."""
    e = to_numpy(edof)
    if e.ndim != 2 or e.shape[1] != 24:
        raise ValueError("edof must have shape (n_elem, 24)")
    n_elem = e.shape[0]
    nz1 = int(e[0, 9]) // 3          # local node 3 = (0, 1, 0) -> node nz + 1
    nyz = int(e[0, 3]) // 3          # local node 1 = (1, 0, 0) -> node (ny + 1)(nz + 1)
    nz = nz1 - 1
    if nz < 1 or nyz % nz1:
        raise ValueError("edof table is not a structured hex8 grid")
    ny = nyz // nz1 - 1
    if ny < 1 or n_elem % (ny * nz):
        raise ValueError("edof table is not a structured hex8 grid")
    nx = n_elem // (ny * nz)
    ref = _edof_table_3d(nx, ny, nz)
    if not np.array_equal(ref, e.astype(np.int64)):
        raise ValueError("edof table does not follow the structured hex8 numbering")
    return nx, ny, nz


class NativeMesh:
    def __init__(self, dims, free: np.ndarray, ke: np.ndarray):
        _lib.require_cuda()
        self.dims = tuple(int(d) for d in dims)
        self.free = np.ascontiguousarray(free, dtype=np.int32)
        self.ke = np.ascontiguousarray(ke, dtype=np.float64)
        nx, ny, nz = self.dims
        self.ndof = 3 * (nx + 1) * (ny + 1) * (nz + 1)
        self.n_elem = nx * ny * nz
        self.n_free = int(self.free.size)
        h = ctypes.c_void_p()
        _lib.call(
            "simpfem_mesh_create", nx, ny, nz, self.free.ctypes.data_as(ctypes.c_void_p),
            self.n_free, self.ke.ctypes.data_as(ctypes.c_void_p), ctypes.byref(h),
        )
        self.handle = h
        import torch

        self.free_t = torch.as_tensor(self.free.astype(np.int64), device="cuda")

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value and _lib._lib is not None:
            try:
                _lib._lib.simpfem_mesh_destroy(h)
            except Exception:  # pragma: no cover
                pass


# A mesh handle holds scratch vectors and the reduction workspace its
# operators use, so handles shared between solvers must not run concurrently.
# Solvers meant to run at the same time (BatchedFloorPolicy workers) build
# their operators inside ``mesh_namespace(tag)`` and get private handles.
_NAMESPACE = contextvars.ContextVar("simpfem_mesh_namespace", default=None)


@contextlib.contextmanager
def mesh_namespace(tag):
    token = _NAMESPACE.set(tag)
    try:
        yield
    finally:
        _NAMESPACE.reset(token)


def get_mesh(dims, free, ke=None) -> NativeMesh:
    free = np.ascontiguousarray(to_numpy(free), dtype=np.int32)
    ke = KE_UNIT_3D if ke is None else np.asarray(to_numpy(ke), dtype=np.float64)
    key = (_NAMESPACE.get(), tuple(int(d) for d in dims), hashlib.sha1(free.tobytes()).hexdigest(),
           hashlib.sha1(np.ascontiguousarray(ke).tobytes()).hexdigest())
    m = _MESHES.get(key)
    if m is None:
        m = NativeMesh(dims, free, ke)
        _MESHES[key] = m
    return m
