"""FusedMatvec: the reference's fused gather / KE u / scatter operator
(gpu_fem/cuda_fused_matvec.py:260-416) over the library's sweep kernels.

Same constructor, methods and dtype contract: FP32 vectors and moduli;
``dtype="fp32"`` is the FP32 element product, ``dtype="bf16"`` rounds u and KE
to bfloat16 (round to nearest even) and accumulates in FP32, as the reference's
WMMA kernel does.  ``matvec_full`` returns K u on every DOF (fixed rows
included, like the reference's scatter into the full vector); ``matvec``
restricts to the given free DOFs.  The structured grid is recovered from the
edof table once; the operator itself runs as ``simpfem_matvec_full`` on a mesh
handle whose every DOF is free.
"""

from __future__ import annotations

import numpy as np

from . import _lib
from ._native import get_mesh, grid_from_edof, to_numpy


class FusedMatvec:
    """Drop-in replacement for ``MatrixFreeKff.matvec(u_free, E_e)`` in FP32 / BF16."""

    KE_SIZE = 24
    # launch constants of the reference's kernels, kept for callers that print them
    BLOCK_X_FP32 = 128
    WARPS_PER_BLOCK_BF16 = 8
    ELEMS_PER_WARP_BF16 = 16
    BLOCK_X_BF16 = 32 * WARPS_PER_BLOCK_BF16
    ELEMS_PER_BLOCK_BF16 = WARPS_PER_BLOCK_BF16 * ELEMS_PER_WARP_BF16
    BLOCK_X = BLOCK_X_FP32

    def __init__(self, edof_gpu, KE_unit_gpu, ndof: int):
        torch = _lib.require_cuda()
        shape = tuple(edof_gpu.shape)
        if len(shape) != 2 or shape[1] != self.KE_SIZE:
            raise ValueError(f"FusedMatvec currently supports ke_size=24 only, got {shape[-1]}")
        dims = grid_from_edof(edof_gpu)
        self._dims = dims
        self._ndof = int(ndof)
        self._n_elem = int(shape[0])
        ke = np.asarray(to_numpy(KE_unit_gpu), dtype=np.float64)
        self._mesh = get_mesh(dims, np.arange(self._ndof, dtype=np.int32), ke)
        if self._mesh.ndof != self._ndof:
            raise ValueError("ndof does not match the mesh of the edof table")
        self._bf16_available = True
        self._y_full = torch.zeros(self._ndof, dtype=torch.float32, device="cuda")

    def _launch(self, dtype: str, u_full, y_full, E_f32) -> None:
        if dtype == "fp32":
            dt = _lib.F32
        elif dtype == "bf16":
            dt = _lib.BF16
        else:
            raise ValueError(f"Unknown dtype '{dtype}' — use 'fp32' or 'bf16'")
        _lib.call("simpfem_matvec_full", self._mesh.handle, dt, _lib.ptr(E_f32), _lib.ptr(u_full),
                  _lib.ptr(y_full), _lib.stream_ptr())

    def matvec(self, u_free, E_e, free_gpu, *, dtype: str = "fp32"):
        """y_free = K_ff u_free in FP32 (u at fixed DOFs taken as zero)."""
        torch = _lib.require_cuda()
        free = _lib.as_cuda(free_gpu, torch.int64)
        u_full = torch.zeros(self._ndof, dtype=torch.float32, device="cuda")
        u_full[free] = _lib.as_cuda(u_free, torch.float32)
        E = _lib.as_cuda(E_e, torch.float32)
        y_full = self._y_full
        self._launch(dtype, u_full, y_full, E)
        return y_full[free]

    def matvec_full(self, u_full_in, E_e, *, dtype: str = "fp32"):
        """y_full = K u_full in FP32; the caller keeps u_full zero at fixed DOFs."""
        torch = _lib.require_cuda()
        u_full = _lib.as_cuda(u_full_in, torch.float32)
        if u_full.numel() != self._ndof:
            raise ValueError("u_full must have ndof entries")
        E = _lib.as_cuda(E_e, torch.float32)
        y_full = self._y_full
        self._launch(dtype, u_full, y_full, E)
        return y_full.clone()
