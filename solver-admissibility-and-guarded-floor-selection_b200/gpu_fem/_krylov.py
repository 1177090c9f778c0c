"""FGMRES / PCG on the device for operator and preconditioner pairs given as callables.

The reference's ``_cupy_fgmres`` (gpu_fem/multigrid_v4.py:416-534) and
``_cupy_pcg`` (gpu_fem/solver_v2.py:551-623) accept any pair of callables.  When
the pair is a hierarchy's own fine operator and ``apply`` the library runs the
whole solve itself; every other pair comes here: the library's device Arnoldi
basis, Givens rotations, back-solve and deterministic reductions
(``simpfem_fgmres_op`` / ``simpfem_pcg_op``) call back into Python only to apply
the two operators, handing over device vectors that are wrapped as torch
tensors without a copy.  The callbacks run on the calling thread and their
torch work lands on the current stream, which is also the solve's stream.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

# int apply(void* ctx, const double* x, double* y, void* stream)
_APPLY_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p)


class _DeviceVector:
    """A device vector of n doubles exposed through the CUDA array interface."""

    def __init__(self, addr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (int(addr), False),
                                         "version": 3, "strides": None}


def _callback(fn, n: int, errors: list):
    torch = _lib.require_cuda()

    def apply(_ctx, x_addr, y_addr, _stream):
        try:
            x = torch.as_tensor(_DeviceVector(x_addr, n), device="cuda")
            y = torch.as_tensor(_DeviceVector(y_addr, n), device="cuda")
            out = _lib.as_cuda(fn(x), torch.float64).reshape(-1)
            if out.numel() != n:
                raise ValueError(f"operator returned {out.numel()} entries for a system of {n}")
            y.copy_(out)
            return 0
        except BaseException as e:  # raised again once the library returns
            errors.append(e)
            return 1

    return _APPLY_FN(apply)


def _run(name: str, A_op, M_op, b, x0, head: tuple, tail: tuple):
    torch = _lib.require_cuda()
    bb = _lib.as_cuda(b, torch.float64).reshape(-1)
    n = int(bb.numel())
    x = torch.empty_like(bb)
    x0t = _lib.as_cuda(x0, torch.float64).reshape(-1) if x0 is not None else None
    errors: list = []
    cb_a, cb_m = _callback(A_op, n, errors), _callback(M_op, n, errors)
    hlen, it, conv = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    hist, cap = tail
    try:
        _lib.call(name, n, ctypes.cast(cb_a, ctypes.c_void_p), ctypes.cast(cb_m, ctypes.c_void_p), None,
                  _lib.ptr(bb), _lib.ptr(x0t) if x0t is not None else None, _lib.ptr(x), *head,
                  hist.ctypes.data_as(ctypes.c_void_p), cap, ctypes.byref(hlen), ctypes.byref(it),
                  ctypes.byref(conv), _lib.stream_ptr())
    except _lib.SimpfemError:
        if errors:
            raise errors[0]
        raise
    return x, int(it.value), bool(conv.value), [float(v) for v in hist[: min(hlen.value, cap)]]


def fgmres(A_op, b, M_op, x0=None, tol=1e-6, maxiter=200, restart=32, history=None):
    """(x, total_iters, converged) with the reference's history rule."""
    cap = int(maxiter) + int(maxiter) // max(int(restart), 1) + 4
    hist = np.zeros(cap, dtype=np.float64)
    x, it, conv, h = _run("simpfem_fgmres_op", A_op, M_op, b, x0, (float(tol), int(maxiter), int(restart)),
                          (hist, cap))
    if history is not None:
        history.extend(h)
    return x, it, conv


def pcg(A_op, b, M_op, x0=None, tol=1e-5, maxiter=1000, history=None):
    """(x, iters, converged); iters counts preconditioner applications."""
    cap = max(int(maxiter), 1) + 4
    hist = np.zeros(cap, dtype=np.float64)
    x, it, conv, h = _run("simpfem_pcg_op", A_op, M_op, b, x0, (float(tol), int(maxiter)), (hist, cap))
    if history is not None:
        history.extend(h)
    return x, it, conv
