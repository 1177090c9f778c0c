"""The cupy calls the reference's phase-5 drivers make around the solve, on torch.

The drivers (run_gmg_floor_detector_prospective.py, _density_field.py,
run_gmg_fixed_floor_controls.py, run_gmg_floor_rule_check.py) do their linear
algebra through ``gpu_fem`` and ``_build_components``; cupy only builds the
moduli, takes norms and dot products (read back with ``.get()``), synchronises
and snapshots memory
(run_gmg_floor_detector_prospective.py:101-112, :204-248).  Those drivers put
``<root>/src`` first on ``sys.path``; with this directory as that ``src``, their
``import cupy`` resolves here and the calls act on torch tensors on the current
CUDA device, which is what this library's ``gpu_fem`` takes and returns.  Only
that surface is provided: anything else raises AttributeError.
"""

from __future__ import annotations

import numpy as np
import torch

float64 = torch.float64
float32 = torch.float32
int32 = torch.int32
int64 = torch.int64
bool_ = torch.bool


def asarray(a, dtype=None):
    if torch.is_tensor(a):
        return a.to(device="cuda", dtype=dtype) if dtype is not None else a.to(device="cuda")
    return torch.as_tensor(np.asarray(a), dtype=dtype, device="cuda")


def zeros(shape, dtype=float64):
    return torch.zeros(shape, dtype=dtype, device="cuda")


class _DeviceScalar(torch.Tensor):
    """A 0-d device result with cupy's ``.get()``, the copy to the host as a numpy
    scalar (run_gmg_fixed_floor_controls.py:128 reads the compliance so)."""

    def get(self):
        return self.detach().cpu().numpy()


def dot(a, b):
    return torch.dot(a.reshape(-1), b.reshape(-1)).as_subclass(_DeviceScalar)


def asnumpy(a):
    return a.detach().cpu().numpy() if torch.is_tensor(a) else np.asarray(a)


class linalg:
    @staticmethod
    def norm(x, ord=None):
        return torch.linalg.vector_norm(x.reshape(-1), ord=2 if ord is None else ord)


class _NullStream:
    @staticmethod
    def synchronize():
        torch.cuda.synchronize()


class _Runtime:
    @staticmethod
    def memGetInfo():
        return torch.cuda.mem_get_info()


class cuda:
    class Stream:
        null = _NullStream()

    runtime = _Runtime()


class _MemoryPool:
    """torch's caching allocator in place of cupy's pool: bytes in use and held."""

    def used_bytes(self) -> int:
        return int(torch.cuda.memory_allocated())

    def total_bytes(self) -> int:
        return int(torch.cuda.memory_reserved())


class _PinnedMemoryPool:
    def n_free_blocks(self) -> int:
        return 0


def get_default_memory_pool():
    return _MemoryPool()


def get_default_pinned_memory_pool():
    return _PinnedMemoryPool()
