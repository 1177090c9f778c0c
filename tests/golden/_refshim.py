"""Load the reference ``gpu_fem`` package on CPU for fixture generation only.

The reference computes with CuPy on a GPU.  Its arithmetic is plain BLAS /
sparse-BLAS with standard semantics, so a numpy-backed stand-in for the
handful of ``cupy`` / ``cupyx.scipy`` names it touches lets the reference's
own unmodified Python (``MatrixFreeKff``, ``GalerkinMatFreeGMG``,
``_cupy_fgmres`` ...) run on the host.  This module is used only by
``make_golden.py`` in this folder, which runs where the reference source tree
is readable; nothing in the tests, the package or the benchmark imports it.
"""

from __future__ import annotations

import importlib
import importlib.util
import os
import sys
import types

import numpy as np
import scipy.linalg
import scipy.sparse

def _ref_root() -> str:
    root = os.environ.get("SIMPFEM_REFERENCE_ROOT")
    if not root or not os.path.isdir(os.path.join(root, "src", "gpu_fem")):
        raise RuntimeError("set SIMPFEM_REFERENCE_ROOT to a checkout of the reference project "
                           "(the folder holding src/gpu_fem and experiments/)")
    return root


class _Pool:
    def free_all_blocks(self):
        return None

    def used_bytes(self):
        return 0

    def total_bytes(self):
        return 0

    def n_free_blocks(self):
        return 0


def _make_cupy_module() -> types.ModuleType:
    cp = types.ModuleType("cupy")
    for name in dir(np):
        if not name.startswith("__"):
            setattr(cp, name, getattr(np, name))
    cp.ndarray = np.ndarray
    cp.__version__ = "13.0.0"
    cp.asnumpy = np.asarray
    cp.linalg = np.linalg
    cp.get_default_memory_pool = lambda: _Pool()
    cp.get_default_pinned_memory_pool = lambda: _Pool()

    cuda = types.SimpleNamespace()
    cuda.Stream = types.SimpleNamespace(null=types.SimpleNamespace(synchronize=lambda: None))
    cuda.runtime = types.SimpleNamespace(memGetInfo=lambda: (0, 0))
    cp.cuda = cuda

    class _RS:
        def __init__(self, seed):
            self._rs = np.random.RandomState(seed)

        def standard_normal(self, n, dtype=np.float64):
            return self._rs.standard_normal(n).astype(dtype)

    cp.random = types.SimpleNamespace(RandomState=_RS)

    class _Scalar(np.ndarray):
        """0-d result with CuPy's ``.get()`` (device -> host copy)."""

        def get(self):
            return np.asarray(self)

    cp.dot = lambda a, b, out=None: np.asarray(np.dot(a, b)).view(_Scalar)
    return cp


def install() -> None:
    """Register the stand-ins and an import-safe ``gpu_fem`` package object."""
    sys.dont_write_bytecode = True
    if "gpu_fem" in sys.modules and getattr(sys.modules["gpu_fem"], "_refshim", False):
        return
    sys.modules["cupy"] = _make_cupy_module()
    cupyx = types.ModuleType("cupyx")
    cupyx_scipy = types.ModuleType("cupyx.scipy")
    cupyx_sparse = types.ModuleType("cupyx.scipy.sparse")
    for name in dir(scipy.sparse):
        if not name.startswith("__"):
            setattr(cupyx_sparse, name, getattr(scipy.sparse, name))
    cupyx_linalg = types.ModuleType("cupyx.scipy.linalg")
    cupyx_linalg.solve_triangular = scipy.linalg.solve_triangular
    cupyx.scipy = cupyx_scipy
    cupyx_scipy.sparse = cupyx_sparse
    cupyx_scipy.linalg = cupyx_linalg
    sys.modules.update(
        {
            "cupyx": cupyx,
            "cupyx.scipy": cupyx_scipy,
            "cupyx.scipy.sparse": cupyx_sparse,
            "cupyx.scipy.linalg": cupyx_linalg,
        }
    )
    # The shipped package __init__ pulls in modules that fail at import time;
    # register an empty package object whose __path__ points at the sources.
    pkg = types.ModuleType("gpu_fem")
    pkg.__path__ = [os.path.join(_ref_root(), "src", "gpu_fem")]
    pkg._refshim = True
    sys.modules["gpu_fem"] = pkg
    paths = importlib.import_module("gpu_fem.paths")
    paths.ensure_local_paths = lambda *a, **k: None


def load(name: str):
    install()
    return importlib.import_module(f"gpu_fem.{name}")


_COPY_ROOT = None


def _copy_root() -> str:
    """Scratch folder for copies of the reference's scripts: SIMPFEM_REFERENCE_COPY,
    else a fresh temporary folder per process."""
    global _COPY_ROOT
    if _COPY_ROOT is None:
        import tempfile

        _COPY_ROOT = os.environ.get("SIMPFEM_REFERENCE_COPY") or tempfile.mkdtemp(prefix="simpfem_refcopy_")
    return _COPY_ROOT


def _copied_script(rel: str) -> str:
    """Copy one reference script under the scratch folder and return the copy's path.

    The experiment scripts derive their root folder from their own location
    and create scratch folders beneath it at import time; running a copy keeps
    every such write out of the read-only reference tree.
    """
    import shutil

    src = os.path.join(_ref_root(), rel)
    dst = os.path.join(_copy_root(), rel)
    os.makedirs(os.path.dirname(dst), exist_ok=True)
    shutil.copyfile(src, dst)
    return dst


def load_paper4_runner():
    install()
    path = _copied_script(os.path.join("experiments", "paper4", "run_experiments_e1_e10.py"))
    spec = importlib.util.spec_from_file_location("paper4_runner", path)
    module = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(module)
    return module


def load_driver_module(rel: str):
    """Import a reference experiment driver (from a copy) without running its main()."""
    install()
    path = _copied_script(rel)
    _copied_script(os.path.join("experiments", "paper4", "run_experiments_e1_e10.py"))
    spec = importlib.util.spec_from_file_location("ref_driver_" + os.path.basename(rel)[:-3], path)
    module = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(module)
    return module


def run_driver(rel: str, argv: list[str]) -> None:
    """Run a reference experiment driver unchanged (from a copy) with ``argv``."""
    import runpy

    install()
    path = _copied_script(rel)
    _copied_script(os.path.join("experiments", "paper4", "run_experiments_e1_e10.py"))
    old = sys.argv
    sys.argv = [path] + list(argv)
    try:
        runpy.run_path(path, run_name="__main__")
    finally:
        sys.argv = old
