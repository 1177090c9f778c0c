"""The allocation-free true-residual guard against the allocating one.

simpfem_true_residual_noalloc serves callers whose host framework owns all
device memory and forbids a library's own cudaMalloc/cudaFree; it must give the
same guard value as simpfem_true_residual (which keeps work buffers in the mesh
handle) on the same state, call after call, and return b - K(E) x in the
caller's buffer.  Collected last on purpose (file name), and written to pass both
alone in a fresh process and after the other GPU tests.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_true_residual_noalloc_matches_allocating_entry(cuda):
    torch = cuda
    from gpu_fem import _lib, presets
    from gpu_fem.bc_generator import generate_bc
    from gpu_fem.pub_simp_solver import KE_UNIT_3D, _edof_table_3d
    from gpu_fem.solver_v2 import MatrixFreeKff

    spec = presets.get_preset("cantilever_3d")
    bc = generate_bc(spec)
    free = bc.free_dofs.astype(np.int32)
    mf = MatrixFreeKff(torch.as_tensor(_edof_table_3d(spec.nelx, spec.nely, spec.nelz), device="cuda"),
                       KE_UNIT_3D, free, len(free), bc.ndof)
    rng = np.random.default_rng(21)
    n_elem = spec.nelx * spec.nely * spec.nelz
    E = torch.as_tensor(1e-3 + rng.random(n_elem), device="cuda")
    free_t = torch.as_tensor(free.astype(np.int64), device="cuda")
    stream = _lib.stream_ptr()
    for trial in range(2):
        x_free = torch.as_tensor(rng.standard_normal(len(free)), device="cuda")
        b_free = torch.as_tensor(bc.F[free] + 1e-3 * rng.standard_normal(len(free)), device="cuda")
        ref = ctypes.c_double()
        _lib.call("simpfem_true_residual", mf.mesh.handle, _lib.ptr(E), _lib.ptr(b_free), _lib.ptr(x_free),
                  ctypes.byref(ref), stream)
        x_full = torch.zeros(bc.ndof, dtype=torch.float64, device="cuda")
        b_full = torch.zeros(bc.ndof, dtype=torch.float64, device="cuda")
        x_full[free_t] = x_free
        b_full[free_t] = b_free
        r_full = torch.full((bc.ndof,), float("nan"), dtype=torch.float64, device="cuda")
        for call in range(2):
            out = ctypes.c_double()
            _lib.call("simpfem_true_residual_noalloc", mf.mesh.handle, _lib.ptr(E), _lib.ptr(b_full),
                      _lib.ptr(x_full), _lib.ptr(r_full), ctypes.byref(out), stream)
            assert abs(out.value - ref.value) <= 1e-12 * ref.value, (trial, call, out.value, ref.value)
            r_expected = b_free - mf.matvec(x_free, E)
            r = r_full[free_t]
            assert float(torch.linalg.norm(r - r_expected)) <= 1e-13 * float(torch.linalg.norm(r_expected))
            fixed = torch.ones(bc.ndof, dtype=torch.bool, device="cuda")
            fixed[free_t] = False
            assert bool(torch.all(r_full[fixed] == 0))
