"""The allocation-free true-residual guard against the allocating one.

simpfem_true_residual_noalloc serves callers whose host framework owns all
device memory and forbids a library's own cudaMalloc/cudaFree; it must give the
same guard value as simpfem_true_residual (which keeps work buffers in the mesh
handle) on the same state, call after call, return b - K(E) x in the caller's
buffer, ignore loads the caller leaves at constrained DOFs, allocate nothing
(checked on a fresh mesh handle by the library's allocation counter and the
device's free memory), and reject a null argument or a mesh above its
8,388,608-DOF maximum before launching anything.  Collected last on purpose
(file name), and written to pass both alone in a fresh process and after the
other GPU tests.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case():
    from gpu_fem import presets
    from gpu_fem.bc_generator import generate_bc

    spec = presets.get_preset("cantilever_3d")
    return spec, generate_bc(spec)


def _fresh_mesh(spec, free):
    """A mesh handle made directly through the C ABI (no cached handle)."""
    from gpu_fem import _lib
    from gpu_fem.pub_simp_solver import KE_UNIT_3D

    h = ctypes.c_void_p()
    ke = np.ascontiguousarray(KE_UNIT_3D, dtype=np.float64)
    _lib.call("simpfem_mesh_create", spec.nelx, spec.nely, spec.nelz, free.ctypes.data_as(ctypes.c_void_p),
              len(free), ke.ctypes.data_as(ctypes.c_void_p), ctypes.byref(h))
    return h


def test_true_residual_noalloc_matches_allocating_entry(cuda):
    torch = cuda
    from gpu_fem import _lib
    from gpu_fem.pub_simp_solver import KE_UNIT_3D, _edof_table_3d
    from gpu_fem.solver_v2 import MatrixFreeKff

    spec, bc = _case()
    free = bc.free_dofs.astype(np.int32)
    mf = MatrixFreeKff(torch.as_tensor(_edof_table_3d(spec.nelx, spec.nely, spec.nelz), device="cuda"),
                       KE_UNIT_3D, free, len(free), bc.ndof)
    rng = np.random.default_rng(21)
    n_elem = spec.nelx * spec.nely * spec.nelz
    E = torch.as_tensor(1e-3 + rng.random(n_elem), device="cuda")
    free_t = torch.as_tensor(free.astype(np.int64), device="cuda")
    fixed = torch.ones(bc.ndof, dtype=torch.bool, device="cuda")
    fixed[free_t] = False
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
        if trial == 1:
            # loads left at constrained DOFs (reactions, say) do not enter the guard
            b_full[fixed] = torch.as_tensor(rng.standard_normal(int(fixed.sum())), device="cuda")
        r_full = torch.full((bc.ndof,), float("nan"), dtype=torch.float64, device="cuda")
        for call in range(2):
            out = ctypes.c_double()
            _lib.call("simpfem_true_residual_noalloc", mf.mesh.handle, _lib.ptr(E), _lib.ptr(b_full),
                      _lib.ptr(x_full), _lib.ptr(r_full), ctypes.byref(out), stream)
            assert abs(out.value - ref.value) <= 1e-12 * ref.value, (trial, call, out.value, ref.value)
            r_expected = b_free - mf.matvec(x_free, E)
            r = r_full[free_t]
            assert float(torch.linalg.norm(r - r_expected)) <= 1e-13 * float(torch.linalg.norm(r_expected))
            assert bool(torch.all(r_full[fixed] == 0))


def test_true_residual_noalloc_allocates_nothing(cuda):
    torch = cuda
    from gpu_fem import _lib

    spec, bc = _case()
    free = np.ascontiguousarray(bc.free_dofs, dtype=np.int32)
    rng = np.random.default_rng(5)
    n_elem = spec.nelx * spec.nely * spec.nelz
    E = torch.as_tensor(1e-3 + rng.random(n_elem), device="cuda")
    b = torch.zeros(bc.ndof, dtype=torch.float64, device="cuda")
    x = torch.zeros(bc.ndof, dtype=torch.float64, device="cuda")
    free_t = torch.as_tensor(free.astype(np.int64), device="cuda")
    b[free_t] = torch.as_tensor(rng.standard_normal(len(free)), device="cuda")
    x[free_t] = torch.as_tensor(rng.standard_normal(len(free)), device="cuda")
    r = torch.empty(bc.ndof, dtype=torch.float64, device="cuda")
    stream = _lib.stream_ptr()
    lib = _lib.load()
    warm = _fresh_mesh(spec, free)
    fresh = _fresh_mesh(spec, free)
    try:
        out = ctypes.c_double()
        # one call on another handle first: loads the library's kernels and looks up
        # the scratch array's address, which happen once per process and device
        _lib.call("simpfem_true_residual_noalloc", warm, _lib.ptr(E), _lib.ptr(b), _lib.ptr(x), _lib.ptr(r),
                  ctypes.byref(out), stream)
        torch.cuda.synchronize()
        allocs0 = int(lib.simpfem_device_alloc_count())
        free0 = torch.cuda.mem_get_info()[0]
        values = []
        for _ in range(2):
            _lib.call("simpfem_true_residual_noalloc", fresh, _lib.ptr(E), _lib.ptr(b), _lib.ptr(x), _lib.ptr(r),
                      ctypes.byref(out), stream)
            values.append(out.value)
        torch.cuda.synchronize()
        assert int(lib.simpfem_device_alloc_count()) == allocs0
        # any cudaMalloc takes at least a 2 MiB page from the device
        assert free0 - torch.cuda.mem_get_info()[0] < 2 << 20
        assert values[0] == values[1] and np.isfinite(values[0])
    finally:
        lib.simpfem_mesh_destroy(warm)
        lib.simpfem_mesh_destroy(fresh)


def test_true_residual_noalloc_rejects_bad_arguments(cuda):
    torch = cuda
    from gpu_fem import _lib

    spec, bc = _case()
    free = np.ascontiguousarray(bc.free_dofs, dtype=np.int32)
    v = torch.zeros(bc.ndof, dtype=torch.float64, device="cuda")
    E = torch.ones(spec.nelx * spec.nely * spec.nelz, dtype=torch.float64, device="cuda")
    out = ctypes.c_double(-1.0)
    stream = _lib.stream_ptr()
    lib = _lib.load()
    h = _fresh_mesh(spec, free)
    try:
        for args in ((None, _lib.ptr(E), _lib.ptr(v), _lib.ptr(v), _lib.ptr(v)),
                     (h, None, _lib.ptr(v), _lib.ptr(v), _lib.ptr(v)),
                     (h, _lib.ptr(E), _lib.ptr(v), _lib.ptr(v), None)):
            with pytest.raises(_lib.SimpfemError, match="EINVAL"):
                _lib.call("simpfem_true_residual_noalloc", *args, ctypes.byref(out), stream)
        with pytest.raises(_lib.SimpfemError, match="EINVAL"):
            _lib.call("simpfem_true_residual_noalloc", h, _lib.ptr(E), _lib.ptr(v), _lib.ptr(v), _lib.ptr(v), None,
                      stream)
    finally:
        lib.simpfem_mesh_destroy(h)
    # 141^3 elements: 142^3 nodes, 8,590,536 DOFs, above the 8,388,608 maximum.  The
    # mesh is made with no free DOF (it only needs its grid); the call must refuse
    # it before any launch, so the small vectors passed are never read.
    big = ctypes.c_void_p()
    from gpu_fem.pub_simp_solver import KE_UNIT_3D

    ke = np.ascontiguousarray(KE_UNIT_3D, dtype=np.float64)
    _lib.call("simpfem_mesh_create", 141, 141, 141, None, 0, ke.ctypes.data_as(ctypes.c_void_p), ctypes.byref(big))
    try:
        launches0 = int(lib.simpfem_launch_count())
        with pytest.raises(_lib.SimpfemError, match="no-alloc maximum"):
            _lib.call("simpfem_true_residual_noalloc", big, _lib.ptr(E), _lib.ptr(v), _lib.ptr(v), _lib.ptr(v),
                      ctypes.byref(out), stream)
        assert int(lib.simpfem_launch_count()) == launches0
        assert out.value == -1.0
    finally:
        lib.simpfem_mesh_destroy(big)
