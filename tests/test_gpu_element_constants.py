"""The element stiffness a mesh is created with is the one its operator applies.

The sweep kernels read the unit element stiffness (its Walsh blocks) from each
device's constant bank, so the meshes alive on a device share one stiffness.
simpfem_mesh_create must refuse a stiffness that differs from the one of the
meshes alive on the device (instead of silently changing their operator), and
once none is left the next mesh installs its own.  Checked with the hex8
stiffness at nu = 0.3 (the reference's KE_UNIT_3D) and nu = 0.25 against an
element-by-element numpy product; the second half runs in a fresh process so
that no other test's mesh is alive.
"""

import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_SCRIPT = r"""
import ctypes, sys
import numpy as np
import torch
sys.path[:0] = [{root!r}, {pkg!r}]
from gpu_fem import _lib
from oracle.solver import edof_table, ke_unit_3d

def create(ke, dims, free):
    h = ctypes.c_void_p()
    ke = np.ascontiguousarray(ke, dtype=np.float64)
    st = _lib.load().simpfem_mesh_create(*dims, free.ctypes.data_as(ctypes.c_void_p), len(free),
                                         ke.ctypes.data_as(ctypes.c_void_p), ctypes.byref(h))
    return st, h

def check(h, ke, dims, free):
    nx, ny, nz = dims
    ndof = 3 * (nx + 1) * (ny + 1) * (nz + 1)
    rng = np.random.default_rng(3)
    E = 0.1 + rng.random(nx * ny * nz)
    u = rng.standard_normal(len(free))
    full = np.zeros(ndof); full[free] = u
    ed = edof_table(nx, ny, nz)
    y = np.zeros(ndof)
    np.add.at(y, ed, (ke @ full[ed].T * E[None, :]).T)
    Et, ut = torch.as_tensor(E, device="cuda"), torch.as_tensor(u, device="cuda")
    yt = torch.empty(len(free), dtype=torch.float64, device="cuda")
    _lib.call("simpfem_matvec", h, _lib.F64, _lib.ptr(Et), _lib.ptr(ut), _lib.ptr(yt), _lib.stream_ptr())
    err = np.linalg.norm(yt.cpu().numpy() - y[free]) / np.linalg.norm(y[free])
    assert err <= 1e-13, err

dims = (5, 3, 4)
ndof = 3 * 6 * 4 * 5
free = np.arange(3 * 4 * 5, ndof, dtype=np.int32)   # x = 0 face clamped
lib = _lib.load()
k25, k30 = ke_unit_3d(nu=0.25), ke_unit_3d(nu=0.3)
st, hb = create(k25, dims, free); assert st == 0
check(hb, k25, dims, free)
st, ha = create(k30, dims, free); assert st == 1, st      # refused while the nu=0.25 mesh lives
assert b"differs" in lib.simpfem_last_error()
st, hb2 = create(k25, dims, free); assert st == 0         # the same stiffness is shared
check(hb2, k25, dims, free)
lib.simpfem_mesh_destroy(hb); lib.simpfem_mesh_destroy(hb2)
st, ha = create(k30, dims, free); assert st == 0          # none left: nu = 0.3 installs
check(ha, k30, dims, free)
lib.simpfem_mesh_destroy(ha)
print("ok")
"""


def test_mismatched_stiffness_refused_in_process(cuda):
    from gpu_fem import _lib
    from gpu_fem.pub_simp_solver import KE_UNIT_3D
    from oracle.solver import ke_unit_3d

    free = np.arange(36, 360, dtype=np.int32)
    lib = _lib.load()
    ha, hb = ctypes.c_void_p(), ctypes.c_void_p()
    ke = np.ascontiguousarray(KE_UNIT_3D, dtype=np.float64)
    _lib.call("simpfem_mesh_create", 5, 3, 4, free.ctypes.data_as(ctypes.c_void_p), len(free),
              ke.ctypes.data_as(ctypes.c_void_p), ctypes.byref(ha))
    try:
        k25 = np.ascontiguousarray(ke_unit_3d(nu=0.25))
        with pytest.raises(_lib.SimpfemError, match="EINVAL.*differs"):
            _lib.call("simpfem_mesh_create", 5, 3, 4, free.ctypes.data_as(ctypes.c_void_p), len(free),
                      k25.ctypes.data_as(ctypes.c_void_p), ctypes.byref(hb))
    finally:
        lib.simpfem_mesh_destroy(ha)


def test_each_stiffness_applied_in_a_fresh_process(cuda):
    code = _SCRIPT.format(root=ROOT, pkg=os.path.join(ROOT, "solver-admissibility-and-guarded-floor-selection_b200"))
    res = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert res.returncode == 0 and res.stdout.strip().endswith("ok"), res.stdout + res.stderr
