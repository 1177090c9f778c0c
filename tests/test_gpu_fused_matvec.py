"""FusedMatvec (the reference's fused FP32 / BF16 operator class) against the
oracle's restatement of its arithmetic.

Both dtypes accumulate in float32 on the GPU and float64 in the oracle; with
the same bfloat16 rounding of u and KE the results agree to 1e-5 of the
largest entry.  matvec_full covers every DOF (fixed rows included, as the
reference's scatter does), matvec the free rows only.
"""

import numpy as np
import pytest

from oracle import solver as osol

pytestmark = pytest.mark.gpu


def _setup(cuda, dims):
    from gpu_fem.cuda_fused_matvec import FusedMatvec
    from gpu_fem.pub_simp_solver import KE_UNIT_3D, _edof_table_3d

    edof = cuda.as_tensor(_edof_table_3d(*dims).astype(np.int64), device="cuda")
    ndof = 3 * (dims[0] + 1) * (dims[1] + 1) * (dims[2] + 1)
    return FusedMatvec(edof, cuda.as_tensor(KE_UNIT_3D, device="cuda"), ndof), ndof, KE_UNIT_3D


@pytest.mark.parametrize("dims", [(12, 6, 4), (24, 12, 6), (31, 9, 17)])
@pytest.mark.parametrize("dtype", ["fp32", "bf16"])
def test_matvec_full_matches_oracle(cuda, dims, dtype):
    fm, ndof, ke = _setup(cuda, dims)
    rng = np.random.default_rng(sum(dims))
    u = rng.standard_normal(ndof).astype(np.float32)
    E = (1e-3 + rng.random(dims[0] * dims[1] * dims[2])).astype(np.float32)
    y = fm.matvec_full(cuda.as_tensor(u, device="cuda"), cuda.as_tensor(E, device="cuda"), dtype=dtype)
    ref = osol.fused_matvec_full(*dims, u, E, ke, dtype)
    assert y.dtype == cuda.float32 and y.shape == (ndof,)
    np.testing.assert_allclose(y.cpu().numpy(), ref, rtol=0, atol=1e-5 * np.abs(ref).max())


def test_matvec_restricts_to_free_dofs(cuda):
    dims = (24, 12, 6)
    fm, ndof, ke = _setup(cuda, dims)
    free = np.arange(3 * 7 * 13, ndof)  # x = 0 face clamped
    rng = np.random.default_rng(2)
    u_free = rng.standard_normal(free.size).astype(np.float32)
    E = (1e-3 + rng.random(dims[0] * dims[1] * dims[2])).astype(np.float32)
    y = fm.matvec(cuda.as_tensor(u_free, device="cuda"), cuda.as_tensor(E, device="cuda"),
                  cuda.as_tensor(free.astype(np.int32), device="cuda"))
    u_full = np.zeros(ndof, dtype=np.float32)
    u_full[free] = u_free
    ref = osol.fused_matvec_full(*dims, u_full, E, ke, "fp32")[free]
    np.testing.assert_allclose(y.cpu().numpy(), ref, rtol=0, atol=1e-5 * np.abs(ref).max())


def test_bf16_differs_from_fp32_by_rounding_only(cuda):
    dims = (12, 6, 4)
    fm, ndof, ke = _setup(cuda, dims)
    u = np.random.default_rng(9).standard_normal(ndof).astype(np.float32)
    E = np.ones(dims[0] * dims[1] * dims[2], dtype=np.float32)
    uu, EE = cuda.as_tensor(u, device="cuda"), cuda.as_tensor(E, device="cuda")
    a = fm.matvec_full(uu, EE, dtype="fp32").cpu().numpy()
    b = fm.matvec_full(uu, EE, dtype="bf16").cpu().numpy()
    rel = np.abs(a - b).max() / np.abs(a).max()
    assert 1e-5 < rel < 3e-2  # bfloat16 has an 8-bit significand


def test_invalid_arguments(cuda):
    from gpu_fem.cuda_fused_matvec import FusedMatvec

    fm, ndof, ke = _setup(cuda, (12, 6, 4))
    with pytest.raises(ValueError):
        fm.matvec_full(cuda.zeros(ndof, device="cuda"), cuda.ones(288, device="cuda"), dtype="fp16")
    with pytest.raises(ValueError):
        FusedMatvec(cuda.zeros((10, 8), dtype=cuda.int64, device="cuda"), cuda.as_tensor(ke, device="cuda"), 30)
