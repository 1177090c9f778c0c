"""Coarsest-level dense factorisation (simpfem_dense_cholesky_inverse) against numpy.

The reference factors the coarsest matrix with cp.linalg.cholesky and treats a
failed factorisation (LinAlgError from a non-positive pivot, or a non-finite
factor) as the trigger for its eps*I regularisation
(gpu_fem/multigrid_v4.py:1308-1337).  The library returns L^{-1} instead of L;
these tests check it against numpy.linalg.inv(numpy.linalg.cholesky(A)) on
ragged sizes around the 32-row leaf and 64-row GEMM tile, and that the failure
signal fires where the reference's would.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _factor(torch, A):
    from gpu_fem import _lib

    n = A.shape[0]
    Ad = torch.as_tensor(np.ascontiguousarray(A), device="cuda")
    Li = torch.full((n, n), float("nan"), dtype=torch.float64, device="cuda")
    info = ctypes.c_int(-7)
    _lib.call("simpfem_dense_cholesky_inverse", n, _lib.ptr(Ad), _lib.ptr(Li), ctypes.byref(info),
              _lib.stream_ptr())
    return Li.cpu().numpy(), info.value


@pytest.mark.parametrize("n", [1, 5, 31, 32, 33, 64, 65, 100, 257, 1000, 2049])
def test_inverse_factor_matches_numpy(cuda, n):
    rng = np.random.default_rng(n)
    Q = rng.standard_normal((n, n))
    A = Q @ Q.T / n + np.diag(rng.uniform(0.5, 2.0, n))
    Li, info = _factor(cuda, A)
    ref = np.linalg.inv(np.linalg.cholesky(A))
    assert info == 0
    # fp64 round-off of a well-conditioned factor and inverse
    assert np.abs(Li - ref).max() <= 1e-12 * np.abs(ref).max()
    assert np.all(np.triu(Li, 1) == 0.0)


def test_ill_conditioned_solve(cuda):
    # SIMP-like spread of scales (1e-9 .. 1): the product L^{-T} L^{-1} b still
    # solves A x = b to a backward error near machine precision
    n = 700
    rng = np.random.default_rng(1)
    Q = rng.standard_normal((n, n))
    s = 10.0 ** rng.uniform(-9, 0, n)
    A = (Q @ Q.T / n + np.eye(n)) * np.sqrt(np.outer(s, s))
    b = rng.standard_normal(n)
    Li, info = _factor(cuda, A)
    assert info == 0
    x = Li.T @ (Li @ b)
    assert np.linalg.norm(A @ x - b) <= 1e-8 * np.linalg.norm(b)


def test_non_spd_reports_first_bad_pivot(cuda):
    n = 200
    rng = np.random.default_rng(2)
    Q = rng.standard_normal((n, n))
    A = Q @ Q.T / n + np.eye(n)
    A[40, 40] = -1.0e6
    _, info = _factor(cuda, A)
    assert info == 41


def test_non_finite_input_fails(cuda):
    n = 96
    A = np.eye(n)
    A[70, 3] = A[3, 70] = np.nan
    _, info = _factor(cuda, A)
    assert info != 0
