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


def _banded_spd(n, bw, seed, scales=None):
    rng = np.random.default_rng(seed)
    A = np.zeros((n, n))
    for d in range(1, bw + 1):
        v = rng.standard_normal(n - d)
        A[np.arange(d, n), np.arange(n - d)] = v
        A[np.arange(n - d), np.arange(d, n)] = v
    A[np.arange(n), np.arange(n)] = 2.0 * bw + 1.0 + rng.uniform(0.0, 1.0, n)  # diagonally dominant
    if scales is not None:
        A *= np.sqrt(np.outer(scales, scales))
    return A


@pytest.mark.parametrize("n,bw", [(300, 1), (500, 37), (1000, 219), (1000, 999), (3960, 219), (2049, 64)])
def test_banded_inverse_factor_matches_numpy(cuda, n, bw):
    """The coarsest matrix is banded; the recursion multiplies only the band's
    non-zero blocks, measured from the data (bw = n - 1 is the dense case)."""
    A = _banded_spd(n, bw, n + bw)
    Li, info = _factor(cuda, A)
    ref = np.linalg.inv(np.linalg.cholesky(A))
    assert info == 0
    assert np.abs(Li - ref).max() <= 1e-12 * np.abs(ref).max()
    assert np.all(np.triu(Li, 1) == 0.0)


def test_banded_with_one_wide_row_and_scales(cuda):
    # one entry far below the band widens the measured band to that row's reach;
    # SIMP-like scales (1e-9 .. 1) as on a coarse level with void regions
    n, bw = 1500, 40
    rng = np.random.default_rng(5)
    A = _banded_spd(n, bw, 6, scales=10.0 ** rng.uniform(-9, 0, n))
    A[1200, 100] = A[100, 1200] = 0.5 * np.sqrt(A[1200, 1200] * A[100, 100])
    b = rng.standard_normal(n)
    Li, info = _factor(cuda, A)
    assert info == 0
    x = Li.T @ (Li @ b)
    assert np.linalg.norm(A @ x - b) <= 1e-8 * np.linalg.norm(b)


@pytest.mark.parametrize("n,bw", [(600, 300), (1000, 219), (1600, 760)])
def test_band_path_repeatable(cuda, n, bw):
    """The band path (one thread-block cluster exchanging tiles through shared
    memory and L2) gives the same bits on every run, at band widths below, at and
    beyond the cluster's eight tile rows, up to its widest band (24 tiles)."""
    A = _banded_spd(n, bw, 11 * n + bw)
    ref = np.linalg.inv(np.linalg.cholesky(A))
    first = None
    for _ in range(8):
        Li, info = _factor(cuda, A)
        assert info == 0
        assert np.abs(Li - ref).max() <= 1e-12 * np.abs(ref).max()
        if first is None:
            first = Li
        else:
            assert np.array_equal(Li, first)


def test_wide_band_takes_the_recursion(cuda):
    # 26 tiles below the diagonal: beyond the band path, the recursion factors it
    n, bw = 1200, 820
    A = _banded_spd(n, bw, 3)
    Li, info = _factor(cuda, A)
    ref = np.linalg.inv(np.linalg.cholesky(A))
    assert info == 0
    assert np.abs(Li - ref).max() <= 1e-12 * np.abs(ref).max()
