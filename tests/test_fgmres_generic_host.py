"""The generic form of _cupy_fgmres (any operator / preconditioner pair that is
not a hierarchy's own fine operator and apply; multigrid_v4.py:416-534) run
on host tensors through stand-ins for the device helpers, against the
oracle's restatement: restart cycles, lucky breakdown, the zero right-hand
side and the history rule (beta / ||b|| at each (re)start, |g_{j+1}| / ||b||
after each iteration) identical to round-off."""

import numpy as np
import pytest

from gpu_fem import _lib
from gpu_fem import multigrid_v4 as mg
from oracle import solver as osol


@pytest.fixture
def host_tensors(monkeypatch):
    import torch

    monkeypatch.setattr(_lib, "require_cuda", lambda: torch)
    monkeypatch.setattr(_lib, "as_cuda", lambda x, dtype: torch.as_tensor(np.asarray(x), dtype=dtype).clone())
    monkeypatch.setattr(mg, "_native_gmg", lambda A, M: None)
    return torch


def _system(n, seed):
    rng = np.random.default_rng(seed)
    Q = rng.standard_normal((n, n))
    A = Q @ Q.T + n * np.eye(n)           # SPD
    A[0, 1] += 0.5                         # and slightly non-symmetric
    d = 1.0 / np.diag(A)
    return A, d, rng.standard_normal(n)


@pytest.mark.parametrize("restart,maxiter,tol", [(5, 40, 1e-10), (30, 30, 1e-12), (3, 7, 1e-14)])
def test_generic_fgmres_matches_oracle(host_tensors, restart, maxiter, tol):
    torch = host_tensors
    A, d, b = _system(24, restart)
    At, dt = torch.as_tensor(A), torch.as_tensor(d)
    hist, ref_hist = [], []
    x, it, conv = mg._cupy_fgmres(lambda v: At @ v, torch.as_tensor(b), lambda v: dt * v, tol=tol,
                                  maxiter=maxiter, restart=restart, history=hist)
    xr, itr, convr = osol.fgmres(lambda v: A @ v, b, lambda v: d * v, tol=tol, maxiter=maxiter, restart=restart,
                                 history=ref_hist)
    assert (it, conv) == (itr, convr)
    assert len(hist) == len(ref_hist)
    # relative residuals: equal to 1e-10 relative down to 1e-14 absolute (round-off at convergence)
    np.testing.assert_allclose(hist, ref_hist, rtol=1e-10, atol=1e-14)
    np.testing.assert_allclose(x.numpy(), xr, rtol=1e-10, atol=1e-12 * np.abs(xr).max())


def test_generic_fgmres_zero_rhs_and_lucky_breakdown(host_tensors):
    torch = host_tensors
    x, it, conv = mg._cupy_fgmres(lambda v: v, torch.zeros(6, dtype=torch.float64), lambda v: v, history=[])
    assert (it, conv) == (0, True) and float(torch.linalg.norm(x)) == 0.0
    # identity operator, identity preconditioner: one iteration is exact
    hist = []
    b = torch.arange(1.0, 7.0, dtype=torch.float64)
    x, it, conv = mg._cupy_fgmres(lambda v: v, b, lambda v: v, tol=1e-12, maxiter=10, restart=5, history=hist)
    assert conv and it == 1 and torch.allclose(x, b)
    assert hist[0] == 1.0 and hist[1] <= 1e-15
