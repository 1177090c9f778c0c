"""_cupy_fgmres / _cupy_pcg with operator and preconditioner pairs that are not a
hierarchy's own (multigrid_v4.py:416-534, solver_v2.py:551-623): the library's
device Krylov core with the two callables applied through callbacks
(simpfem_fgmres_op / simpfem_pcg_op), against the oracle's restatement --
restart cycles, lucky breakdown, the zero right-hand side and the history rule
(beta / ||b|| at each (re)start, |g_{j+1}| / ||b|| after each iteration)
identical to round-off."""

import numpy as np
import pytest

from oracle import solver as osol

pytestmark = pytest.mark.gpu


def _system(n, seed, symmetric=False):
    rng = np.random.default_rng(seed)
    Q = rng.standard_normal((n, n))
    A = Q @ Q.T + n * np.eye(n)           # SPD
    if not symmetric:
        A[0, 1] += 0.5                     # and slightly non-symmetric
    d = 1.0 / np.diag(A)
    return A, d, rng.standard_normal(n)


@pytest.mark.parametrize("restart,maxiter,tol", [(5, 40, 1e-10), (30, 30, 1e-12), (3, 7, 1e-14)])
def test_callback_fgmres_matches_oracle(cuda, restart, maxiter, tol):
    torch = cuda
    from gpu_fem.multigrid_v4 import _cupy_fgmres

    A, d, b = _system(24, restart)
    At, dt = torch.as_tensor(A, device="cuda"), torch.as_tensor(d, device="cuda")
    hist, ref_hist = [], []
    x, it, conv = _cupy_fgmres(lambda v: At @ v, torch.as_tensor(b, device="cuda"), lambda v: dt * v, tol=tol,
                               maxiter=maxiter, restart=restart, history=hist)
    xr, itr, convr = osol.fgmres(lambda v: A @ v, b, lambda v: d * v, tol=tol, maxiter=maxiter, restart=restart,
                                 history=ref_hist)
    assert (it, conv) == (itr, convr)
    assert len(hist) == len(ref_hist)
    np.testing.assert_allclose(hist, ref_hist, rtol=1e-10, atol=1e-14)
    np.testing.assert_allclose(x.cpu().numpy(), xr, rtol=1e-10, atol=1e-12 * np.abs(xr).max())


def test_callback_fgmres_initial_guess_zero_rhs_and_breakdown(cuda):
    torch = cuda
    from gpu_fem.multigrid_v4 import _cupy_fgmres

    x, it, conv = _cupy_fgmres(lambda v: v, torch.zeros(6, dtype=torch.float64, device="cuda"), lambda v: v,
                               history=[])
    assert (it, conv) == (0, True) and float(torch.linalg.norm(x)) == 0.0
    # identity operator, identity preconditioner: one iteration is exact (lucky breakdown)
    hist = []
    b = torch.arange(1.0, 7.0, dtype=torch.float64, device="cuda")
    x, it, conv = _cupy_fgmres(lambda v: v, b, lambda v: v, tol=1e-12, maxiter=10, restart=5, history=hist)
    assert conv and it == 1 and torch.allclose(x, b)
    assert hist[0] == 1.0 and hist[1] <= 1e-15
    # an initial guess is used as given
    A, d, bb = _system(16, 7)
    x0 = np.random.default_rng(8).standard_normal(16)
    At, dt = torch.as_tensor(A, device="cuda"), torch.as_tensor(d, device="cuda")
    hist, ref_hist = [], []
    x, it, conv = _cupy_fgmres(lambda v: At @ v, torch.as_tensor(bb, device="cuda"), lambda v: dt * v,
                               x0=torch.as_tensor(x0, device="cuda"), tol=1e-11, maxiter=30, restart=6, history=hist)
    xr, itr, convr = osol.fgmres(lambda v: A @ v, bb, lambda v: d * v, x0=x0, tol=1e-11, maxiter=30, restart=6,
                                 history=ref_hist)
    assert (it, conv) == (itr, convr)
    np.testing.assert_allclose(hist, ref_hist, rtol=1e-10, atol=1e-14)


@pytest.mark.parametrize("maxiter,tol", [(50, 1e-12), (4, 1e-14)])
def test_callback_pcg_matches_oracle(cuda, maxiter, tol):
    torch = cuda
    from gpu_fem.solver_v2 import _cupy_pcg

    A, d, b = _system(20, maxiter, symmetric=True)
    At, dt = torch.as_tensor(A, device="cuda"), torch.as_tensor(d, device="cuda")
    hist, ref_hist = [], []
    # a matrix operand as well as a callable (the reference accepts both)
    x, it, conv = _cupy_pcg(At, torch.as_tensor(b, device="cuda"), lambda v: dt * v, tol=tol, maxiter=maxiter,
                            history=hist)
    xr, itr, convr = osol.pcg(lambda v: A @ v, b, lambda v: d * v, tol=tol, maxiter=maxiter, history=ref_hist)
    assert (it, conv) == (itr, convr)
    np.testing.assert_allclose(hist, ref_hist, rtol=1e-9, atol=1e-14)
    np.testing.assert_allclose(x.cpu().numpy(), xr, rtol=1e-9, atol=1e-11 * np.abs(xr).max())


def test_callback_failure_surfaces(cuda):
    torch = cuda
    from gpu_fem.multigrid_v4 import _cupy_fgmres

    def bad(v):
        raise FloatingPointError("operator failed")

    with pytest.raises(FloatingPointError):
        _cupy_fgmres(bad, torch.ones(5, dtype=torch.float64, device="cuda"), lambda v: v, tol=1e-8, maxiter=5,
                     restart=5)
    # the library stays usable afterwards
    x, it, conv = _cupy_fgmres(lambda v: 2.0 * v, torch.ones(5, dtype=torch.float64, device="cuda"), lambda v: v,
                               tol=1e-12, maxiter=5, restart=5)
    assert conv and torch.allclose(x, torch.full((5,), 0.5, dtype=torch.float64, device="cuda"))
