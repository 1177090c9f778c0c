"""Checkpointed guard: the FP64 true residual of the probe's iterate at r50,
read inside FGMRES (simpfem_fgmres_checked with check_true_residual), and the
policy option that lets the preserve/escalate rule read true residuals.

* the true residual the check reports equals the guard's own recomputation on
  the iterate the solve returns when the check stops it there (1e-10);
* a check that only observes leaves the solve bit-identical (history, count,
  final true residual);
* GuardedFloorPolicy(checkpoint_guard=True) records the true residuals at r50
  and at the probe's end, classifies on them, and every answer is guarded.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DIMS = (40, 20, 20)
POLICY = dict(penal=3.0, tol=1e-6, restart=300, maxiter=300, probe_iters=100, probe_r50=50,
              raised_rho_mins=(1e-3, 1e-2), cycle_precision="fp32")


def _policy(checkpoint):
    from gpu_fem.paper4 import PLAIN_JACOBI_STACK
    from gpu_fem.policy import GuardedFloorPolicy
    from gpu_fem.presets import cantilever_spec

    return GuardedFloorPolicy(cantilever_spec(*DIMS), stack=dict(PLAIN_JACOBI_STACK, fine_smoother="fp32"),
                              checkpoint_guard=checkpoint, **POLICY)


def _mask(seed, p):
    return (np.random.default_rng(seed).random(int(np.prod(DIMS))) >= p).astype(np.float64)


def test_checkpoint_true_residual_matches_guard(cuda):
    pol = _policy(False)
    d = cuda.as_tensor(_mask(5, 0.78), device="cuda")
    seen = []
    a = pol.solve_at_floor(d, 1e-12, maxiter=100, history=[], check=(50, lambda h, t: seen.append(t) or True, True))
    assert a.iters == 50 and len(seen) == 1
    assert seen[0] == pytest.approx(a.final_rel_residual, rel=1e-10)


def test_observing_check_changes_nothing(cuda):
    pol = _policy(False)
    d = cuda.as_tensor(_mask(5, 0.78), device="cuda")
    h0: list = []
    a = pol.solve_at_floor(d, 1e-12, maxiter=100, history=h0)
    h1: list = []
    seen = []
    b = pol.solve_at_floor(d, 1e-12, maxiter=100, history=h1, check=(50, lambda h, t: seen.append(t) and False, True))
    assert h0 == h1 and a.iters == b.iters and a.final_rel_residual == b.final_rel_residual
    assert len(seen) == (1 if a.iters > 50 else 0)


@pytest.mark.parametrize("seed,p", [(1, 0.2), (3, 0.7), (5, 0.78)])
def test_checkpoint_policy_rows(cuda, seed, p):
    pol = _policy(True)
    r = pol.run(cuda.as_tensor(_mask(seed, p), device="cuda"))
    assert r["checkpoint_guard"] == 1
    assert np.isfinite(r["probe_true_r50"]) and np.isfinite(r["probe_true_r100"])
    if r["probe_iters"] <= 50:
        assert r["probe_true_r50"] == r["probe_true_r100"]
    assert r["solve_converged"] == 1 and r["solve_final_rel_residual"] <= 1e-6
