"""Host control of the learned floor policy (LearnedFloorPolicy.run), without a
GPU: the proposer's pooling and softmax and the solves are replaced by scripted
stand-ins, so the decision at r50 and the attempt order are exercised on their
own -- a confident proposal stops the probe at r50 and tries its rung first,
the plain rule's rung last; an unconfident one lets the probe run on and the
plain r50/r100 rule decide; the high-residual rule stops the probe whatever
the network says; a probe that converges before r50 is reused; a wrong
proposal costs extra solves, and the FP64 guard still judges every answer."""

import numpy as np
import pytest

from gpu_fem.floor_proposer import LearnedFloorPolicy
from gpu_fem.policy import FloorAttempt


def _hist(r50, r_end, n):
    h = list(np.geomspace(1.0, r50, 51)) if n >= 50 else list(np.geomspace(1.0, r_end, n + 1))
    if n > 50:
        h += list(np.geomspace(r50, r_end, n - 49))[1:]
    return h


def _policy(script, prob, min_confidence=0.5):
    """script[rho_min] -> successive (iters, reported, true_rel, r50, r_end);
    prob: the proposer's softmax at r50."""
    p = object.__new__(LearnedFloorPolicy)
    p.penal, p.tol, p.restart, p.maxiter = 4.5, 1e-6, 300, 300
    p.probe_iters, p.probe_r50 = 100, 50
    p.baseline_rho_min, p.raised_rho_mins = 1e-12, [1e-3, 1e-2]
    p.thresholds = dict(high_residual_threshold=1e-2, plateau_residual_threshold=1e-4, plateau_ratio_threshold=0.6)
    p.severity_jump_r50_threshold, p.severity_jump_rho_min = 0.0, 1e-2
    p.reuse_probe, p.checkpoint_guard, p.last_x = True, False, None
    p.min_confidence = min_confidence
    p.dims = (4, 4, 4)
    seen = {"features": None}
    calls = []
    queue = {k: list(v) for k, v in script.items()}

    def solve_at_floor(density, rho_min, *, maxiter, history, binary=False, x0=None, check=None):
        iters, reported, true_rel, r50, r_end = queue[rho_min].pop(0)
        iters = min(iters, maxiter)
        h = _hist(r50, r_end, iters)
        if check is not None and iters > check[0]:
            # the library runs the check once the solve has done check[0] iterations
            if check[1](h[: check[0] + 1]):
                h, iters, reported = h[: check[0] + 1], check[0], False
                true_rel = 1.0
        history.extend(h)
        calls.append(rho_min)
        p.last_x = ("x", rho_min, len(calls))
        return FloorAttempt(rho_min, iters, reported, true_rel <= 1e-6, true_rel, 0.1, 0.2 * iters, list(h))

    def propose(pooled, features):
        seen["features"] = features
        return np.asarray(prob, dtype=np.float64)

    p.solve_at_floor = solve_at_floor
    p._pool = lambda density: "pooled"
    p._propose = propose
    p._sync = lambda: None
    return p, calls, seen


def test_confident_proposal_stops_at_r50_and_tries_its_rung_first():
    p, calls, seen = _policy({1e-12: [(100, False, 3e-5, 5e-3, 2e-4)], 1e-2: [(40, True, 8e-7, 1e-4, 9e-7)]},
                             prob=[0.05, 0.15, 0.8])
    r = p.run(None)
    assert calls == [1e-12, 1e-2]
    assert (r["stopped_at_r50"], r["trigger"], r["proposal"]) == ("learned", "learned", 2)
    assert r["probe_iters"] == 50 and r["attempted_rho_mins"] == "1e-02" and r["solve_converged"] == 1
    # features: log10(r50) / 4 and the iteration reaching 1e-2 over 50
    assert seen["features"][0] == pytest.approx(np.log10(5e-3) / 4.0)


def test_wrong_proposal_costs_solves_and_the_plain_rung_comes_last():
    p, calls, _ = _policy({1e-12: [(100, False, 3e-5, 5e-3, 2e-4), (300, True, 9e-7, 1e-3, 9e-7)],
                           1e-3: [(300, False, 5e-6, 1e-3, 5e-6)], 1e-2: [(300, False, 4e-6, 1e-3, 4e-6)]},
                          prob=[0.1, 0.8, 0.1])
    r = p.run(None)
    # proposed 1e-3, then the raised rung above it, then the baseline floor
    assert calls == [1e-12, 1e-3, 1e-2, 1e-12]
    assert r["attempted_rho_mins"] == "1e-03;1e-02;1e-12"
    assert (r["recommended_rho_min"], r["solve_converged"], r["n_setups"]) == (1e-12, 1, 4)


def test_unconfident_proposal_lets_the_plain_rule_decide():
    p, calls, _ = _policy({1e-12: [(100, False, 3e-6, 5e-3, 2e-5), (300, True, 9e-7, 5e-3, 9e-7)]},
                          prob=[0.3, 0.4, 0.3])
    r = p.run(None)
    assert r["stopped_at_r50"] == "" and r["proposal"] == 0 and r["trigger"] == "keep"
    assert calls == [1e-12, 1e-12] and r["probe_iters"] == 100 and r["solve_converged"] == 1


def test_high_residual_rule_stops_whatever_the_network_says():
    p, calls, _ = _policy({1e-12: [(100, False, 1e-2, 3e-2, 2e-2)], 1e-3: [(60, True, 7e-7, 1e-4, 9e-7)]},
                          prob=[0.9, 0.05, 0.05])
    r = p.run(None)
    assert (r["stopped_at_r50"], r["trigger"], r["proposal"]) == ("high_residual", "high_residual", 0)
    # no baseline rung after a high-residual stop
    assert calls == [1e-12, 1e-3] and r["attempted_rho_mins"] == "1e-03"


def test_probe_converged_before_r50_is_reused():
    p, calls, seen = _policy({1e-12: [(20, True, 6e-7, 1e-6, 8e-7)]}, prob=[0.0, 0.0, 1.0])
    r = p.run(None)
    assert calls == [1e-12] and seen["features"] is None
    assert (r["selected_reused_probe"], r["recommended_rho_min"], r["n_setups"]) == (1, 1e-12, 1)
    assert p.last_x == ("x", 1e-12, 1)
