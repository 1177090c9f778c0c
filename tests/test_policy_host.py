"""Host control of the guarded floor policy (GuardedFloorPolicy.run), without a
GPU: the solves are replaced by a scripted stand-in that returns chosen
residual histories, iteration counts and true residuals per floor, so every
branch of the reference driver's sequence (run_gmg_floor_detector_prospective.py
:263-354) is exercised -- probe kept and reused, probe kept then a full solve,
keep -> guard failed -> fallback ladder (a false keep), high-r50 and plateau
escalations, the severity jump, an exhausted ladder, and the checkpointed
guard reading true residuals."""

import numpy as np
import pytest

from gpu_fem.policy import FloorAttempt, GuardedFloorPolicy


def _hist(r50, r_end, n):
    """A residual history of n + 1 entries through r50 at index 50 and r_end at the end."""
    h = list(np.geomspace(1.0, r50, 51)) if n >= 50 else list(np.geomspace(1.0, r_end, n + 1))
    if n > 50:
        h += list(np.geomspace(r50, r_end, n - 49))[1:]
    return h


def _policy(script, **kw):
    """script[rho_min] -> list of (iters, reported, true_rel, r50, r_end) per successive solve at that floor."""
    p = object.__new__(GuardedFloorPolicy)
    p.penal, p.tol, p.restart, p.maxiter = 4.5, 1e-6, 300, 300
    p.probe_iters, p.probe_r50 = 100, 50
    p.baseline_rho_min = 1e-12
    p.raised_rho_mins = list(kw.get("ladder", (1e-3, 1e-2)))
    p.thresholds = dict(high_residual_threshold=1e-2, plateau_residual_threshold=1e-4, plateau_ratio_threshold=0.6)
    p.severity_jump_r50_threshold = kw.get("severity", 0.0)
    p.severity_jump_rho_min = 1e-2
    p.reuse_probe = True
    p.checkpoint_guard = kw.get("checkpoint", False)
    p.last_x = None
    calls = []
    queue = {k: list(v) for k, v in script.items()}

    def solve_at_floor(density, rho_min, *, maxiter, history, binary=False, x0=None, check=None):
        iters, reported, true_rel, r50, r_end = queue[rho_min].pop(0)
        iters = min(iters, maxiter)
        h = _hist(r50, r_end, iters)
        history.extend(h)
        if check is not None and iters >= check[0]:
            check[1](h[: check[0] + 1], kw.get("true_r50", r50))
        calls.append((rho_min, maxiter))
        p.last_x = ("x", rho_min, len(calls))
        return FloorAttempt(rho_min, iters, reported, true_rel <= 1e-6, true_rel, 0.1, 0.2 * iters, list(h))

    p.solve_at_floor = solve_at_floor
    return p, calls


def test_probe_kept_and_reused():
    p, calls = _policy({1e-12: [(30, True, 5e-7, 1e-6, 9e-7)]})
    r = p.run(None)
    assert calls == [(1e-12, 100)]
    assert (r["trigger"], r["recommended_rho_min"], r["attempted_rho_mins"]) == ("keep", 1e-12, "1e-12")
    assert r["selected_reused_probe"] == 1 and r["n_setups"] == 1 and r["solve_converged"] == 1
    assert r["total_iters"] == 30 and p.last_x == ("x", 1e-12, 1)


def test_probe_kept_at_its_cap_then_full_solve():
    p, calls = _policy({1e-12: [(100, False, 3e-6, 1e-3, 2e-5), (140, True, 8e-7, 1e-3, 9e-7)]})
    r = p.run(None)
    assert calls == [(1e-12, 100), (1e-12, 300)]
    assert r["trigger"] == "keep" and r["solve_converged"] == 1 and r["selected_reused_probe"] == 0
    assert r["n_setups"] == 2 and r["total_iters"] == 240 and r["solve_iters"] == 140


def test_keep_guard_failed_falls_back_to_the_ladder():
    p, calls = _policy({1e-12: [(100, False, 1e-4, 1e-3, 2e-5), (300, False, 2e-6, 1e-3, 1e-6)],
                        1e-3: [(40, True, 7e-7, 1e-4, 9e-7)]})
    r = p.run(None)
    assert calls == [(1e-12, 100), (1e-12, 300), (1e-3, 300)]
    assert r["trigger"] == "keep" and r["post_solve_fallback_triggered"] == 1 and r["detector_false_keep"] == 1
    assert (r["recommended_rho_min"], r["attempted_rho_mins"], r["solve_converged"]) == (1e-3, "1e-12;1e-03", 1)
    assert r["failed_ladder_solve_time_s"] == pytest.approx(0.2 * 300)


def test_high_r50_escalates_through_the_ladder():
    p, calls = _policy({1e-12: [(100, False, 1e-2, 2e-2, 1.5e-2)],
                        1e-3: [(300, False, 3e-6, 1e-3, 2e-6)], 1e-2: [(60, True, 6e-7, 1e-4, 8e-7)]})
    r = p.run(None)
    assert calls == [(1e-12, 100), (1e-3, 300), (1e-2, 300)]
    assert (r["trigger"], r["predicted_raise_floor"], r["post_solve_fallback_triggered"]) == ("high_r50", 1, 0)
    assert (r["recommended_rho_min"], r["attempted_rho_mins"], r["n_floor_attempts"]) == (1e-2, "1e-03;1e-02", 2)


def test_plateau_escalates():
    # r50 = 2e-4 below the high threshold; r100 = 1.5e-4 >= 1e-4 and r100 / r50 = 0.75 >= 0.6
    p, calls = _policy({1e-12: [(100, False, 1e-4, 2e-4, 1.5e-4)], 1e-3: [(50, True, 9e-7, 1e-4, 9e-7)]})
    r = p.run(None)
    assert r["trigger"] == "plateau" and r["recommended_rho_min"] == 1e-3 and r["solve_converged"] == 1
    assert r["probe_r100_over_r50"] == pytest.approx(0.75)


def test_exhausted_ladder_reports_the_last_floor_unconverged():
    p, calls = _policy({1e-12: [(100, False, 1e-2, 2e-2, 1.5e-2)],
                        1e-3: [(300, False, 3e-6, 1e-3, 2e-6)], 1e-2: [(300, False, 2e-6, 1e-3, 2e-6)]})
    r = p.run(None)
    assert (r["recommended_rho_min"], r["solve_converged"], r["solve_iters"]) == (1e-2, 0, 300)
    assert r["attempted_rho_mins"] == "1e-03;1e-02"


def test_severity_jump_skips_the_lower_rungs():
    p, calls = _policy({1e-12: [(100, False, 1e-1, 2e-1, 1.9e-1)], 1e-2: [(60, True, 6e-7, 1e-4, 8e-7)]},
                       severity=0.1)
    r = p.run(None)
    assert calls == [(1e-12, 100), (1e-2, 300)]
    assert r["severity_jump_triggered"] == 1 and r["attempted_rho_mins"] == "1e-02"


def test_checkpoint_guard_classifies_on_true_residuals():
    # the FGMRES estimate at r50 says keep (1e-3), the recomputed true residual
    # there says high (5e-2): the checkpointed rule escalates
    p, calls = _policy({1e-12: [(100, False, 4e-2, 1e-3, 2e-5)], 1e-3: [(50, True, 9e-7, 1e-4, 9e-7)]},
                       checkpoint=True, true_r50=5e-2)
    r = p.run(None)
    assert r["checkpoint_guard"] == 1 and r["probe_true_r50"] == 5e-2 and r["probe_true_r100"] == 4e-2
    assert r["trigger"] == "high_r50" and r["recommended_rho_min"] == 1e-3
    q, _ = _policy({1e-12: [(100, False, 4e-2, 1e-3, 2e-5), (300, True, 5e-7, 1e-3, 9e-7)]})
    assert q.run(None)["trigger"] == "keep"
