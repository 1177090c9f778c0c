"""The SIMP loop entry's control flow against the reference's own loop, on CPU.

tests/golden/simp_control_16x8x6.json (make_simp_control_golden.py) holds the
reference's run_simp_surrogate_gpu run with the stand-ins of
tests/golden/simp_control_fakes.py in place of its numeric steps, in two
scenarios: "controlled" (projection, schedule-only controller with its radius
changes and restarts from the best design, a passive mask, a surrogate on every
fourth iteration; 72 iterations) and "plain" (the unprojected OC step until the
convergence test stops the loop).  Here gpu_fem.simp_gpu.run_simp_surrogate_gpu
runs on the host with the same stand-ins (its device hooks -- _lib, _DEVICE,
cone_filter, heaviside, _oc_step, OCUpdater -- pointed at them) and this
package's ScheduleOnlyController, so both loops see identical numbers: every
params_log row must equal the reference's key for key in its order (floats to
1e-12 relative: grayness and volume are torch reductions here, numpy ones
there), and so must the result's scalars, rho_final and the stand-in solver's
sequence of solves and invalidations.
"""

import json
import math
import os
import sys
import types

import numpy as np
import pytest
import torch

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, GOLDEN)
import simp_control_fakes as fakes  # noqa: E402


def _host_tensor(x, dtype):
    t = x if torch.is_tensor(x) else torch.as_tensor(np.asarray(x))
    return t.to(dtype).contiguous()


@pytest.fixture
def host_loop(monkeypatch):
    from gpu_fem import simp_gpu

    def cone_filter(x, dims, rmin, transpose=False):
        H = fakes.filter_matrix(*dims, rmin)
        return torch.from_numpy((H.T if transpose else H) @ x.numpy())

    def heaviside(x, beta, eta, derivative=False):
        return torch.from_numpy(fakes.project(x.numpy(), beta, eta))

    def oc_step(oc, cache, dims, rmin, rho, rho_f, dc, beta, eta, volfrac, move, projected):
        rn, change = fakes.oc_step(rho.numpy(), rho_f.numpy(), dc.numpy(), beta, eta, volfrac, move,
                                   fakes.filter_matrix(*dims, rmin), projected)
        return torch.from_numpy(np.array(rn, dtype=np.float64)), change

    monkeypatch.setattr(simp_gpu, "_lib", types.SimpleNamespace(require_cuda=lambda: torch, as_cuda=_host_tensor))
    monkeypatch.setattr(simp_gpu, "_DEVICE", "cpu")
    monkeypatch.setattr(simp_gpu, "OCUpdater", lambda: None)
    monkeypatch.setattr(simp_gpu, "cone_filter", cone_filter)
    monkeypatch.setattr(simp_gpu, "heaviside", heaviside)
    monkeypatch.setattr(simp_gpu, "_oc_step", oc_step)
    return simp_gpu


def _same(a, b, where):
    if isinstance(b, bool) or isinstance(a, bool):
        assert bool(a) == bool(b) and type(a) is type(b), where
    elif isinstance(b, float) or isinstance(a, float):
        a, b = float(a), float(b)
        if math.isnan(b) or math.isinf(b):
            assert (math.isnan(a) and math.isnan(b)) or a == b, (where, a, b)
        else:
            assert abs(a - b) <= 1e-12 * max(abs(b), 1e-300), (where, a, b)
    else:
        assert a == b, (where, a, b)


@pytest.mark.parametrize("name", list(fakes.SCENARIOS))
def test_loop_control_flow_matches_reference(host_loop, name):
    from gpu_fem.pub_baseline_controller import ScheduleOnlyController

    with open(os.path.join(GOLDEN, "simp_control_16x8x6.json")) as f:
        g = json.load(f)[name]
    sc = fakes.SCENARIOS[name]
    fixed, free, F, ndof = fakes.problem()
    fakes.EVENTS.clear()
    res = host_loop.run_simp_surrogate_gpu(
        host_loop.TO3DParams(**sc["params"]), fixed, free, F, ndof, fakes.EchoSurrogate() if sc["surrogate"] else None,
        fakes.router, device="auto", param_controller=ScheduleOnlyController() if sc["controller"] else None,
        passive_mask=fakes.passive_mask() if sc["passive"] else None, solver_class=fakes.FakeSolver,
        solver_kwargs=dict(fakes.SOLVER_KWARGS))
    log = [{k: v for k, v in row.items() if k != "iter_wall_sec"} for row in res["params_log"]]
    assert len(log) == len(g["params_log"])
    for k, (a, b) in enumerate(zip(log, g["params_log"])):
        assert list(a) == list(b), k
        for key in b:
            _same(a[key], b[key], (name, k + 1, key))
    for key, value in g["scalars"].items():
        _same(res[key], value, (name, key))
    np.testing.assert_allclose(res["rho_final"], np.array(g["rho_final"]), rtol=1e-12, atol=0)
    events = [e if isinstance(e, str) else list(e) for e in fakes.EVENTS]
    assert events == g["events"]


def test_scenarios_reach_the_branches():
    """The golden runs take every branch the test is meant to cover."""
    with open(os.path.join(GOLDEN, "simp_control_16x8x6.json")) as f:
        g = json.load(f)
    ctl, plain = g["controlled"], g["plain"]
    assert any(row["used_surrogate"] for row in ctl["params_log"])
    assert len({row["rmin"] for row in ctl["params_log"]}) >= 4
    assert {row["beta"] for row in ctl["params_log"]} >= {1.0, 4.0, 16.0, 32.0}
    restarts = ctl["events"].count("invalidate") - (len({row["rmin"] for row in ctl["params_log"]}) - 1)
    assert restarts > 0 and ctl["scalars"]["best_is_valid"]
    assert plain["scalars"]["n_iter"] < fakes.SCENARIOS["plain"]["params"]["max_iter"]
    assert plain["params_log"][-1]["change"] < fakes.SCENARIOS["plain"]["params"]["tol"]


def test_oc_step_wiring(monkeypatch):
    """The real _oc_step: the projected form goes to simpfem_oc_update_projected with
    the loop's arguments; the unprojected one to simpfem_oc_update with H^T dc and the
    volume weights H^T 1, computed once per radius."""
    from gpu_fem import simp_gpu

    calls = []

    def cone_filter(x, dims, rmin, transpose=False):
        calls.append(("filter", rmin, transpose, float(x.sum())))
        return x * (2.0 if transpose else 1.0)

    class OC:
        def projected(self, *args):
            calls.append(("projected",) + tuple(a if not torch.is_tensor(a) else float(a.sum()) for a in args))
            return torch.zeros(3), 0.5, 1.0, 7

        def __call__(self, rho, dc_design, weights, volfrac, move):
            calls.append(("oc", float(dc_design.sum()), float(weights.sum()), volfrac, move))
            return torch.ones(3), 0.25, 1.0, 7

    monkeypatch.setattr(simp_gpu, "_lib", types.SimpleNamespace(require_cuda=lambda: torch, as_cuda=_host_tensor))
    monkeypatch.setattr(simp_gpu, "_DEVICE", "cpu")
    monkeypatch.setattr(simp_gpu, "cone_filter", cone_filter)
    rho, rho_f, dc = torch.full((3,), 0.25, dtype=torch.float64), torch.full((3,), 0.5, dtype=torch.float64), \
        torch.full((3,), -1.0, dtype=torch.float64)
    cache = {}
    out = simp_gpu._oc_step(OC(), cache, (3, 1, 1), 1.5, rho, rho_f, dc, 4.0, 0.5, 0.3, 0.2, True)
    assert out[1] == 0.5 and calls[-1][0] == "projected" and calls[-1][1:] == ((3, 1, 1), 1.5, 0.75, 1.5, -3.0,
                                                                                 4.0, 0.5, 0.3, 0.2)
    assert not cache
    calls.clear()
    for rmin in (1.5, 1.5, 1.4):
        rho_new, change = simp_gpu._oc_step(OC(), cache, (3, 1, 1), rmin, rho, rho_f, dc, 4.0, 0.5, 0.3, 0.2, False)
        assert change == 0.25 and torch.equal(rho_new, torch.ones(3))
    # weights H^T 1 for 1.5, then only H^T dc, then new weights for 1.4
    assert [c[:3] for c in calls if c[0] == "filter"] == [
        ("filter", 1.5, True), ("filter", 1.5, True), ("filter", 1.5, True), ("filter", 1.4, True),
        ("filter", 1.4, True)]
    assert [c for c in calls if c[0] == "oc"] == [("oc", -6.0, 6.0, 0.3, 0.2)] * 3
    assert list(cache) == [1.4]
