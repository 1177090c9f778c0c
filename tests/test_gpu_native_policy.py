"""The guarded floor policy run in the library (simpfem_policy_run / _batch)
against the Python policy that drives the same kernels step by step.

* plain policy, canonical stack, Bernoulli states of the 24 x 12 x 6 cantilever
  (penal 4.5, probe 30 / r50 15, ladder {1e-3, 1e-2}: keeps, raises and a
  fallback occur): every decision field and iteration count identical, the
  solutions equal to 1e-12 relative, the FP64 guard met by every accepted answer;
* the learned policy (committed proposer, mixed-precision Jacobi hierarchy) on
  unfiltered masks that stop at r50: the same;
* the batch over three workers equals BatchedFloorPolicy.run_many, and a batch
  over two meshes equals the same states run one after another per mesh;
* two hierarchies on one mesh handle are refused.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KEYS = ("trigger", "recommended_rho_min", "attempted_rho_mins", "solve_converged", "solver_reported_converged",
        "solve_iters", "probe_iters", "total_iters", "n_setups", "predicted_raise_floor",
        "post_solve_fallback_triggered", "selected_reused_probe")


def _states(n_elem, seeds=(3, 5), probs=(0.2, 0.35, 0.6)):
    out = []
    for seed in seeds:
        field = np.random.default_rng(seed).random(n_elem)
        for p in probs:
            out.append((field < p).astype(np.float64))
    return out


def _same(a, b, keys=KEYS):
    for k in keys:
        assert a[k] == b[k], (k, a[k], b[k], a, b)
    assert a["probe_r50"] == pytest.approx(b["probe_r50"], rel=1e-12)


def _close(x, y):
    import torch

    assert float(torch.linalg.norm(x - y)) <= 1e-12 * float(torch.linalg.norm(y))


def _plain(preset="cantilever_3d", **kw):
    from gpu_fem.policy import GuardedFloorPolicy

    args = dict(penal=4.5, raised_rho_mins=(1e-3, 1e-2), probe_iters=30, probe_r50=15, maxiter=60)
    args.update(kw)
    return GuardedFloorPolicy(preset, **args)


def test_native_plain_policy_matches_python(cuda):
    torch = cuda
    from gpu_fem.policy import run_native

    py, nat = _plain(), _plain()
    n = py.spec.nelx * py.spec.nely * py.spec.nelz
    triggers = set()
    for d in _states(n):
        dt = torch.as_tensor(d, device="cuda")
        a = py.run(dt, binary=True)
        xa = py.last_x.clone()
        b = run_native(nat, dt, binary=True)
        _same(a, b)
        _close(nat.last_x, xa)
        assert b["solve_converged"] == 1 and b["solve_final_rel_residual"] <= 1e-6
        triggers.add(b["trigger"])
    assert {"keep", "high_r50"} <= triggers


def test_native_learned_policy_matches_python(cuda):
    torch = cuda
    from gpu_fem.floor_proposer import FloorProposerNet, LearnedFloorPolicy
    from gpu_fem.paper4 import PLAIN_JACOBI_STACK
    from gpu_fem.policy import run_native
    from gpu_fem.presets import cantilever_spec

    stack = dict(PLAIN_JACOBI_STACK, fine_smoother="fp32")

    def make():
        return LearnedFloorPolicy(cantilever_spec(40, 20, 20), proposer=FloorProposerNet.load(max_batch=1),
                                  penal=3.0, raised_rho_mins=(1e-3, 1e-2), stack=stack, cycle_precision="fp32")

    py, nat = make(), make()
    stops = 0
    for d in _states(40 * 20 * 20, seeds=(11, 12), probs=(0.3, 0.55, 0.7)):
        dt = torch.as_tensor(d, device="cuda")
        a = py.run(dt)
        xa = py.last_x.clone()
        b = run_native(nat, dt)
        _same(a, b, KEYS[:-2] + ("selected_reused_probe",))
        assert a["stopped_at_r50"] == b["stopped_at_r50"] and a["proposal"] == b["proposal"]
        _close(nat.last_x, xa)
        assert b["solve_converged"] == 1
        stops += bool(b["stopped_at_r50"])
    assert stops >= 1


def test_native_batch_matches_threaded_batch(cuda):
    torch = cuda
    from gpu_fem.policy import BatchedFloorPolicy

    kw = dict(penal=4.5, raised_rho_mins=(1e-3, 1e-2), probe_iters=30, probe_r50=15, maxiter=60)
    py = BatchedFloorPolicy(3, "cantilever_3d", **kw)
    nat = BatchedFloorPolicy(3, "cantilever_3d", **kw)
    n = py.workers[0].spec.nelx * py.workers[0].spec.nely * py.workers[0].spec.nelz
    dens = [torch.as_tensor(d, device="cuda") for d in _states(n, seeds=(3, 5, 7))]
    xs = []
    rows = py.run_many(dens, binary=True, on_result=lambda k, w, r: xs.append((k, w.last_x.clone())))
    xs = dict(xs)
    rows_n = nat.run_many_native(dens, binary=True)
    torch.cuda.synchronize()
    for k, (a, b) in enumerate(zip(rows, rows_n)):
        _same(a, b)
        _close(nat.last_xs[k], xs[k])


def test_native_batch_over_two_meshes(cuda):
    torch = cuda
    import ctypes

    from gpu_fem import _lib
    from gpu_fem._native import mesh_namespace
    from gpu_fem.policy import native_opts, native_row, run_native
    from gpu_fem.presets import cantilever_spec

    def pair(dims, tag):
        with mesh_namespace(("two-mesh", tag)):
            return _plain(cantilever_spec(*dims))

    a, b = pair((24, 12, 6), "a"), pair((16, 8, 8), "b")
    ra, rb = pair((24, 12, 6), "ra"), pair((16, 8, 8), "rb")
    sa = _states(24 * 12 * 6, seeds=(3,))
    sb = _states(16 * 8 * 8, seeds=(4,))
    order = [(a, ra, d) for d in sa] + [(b, rb, d) for d in sb]
    order = [order[i] for i in (0, 3, 1, 4, 2, 5)]  # interleave the meshes
    dens = [torch.as_tensor(d, device="cuda") for _, _, d in order]
    xs = [torch.empty_like(p.F_free_gpu) for p, _, _ in order]
    states = (_lib.PolicyState * len(order))()
    for k, (p, _, _) in enumerate(order):
        states[k].g = p.gmg._h.value
        states[k].density = _lib.ptr(dens[k])
        states[k].b_free = _lib.ptr(p.F_free_gpu)
        states[k].x_free = _lib.ptr(xs[k])
    results = (_lib.PolicyResult * len(order))()
    o = native_opts(a, binary=True)
    _lib.call("simpfem_policy_batch", ctypes.byref(o), states, len(order), results, _lib.stream_ptr())
    torch.cuda.synchronize()
    for k, (_, ref, _) in enumerate(order):
        row = run_native(ref, dens[k], binary=True)  # the same states, one after another per mesh
        _same(native_row(results[k]), row)
        _close(xs[k], ref.last_x)


def test_native_batch_refuses_a_shared_mesh(cuda):
    torch = cuda
    import ctypes

    from gpu_fem import _lib
    from gpu_fem.policy import native_opts

    p, q = _plain(), _plain()  # default namespace: both on the same cached mesh handle
    n = p.spec.nelx * p.spec.nely * p.spec.nelz
    d = torch.ones(n, dtype=torch.float64, device="cuda")
    states = (_lib.PolicyState * 2)()
    for k, pol in enumerate((p, q)):
        states[k].g = pol.gmg._h.value
        states[k].density = _lib.ptr(d)
        states[k].b_free = _lib.ptr(pol.F_free_gpu)
        states[k].x_free = None
    results = (_lib.PolicyResult * 2)()
    with pytest.raises(_lib.SimpfemError, match="share one mesh"):
        _lib.call("simpfem_policy_batch", ctypes.byref(native_opts(p, binary=True)), states, 2, results,
                  _lib.stream_ptr())
