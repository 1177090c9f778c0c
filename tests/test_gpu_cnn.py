"""The learned floor proposer's CUDA kernels (csrc/cnn.cu) against the oracle,
and the policy built on it.

Pooling, forward probabilities, loss and every parameter gradient are compared
with oracle/cnn.py on the same parameters and inputs: the oracle accumulates in
float64 and the kernels in float32 over at most 34 * 27 = 918 terms per output,
so probabilities and the loss agree to 2e-5 and each parameter tensor's
gradient to 1e-3 of that tensor's largest entry.  Training is checked for
bitwise reproducibility and for learning a separable labelling.  The checked
FGMRES (simpfem_fgmres_checked) is checked to stop exactly at its check; the
learned policy to follow the plain policy when the proposal is the plain
policy's own choice (same floor, no more attempts or iterations) and to return
only guarded answers under every proposal.
"""

import ctypes

import numpy as np
import pytest

from oracle import cnn

pytestmark = pytest.mark.gpu


def _net(cuda, params=None, max_batch=64):
    from gpu_fem.floor_proposer import FloorProposerNet

    return FloorProposerNet(max_batch=max_batch, params=params, seed=0)


def _params(seed):
    rng = np.random.default_rng(seed)
    theta = cnn.init_params(seed)
    # non-zero biases so every bias path carries signal
    offs = np.cumsum([0] + [int(np.prod(s)) for s in cnn.param_shapes()])
    for i, s in enumerate(cnn.param_shapes()):
        if len(s) == 1:
            theta[offs[i]:offs[i + 1]] = rng.standard_normal(s[0]) * 0.05
    return theta.astype(np.float32)


def _inputs(seed, n):
    rng = np.random.default_rng(seed)
    x = rng.random((n, 1, 16, 16, 16)).astype(np.float32)
    f = (rng.standard_normal((n, 2)) * 0.5).astype(np.float32)
    lab = rng.integers(0, 3, n).astype(np.int32)
    return x, f, lab


def test_param_count_matches_oracle(cuda):
    from gpu_fem import _lib

    assert _lib.lib().simpfem_cnn_n_params() == cnn.n_params()


@pytest.mark.parametrize("dims", [(40, 20, 20), (80, 40, 20), (13, 7, 21), (16, 16, 16), (160, 80, 40)])
def test_pool16_matches_oracle(cuda, dims):
    from gpu_fem.floor_proposer import FloorProposerNet

    d = np.random.default_rng(sum(dims)).random(int(np.prod(dims)))
    got = FloorProposerNet.pool(cuda.as_tensor(d, device="cuda"), dims).cpu().numpy().reshape(16, 16, 16)
    np.testing.assert_allclose(got, cnn.pool16(d, dims), rtol=1e-6, atol=0)


@pytest.mark.parametrize("n", [1, 5, 64])
def test_forward_matches_oracle(cuda, n):
    theta = _params(3)
    x, f, _ = _inputs(n, n)
    net = _net(cuda, theta)
    prob = net.forward(cuda.as_tensor(x, device="cuda"), cuda.as_tensor(f, device="cuda")).cpu().numpy()
    logits, _ = cnn.forward(theta, x, f)
    e = np.exp(logits - logits.max(axis=1, keepdims=True))
    ref = e / e.sum(axis=1, keepdims=True)
    np.testing.assert_allclose(prob, ref, atol=2e-5, rtol=0)
    np.testing.assert_allclose(prob.sum(axis=1), 1.0, atol=1e-6)


@pytest.mark.parametrize("n,seed", [(1, 11), (6, 12), (48, 13)])
def test_loss_and_gradient_match_oracle(cuda, n, seed):
    theta = _params(seed)
    x, f, lab = _inputs(seed + 100, n)
    net = _net(cuda, theta)
    loss, g = net.loss_grad(cuda.as_tensor(x, device="cuda"), cuda.as_tensor(f, device="cuda"),
                            cuda.as_tensor(lab, device="cuda"), want_grad=True)
    ref_loss, ref_g = cnn.loss_and_grad(theta, x, f, lab)
    assert abs(loss - ref_loss) <= 2e-5 * max(1.0, abs(ref_loss))
    offs = np.cumsum([0] + [int(np.prod(s)) for s in cnn.param_shapes()])
    for i in range(len(offs) - 1):
        got, ref = g[offs[i]:offs[i + 1]], ref_g[offs[i]:offs[i + 1]]
        scale = float(np.abs(ref).max())
        assert scale > 0, f"parameter tensor {i} has no gradient signal"
        err = float(np.abs(got - ref).max())
        assert err <= 1e-3 * scale, f"parameter tensor {i}: max error {err:.3e} vs scale {scale:.3e}"


def test_adam_step_matches_formula(cuda):
    theta = _params(5)
    x, f, lab = _inputs(6, 8)
    net = _net(cuda, theta)
    _, g = net.loss_grad(cuda.as_tensor(x, device="cuda"), cuda.as_tensor(f, device="cuda"),
                         cuda.as_tensor(lab, device="cuda"), want_grad=True)
    net.adam_step(1e-3)
    got = net.get_params()
    g64 = g.astype(np.float64)
    m = 0.1 * g64
    v = 0.001 * g64 * g64
    ref = theta - 1e-3 * (m / 0.1) / (np.sqrt(v / 0.001) + 1e-8)
    np.testing.assert_allclose(got, ref, atol=1e-6, rtol=1e-5)


def test_training_is_reproducible_and_learns(cuda):
    rng = np.random.default_rng(21)
    n = 384
    fill = rng.uniform(0.05, 0.95, n)
    x = (rng.random((n, 1, 16, 16, 16)) < fill[:, None, None, None, None]).astype(np.float32)
    f = np.stack([np.log10(fill) / 4, rng.random(n)], axis=1).astype(np.float32)
    lab = np.digitize(fill, [0.35, 0.65]).astype(np.int64)  # three classes by fill fraction
    xd, fd = cuda.as_tensor(x, device="cuda"), cuda.as_tensor(f, device="cuda")
    runs = []
    for _ in range(2):
        net = _net(cuda, None, max_batch=64)
        curve = net.train(xd, fd, lab, epochs=12, batch=64, lr=3e-3, seed=4)
        runs.append((curve, net.get_params(), net))
    assert runs[0][0] == runs[1][0]
    assert np.array_equal(runs[0][1], runs[1][1])
    curve = runs[0][0]
    assert curve[-1] < 0.5 * curve[0], curve
    acc = float(np.mean(runs[0][2].forward(xd, fd).argmax(1).cpu().numpy() == lab))
    assert acc >= 0.9, acc


def test_batch_limits_and_argument_checks(cuda):
    from gpu_fem import _lib

    net = _net(cuda, None, max_batch=4)
    with pytest.raises(ValueError):
        net.set_params(np.zeros(10, dtype=np.float32))
    x = cuda.zeros((5, 4096), dtype=cuda.float32, device="cuda")
    f = cuda.zeros((5, 2), dtype=cuda.float32, device="cuda")
    p = cuda.empty((5, 3), dtype=cuda.float32, device="cuda")
    for bad in (0, 5):
        rc = _lib.lib().simpfem_cnn_forward(net._h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(f.data_ptr()),
                                            bad, ctypes.c_void_p(p.data_ptr()), _lib.stream_ptr())
        assert rc != 0
    # the python wrapper splits larger inputs into max_batch chunks
    assert net.forward(x, f).shape == (5, 3)
    with pytest.raises(ValueError):
        net.loss_grad(x[:4], f[:4], cuda.tensor([0, 1, 3, 0], dtype=cuda.int32, device="cuda"))


def _constant_proposer(cuda, rung):
    """Parameters whose softmax puts ~1 on ``rung`` for every input."""
    theta = np.zeros(cnn.n_params(), dtype=np.float32)
    theta[-3 + rung] = 20.0
    return _net(cuda, theta, max_batch=4)


def _states(dims, seeds, probs, radius=1.5):
    """Seeded void masks, cone-filtered unless ``radius`` <= 1 (the identity)."""
    from gpu_fem.pub_simp_solver import _build_density_filter

    H = _build_density_filter(dims[0], dims[1], radius, dims[2]) if radius > 1.0 else None
    out = []
    for s, p in zip(seeds, probs):
        solid = (np.random.default_rng(s).random(int(np.prod(dims))) >= p).astype(np.float64)
        out.append(solid if H is None else np.asarray(H @ solid))
    return out


POLICY = dict(penal=3.0, tol=1e-6, restart=300, maxiter=300, probe_iters=100, probe_r50=50,
              raised_rho_mins=(1e-3, 1e-2), cycle_precision="fp32")


def _policies(cuda, dims, proposer):
    from gpu_fem.floor_proposer import LearnedFloorPolicy
    from gpu_fem.paper4 import PLAIN_JACOBI_STACK
    from gpu_fem.policy import GuardedFloorPolicy
    from gpu_fem.presets import cantilever_spec

    stack = dict(PLAIN_JACOBI_STACK, fine_smoother="fp32")
    spec = cantilever_spec(*dims)
    return (GuardedFloorPolicy(spec, stack=stack, **POLICY),
            LearnedFloorPolicy(spec, proposer=proposer, dims=dims, stack=stack, **POLICY))


# unfiltered masks on 40x20x20: low void fractions keep the baseline floor, high
# ones trip the r50 rule (measured on the mixed-precision Jacobi hierarchy)
MASKS = dict(dims=(40, 20, 20), seeds=range(6), probs=(0.2, 0.4, 0.65, 0.7, 0.75, 0.78), radius=1.0)


def test_checked_fgmres_stops_at_the_check(cuda):
    """simpfem_fgmres_checked: the check sees the history up to its iteration, a
    true return ends the solve there, and the history before it is unchanged."""
    _, pol = _policies(cuda, MASKS["dims"], _constant_proposer(cuda, 0))
    d = cuda.as_tensor(_states(**MASKS)[5], device="cuda")
    full: list = []
    a = pol.solve_at_floor(d, 1e-12, maxiter=100, history=full)
    assert a.iters > 50
    seen = []
    cut: list = []
    b = pol.solve_at_floor(d, 1e-12, maxiter=100, history=cut, check=(50, lambda h: seen.append(list(h)) or True))
    assert len(seen) == 1 and len(seen[0]) == 51
    assert b.iters == 50 and not b.solver_reported_converged and len(cut) == 51
    assert cut == full[:51] == seen[0]
    # the iterate after 50 iterations: its true residual is the one FGMRES reported
    assert b.final_rel_residual == pytest.approx(cut[-1], rel=0.1)
    # a check that returns false changes nothing
    c_hist: list = []
    c = pol.solve_at_floor(d, 1e-12, maxiter=100, history=c_hist, check=(50, lambda h: False))
    assert c.iters == a.iters and c_hist == full and c.final_rel_residual == a.final_rel_residual


def test_learned_policy_follows_plain_choice(cuda):
    """With the proposal set to the plain policy's own selection the learned
    policy selects the same floor with no more attempts, setups or iterations.
    Each state gets fresh hierarchies, so both probes are the same computation
    (a hierarchy's lambda cache carries over from the states it solved before)."""
    from gpu_fem.floor_proposer import rung_index

    dims = MASKS["dims"]
    states = _states(**MASKS)
    nets = [_constant_proposer(cuda, k) for k in range(3)]
    seen = set()
    saved = 0
    for d in states:
        plain, _ = _policies(cuda, dims, nets[0])
        rp = plain.run(cuda.as_tensor(d, device="cuda"))
        k = rung_index(rp["recommended_rho_min"])
        seen.add(k)
        _, learned = _policies(cuda, dims, nets[k])
        rl = learned.run(cuda.as_tensor(d, device="cuda"))
        assert rl["probe_r50"] == rp["probe_r50"]
        assert rl["solve_converged"] >= rp["solve_converged"]
        assert rl["recommended_rho_min"] == rp["recommended_rho_min"]
        assert rl["n_floor_attempts"] <= rp["n_floor_attempts"]
        assert rl["n_setups"] <= rp["n_setups"]
        assert rl["total_iters"] <= rp["total_iters"]
        saved += rp["total_iters"] - rl["total_iters"]
        if rp["probe_r50"] >= 1e-2:
            assert rl["stopped_at_r50"] == "high_residual"
    assert len(seen) >= 2, seen
    assert saved > 0


def test_wrong_proposal_stays_guarded(cuda):
    """Every constant proposal, right or wrong, ends in a guarded answer."""
    dims = MASKS["dims"]
    states = _states(dims, (40, 41, 42), (0.3, 0.68, 0.74), radius=1.0)
    for k in range(3):
        _, learned = _policies(cuda, dims, _constant_proposer(cuda, k))
        for d in states:
            r = learned.run(cuda.as_tensor(d, device="cuda"))
            assert r["solve_converged"] == 1
            assert r["solve_final_rel_residual"] <= 1e-6
            if r["probe_iters"] >= 50:  # the probe reached the decision point
                assert r["proposal"] == k


def test_trained_proposer_gains_over_plain_policy(cuda):
    """The committed network (gpu_fem/data/floor_proposer.npz, with the confidence
    threshold calibrated on fresh states) against the plain probe-and-ladder and
    against the r50 rule stop without the network, on the first 128 held-out
    states of the training script's generator (seed 1: half cone-filtered, half
    unfiltered masks, 40x20x20 and 80x40x20): every answer the plain policy guards
    is guarded, the learned policy needs fewer outer iterations than the plain one,
    no more than the rule stop alone (2 % slack on this subset; on all 512 held-out
    states it needs 1.7 % fewer, floor_proposer_eval.json), and selects the plain
    policy's floor on at least 95 % of the states."""
    import os
    import sys

    from gpu_fem.floor_proposer import DEFAULT_WEIGHTS, FloorProposerNet, LearnedFloorPolicy
    from gpu_fem.paper4 import PLAIN_JACOBI_STACK
    from gpu_fem.policy import GuardedFloorPolicy
    from gpu_fem.presets import cantilever_spec

    pkg = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                       "solver-admissibility-and-guarded-floor-selection_b200")
    if pkg not in sys.path:
        sys.path.insert(0, pkg)
    import train_floor_proposer as tfp

    net = FloorProposerNet.load(DEFAULT_WEIGHTS, max_batch=4)
    zero = _constant_proposer(cuda, 0)
    states = tfp.make_states(512, seed=1)[:128]
    stack = dict(PLAIN_JACOBI_STACK, fine_smoother="fp32")
    tot = {"plain": [0, 0, 0], "rule": [0, 0, 0], "learned": [0, 0, 0]}
    for dims in tfp.MESHES:
        spec = cantilever_spec(*dims)
        pols = {"plain": GuardedFloorPolicy(spec, stack=stack, **tfp.POLICY),
                "rule": LearnedFloorPolicy(spec, proposer=zero, dims=dims, stack=stack, **tfp.POLICY),
                "learned": LearnedFloorPolicy(spec, proposer=net, dims=dims, stack=stack, **tfp.POLICY)}
        for st in states:
            if st["dims"] != dims:
                continue
            dd = cuda.as_tensor(st["density"], device="cuda")
            rows = {k: p.run(dd) for k, p in pols.items()}
            for k, r in rows.items():
                tot[k][0] += r["total_iters"]
                tot[k][1] += r["solve_converged"]
                tot[k][2] += int(r["recommended_rho_min"] == rows["plain"]["recommended_rho_min"])
    print("outer iterations / guarded / same floor as plain:", tot)
    assert tot["learned"][1] >= tot["plain"][1]
    assert tot["learned"][0] < tot["plain"][0]
    assert tot["learned"][0] <= 1.02 * tot["rule"][0]
    assert tot["learned"][2] >= 0.95 * len(states)
