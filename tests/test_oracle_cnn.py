"""The CPU restatement of the learned floor proposer (oracle/cnn.py).

Its analytic gradient is checked against central finite differences (with the
bfloat16 weight rounding switched off, since rounding makes the loss
piecewise constant in the weights), against torch autograd on the CPU (with the
rounding on: the rounded weights are the leaves), and its adaptive average
pooling against torch.nn.functional.adaptive_avg_pool3d.
"""

import numpy as np
import pytest

from oracle import cnn


def test_param_count():
    assert cnn.n_params() == 49017


def test_gradient_matches_finite_differences(monkeypatch):
    monkeypatch.setattr(cnn, "bf16", lambda w: np.asarray(w, dtype=np.float64))
    rng = np.random.default_rng(0)
    theta = cnn.init_params(1).astype(np.float64)
    theta[cnn.n_params() - 3:] = rng.standard_normal(3) * 0.1  # non-zero dense bias
    x = rng.random((2, 1, 16, 16, 16))
    f = rng.standard_normal((2, 2))
    lab = np.array([0, 2])

    l0, g = cnn.loss_and_grad(theta, x, f, lab)
    assert np.isfinite(l0)
    offs = np.cumsum([0] + [int(np.prod(s)) for s in cnn.param_shapes()])
    h = 1e-6
    for t in range(len(offs) - 1):
        # the largest-gradient entry of each parameter tensor and one other
        seg = g[offs[t]:offs[t + 1]]
        for k in {int(np.argmax(np.abs(seg))), int(rng.integers(0, seg.size))}:
            i = offs[t] + k
            tp, tm = theta.copy(), theta.copy()
            tp[i] += h
            tm[i] -= h
            fd = (cnn.loss_and_grad(tp, x, f, lab)[0] - cnn.loss_and_grad(tm, x, f, lab)[0]) / (2 * h)
            assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(g[i]), (t, k, fd, g[i])


def test_gradient_matches_torch_autograd():
    torch = pytest.importorskip("torch")
    F = torch.nn.functional
    rng = np.random.default_rng(3)
    theta = cnn.init_params(2)
    theta[cnn.n_params() - 3:] = rng.standard_normal(3).astype(np.float32) * 0.1
    x = rng.random((3, 1, 16, 16, 16))
    f = rng.standard_normal((3, 2))
    lab = np.array([2, 0, 1])
    loss, g = cnn.loss_and_grad(theta, x, f, lab)

    ps = cnn.unpack(theta)
    leaves = []
    for i, p in enumerate(ps):
        v = cnn.bf16(p) if p.ndim > 1 else p
        leaves.append(torch.tensor(np.asarray(v, dtype=np.float64), requires_grad=True))
    h = torch.tensor(x)
    for li, (_, _, stride) in enumerate(cnn.LAYERS):
        h = F.relu(F.conv3d(h, leaves[2 * li], leaves[2 * li + 1], stride=stride, padding=1))
    z = torch.cat([h.mean(dim=(2, 3, 4)), torch.tensor(f)], dim=1)
    logits = z @ leaves[-2].T + leaves[-1]
    tl = F.cross_entropy(logits, torch.tensor(lab))
    tl.backward()
    ref = np.concatenate([lf.grad.numpy().ravel() for lf in leaves])
    assert abs(float(tl) - loss) <= 1e-12 * max(1.0, abs(loss))
    np.testing.assert_allclose(g, ref, rtol=1e-9, atol=1e-12)


def test_bf16_rounding_ties_to_even():
    vals = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 1e-30], dtype=np.float32)
    out = cnn.bf16(vals)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: even mantissa (1.0); 1 + 3*2^-8 rounds up to 1 + 2^-6
    assert out[0] == 1.0 and out[1] == 1.0 and out[2] == np.float32(1.0 + 2 ** -6) and out[3] == -2.5
    assert (out.view(np.uint32) & 0xFFFF).max() == 0


@pytest.mark.parametrize("dims", [(40, 20, 20), (80, 40, 20), (13, 7, 21), (16, 16, 16)])
def test_pool16_matches_torch(dims):
    torch = pytest.importorskip("torch")
    d = np.random.default_rng(sum(dims)).random(int(np.prod(dims)))
    ref = torch.nn.functional.adaptive_avg_pool3d(torch.tensor(d.reshape(1, 1, *dims)), 16)[0, 0].numpy()
    np.testing.assert_allclose(cnn.pool16(d, dims), ref, rtol=1e-6)
