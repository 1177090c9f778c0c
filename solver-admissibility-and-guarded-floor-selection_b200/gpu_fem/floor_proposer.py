"""Learned floor proposer: a small 3D CNN that proposes the admissible floor rung.

No counterpart in the reference.  The network (kernels in csrc/cnn.cu, declared
in include/simpfem.h) reads the density field average-pooled to 16^3 and two
probe features -- log10(r50) / 4, and the iteration count at which the probe's
relative residual first reached the high-residual threshold (1e-2), divided by
the r50 index (1 when it had not by then) -- and outputs a softmax over the rungs
{1e-12, 1e-3, 1e-2}.  It is trained on the GPU by the project's own forward and
backward kernels on states and outcomes the solver itself generates: each
training state is labelled with the rung the plain probe-and-ladder policy
selects for it.

``LearnedFloorPolicy`` decides at the probe's r50 point (a host check inside the
native FGMRES, simpfem_fgmres_checked): when r50 is above the high-residual
threshold the plain rule raises the floor whatever r100 shows, so the probe stops
there; when the proposer is confident of a raised rung the probe also stops and
the ladder starts at that rung; otherwise the probe runs to r100 and the plain
rule decides exactly as in GuardedFloorPolicy.  Skipped rungs are tried last, so
a wrong proposal costs time (or selects a higher floor than the plain policy
would), never an unguarded answer: the FP64 recomputed-residual guard judges
every attempt.
"""

from __future__ import annotations

import ctypes
import os
import time
from typing import Optional, Sequence

import numpy as np

from . import _lib
from .policy import GuardedFloorPolicy, _classify

RUNGS = (1e-12, 1e-3, 1e-2)
VOX = 16 ** 3
DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "floor_proposer.npz")


def probe_features(r50: float, history: Sequence[float], r50_index: int,
                   high: float = 1e-2) -> tuple[float, float]:
    """(log10(r50) / 4, iterations to reach ``high`` / r50_index) from the probe's
    relative-residual history (entry k = after k iterations)."""
    hit = next((k for k, v in enumerate(list(history)[:r50_index + 1]) if v <= high), r50_index)
    return float(np.log10(max(float(r50), 1e-16)) / 4.0), float(hit) / float(r50_index)


def rung_index(rho_min: float) -> int:
    return int(np.argmin([abs(np.log10(rho_min) - np.log10(r)) for r in RUNGS]))


def he_init(seed: int, n: int) -> np.ndarray:
    """He-normal weights and zero biases in the library's parameter layout."""
    rng = np.random.default_rng(seed)
    out = []
    for cin, cout in ((1, 16), (16, 16), (16, 32), (32, 32)):
        out += [rng.standard_normal(cout * cin * 27) * np.sqrt(2.0 / (cin * 27)), np.zeros(cout)]
    out += [rng.standard_normal(3 * 34) * np.sqrt(2.0 / 34), np.zeros(3)]
    theta = np.concatenate(out).astype(np.float32)
    if theta.size != n:
        raise RuntimeError("parameter layout mismatch")
    return theta


class FloorProposerNet:
    """The CNN's parameters and workspaces on the GPU (``simpfem_cnn`` handle)."""

    def __init__(self, max_batch: int = 256, params: Optional[np.ndarray] = None, seed: int = 0):
        _lib.require_cuda()
        self.n_params = int(_lib.lib().simpfem_cnn_n_params())
        self.max_batch = int(max_batch)
        h = ctypes.c_void_p()
        _lib.call("simpfem_cnn_create", self.max_batch, ctypes.byref(h))
        self._h = h
        self.set_params(he_init(seed, self.n_params) if params is None else params)
        self.min_confidence = 0.5

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.lib().simpfem_cnn_destroy(h)
            except Exception:
                pass

    def set_params(self, theta) -> None:
        t = np.ascontiguousarray(theta, dtype=np.float32)
        if t.size != self.n_params:
            raise ValueError(f"expected {self.n_params} parameters, got {t.size}")
        _lib.call("simpfem_cnn_set_params", self._h, t.ctypes.data_as(ctypes.c_void_p), self.n_params)

    def get_params(self) -> np.ndarray:
        t = np.empty(self.n_params, dtype=np.float32)
        _lib.call("simpfem_cnn_get_params", self._h, t.ctypes.data_as(ctypes.c_void_p), self.n_params)
        return t

    @staticmethod
    def pool(density, dims):
        """(16^3,) float32 device tensor: the density average-pooled to 16^3."""
        torch = _lib.require_cuda()
        d = _lib.as_cuda(density, torch.float64)
        if d.numel() != int(np.prod(dims)):
            raise ValueError("density size does not match dims")
        out = torch.empty(VOX, dtype=torch.float32, device="cuda")
        _lib.call("simpfem_cnn_pool16", int(dims[0]), int(dims[1]), int(dims[2]), _lib.ptr(d), _lib.ptr(out),
                  _lib.stream_ptr())
        return out

    def forward(self, x, feats):
        """Softmax probabilities (N, 3) for inputs x (N, 16^3) and feats (N, 2)."""
        torch = _lib.require_cuda()
        x = _lib.as_cuda(x, torch.float32).reshape(-1, VOX).contiguous()
        f = _lib.as_cuda(feats, torch.float32).reshape(-1, 2).contiguous()
        if f.shape[0] != x.shape[0]:
            raise ValueError("x and feats must hold the same number of samples")
        n = x.shape[0]
        probs = []
        for s in range(0, n, self.max_batch):
            e = min(n, s + self.max_batch)
            p = torch.empty((e - s, 3), dtype=torch.float32, device="cuda")
            _lib.call("simpfem_cnn_forward", self._h, _lib.ptr(x[s:e]), _lib.ptr(f[s:e]), e - s, _lib.ptr(p),
                      _lib.stream_ptr())
            probs.append(p)
        return torch.cat(probs)

    def loss_grad(self, x, feats, labels, want_grad: bool = False):
        """Mean cross-entropy of one batch (<= max_batch samples); the gradient stays
        on the device for adam_step and is also returned when ``want_grad``."""
        torch = _lib.require_cuda()
        x = _lib.as_cuda(x, torch.float32).reshape(-1, VOX).contiguous()
        f = _lib.as_cuda(feats, torch.float32).reshape(-1, 2).contiguous()
        y = _lib.as_cuda(labels, torch.int32).contiguous()
        if y.numel() != x.shape[0] or f.shape[0] != x.shape[0]:
            raise ValueError("x, feats and labels must hold the same number of samples")
        if y.numel() and (int(y.min()) < 0 or int(y.max()) >= len(RUNGS)):
            raise ValueError("labels must index the rungs 0..2")
        loss = ctypes.c_float()
        g = np.empty(self.n_params, dtype=np.float32) if want_grad else None
        _lib.call("simpfem_cnn_loss_grad", self._h, _lib.ptr(x), _lib.ptr(f), _lib.ptr(y), int(x.shape[0]),
                  g.ctypes.data_as(ctypes.c_void_p) if want_grad else None, ctypes.byref(loss), _lib.stream_ptr())
        return float(loss.value), g

    def adam_step(self, lr: float, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8) -> None:
        _lib.call("simpfem_cnn_adam_step", self._h, float(lr), float(beta1), float(beta2), float(eps),
                  _lib.stream_ptr())

    def train(self, x, feats, labels, *, epochs: int = 30, batch: int = 128, lr: float = 2e-3, seed: int = 0,
              class_balance: bool = True) -> list:
        """Mini-batch Adam on (x, feats, labels); returns the mean loss per epoch.
        With class_balance, each epoch draws every present class equally often."""
        torch = _lib.require_cuda()
        x = _lib.as_cuda(x, torch.float32).reshape(-1, VOX)
        f = _lib.as_cuda(feats, torch.float32).reshape(-1, 2)
        y = np.asarray(labels, dtype=np.int64)
        rng = np.random.default_rng(seed)
        batch = min(batch, self.max_batch)
        hist = []
        for _ in range(epochs):
            if class_balance:
                groups = [np.flatnonzero(y == k) for k in range(3) if np.any(y == k)]
                per = max(len(g) for g in groups)
                order = np.concatenate([rng.choice(g, per, replace=len(g) < per) for g in groups])
                rng.shuffle(order)
            else:
                order = rng.permutation(len(y))
            losses = []
            for s in range(0, len(order) - batch + 1, batch):
                idx = torch.as_tensor(order[s:s + batch], device="cuda")
                lab = torch.as_tensor(y[order[s:s + batch]], dtype=torch.int32, device="cuda")
                loss, _ = self.loss_grad(x[idx], f[idx], lab)
                self.adam_step(lr)
                losses.append(loss)
            hist.append(float(np.mean(losses)) if losses else float("nan"))
        return hist

    def save(self, path: str, **meta) -> None:
        os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
        np.savez_compressed(path, params=self.get_params(), **{k: np.asarray(v) for k, v in meta.items()})

    @classmethod
    def load(cls, path: str = DEFAULT_WEIGHTS, max_batch: int = 256) -> "FloorProposerNet":
        """The network saved at ``path``; its ``min_confidence`` is the threshold
        calibrated with it (0.5 when the file holds none)."""
        with np.load(path) as z:
            net = cls(max_batch=max_batch, params=z["params"])
            if "min_confidence" in z.files:
                net.min_confidence = float(z["min_confidence"])
            return net


class LearnedFloorPolicy(GuardedFloorPolicy):
    """GuardedFloorPolicy that decides at r50 with the proposer.

    ``proposer`` is a FloorProposerNet; ``dims`` the element grid of the preset
    (for pooling); ``min_confidence``: proposals whose softmax probability is
    below it count as rung 0 (the probe continues and the plain rule decides);
    None takes the threshold calibrated with the network (``proposer.min_confidence``).
    Attempt order after a stop at r50: the proposed rung (at least 1e-3), the
    raised rungs above it, the raised rungs below it, and -- when the stop was the
    proposer's and not the high-residual rule's -- the baseline floor last."""

    def __init__(self, preset, *, proposer: FloorProposerNet, dims: Optional[Sequence[int]] = None,
                 min_confidence: Optional[float] = None, **kwargs):
        super().__init__(preset, **kwargs)
        if dims is None:
            dims = (self.spec.nelx, self.spec.nely, self.spec.nelz)
        rungs = [self.baseline_rho_min] + list(self.raised_rho_mins)
        if tuple(rungs) != RUNGS:
            raise ValueError("the proposer is trained on the rungs 1e-12 | 1e-3, 1e-2")
        if self.severity_jump_r50_threshold > 0.0:
            raise ValueError("the severity jump is not combined with the learned proposal")
        self.proposer = proposer
        self.dims = tuple(int(d) for d in dims)
        self.min_confidence = float(proposer.min_confidence if min_confidence is None else min_confidence)

    # device steps of the decision (a host test replaces them)
    def _pool(self, density):
        """The density average-pooled to 16^3 on the device."""
        return self.proposer.pool(density, self.dims)

    def _propose(self, pooled, features) -> np.ndarray:
        """Softmax over the rungs for one pooled density and its two probe features."""
        torch = _lib.require_cuda()
        prob = self.proposer.forward(pooled.reshape(1, -1),
                                     torch.tensor([features], dtype=torch.float32, device="cuda"))
        return prob[0].cpu().numpy()

    def _sync(self) -> None:
        _lib.require_cuda().cuda.current_stream().synchronize()

    def run(self, density, *, binary: bool = False) -> dict:
        rungs = [self.baseline_rho_min] + list(self.raised_rho_mins)
        high = self.thresholds["high_residual_threshold"]
        t0 = time.perf_counter()
        x = self._pool(density)
        self._sync()
        pool_time = time.perf_counter() - t0
        dec = {"prob": None, "proposed": None, "stop": None}

        def at_r50(history):
            r50 = history[min(self.probe_r50, len(history) - 1)]
            prob = self._propose(x, probe_features(r50, history, self.probe_r50, high))
            k = int(np.argmax(prob))
            dec["prob"] = prob
            dec["proposed"] = k if float(prob[k]) >= self.min_confidence else 0
            dec["stop"] = "high_residual" if r50 >= high else ("learned" if dec["proposed"] >= 1 else None)
            return dec["stop"] is not None

        probe_history: list = []
        probe = self.solve_at_floor(density, self.baseline_rho_min, maxiter=self.probe_iters, history=probe_history,
                                    binary=binary, check=(self.probe_r50, at_r50))
        probe_x = self.last_x
        r50 = probe_history[min(self.probe_r50, len(probe_history) - 1)]
        raised = list(range(1, len(rungs)))
        if dec["stop"] is not None:
            r100 = float("nan")
            raise_floor, trigger = True, dec["stop"]
            start = max(1, dec["proposed"])
            seq = [k for k in raised if k >= start] + [k for k in raised if k < start]
            if dec["stop"] == "learned":
                seq.append(0)  # the plain rule might have kept the floor: its rung comes last
        else:
            # the probe ran past r50 (or converged before it): the plain rule decides
            r100 = probe_history[min(self.probe_iters, len(probe_history) - 1)]
            raise_floor, trigger = _classify(r50, r100, **self.thresholds)
            seq = raised if raise_floor else [0] + raised
        attempts: list = []
        attempted: list = []
        sel = None
        for k in seq:
            rho_min = rungs[k]
            attempted.append(rho_min)
            if self.reuse_probe and rho_min == probe.rho_min and probe.solver_reported_converged:
                a = probe
            else:
                a = self.solve_at_floor(density, rho_min, maxiter=self.maxiter, history=[], binary=binary)
            attempts.append(a)
            sel = a
            if a.true_converged:
                break
        if sel is probe:
            self.last_x = probe_x
        failed = [a for a in attempts if a is not sel]
        return {
            "probe_r50": r50, "probe_r100": r100, "probe_iters": probe.iters, "probe_history": probe_history,
            "probe_setup_time_s": probe.setup_time_s, "probe_solve_time_s": probe.solve_time_s,
            "selected_reused_probe": int(sel is probe),
            "selected_setup_time_s": sel.setup_time_s if sel else float("nan"),
            "selected_solve_time_s": sel.solve_time_s if sel else float("nan"),
            "failed_ladder_setup_time_s": sum(a.setup_time_s for a in failed),
            "failed_ladder_solve_time_s": sum(a.solve_time_s for a in failed),
            "solver_reported_converged": int(bool(sel and sel.solver_reported_converged)),
            "trigger": trigger, "predicted_raise_floor": int(raise_floor), "stopped_at_r50": dec["stop"] or "",
            "proposal": -1 if dec["proposed"] is None else dec["proposed"],
            "proposal_prob": [] if dec["prob"] is None else dec["prob"].tolist(),
            "recommended_rho_min": sel.rho_min if sel else float("nan"),
            "attempted_rho_mins": ";".join(f"{v:.0e}" for v in attempted),
            "n_floor_attempts": len(attempted),
            "solve_converged": int(bool(sel and sel.true_converged)),
            "solve_iters": sel.iters if sel else self.maxiter,
            "solve_final_rel_residual": sel.final_rel_residual if sel else float("nan"),
            "n_setups": 1 + sum(1 for a in attempts if a is not probe),
            "total_iters": probe.iters + sum(a.iters for a in attempts if a is not probe),
            "policy_time_s": pool_time + probe.setup_time_s + probe.solve_time_s
            + sum(a.setup_time_s + a.solve_time_s for a in attempts if a is not probe),
            "recorded_policy_time_s": probe.setup_time_s + probe.solve_time_s
            + sum(a.setup_time_s + a.solve_time_s for a in attempts if a is not probe),
            "attempts": attempts,
        }
