"""Generate, label, train and evaluate the learned floor proposer on one GPU.

    python train_floor_proposer.py [--train 4096] [--heldout 512] [--epochs 40] [--out gpu_fem/data]

States: cantilever meshes 40x20x20 and 80x40x20, elements void with probability
p (seeded Bernoulli); half the states are cone-filtered with p ~ U[0.1, 0.6] and
radius r ~ U[1.2, 2.5] (rounded to 0.1), half are unfiltered masks with
p ~ U[0.1, 0.8] (on the filtered half the probe converges at 1e-12 on every
state, so those states alone hold no escalation to learn); SIMP p = 3, floors
{1e-12 | 1e-3, 1e-2}.  Each training state is solved by the plain guarded policy
(mixed-precision hierarchy, damped-Jacobi V-cycle, probe 100 / r50 at 50,
FGMRES restart 300, tol 1e-6; gpu_fem.policy.BatchedFloorPolicy) and labelled
with the rung that policy selects; the features are the density pooled to 16^3,
the probe's r50 and the iteration at which it reached 1e-2.  The network is
trained with the library's own CUDA forward/backward kernels (class-balanced
mini-batch Adam); then the held-out states are solved one at a time by the plain
policy and by LearnedFloorPolicy and compared: floor attempts, setups, outer
iterations, policy time, selected floor, guarded answers.  Writes
floor_proposer.npz (parameters) and floor_proposer_eval.json (dataset, training
curve, held-out comparison).
"""

from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)

MESHES = ((40, 20, 20), (80, 40, 20))
POLICY = dict(penal=3.0, tol=1e-6, restart=300, maxiter=300, probe_iters=100, probe_r50=50,
              raised_rho_mins=(1e-3, 1e-2), cycle_precision="fp32")

_FILTERS: dict = {}


def cone_filter(solid: np.ndarray, dims, r: float) -> np.ndarray:
    """The solver package's cone density filter (row-normalised), cached per grid and radius."""
    from gpu_fem.pub_simp_solver import _build_density_filter

    key = (tuple(dims), r)
    if key not in _FILTERS:
        _FILTERS[key] = _build_density_filter(dims[0], dims[1], r, dims[2])
    return np.asarray(_FILTERS[key] @ solid)


def make_states(n: int, seed: int):
    """Even-indexed states: the filtered generator (void p ~ U[0.1, 0.6], cone
    radius ~ U[1.2, 2.5] on a 0.1 grid).  Odd-indexed states: unfiltered solid
    masks (radius 1, the identity filter) with void p ~ U[0.1, 0.8], where the
    probe's r50 rule and the ladder's escalations actually occur."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        dims = MESHES[(i // 2) % len(MESHES)]
        if i % 2 == 0:
            p = float(rng.uniform(0.1, 0.6))
            r = round(float(rng.uniform(1.2, 2.5)), 1)
        else:
            p = float(rng.uniform(0.1, 0.8))
            r = 1.0
        solid = (rng.random(int(np.prod(dims))) >= p).astype(np.float64)
        dens = solid if r <= 1.0 else cone_filter(solid, dims, r)
        out.append(dict(dims=dims, p=p, r=r, density=dens))
    return out


def _stack():
    from gpu_fem.paper4 import PLAIN_JACOBI_STACK

    return dict(PLAIN_JACOBI_STACK, fine_smoother="fp32")


def solve_plain(states, width: int):
    import torch

    from gpu_fem.policy import BatchedFloorPolicy
    from gpu_fem.presets import cantilever_spec

    rows = [None] * len(states)
    for dims in MESHES:
        idx = [i for i, s in enumerate(states) if s["dims"] == dims]
        if not idx:
            continue
        bp = BatchedFloorPolicy(width, cantilever_spec(*dims), stack=_stack(), **POLICY)
        res = bp.run_many([torch.as_tensor(states[i]["density"], device="cuda") for i in idx])
        for i, r in zip(idx, res):
            rows[i] = r
    return rows


def features(states, rows):
    import torch

    from gpu_fem.floor_proposer import FloorProposerNet, probe_features, rung_index

    x = torch.stack([FloorProposerNet.pool(torch.as_tensor(s["density"], device="cuda"), s["dims"]) for s in states])
    f = torch.tensor([probe_features(r["probe_r50"], r["probe_history"], POLICY["probe_r50"]) for r in rows],
                     dtype=torch.float32, device="cuda")
    y = np.array([rung_index(r["recommended_rho_min"]) for r in rows], dtype=np.int64)
    return x, f, y


def evaluate(net, held):
    """Held-out states through the plain and the learned policy, one state at a
    time on one stream each (same hierarchy configuration), in the same order."""
    import torch

    from gpu_fem.floor_proposer import LearnedFloorPolicy
    from gpu_fem.policy import GuardedFloorPolicy
    from gpu_fem.presets import cantilever_spec

    plain_rows, learned_rows = [None] * len(held), [None] * len(held)
    for dims in MESHES:
        idx = [i for i, s in enumerate(held) if s["dims"] == dims]
        if not idx:
            continue
        spec = cantilever_spec(*dims)
        plain = GuardedFloorPolicy(spec, stack=_stack(), **POLICY)
        learned = LearnedFloorPolicy(spec, proposer=net, dims=dims, stack=_stack(), **POLICY)
        for i in idx:
            d = torch.as_tensor(held[i]["density"], device="cuda")
            plain_rows[i] = plain.run(d)
            learned_rows[i] = learned.run(d)
    return plain_rows, learned_rows


def compare(plain_rows, learned_rows, mask=None):
    sel = [k for k in range(len(plain_rows)) if mask is None or mask[k]]
    P = [plain_rows[k] for k in sel]
    L = [learned_rows[k] for k in sel]

    def tot(rows, key):
        return float(np.sum([r[key] for r in rows]))

    return {
        "states": len(sel),
        "floor_attempts": [tot(P, "n_floor_attempts"), tot(L, "n_floor_attempts")],
        "setups": [tot(P, "n_setups"), tot(L, "n_setups")],
        "outer_iterations": [tot(P, "total_iters"), tot(L, "total_iters")],
        "policy_time_s": [tot(P, "recorded_policy_time_s"), tot(L, "policy_time_s")],
        "same_selected_floor": float(np.mean([p["recommended_rho_min"] == q["recommended_rho_min"]
                                              for p, q in zip(P, L)])) if sel else float("nan"),
        "higher_floor_than_plain": int(sum(q["recommended_rho_min"] > p["recommended_rho_min"] for p, q in zip(P, L))),
        "lower_floor_than_plain": int(sum(q["recommended_rho_min"] < p["recommended_rho_min"] for p, q in zip(P, L))),
        "guarded": [int(sum(r["solve_converged"] for r in P)), int(sum(r["solve_converged"] for r in L))],
    }


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=4096)
    ap.add_argument("--heldout", type=int, default=512)
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--width", type=int, default=4)
    ap.add_argument("--out", default=os.path.join(HERE, "gpu_fem", "data"))
    a = ap.parse_args()
    import torch

    from gpu_fem.floor_proposer import FloorProposerNet

    t0 = time.time()
    train = make_states(a.train, seed=0)
    held = make_states(a.heldout, seed=1)
    t_gen = time.time() - t0
    t0 = time.time()
    rows_train = solve_plain(train, a.width)
    t_label = time.time() - t0
    xtr, ftr, ytr = features(train, rows_train)
    net = FloorProposerNet(max_batch=256, seed=0)
    t0 = time.time()
    curve = net.train(xtr, ftr, ytr, epochs=a.epochs, batch=128, lr=2e-3, seed=0)
    torch.cuda.synchronize()
    t_train = time.time() - t0
    pred_tr = net.forward(xtr, ftr).argmax(1).cpu().numpy()

    t0 = time.time()
    plain_rows, learned_rows = evaluate(net, held)
    t_eval = time.time() - t0
    xho, fho, yho = features(held, plain_rows)
    pred_ho = net.forward(xho, fho).argmax(1).cpu().numpy()
    escalated = [r["predicted_raise_floor"] == 1 or r["n_floor_attempts"] > 1 for r in plain_rows]
    summary = {
        "states": {"train": a.train, "heldout": a.heldout, "meshes": MESHES,
                   "generator": {"filtered": {"void_p": [0.1, 0.6], "filter_r": [1.2, 2.5]},
                                 "unfiltered": {"void_p": [0.1, 0.8]}},
                   "simp_p": 3.0, "policy": dict(POLICY),
                   "label_counts_train": np.bincount(ytr, minlength=3).tolist(),
                   "label_counts_heldout": np.bincount(yho, minlength=3).tolist()},
        "seconds": {"generate_cpu": t_gen, "label_gpu": t_label, "train_gpu": t_train, "evaluate_gpu": t_eval},
        "training": {"epochs": a.epochs, "batch": 128, "lr": 2e-3, "loss_curve": curve,
                     "train_accuracy": float(np.mean(pred_tr == ytr)),
                     "heldout_accuracy": float(np.mean(pred_ho == yho)),
                     "heldout_confusion": np.histogram2d(yho, pred_ho, bins=[3, 3], range=[[0, 3], [0, 3]])[0]
                     .astype(int).tolist()},
        "heldout_plain_vs_learned": {
            "all": compare(plain_rows, learned_rows),
            "plain_escalated": compare(plain_rows, learned_rows, escalated),
            "plain_kept": compare(plain_rows, learned_rows, [not e for e in escalated]),
            "learned_stopped_at_r50": compare(plain_rows, learned_rows,
                                              [bool(r["stopped_at_r50"]) for r in learned_rows]),
        },
    }
    os.makedirs(a.out, exist_ok=True)
    net.save(os.path.join(a.out, "floor_proposer.npz"), train_accuracy=summary["training"]["train_accuracy"],
             heldout_accuracy=summary["training"]["heldout_accuracy"])
    with open(os.path.join(a.out, "floor_proposer_eval.json"), "w") as fh:
        json.dump(summary, fh, indent=1)
    print(json.dumps({k: v for k, v in summary.items() if k != "training"}, indent=1))
    print(json.dumps({k: v for k, v in summary["training"].items() if k != "loss_curve"}))


if __name__ == "__main__":
    main()
