"""Generate, label, train and evaluate the learned floor proposer on one GPU.

    python train_floor_proposer.py [--train 4096] [--val 512] [--heldout 512] [--epochs 30] [--out gpu_fem/data]

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
mini-batch Adam) on all but the last --val training states, which choose the
epoch (lowest validation loss).  The held-out states are then solved one at a
time by the plain policy, by the r50 rule stop alone (no network) and by
LearnedFloorPolicy, and compared: floor attempts, setups, outer iterations,
policy time, selected floor, guarded answers.  Writes
floor_proposer.npz (parameters) and floor_proposer_eval.json (dataset, training
curve, held-out comparison).

    python train_floor_proposer.py --calibrate 256

keeps the saved network and picks its confidence threshold (the softmax
probability below which a proposal counts as "keep the probe running") on 256
fresh states: the threshold with the fewest outer iterations among those that
guard as many answers as the plain policy.  It is saved with the parameters
(LearnedFloorPolicy uses it by default) and the held-out states are compared
again with it.
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
    """Held-out states through three policies, one state at a time on one stream
    each (same hierarchy configuration, same order): the plain policy; the r50
    rule stop alone (LearnedFloorPolicy with a proposer that always says rung 0,
    so the probe stops at r50 only when r50 is above the high threshold); and the
    learned policy with the trained network."""
    import torch

    from gpu_fem.floor_proposer import FloorProposerNet, LearnedFloorPolicy
    from gpu_fem.policy import GuardedFloorPolicy
    from gpu_fem.presets import cantilever_spec

    zero = FloorProposerNet(max_batch=4, params=np.zeros(net.n_params, dtype=np.float32))
    rows = {"plain": [None] * len(held), "rule": [None] * len(held), "learned": [None] * len(held)}
    for dims in MESHES:
        idx = [i for i, s in enumerate(held) if s["dims"] == dims]
        if not idx:
            continue
        spec = cantilever_spec(*dims)
        pols = {"plain": GuardedFloorPolicy(spec, stack=_stack(), **POLICY),
                "rule": LearnedFloorPolicy(spec, proposer=zero, dims=dims, stack=_stack(), **POLICY),
                "learned": LearnedFloorPolicy(spec, proposer=net, dims=dims, stack=_stack(), **POLICY)}
        for i in idx:
            d = torch.as_tensor(held[i]["density"], device="cuda")
            for k, pol in pols.items():
                rows[k][i] = pol.run(d)
    return rows


def calibrate(net, states, thresholds):
    """Total outer iterations and guarded answers of the plain policy, the r50 rule
    stop alone and the learned policy at each confidence threshold on ``states``
    (one state at a time, as in ``evaluate``)."""
    import torch

    from gpu_fem.floor_proposer import FloorProposerNet, LearnedFloorPolicy
    from gpu_fem.policy import GuardedFloorPolicy
    from gpu_fem.presets import cantilever_spec

    zero = FloorProposerNet(max_batch=4, params=np.zeros(net.n_params, dtype=np.float32))
    arms = ["plain", "rule"] + [f"learned@{t:g}" for t in thresholds]
    tot = {a: {"outer_iterations": 0, "guarded": 0, "same_floor_as_plain": 0} for a in arms}
    for dims in MESHES:
        idx = [i for i, st in enumerate(states) if st["dims"] == dims]
        if not idx:
            continue
        spec = cantilever_spec(*dims)
        pols = {"plain": GuardedFloorPolicy(spec, stack=_stack(), **POLICY),
                "rule": LearnedFloorPolicy(spec, proposer=zero, dims=dims, stack=_stack(), **POLICY)}
        for t in thresholds:
            pols[f"learned@{t:g}"] = LearnedFloorPolicy(spec, proposer=net, dims=dims, min_confidence=t,
                                                        stack=_stack(), **POLICY)
        for i in idx:
            d = torch.as_tensor(states[i]["density"], device="cuda")
            rows = {a: pol.run(d) for a, pol in pols.items()}
            for a, r in rows.items():
                tot[a]["outer_iterations"] += int(r["total_iters"])
                tot[a]["guarded"] += int(r["solve_converged"])
                tot[a]["same_floor_as_plain"] += int(r["recommended_rho_min"] == rows["plain"]["recommended_rho_min"])
    return tot


def compare(rows, mask=None):
    """Totals per policy over the states in ``mask`` (all by default); floors are
    compared with the plain policy's selection."""
    plain = rows["plain"]
    sel = [k for k in range(len(plain)) if mask is None or mask[k]]

    def tot(arm, key):
        return float(np.sum([rows[arm][k][key] for k in sel]))

    out = {"states": len(sel)}
    for arm in rows:
        tkey = "recorded_policy_time_s" if arm == "plain" else "policy_time_s"
        out[arm] = {
            "floor_attempts": tot(arm, "n_floor_attempts"),
            "setups": tot(arm, "n_setups"),
            "outer_iterations": tot(arm, "total_iters"),
            "policy_time_s": tot(arm, tkey),
            "guarded": int(tot(arm, "solve_converged")),
            "same_floor_as_plain": int(sum(rows[arm][k]["recommended_rho_min"] == plain[k]["recommended_rho_min"]
                                           for k in sel)),
            "higher_floor_than_plain": int(sum(rows[arm][k]["recommended_rho_min"] > plain[k]["recommended_rho_min"]
                                               for k in sel)),
        }
    return out


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=4096)
    ap.add_argument("--heldout", type=int, default=512)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--val", type=int, default=512)
    ap.add_argument("--width", type=int, default=4)
    ap.add_argument("--out", default=os.path.join(HERE, "gpu_fem", "data"))
    ap.add_argument("--calibrate", type=int, default=0, metavar="N",
                    help="only calibrate the saved network's confidence threshold on N fresh states "
                         "(seed 2) and re-evaluate the held-out states with it")
    a = ap.parse_args()
    import torch

    from gpu_fem.floor_proposer import FloorProposerNet

    if a.calibrate:
        path = os.path.join(a.out, "floor_proposer.npz")
        net = FloorProposerNet.load(path, max_batch=4)
        thresholds = (0.5, 0.7, 0.9, 0.97, 0.995)
        cal = calibrate(net, make_states(a.calibrate, seed=2), thresholds)
        # the threshold with the fewest outer iterations among those guarding as many
        # answers as the plain policy; ties go to the higher (more conservative) one
        ok = [t for t in thresholds if cal[f"learned@{t:g}"]["guarded"] >= cal["plain"]["guarded"]]
        best = min(ok, key=lambda t: (cal[f"learned@{t:g}"]["outer_iterations"], -t)) if ok else 1.0
        net.min_confidence = float(best)
        held = make_states(a.heldout, seed=1)
        rows = evaluate(net, held)
        escalated = [r["predicted_raise_floor"] == 1 or r["n_floor_attempts"] > 1 for r in rows["plain"]]
        with open(os.path.join(a.out, "floor_proposer_eval.json")) as fh:
            summary = json.load(fh)
        summary["calibration"] = {"states": a.calibrate, "seed": 2, "thresholds": list(thresholds),
                                  "totals": cal, "chosen_min_confidence": best}
        summary["heldout_policies_calibrated"] = {
            "min_confidence": best,
            "all": compare(rows),
            "plain_escalated": compare(rows, escalated),
            "plain_kept": compare(rows, [not e for e in escalated]),
        }
        with np.load(path) as z:
            meta = {k: z[k] for k in z.files if k not in ("params", "min_confidence")}
        net.save(path, min_confidence=best, **meta)
        with open(os.path.join(a.out, "floor_proposer_eval.json"), "w") as fh:
            json.dump(summary, fh, indent=1)
        print(json.dumps({"calibration": summary["calibration"],
                          "heldout": summary["heldout_policies_calibrated"]}, indent=1))
        return

    t0 = time.time()
    train = make_states(a.train, seed=0)
    held = make_states(a.heldout, seed=1)
    t_gen = time.time() - t0
    t0 = time.time()
    rows_train = solve_plain(train, a.width)
    t_label = time.time() - t0
    xtr, ftr, ytr = features(train, rows_train)
    # the last --val training states choose the epoch (lowest validation loss)
    nfit = len(train) - a.val
    net = FloorProposerNet(max_batch=256, seed=0)
    t0 = time.time()
    curve, val_curve = [], []
    best = (float("inf"), -1, None)
    for ep in range(a.epochs):
        curve += net.train(xtr[:nfit], ftr[:nfit], ytr[:nfit], epochs=1, batch=128, lr=2e-3, seed=ep)
        pv = net.forward(xtr[nfit:], ftr[nfit:]).double().cpu().numpy()
        vl = float(-np.mean(np.log(np.maximum(pv[np.arange(a.val), ytr[nfit:]], 1e-30))))
        val_curve.append(vl)
        if vl < best[0]:
            best = (vl, ep, net.get_params())
    net.set_params(best[2])
    torch.cuda.synchronize()
    t_train = time.time() - t0
    pred_tr = net.forward(xtr[:nfit], ftr[:nfit]).argmax(1).cpu().numpy()
    pred_val = net.forward(xtr[nfit:], ftr[nfit:]).argmax(1).cpu().numpy()

    t0 = time.time()
    rows = evaluate(net, held)
    t_eval = time.time() - t0
    xho, fho, yho = features(held, rows["plain"])
    pred_ho = net.forward(xho, fho).argmax(1).cpu().numpy()
    escalated = [r["predicted_raise_floor"] == 1 or r["n_floor_attempts"] > 1 for r in rows["plain"]]

    def confusion(y, p):
        return np.histogram2d(y, p, bins=[3, 3], range=[[0, 3], [0, 3]])[0].astype(int).tolist()

    summary = {
        "states": {"train": nfit, "validation": a.val, "heldout": a.heldout, "meshes": MESHES,
                   "generator": {"filtered": {"void_p": [0.1, 0.6], "filter_r": [1.2, 2.5]},
                                 "unfiltered": {"void_p": [0.1, 0.8]}},
                   "simp_p": 3.0, "policy": dict(POLICY),
                   "label_counts_train": np.bincount(ytr[:nfit], minlength=3).tolist(),
                   "label_counts_validation": np.bincount(ytr[nfit:], minlength=3).tolist(),
                   "label_counts_heldout": np.bincount(yho, minlength=3).tolist()},
        "seconds": {"generate_cpu": t_gen, "label_gpu": t_label, "train_gpu": t_train, "evaluate_gpu": t_eval},
        "training": {"epochs": a.epochs, "chosen_epoch": best[1], "batch": 128, "lr": 2e-3,
                     "loss_curve": curve, "validation_loss_curve": val_curve,
                     "train_accuracy": float(np.mean(pred_tr == ytr[:nfit])),
                     "validation_accuracy": float(np.mean(pred_val == ytr[nfit:])),
                     "heldout_accuracy": float(np.mean(pred_ho == yho)),
                     "heldout_confusion": confusion(yho, pred_ho)},
        "heldout_policies": {
            "all": compare(rows),
            "plain_escalated": compare(rows, escalated),
            "plain_kept": compare(rows, [not e for e in escalated]),
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
