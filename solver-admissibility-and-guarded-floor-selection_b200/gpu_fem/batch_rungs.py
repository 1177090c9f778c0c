"""States of uneven mesh sizes in flight together, each solved at every floor rung.

The batching workload of the floor study: cantilever states drawn from several
meshes (default 45 x 30 x 30, 60 x 30 x 30, 80 x 40 x 20), void probability
{0.2, 0.35, 0.5} by seed, cone filter 1.5, SIMP p = 3; every state solved at each
rung {1e-12, 1e-3, 1e-2} with the FP64 recomputed-residual guard
(GuardedFloorPolicy.solve_at_floor, the reference driver's solve_at_floor,
experiments/phase5/run_gmg_floor_detector_prospective.py:220-261).

``RungBatch`` keeps ``width`` workers per mesh, each with its own hierarchy,
mesh handle, CUDA stream and host thread; states go round-robin to the workers
of their mesh and every worker takes its states in order, so results are
deterministic.  All meshes' workers run at once, so states of different sizes
share the GPU.  (No single persistent launch or captured graph: each worker
launches its own kernels; the library synchronises only the worker's stream.)

    python batch_rungs.py [--states 128] [--width 2] [--no-fp64]
"""

from __future__ import annotations

import argparse
import json
import os
import sys
import threading
import time

import numpy as np

if __package__ in (None, ""):
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    __package__ = "gpu_fem"  # noqa: A001

from . import _lib  # noqa: E402

MESHES = ((45, 30, 30), (60, 30, 30), (80, 40, 20))
PROBS = (0.2, 0.35, 0.5)
RUNGS = (1e-12, 1e-3, 1e-2)


def make_states(n_states: int, meshes=MESHES, radius: float = 1.5):
    """State s: mesh s mod len(meshes), void probability PROBS[s mod 3], seed s."""
    from .pub_simp_solver import _build_density_filter

    filters = {}
    out = []
    for s in range(n_states):
        dims = tuple(meshes[s % len(meshes)])
        if dims not in filters:
            filters[dims] = _build_density_filter(dims[0], dims[1], radius, dims[2])
        p = PROBS[s % len(PROBS)]
        solid = (np.random.default_rng(s).random(int(np.prod(dims))) >= p).astype(np.float64)
        out.append((s, dims, np.asarray(filters[dims] @ solid)))
    return out


def _kwargs(precision: str) -> dict:
    from .paper4 import PLAIN_JACOBI_STACK

    stack = dict(PLAIN_JACOBI_STACK, fine_smoother="fp32" if precision == "mixed" else "fp64")
    return dict(penal=3.0, tol=1e-6, restart=300, maxiter=300, probe_iters=100, probe_r50=50,
                raised_rho_mins=(1e-3, 1e-2), stack=stack,
                cycle_precision="fp32" if precision == "mixed" else "fp64")


class RungBatch:
    def __init__(self, meshes=MESHES, width: int = 2, precision: str = "mixed"):
        torch = _lib.require_cuda()
        from ._native import mesh_namespace
        from .policy import GuardedFloorPolicy
        from .presets import cantilever_spec

        if int(width) < 1:
            raise ValueError("width must be >= 1")
        self.width = int(width)
        self.workers = {}
        for dims in meshes:
            dims = tuple(int(d) for d in dims)
            ws = []
            for w in range(self.width):
                with mesh_namespace(("rung-batch", id(self), dims, w)):
                    pol = GuardedFloorPolicy(cantilever_spec(*dims), **_kwargs(precision))
                ws.append((pol, torch.cuda.Stream()))
            _lib.call("simpfem_mesh_tune", ws[0][0].mf_op.mesh.handle, _lib.stream_ptr())
            self.workers[dims] = ws
        torch.cuda.current_stream().synchronize()

    def run(self, states, rungs=RUNGS) -> list:
        """Rows (state, dims, rung, iterations, guarded, true residual, seconds) in
        state order, rungs in the given order per state."""
        torch = _lib.require_cuda()
        jobs = {}
        for idx, (sid, dims, dens) in enumerate(states):
            ws = self.workers[tuple(dims)]
            k = sum(1 for j in range(idx) if tuple(states[j][1]) == tuple(dims))
            jobs.setdefault((tuple(dims), k % self.width), []).append((idx, sid, dens))
        rows = [None] * len(states)
        errors = []
        caller = torch.cuda.current_stream()

        def work(key):
            dims, w = key
            pol, stream = self.workers[dims][w]
            try:
                stream.wait_stream(caller)
                with torch.cuda.stream(stream):
                    for idx, sid, dens in jobs[key]:
                        d = torch.as_tensor(dens, device="cuda")
                        out = []
                        for rho_min in rungs:
                            a = pol.solve_at_floor(d, rho_min, maxiter=pol.maxiter, history=[])
                            out.append({"state": sid, "dims": list(dims), "rho_min": rho_min, "iters": a.iters,
                                        "guarded": int(a.true_converged), "true_rel_residual": a.final_rel_residual,
                                        "seconds": a.setup_time_s + a.solve_time_s})
                        rows[idx] = out
            except BaseException as e:  # raised again on the calling thread
                errors.append(e)

        threads = [threading.Thread(target=work, args=(key,)) for key in jobs]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        for ws in self.workers.values():
            for _, stream in ws:
                caller.wait_stream(stream)
        if errors:
            raise errors[0]
        return [r for rs in rows for r in rs]


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--states", type=int, default=128)
    ap.add_argument("--width", type=int, default=2, help="workers per mesh")
    ap.add_argument("--no-fp64", action="store_true", help="skip the one-at-a-time FP64 comparison")
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    torch = _lib.require_cuda()
    states = make_states(a.states)
    warm = make_states(len(MESHES) * a.width)
    batch = RungBatch(width=a.width)
    batch.run(warm)  # every worker sees one state first
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    rows = batch.run(states)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    res = {"workload": "cantilever states of meshes 45x30x30, 60x30x30, 80x40x20 (void p 0.2/0.35/0.5 by seed, "
                       "cone filter 1.5), each solved at rungs 1e-12, 1e-3, 1e-2 with the FP64 guard",
           "states": a.states, "solves": len(rows), "width_per_mesh": a.width,
           "mixed_batched": {"solves_per_s": len(rows) / (ms / 1e3), "ms": ms,
                             "guarded": sum(r["guarded"] for r in rows),
                             "mean_iters": float(np.mean([r["iters"] for r in rows]))}}
    if not a.no_fp64:
        from .policy import GuardedFloorPolicy
        from .presets import cantilever_spec

        pols = {dims: GuardedFloorPolicy(cantilever_spec(*dims), **_kwargs("fp64")) for dims in MESHES}
        for sid, dims, dens in warm[:len(MESHES)]:
            pols[tuple(dims)].solve_at_floor(torch.as_tensor(dens, device="cuda"), 1e-12, maxiter=300, history=[])
        torch.cuda.synchronize()
        e0.record()
        n64, g64, it64 = 0, 0, []
        for sid, dims, dens in states:
            d = torch.as_tensor(dens, device="cuda")
            for rho_min in RUNGS:
                at = pols[tuple(dims)].solve_at_floor(d, rho_min, maxiter=300, history=[])
                n64 += 1
                g64 += int(at.true_converged)
                it64.append(at.iters)
        e1.record()
        torch.cuda.synchronize()
        ms64 = e0.elapsed_time(e1)
        res["fp64_sequential"] = {"solves_per_s": n64 / (ms64 / 1e3), "ms": ms64, "guarded": g64,
                                  "mean_iters": float(np.mean(it64))}
        res["speedup"] = res["mixed_batched"]["solves_per_s"] / res["fp64_sequential"]["solves_per_s"]
    print(json.dumps(res))
    if a.out:
        with open(a.out, "w") as fh:
            json.dump(dict(res, rows=rows), fh, indent=0)


if __name__ == "__main__":
    main()
