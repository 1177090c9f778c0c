"""Benchmark: guarded solves/s to true relative residual 1e-6 on the 512k-element
cantilever (160 x 80 x 40), mixed precision vs FP64, one B200 per rank.

A step is one guarded solve of one state: probe at rho_min = 1e-12, r50/r100
preserve/escalate rule, floor ladder {1e-12 | 1e-3, 1e-2}, FP64 recomputed
true-residual guard (gpu_fem.policy.GuardedFloorPolicy).  States follow the
synthetic generator of the workload: element void with probability
p in {0.2, 0.35, 0.5} (seeded Bernoulli), otherwise solid, cone filter of
radius 1.5, E = 1e-12 + (1 - 1e-12) rho_f^3, unit tip load, x = 0 face clamped.
The hierarchy is the damped-Jacobi V-cycle (4 levels, FGMRES restart 300,
tol 1e-6); ``--stack canonical`` selects the reference drivers' default stack.

The mixed arm (``value``, ``e2e``) is the mixed-precision, batched and learned
form: ``--width`` states in flight per GPU (gpu_fem.policy.BatchedFloorPolicy,
one hierarchy and CUDA stream per worker), each worker a LearnedFloorPolicy
with the committed floor proposer (``--policy plain`` for the probe-and-ladder
alone); ``learned_stops_at_r50`` counts the states whose probe the proposal or
the r50 rule ended early.  The ``fp64`` object is the plain FP64 form from
scratch, one state at a time, on the same states.  ``mixed_width1`` is the mixed
form one state at a time (precision without concurrency); ``like_for_like``
repeats both forms with the probe re-solved at a kept floor, as the reference
driver does.  ``error_vs_oracle`` compares the FP64 and the mixed GPU answers of
the first two timed states with the oracle's complete solves of the same states,
whose time is the ``cpu_baseline``; ``--impl reference`` solves those same states.
Two rooflines: the FP32 fused smoothing step and the FP64 operator product,
each launch timed alone after 256 MB of pseudo-random writes evict the L2.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--width B] [--policy learned|plain]
                    [--impl native|reference]
    python bench.py --kernel smoother-step|operator|dense|policy [--grid NX NY NZ] [--reps R]
                    [--precision fp32|fp64] [--stack plain|canonical] [--dense-n N --band BW]

N > 1 (torchrun): ranks solve disjoint states, no collective on the data path;
the reported value is all states / max-over-ranks time.
"""

from __future__ import annotations

import argparse
import ctypes
import datetime
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "solver-admissibility-and-guarded-floor-selection_b200")
sys.path.insert(0, PKG)
sys.path.insert(0, ROOT)

NX, NY, NZ = 160, 80, 40
PROBS = (0.2, 0.35, 0.5)
METRIC = "guarded solves/s & s/solve to true resid 1e-6 @512k elems: mixed vs FP64, 1 B200"


def _args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=48)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="native", choices=["native", "reference"])
    ap.add_argument("--stack", default="plain", choices=["plain", "canonical"])
    ap.add_argument("--width", type=int, default=8, help="states in flight per GPU in the mixed arm")
    ap.add_argument("--policy", default="learned", choices=["learned", "plain", "rule"],
                    help="mixed arm: learned floor proposal (decides at r50), the plain probe-and-ladder, or "
                         "the r50 rule stop alone")
    ap.add_argument("--batch", default="threads", choices=["threads", "native"],
                    help="mixed arm: workers driven from Python threads, or the library's batch entry")
    ap.add_argument("--workload", default="filtered", choices=["filtered", "escalating"],
                    help="filtered: the workload's states; escalating: unfiltered masks, void p 0.5-0.7, whose "
                         "probes escalate")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    # single-kernel launches for timing and ncu captures (no bench line)
    ap.add_argument("--kernel", default=None, choices=["smoother-step", "operator", "dense", "policy"],
                    help="time one library kernel (or one guarded solve) instead of the benchmark")
    ap.add_argument("--grid", type=int, nargs=3, default=[NX, NY, NZ], metavar=("NX", "NY", "NZ"))
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--dense-n", type=int, default=3960)
    ap.add_argument("--band", type=int, default=None)
    ap.add_argument("--restart", type=int, default=300)
    return ap.parse_args()


def run_kernel(args) -> None:
    """One library kernel launched standalone: ``smoother-step`` (the fused fine
    smoothing step, simpfem_gmg_time_smoother_step) and ``operator`` (the FP64
    operator product, simpfem_gmg_time_operator) on the 4-level hierarchy of an
    NX x NY x NZ cantilever with random E in [1e-3, 1.001), each launch timed alone
    from a cold L2; ``dense`` the coarsest factorisation
    (simpfem_dense_cholesky_inverse) of a random SPD matrix, banded with --band;
    ``policy`` one guarded solve after three warm-up states, bracketed by
    cudaProfilerStart/Stop for ncu --profile-from-start off.  Exits 0 on success,
    so the same command line can run under ncu afterwards."""
    import torch

    from gpu_fem import _lib

    nx, ny, nz = args.grid
    ndof, ne = 3 * (nx + 1) * (ny + 1) * (nz + 1), nx * ny * nz
    if args.kernel in ("smoother-step", "operator"):
        from gpu_fem.paper4 import _build_components
        from gpu_fem.presets import cantilever_spec

        st = _stack(args.stack, "mixed" if args.precision == "fp32" else "fp64")
        cyc = "fp32" if args.precision == "fp32" else "fp64"
        gmg = _build_components(cantilever_spec(nx, ny, nz), cycle_precision=cyc, **st)[-1]
        gmg.setup(torch.as_tensor(1e-3 + np.random.default_rng(0).random(ne), device="cuda"))
        avg = ctypes.c_float()
        # the timed launches (one warm launch, then --reps cold ones) are the only ones
        # inside the profiler range, for ncu --profile-from-start off
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        if args.kernel == "smoother-step":
            _lib.call("simpfem_gmg_time_smoother_step", gmg._h, 0, args.reps, ctypes.byref(avg), _lib.stream_ptr())
            s = 4 if args.precision == "fp32" else 8
            alg = (4 if args.stack == "plain" else 6) * s * ndof + s * ne + ndof
        else:
            _lib.call("simpfem_gmg_time_operator", gmg._h, args.reps, ctypes.byref(avg), _lib.stream_ptr())
            alg = 8 * ne + 2 * 8 * ndof + ndof
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        print(json.dumps({"kernel": args.kernel, "grid": [nx, ny, nz], "precision": args.precision,
                          "stack": args.stack, "avg_us": round(avg.value * 1e3, 3),
                          "algorithmic_bytes": alg, "gbs": round(alg / (avg.value * 1e-3) / 1e9, 1)}))
    elif args.kernel == "dense":
        n = args.dense_n
        g = torch.Generator(device="cuda")
        g.manual_seed(0)
        if args.band is None:
            Q = torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g)
            A0 = Q @ Q.T / n + torch.eye(n, dtype=torch.float64, device="cuda")
        else:
            R = torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g)
            i = torch.arange(n, device="cuda")
            A0 = torch.where((i[:, None] - i[None, :]).abs() <= args.band, R, torch.zeros_like(R))
            A0 = torch.tril(A0, -1) + torch.tril(A0, -1).T + torch.diag(
                torch.full((n,), 2.0 * args.band + 2.0, dtype=torch.float64, device="cuda"))
        A, Li = torch.empty_like(A0), torch.empty_like(A0)
        info = ctypes.c_int()
        times = []
        for _ in range(args.reps):
            A.copy_(A0)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            _lib.call("simpfem_dense_cholesky_inverse", n, _lib.ptr(A), _lib.ptr(Li), ctypes.byref(info),
                      _lib.stream_ptr())
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        if info.value != 0:
            raise SystemExit(f"factorisation failed: info {info.value}")
        print(json.dumps({"kernel": "dense", "n": n, "band": args.band, "best_ms": round(min(times), 4),
                          "median_ms": round(statistics.median(times), 4)}))
    else:
        from gpu_fem.policy import GuardedFloorPolicy
        from gpu_fem.presets import cantilever_spec
        from gpu_fem.pub_simp_solver import _build_density_filter

        H = _build_density_filter(nx, ny, 1.5, nz)
        prec = "mixed" if args.precision == "fp32" else "fp64"
        pol = GuardedFloorPolicy(cantilever_spec(nx, ny, nz), penal=3.0, tol=1e-6, restart=args.restart,
                                 maxiter=args.restart, probe_iters=100, probe_r50=50, raised_rho_mins=(1e-3, 1e-2),
                                 stack=_stack(args.stack, prec), cycle_precision="fp32" if prec == "mixed" else "fp64")

        def state(seed):
            solid = (np.random.default_rng(seed).random(ne) >= 0.35).astype(np.float64)
            return torch.as_tensor(np.asarray(H @ solid), device="cuda")

        for seed in range(3):
            pol.run(state(seed))
        d = state(3)
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        r = pol.run(d)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        print(json.dumps({"kernel": "policy", "grid": [nx, ny, nz], "precision": prec,
                          "iters": r["total_iters"], "floor": r["recommended_rho_min"],
                          "setup_ms": round(r["probe_setup_time_s"] * 1e3, 3),
                          "solve_ms": round(r["probe_solve_time_s"] * 1e3, 3), "guarded": r["solve_converged"]}))


def timed_seed_start(warmup: int, width: int) -> int:
    """Index of the first timed state: the batched arm's warm-up takes max(W, 2B) states."""
    return max(warmup, 2 * max(1, width))


def rank_seeds(rank: int, n: int) -> list:
    """State seeds of one rank: disjoint across ranks (replicas shard the states)."""
    return [1000 * rank + i for i in range(n)]


def job_states(per_rank: int, world: int) -> int:
    """States the whole job solves in the timed region (weak scaling)."""
    return per_rank * world


def max_over_ranks(ms: float, world: int, device: str) -> float:
    """The job's time: the slowest rank's device time (one all-reduce MAX)."""
    if world <= 1:
        return ms
    import torch
    import torch.distributed as dist

    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _filter():
    from gpu_fem.pub_simp_solver import _build_density_filter

    return _build_density_filter(NX, NY, 1.5, NZ)


ESCALATING_PROBS = (0.5, 0.6, 0.7)


def make_state(H, seed: int, workload: str = "filtered") -> np.ndarray:
    """The workload's state: void with probability PROBS[seed % 3], cone filter
    r = 1.5; ``escalating``: unfiltered solid masks with void probability
    ESCALATING_PROBS[seed % 3], where the probe's r50 / r100 rule raises floors."""
    if workload == "escalating":
        p = ESCALATING_PROBS[seed % len(ESCALATING_PROBS)]
        return (np.random.default_rng(seed).random(NX * NY * NZ) >= p).astype(np.float64)
    p = PROBS[seed % len(PROBS)]
    solid = (np.random.default_rng(seed).random(NX * NY * NZ) >= p).astype(np.float64)
    return np.asarray(H @ solid)


def _stack(name: str, precision: str) -> dict:
    from gpu_fem.paper4 import CANONICAL_STACK, PLAIN_JACOBI_STACK

    st = dict(CANONICAL_STACK if name == "canonical" else PLAIN_JACOBI_STACK)
    st["fine_smoother"] = "fp32" if precision == "mixed" else "fp64"
    return st


class ClockSampler:
    """SM clocks and throttle reasons sampled every 200 ms while running: NVML
    queries in-process (no child process is started inside the timed region),
    nvidia-smi only when NVML is not importable."""

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = threading.Thread(target=self._run, daemon=True)

    def _nvml_handle(self):
        import pynvml
        import torch

        pynvml.nvmlInit()
        try:
            p = torch.cuda.get_device_properties(self.index)
            bus = f"{p.pci_domain_id:08X}:{p.pci_bus_id:02X}:{p.pci_device_id:02X}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def _run(self):
        try:
            nv, h = self._nvml_handle()
        except Exception:
            nv = None
        if nv is not None:
            bits = (nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                    nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap)
            while not self._stop.is_set():
                try:
                    r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                    self.samples.append([str(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)),
                                         str(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)),
                                         str(nv.nvmlDeviceGetPowerUsage(h) / 1000.0)]
                                        + ["Active" if r & b else "Not Active" for b in bits])
                except Exception:
                    pass
                self._stop.wait(0.2)
            return
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                f = [x.strip() for x in out.stdout.strip().split(",")]
                if len(f) >= 7:
                    self.samples.append(f)
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self) -> dict:
        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [v for v in (num(s[0]) for s in self.samples) if v is not None]
        mx = [v for v in (num(s[1]) for s in self.samples) if v is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[3 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _traffic_per_launch():
    """DRAM bytes per launch of the timed kernel from the committed ncu summary."""
    try:
        with open(os.path.join(ROOT, "profiles", "roofline_traffic.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def run_native(args):
    import torch
    import torch.distributed as dist

    from gpu_fem import _lib
    from gpu_fem.policy import BatchedFloorPolicy, GuardedFloorPolicy
    from gpu_fem.presets import cantilever_spec

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=datetime.timedelta(seconds=300))
    H = _filter()
    spec = cantilever_spec(NX, NY, NZ)
    K, W, B = args.steps, args.warmup, max(1, args.width)
    WB = timed_seed_start(W, B)  # warm-up states for the batched arm: every worker sees at least two
    seeds = rank_seeds(rank, WB + 2 * K)
    states = {s: make_state(H, s, args.workload) for s in seeds}

    def policy_kwargs(precision):
        return dict(penal=3.0, tol=1e-6, restart=300, maxiter=300, probe_iters=100, probe_r50=50,
                    raised_rho_mins=(1e-3, 1e-2), stack=_stack(args.stack, precision),
                    cycle_precision="fp32" if precision == "mixed" else "fp64")

    def policy(precision):
        return GuardedFloorPolicy(spec, **policy_kwargs(precision))

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def timed(pol, seq, host_io: bool):
        dev = {s: torch.as_tensor(states[s], device="cuda") for s in seq} if not host_io else None
        host = {s: torch.as_tensor(states[s]).pin_memory() for s in seq} if host_io else None
        rows = []
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = _lib.lib().simpfem_launch_count()
        e0.record()
        for s in seq:
            if host_io:
                out = pol.run(host[s].to("cuda", non_blocking=True))
                out["x_host"] = pol.last_x.to("cpu")
            else:
                out = pol.run(dev[s])
            rows.append(out)
        e1.record()
        barrier()
        ms = e0.elapsed_time(e1)
        launches = _lib.lib().simpfem_launch_count() - l0
        ms = max_over_ranks(ms, world, "cuda")
        return ms, rows, launches

    def timed_batch(bp, seq, host_io: bool):
        # host_io: pinned host densities in, each solution x back to the host, inside the timed region
        if host_io:
            dens = [torch.as_tensor(states[s]).pin_memory() for s in seq]
            # pinned result buffers; each solution is copied asynchronously on its
            # worker's stream (the stream order keeps it ahead of the next solve)
            xs = [torch.empty(bp.workers[0].F_free_gpu.numel(), dtype=torch.float64).pin_memory() for _ in seq]
        else:
            dens = [torch.as_tensor(states[s], device="cuda") for s in seq]
            xs = []

        def keep_x(k, worker, row):
            xs[k].copy_(worker.last_x, non_blocking=True)

        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = _lib.lib().simpfem_launch_count()
        e0.record()
        if args.batch == "native":
            # the whole batch inside the library (simpfem_policy_batch); solutions copied after
            rows = bp.run_many_native(dens, keep_x=host_io)
            for k in range(len(xs)):
                xs[k].copy_(bp.last_xs[k], non_blocking=True)
        else:
            rows = bp.run_many(dens, on_result=keep_x if host_io else None)
        e1.record()
        barrier()
        ms = e0.elapsed_time(e1)
        launches = _lib.lib().simpfem_launch_count() - l0
        ms = max_over_ranks(ms, world, "cuda")
        return ms, rows, launches

    # mixed precision, B states in flight (one hierarchy and stream per worker)
    learned = None
    if args.policy == "learned":
        from gpu_fem.floor_proposer import DEFAULT_WEIGHTS

        learned = DEFAULT_WEIGHTS
    elif args.policy == "rule":
        learned = "rule"
    mixed = BatchedFloorPolicy(B, spec, learned=learned, **policy_kwargs("mixed"))
    mixed.run_many([torch.as_tensor(states[s], device="cuda") for s in seeds[:WB]])
    timed_seeds = seeds[WB:WB + K]
    with ClockSampler(local) as clk:
        ms_mixed, rows_mixed, launches = timed_batch(mixed, timed_seeds, host_io=False)
    ms_e2e, rows_e2e, _ = timed_batch(mixed, seeds[WB + K:WB + 2 * K], host_io=True)
    # plain FP64 from scratch, one state at a time, on the same states
    fp64 = policy("fp64")
    for s in seeds[:W]:
        fp64.run(torch.as_tensor(states[s], device="cuda"))
    ms_fp64, rows_fp64, _ = timed(fp64, timed_seeds, host_io=False)

    # the same forms with the probe re-solved at a kept floor, as the reference
    # driver does (like for like with the reference arm), and the mixed form one
    # state at a time (what precision buys without concurrency)
    for w in mixed.workers:
        w.reuse_probe = False
    fp64.reuse_probe = False
    ms_mixed_nr, rows_mixed_nr, _ = timed_batch(mixed, timed_seeds, host_io=False)
    ms_fp64_nr, rows_fp64_nr, _ = timed(fp64, timed_seeds, host_io=False)
    for w in mixed.workers:
        w.reuse_probe = True
    fp64.reuse_probe = True
    ms_mixed_w1, rows_mixed_w1, _ = timed(mixed.workers[0], timed_seeds, host_io=False)

    # the mixed solve's error against the FP64 solve of the same state (untimed,
    # after the timed regions): displacement and compliance, first 8 timed states
    w0 = mixed.workers[0]
    F = w0.F_free_gpu
    fp64_err = []
    for s in timed_seeds[:8]:
        d = torch.as_tensor(states[s], device="cuda")
        rm = w0.run(d)
        xm = w0.last_x.clone()
        rf = fp64.run(d)
        xf = fp64.last_x
        cm, cf = float(torch.dot(F, xm)), float(torch.dot(F, xf))
        fp64_err.append((float(torch.linalg.norm(xm - xf) / torch.linalg.norm(xf)), abs(cm - cf) / abs(cf),
                         rm["recommended_rho_min"] == rf["recommended_rho_min"]))
    torch.cuda.synchronize()

    n_states = job_states(K, world)
    value = n_states / (ms_mixed / 1e3)
    e2e_value = n_states / (ms_e2e / 1e3)
    n_free = int(mixed.workers[0].F_free_gpu.numel())

    # roofline of the dominant kernel: the fused fine smoothing step of the cycle
    hbm_peak, peak_kind = _peaks()
    avg = ctypes.c_float()
    _lib.call("simpfem_gmg_time_smoother_step", mixed.workers[0].gmg._h, 0, 50, ctypes.byref(avg),
              _lib.stream_ptr())
    ndof = 3 * (NX + 1) * (NY + 1) * (NZ + 1)
    ne = NX * NY * NZ
    # the FP64 operator product of every FGMRES iteration and of the guard
    avg64 = ctypes.c_float()
    _lib.call("simpfem_gmg_time_operator", fp64.gmg._h, 50, ctypes.byref(avg64), _lib.stream_ptr())
    op_bytes = 8 * ne + 2 * 8 * ndof + ndof  # read E and u, write y (FP64), 1-byte DOF mask
    op_flops = 1152 * ne                     # 2 x 24 x 24 per element, the reference's convention
    # fp32 vectors read u, rhs, dinv (plus d for Chebyshev) and write x (plus d); E (fp32); 1-byte DOF mask
    nvec = 4 if args.stack == "plain" else 6
    alg_bytes = nvec * 4 * ndof + 4 * ne + ndof
    achieved = alg_bytes / (avg.value * 1e-3) / 1e9
    traffic = _traffic_per_launch().get(f"fine_step_{args.stack}_mixed")
    result = {
        "metric": METRIC,
        "value": round(value, 4),
        "unit": "guarded solves/s",
        "n_gpus": world,
        "steps": K,
        "warmup": W,
        "ms_per_step": round(ms_mixed / K, 3),
        "s_per_solve": round(ms_mixed / K / 1e3, 5),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 V-cycle (bf16-stored coarse stencils), f64 FGMRES/Cholesky/guard",
        "data": ("synthetic (seeded void p in {0.2,0.35,0.5}, cone filter r=1.5, SIMP p=3)"
                 if args.workload == "filtered" else
                 "synthetic escalating (seeded unfiltered masks, void p in {0.5,0.6,0.7}, SIMP p=3)"),
        "config": {
            "workload": "guarded SIMP-floor solve, cantilever 160x80x40 (512,000 elements, "
                        f"{n_free} free DOFs), floors 1e-12|1e-3,1e-2, 4-level GMG ({args.stack} stack), "
                        "FGMRES restart 300 tol 1e-6, r50/r100 probe 100 its",
            "global_batch": n_states,
            "batch_width": B,
            "parallelism": f"{B} states in flight per GPU (one stream each, {args.batch}) x {world} replicas",
            "l2": "working set larger than L2 (FGMRES basis + hierarchy > 126 MB); no flush",
        },
        "clocks": clk.summary(),
        "fp64": {
            "value": round(n_states / (ms_fp64 / 1e3), 4),
            "unit": "guarded solves/s",
            "s_per_solve": round(ms_fp64 / K / 1e3, 5),
            "speedup_mixed_over_fp64": round(ms_fp64 / ms_mixed, 3),
        },
        "mixed_width1": {
            "value": round(n_states / (ms_mixed_w1 / 1e3), 4),
            "unit": "guarded solves/s",
            "speedup_over_fp64": round(ms_fp64 / ms_mixed_w1, 3),
            "note": "the mixed form one state at a time: what precision buys without concurrency",
        },
        "like_for_like": {
            "mixed_value": round(n_states / (ms_mixed_nr / 1e3), 4),
            "fp64_value": round(n_states / (ms_fp64_nr / 1e3), 4),
            "unit": "guarded solves/s",
            "speedup_mixed_over_fp64": round(ms_fp64_nr / ms_mixed_nr, 3),
            "all_guarded": all(r["solve_converged"] for r in rows_mixed_nr + rows_fp64_nr),
            "note": "probe re-solved at a kept floor (reuse_probe off), as the reference driver does",
        },
        "solves": [
            {"seed": s, "trigger": r["trigger"], "rho_min": r["recommended_rho_min"],
             "converged": r["solve_converged"], "iters": r["total_iters"],
             "true_residual": r["solve_final_rel_residual"], "fp64_iters": f["total_iters"],
             "fp64_true_residual": f["solve_final_rel_residual"]}
            for s, r, f in zip(timed_seeds, rows_mixed, rows_fp64)
        ],
        "all_guarded": all(r["solve_converged"] for r in rows_mixed + rows_e2e + rows_fp64),
        "error_vs_fp64": {
            "states": len(fp64_err),
            "x_rel_err_max": max(e[0] for e in fp64_err),
            "compliance_rel_err_max": max(e[1] for e in fp64_err),
            "same_floor": all(e[2] for e in fp64_err),
            "note": "mixed vs FP64 solve of the same state, both stopped at true relative residual <= 1e-6",
        },
        "policy": args.policy,
        "workload": args.workload,
        "triggers": {t: sum(1 for r in rows_mixed if r["trigger"] == t) for t in sorted({r["trigger"] for r in rows_mixed})},
        "mixed_total_outer_iterations": int(sum(r["total_iters"] for r in rows_mixed)),
        "learned_stops_at_r50": sum(1 for r in rows_mixed + rows_e2e if r.get("stopped_at_r50")),
        "e2e": {
            "value": round(e2e_value, 4),
            "unit": "guarded solves/s",
            "h2d_bytes_per_step": 8 * ne,
            "d2h_bytes_per_step": 8 * n_free,
        },
        "gpu_launches": int(launches),
        "roofline": {
            "kernel": f"fine_sweep_x2_kernel<EPI_{'JAC' if args.stack == 'plain' else 'CHEB'}> (FP32 fused smoothing step, cold L2)",
            "bound": "hbm",
            "achieved": round(achieved, 1),
            "peak": hbm_peak,
            "peak_kind": peak_kind,
            "unit": "GB/s",
            "frac": round(achieved / hbm_peak, 4),
            "traffic": traffic,
            "algorithmic_bytes_per_launch": alg_bytes,
            "avg_launch_us": round(avg.value * 1e3, 3),
        },
        "roofline_fp64_operator": {
            "kernel": "fine_sweep_kernel<double, EPI_APPLY> (FP64 operator product, cold L2)",
            "bound": "hbm",
            "achieved": round(op_bytes / (avg64.value * 1e-3) / 1e9, 1),
            "peak": hbm_peak,
            "peak_kind": peak_kind,
            "unit": "GB/s",
            "frac": round(op_bytes / (avg64.value * 1e-3) / 1e9 / hbm_peak, 4),
            "traffic": _traffic_per_launch().get("fine_op_fp64"),
            "algorithmic_bytes_per_launch": op_bytes,
            "gflops_reference_convention": round(op_flops / (avg64.value * 1e-3) / 1e9, 1),
            "avg_launch_us": round(avg64.value * 1e3, 3),
        },
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the oracle (the reference's FP64 method on numpy/scipy) solves the first two
        # timed states completely; its answers judge both GPU forms, and its time is
        # the CPU baseline
        n_or = 2
        orc = oracle_solves([states[s] for s in timed_seeds[:n_or]])
        errs = []
        for k, s in enumerate(timed_seeds[:n_or]):
            d = torch.as_tensor(states[s], device="cuda")
            ref = orc["results"][k]
            xo = torch.as_tensor(ref["x"], device="cuda")
            co = float(torch.dot(F, xo))
            for form, pol in (("fp64", fp64), ("mixed", w0)):
                r = pol.run(d)
                x = pol.last_x
                errs.append({"seed": s, "form": form,
                             "x_rel_err": float(torch.linalg.norm(x - xo) / torch.linalg.norm(xo)),
                             "compliance_rel_err": abs(float(torch.dot(F, x)) - co) / abs(co),
                             "same_decisions": r["recommended_rho_min"] == ref["rho_min"]
                             and r["trigger"] == ref["trigger"] and bool(r["solve_converged"]) == ref["converged"],
                             "true_residual": r["solve_final_rel_residual"]})
        result["error_vs_oracle"] = {
            "states": n_or,
            "per_solve": errs,
            "fp64_x_rel_err_max": max(e["x_rel_err"] for e in errs if e["form"] == "fp64"),
            "fp64_compliance_rel_err_max": max(e["compliance_rel_err"] for e in errs if e["form"] == "fp64"),
            "mixed_x_rel_err_max": max(e["x_rel_err"] for e in errs if e["form"] == "mixed"),
            "mixed_compliance_rel_err_max": max(e["compliance_rel_err"] for e in errs if e["form"] == "mixed"),
            "same_decisions": all(e["same_decisions"] for e in errs),
            "note": "GPU answers of the first timed states against the oracle's complete FP64 guarded solves "
                    "of the same states (all stopped at true relative residual <= 1e-6)",
        }
        result["cpu_baseline"] = orc["cpu_baseline"]
    if rank == 0:
        print(json.dumps(result), flush=True)
    if world > 1:
        dist.destroy_process_group()


def oracle_solves(densities) -> dict:
    """The oracle (the reference's FP64 method on numpy/scipy: damped-Jacobi 4-level
    GMG, FGMRES restart 300, the guarded policy with the probe re-solved at a kept
    floor, as the reference driver does) on complete guarded solves of the given
    512k states, in order through one hierarchy, on all host cores."""
    from oracle.gmg import GMG
    from oracle.policy import run_state
    from oracle.solver import Operator, cantilever_bc

    cores = len(os.sched_getaffinity(0))
    free, F = cantilever_bc(NX, NY, NZ)
    op = Operator(NX, NY, NZ, free)
    Ff = F[free]
    g = GMG(op, n_levels=4, fine_smoother="fp64", smoother_type="jacobi")
    results, times = [], []
    for d in densities:
        t0 = time.perf_counter()
        res = run_state(op, g, Ff, lambda rm, d=d: d, penal=3.0, raised=(1e-3, 1e-2), restart=300, maxiter=300)
        times.append(time.perf_counter() - t0)
        sel = res["selected"]
        results.append({"x": sel["x"], "rho_min": sel["rho_min"], "trigger": res["trigger"],
                        "converged": bool(sel["converged"])})
    v = len(times) / sum(times)
    return {"results": results, "times": times,
            "cpu_baseline": {"value": round(v, 6), "unit": "guarded solves/s", "cores": cores, "kind": "port",
                             "sample": f"{len(times)} complete guarded solves of the first timed 512k states "
                                       f"(oracle, numpy/scipy FP64; {', '.join(f'{t:.1f}' for t in times)} s)",
                             "s_per_solve": round(sum(times) / len(times), 2)}}


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle.gmg import GMG
    from oracle.policy import run_state
    from oracle.solver import Operator, cantilever_bc

    H = _filter()
    free, F = cantilever_bc(NX, NY, NZ)
    op = Operator(NX, NY, NZ, free)
    Ff = F[free]
    g = GMG(op, n_levels=4, fine_smoother="fp64", smoother_type="jacobi")
    steps = max(1, min(args.steps, 2))
    # the same states as the native arm's first timed states
    first = timed_seed_start(args.warmup, args.width)
    times = []
    for i in range(steps):
        d = make_state(H, first + i, args.workload)
        t0 = time.perf_counter()
        run_state(op, g, Ff, lambda rm, d=d: d, penal=3.0, raised=(1e-3, 1e-2), restart=300, maxiter=300)
        times.append(time.perf_counter() - t0)
    v = steps / sum(times)
    cores = len(os.sched_getaffinity(0))
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(v, 6), "unit": "guarded solves/s", "n_gpus": world,
        "steps": steps, "warmup": 0, "ms_per_step": round(1e3 * sum(times) / steps, 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "guarded SIMP-floor solve, cantilever 160x80x40 (512,000 elements), damped-Jacobi "
                               "4-level GMG, FGMRES restart 300 tol 1e-6, floors 1e-12|1e-3,1e-2"},
        "cpu_baseline": {"value": round(v, 6), "unit": "guarded solves/s", "cores": cores, "kind": "port",
                         "sample": f"{steps} complete guarded solves of seeds {first}..{first + steps - 1}, the "
                                   "native arm's first timed states (oracle, numpy/scipy FP64)"},
        "e2e": {"value": round(v, 6), "unit": "guarded solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


if __name__ == "__main__":
    a = _args()
    if a.kernel is not None:
        run_kernel(a)
    elif a.impl == "reference":
        run_reference(a)
    else:
        run_native(a)
