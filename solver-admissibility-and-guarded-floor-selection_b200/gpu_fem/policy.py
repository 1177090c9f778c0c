"""The guarded SIMP-floor policy: probe -> preserve/escalate -> floor ladder ->
recomputed true-residual guard.

Follows experiments/phase5/run_gmg_floor_detector_prospective.py:
``_classify`` (:77-90), ``solve_at_floor`` (:220-261), the r50 / r100 probe
read-out (:263-277), the optional severity jump (:278-290), the floor sequence
(:313-349) and the post-solve fallback after a failed keep (:351-354).  The
density-field variant (run_gmg_floor_detector_density_field.py:180-299) is the
same policy with E = rho_min + (1 - rho_min) * density ** penal; the Bernoulli
variant first maps a solid mask to rho = 1 (solid) / rho_min (void).

Every accepted answer passes the FP64 guard ||F - K(E) x|| / ||F|| <= tol,
recomputed from x after the solve.
"""

from __future__ import annotations

import ctypes
import threading
import time
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._native import mesh_namespace
from .multigrid_v4 import _cupy_fgmres
from .paper4 import CANONICAL_STACK, _build_components


def _classify(r50: float, r100: float, *, high_residual_threshold: float, plateau_residual_threshold: float,
              plateau_ratio_threshold: float) -> tuple[bool, str]:
    if r50 >= high_residual_threshold:
        return True, "high_r50"
    ratio = r100 / max(r50, 1e-300)
    if r100 >= plateau_residual_threshold and ratio >= plateau_ratio_threshold:
        return True, "plateau"
    return False, "keep"


@dataclass
class FloorAttempt:
    rho_min: float
    iters: int
    solver_reported_converged: bool
    true_converged: bool
    final_rel_residual: float
    setup_time_s: float
    solve_time_s: float
    history: list = field(default_factory=list)


class GuardedFloorPolicy:
    """One hierarchy reused across states (as the drivers do), so the lambda_max
    cache carries over from state to state exactly like the reference."""

    def __init__(self, preset="cantilever_gpu_medium", *, penal: float = 4.5, tol: float = 1e-6,
                 restart: int = 300, maxiter: int = 300, probe_iters: int = 100, probe_r50: int = 50,
                 baseline_rho_min: float = 1e-12, raised_rho_mins: Sequence[float] = (1e-3,),
                 high_residual_threshold: float = 1e-2, plateau_residual_threshold: float = 1e-4,
                 plateau_ratio_threshold: float = 0.6, severity_jump_r50_threshold: float = 0.0,
                 severity_jump_rho_min: float = 1e-2, stack: Optional[dict] = None, n_levels: int = 4,
                 cycle_precision: str = "fp64", reuse_probe: bool = True, checkpoint_guard: bool = False):
        flags = dict(CANONICAL_STACK if stack is None else stack)
        (self.spec, self.bc, self.free, self.free_gpu, self.edof_gpu, self.F_free_gpu, self.mf_op,
         self.gmg) = _build_components(preset, n_levels=n_levels, cycle_precision=cycle_precision, **flags)
        torch = _lib.require_cuda()
        self.penal = float(penal)
        self.tol = float(tol)
        self.restart = int(restart)
        self.maxiter = int(maxiter)
        self.probe_iters = int(probe_iters)
        self.probe_r50 = int(probe_r50)
        self.baseline_rho_min = float(baseline_rho_min)
        self.raised_rho_mins = [float(v) for v in raised_rho_mins]
        self.thresholds = dict(high_residual_threshold=high_residual_threshold,
                               plateau_residual_threshold=plateau_residual_threshold,
                               plateau_ratio_threshold=plateau_ratio_threshold)
        self.severity_jump_r50_threshold = float(severity_jump_r50_threshold)
        self.severity_jump_rho_min = float(severity_jump_rho_min)
        self.b_norm = float(torch.linalg.norm(self.F_free_gpu))
        self.reuse_probe = bool(reuse_probe)
        # checkpointed guard (the reference README's proposed extension): the probe
        # recomputes the FP64 true residual of its iterate at r50, and the rule reads
        # true residuals at r50 and at the probe's end instead of FGMRES's estimates
        self.checkpoint_guard = bool(checkpoint_guard)
        self.last_x = None

    # ---------------------------------------------------------------- moduli
    def moduli(self, density, rho_min: float, *, binary: bool = False):
        """E = rho_min + (1 - rho_min) * rho ** penal on the device.  ``binary``:
        ``density`` is a solid mask and void elements take rho = rho_min."""
        torch = _lib.require_cuda()
        d = _lib.as_cuda(density, torch.float64)
        if binary:
            rho = torch.where(d != 0, torch.ones_like(d), torch.full_like(d, rho_min))
        else:
            rho = d
        return rho_min + (1.0 - rho_min) * rho ** self.penal

    def solve_at_floor(self, density, rho_min: float, *, maxiter: int, history: list, binary: bool = False,
                       x0=None, check=None) -> FloorAttempt:
        """One guarded solve at ``rho_min``.  ``check`` (iteration, fn): fn(history so
        far) runs once the solve has done that many iterations and may end it there
        (the learned floor policy's decision point; the plain policy passes none)."""
        torch = _lib.require_cuda()
        E_e = self.moduli(density, rho_min, binary=binary)
        # timing syncs wait for this policy's stream only, so policies on other
        # streams (BatchedFloorPolicy) keep running
        stream = torch.cuda.current_stream()
        stream.synchronize()
        t0 = time.perf_counter()
        self.gmg.setup(E_e)
        stream.synchronize()
        setup_time = time.perf_counter() - t0

        def A_op(x):
            return self.mf_op.matvec(x, E_e)

        t0 = time.perf_counter()
        if check is None:
            x, iters, reported = _cupy_fgmres(A_op, self.F_free_gpu, self.gmg.apply, x0=x0, tol=self.tol,
                                              maxiter=maxiter, restart=self.restart, history=history)
        else:
            x, iters, reported = self.gmg._native_fgmres(self.F_free_gpu, x0, self.tol, maxiter, self.restart,
                                                         history, check=check)
        stream.synchronize()
        solve_time = time.perf_counter() - t0
        final = float(torch.linalg.norm(self.F_free_gpu - A_op(x)) / self.b_norm)
        self.last_x = x
        return FloorAttempt(rho_min, int(iters), bool(reported), final <= self.tol, final, setup_time, solve_time,
                            list(history))

    # ---------------------------------------------------------------- policy
    def run(self, density, *, binary: bool = False) -> dict:
        probe_history: list = []
        chk: dict = {}
        check = None
        if self.checkpoint_guard:
            def at_r50(_history, true_rel):
                chk["r50"] = true_rel
                return False  # observe only

            check = (self.probe_r50, at_r50, True)
        probe = self.solve_at_floor(density, self.baseline_rho_min, maxiter=self.probe_iters,
                                    history=probe_history, binary=binary, check=check)
        r50 = probe_history[min(self.probe_r50, len(probe_history) - 1)]
        r100 = probe_history[min(self.probe_iters, len(probe_history) - 1)]
        true_r50 = true_r100 = float("nan")
        if self.checkpoint_guard:
            # a probe that stopped before r50 has one true residual, at its end
            true_r50 = float(chk.get("r50", probe.final_rel_residual))
            true_r100 = float(probe.final_rel_residual)
            raise_floor, trigger = _classify(true_r50, true_r100, **self.thresholds)
        else:
            raise_floor, trigger = _classify(r50, r100, **self.thresholds)
        severity = raise_floor and self.severity_jump_r50_threshold > 0.0 and r50 >= self.severity_jump_r50_threshold
        if raise_floor and severity:
            ladder = [v for v in self.raised_rho_mins if v >= self.severity_jump_rho_min] or [self.severity_jump_rho_min]
        else:
            ladder = self.raised_rho_mins if raise_floor else [self.baseline_rho_min]
        attempts: list[FloorAttempt] = []
        attempted: list[float] = []
        state = {"selected": None, "reused_probe": False}
        probe_x = self.last_x

        def run_sequence(seq):
            for rho_min in seq:
                if rho_min in attempted:
                    continue
                attempted.append(rho_min)
                if self.reuse_probe and rho_min == probe.rho_min and probe.solver_reported_converged:
                    # The probe stopped on the tolerance before its iteration cap, so the
                    # driver's repeat solve at this floor (same E, same hierarchy, larger
                    # cap) is the identical deterministic computation: reuse its result.
                    a = probe
                    state["reused_probe"] = True
                else:
                    a = self.solve_at_floor(density, rho_min, maxiter=self.maxiter, history=[], binary=binary)
                attempts.append(a)
                state["selected"] = a
                if a.true_converged:
                    break

        run_sequence(ladder)
        sel = state["selected"]
        fallback = False
        if (sel is None or not sel.true_converged) and not raise_floor:
            fallback = True
            run_sequence(self.raised_rho_mins)
            sel = state["selected"]
        if state["reused_probe"] and sel is probe:
            self.last_x = probe_x
        failed = [a for a in attempts if a is not sel]
        return {
            "probe_r50": r50,
            "probe_r100": r100,
            "probe_r100_over_r50": r100 / max(r50, 1e-300),
            "checkpoint_guard": int(self.checkpoint_guard),
            "probe_true_r50": true_r50,
            "probe_true_r100": true_r100,
            "probe_setup_time_s": probe.setup_time_s,
            "probe_solve_time_s": probe.solve_time_s,
            "probe_iters": probe.iters,
            "trigger": trigger,
            "predicted_raise_floor": int(raise_floor),
            "severity_jump_triggered": int(severity),
            "post_solve_fallback_triggered": int(fallback),
            "detector_false_keep": int((not raise_floor) and fallback),
            "recommended_rho_min": sel.rho_min if sel else (ladder[-1] if ladder else float("nan")),
            "attempted_rho_mins": ";".join(f"{v:.0e}" for v in attempted),
            "n_floor_attempts": len(attempted),
            "solve_converged": int(bool(sel and sel.true_converged)),
            "solver_reported_converged": int(bool(sel and sel.solver_reported_converged)),
            "solve_iters": sel.iters if sel else self.maxiter,
            "solve_final_rel_residual": sel.final_rel_residual if sel else float("nan"),
            "selected_setup_time_s": sel.setup_time_s if sel else float("nan"),
            "selected_solve_time_s": sel.solve_time_s if sel else float("nan"),
            "failed_ladder_setup_time_s": sum(a.setup_time_s for a in failed),
            "failed_ladder_solve_time_s": sum(a.solve_time_s for a in failed),
            "recorded_policy_time_s": probe.setup_time_s + probe.solve_time_s
            + sum(a.setup_time_s + a.solve_time_s for a in attempts if a is not probe),
            "selected_reused_probe": int(state["reused_probe"]),
            "n_setups": 1 + sum(1 for a in attempts if a is not probe),
            "total_iters": probe.iters + sum(a.iters for a in attempts if a is not probe),
            "probe_history": probe_history,
            "attempts": attempts,
        }


_TRIGGERS = ("keep", "high_r50", "plateau", "learned", "high_residual")


def native_opts(pol: "GuardedFloorPolicy", *, binary: bool = False) -> "_lib.PolicyOpts":
    """The library's policy options (simpfem_policy_opts) of a GuardedFloorPolicy or
    LearnedFloorPolicy."""
    if pol.severity_jump_r50_threshold > 0.0 or pol.checkpoint_guard:
        raise ValueError("the severity jump and the checkpointed guard run in the Python policy only")
    if len(pol.raised_rho_mins) > 6:
        raise ValueError("at most six raised floors")
    o = _lib.PolicyOpts()
    _lib.lib().simpfem_policy_default_opts(ctypes.byref(o))
    o.penal = pol.penal
    o.binary = int(bool(binary))
    o.tol = pol.tol
    o.restart, o.maxiter = pol.restart, pol.maxiter
    o.probe_iters, o.probe_r50 = pol.probe_iters, pol.probe_r50
    o.baseline_rho_min = pol.baseline_rho_min
    o.n_raised = len(pol.raised_rho_mins)
    for k, v in enumerate(pol.raised_rho_mins):
        o.raised_rho_mins[k] = v
    o.high_residual_threshold = pol.thresholds["high_residual_threshold"]
    o.plateau_residual_threshold = pol.thresholds["plateau_residual_threshold"]
    o.plateau_ratio_threshold = pol.thresholds["plateau_ratio_threshold"]
    o.reuse_probe = int(bool(pol.reuse_probe))
    proposer = getattr(pol, "proposer", None)
    if proposer is not None:
        o.proposer = proposer._h.value
        o.min_confidence = pol.min_confidence
    return o


def native_row(r: "_lib.PolicyResult") -> dict:
    """A result row of the library's policy, with the keys of GuardedFloorPolicy.run."""
    attempted = [r.attempted[k] for k in range(r.n_attempts)]
    trig = _TRIGGERS[r.trigger]
    return {
        "probe_r50": r.probe_r50, "probe_r100": r.probe_r100, "probe_iters": r.probe_iters, "trigger": trig,
        "predicted_raise_floor": r.raise_floor, "post_solve_fallback_triggered": r.fallback,
        "detector_false_keep": int((not r.raise_floor) and r.fallback),
        "stopped_at_r50": trig if trig in ("learned", "high_residual") else "", "proposal": r.proposal,
        "recommended_rho_min": r.selected_rho_min, "attempted_rho_mins": ";".join(f"{v:.0e}" for v in attempted),
        "n_floor_attempts": r.n_attempts, "solve_converged": r.converged,
        "solver_reported_converged": r.reported_converged, "solve_iters": r.solve_iters,
        "solve_final_rel_residual": r.final_rel_residual, "selected_reused_probe": r.reused_probe,
        "n_setups": r.n_setups, "total_iters": r.total_iters, "policy_time_s": r.seconds,
    }


def run_native(pol: "GuardedFloorPolicy", density, *, binary: bool = False) -> dict:
    """One guarded solve of ``density`` run entirely in the library (simpfem_policy_run)
    on the current stream; the same decisions and kernels as ``pol.run`` (the guard
    value may differ in its last bits: the library reduces in its fixed order).
    The solution is left in ``pol.last_x``."""
    torch = _lib.require_cuda()
    d = _lib.as_cuda(density, torch.float64)
    x = torch.empty_like(pol.F_free_gpu)
    res = _lib.PolicyResult()
    o = native_opts(pol, binary=binary)
    _lib.call("simpfem_policy_run", pol.gmg._h, ctypes.byref(o), _lib.ptr(d), _lib.ptr(pol.F_free_gpu), _lib.ptr(x),
              ctypes.byref(res), _lib.stream_ptr())
    pol.last_x = x
    return native_row(res)


class BatchedFloorPolicy:
    """Several density states in flight at once on one GPU.

    ``width`` independent GuardedFloorPolicy workers, each with its own
    hierarchy and CUDA stream, are driven by one host thread each (the library
    releases the interpreter lock inside every call and synchronises only its
    own stream).  While one state's hierarchy setup runs its latency-bound
    coarsest factorisation, the other states' cycles fill the GPU.  State k goes
    to worker k mod width and each worker takes its states in order, so results
    are deterministic; every worker carries its own lambda-cache history, as one
    driver hierarchy does.  Every accepted answer still passes the FP64 guard.

    ``learned``: path of floor-proposer weights (gpu_fem.floor_proposer); the
    workers are then LearnedFloorPolicy instances, each with its own network
    handle (a handle's workspaces serve one stream at a time).  "rule": the same
    workers with a network of zeros, i.e. the probe stops at r50 only on the
    plain rule's high-residual trigger.
    """

    def __init__(self, width: int = 3, *args, learned: Optional[str] = None, **kwargs):
        torch = _lib.require_cuda()
        if int(width) < 1:
            raise ValueError("width must be >= 1")
        self.width = int(width)
        self.workers = []
        for i in range(self.width):
            # private mesh handles: scratch and reduction workspaces are per handle
            with mesh_namespace(("batched", id(self), i)):
                if learned is None:
                    self.workers.append(GuardedFloorPolicy(*args, **kwargs))
                else:
                    from .floor_proposer import FloorProposerNet, LearnedFloorPolicy

                    if learned == "rule":
                        # a network of zeros proposes no raised rung: the r50 rule stop alone
                        net = FloorProposerNet(max_batch=1)
                        net.set_params(np.zeros(net.n_params, dtype=np.float32))
                    else:
                        net = FloorProposerNet.load(learned, max_batch=1)
                    self.workers.append(LearnedFloorPolicy(*args, proposer=net, **kwargs))
        self.streams = [torch.cuda.Stream() for _ in range(self.width)]
        # pick the sweep shapes now, on an idle device; every worker's mesh (same
        # grid) then reuses them
        _lib.call("simpfem_mesh_tune", self.workers[0].mf_op.mesh.handle, _lib.stream_ptr())
        torch.cuda.current_stream().synchronize()

    def run_many_native(self, densities, *, binary: bool = False, keep_x: bool = True) -> list:
        """run_many in the library (simpfem_policy_batch): state k goes to worker
        k mod width, each worker's states in order on its own stream and host thread
        inside the library, so the rows (and solutions) are those of run_many.  With
        ``keep_x`` the solutions are in ``self.last_xs`` (one device tensor per state)."""
        torch = _lib.require_cuda()
        n = len(densities)
        dens = [_lib.as_cuda(d, torch.float64) for d in densities]
        xs = [torch.empty_like(self.workers[k % self.width].F_free_gpu) for k in range(n)] if keep_x else []
        states = (_lib.PolicyState * max(n, 1))()
        for k in range(n):
            w = self.workers[k % self.width]
            states[k].g = w.gmg._h.value
            states[k].density = _lib.ptr(dens[k])
            states[k].b_free = _lib.ptr(w.F_free_gpu)
            states[k].x_free = _lib.ptr(xs[k]) if keep_x else None
        results = (_lib.PolicyResult * max(n, 1))()
        o = native_opts(self.workers[0], binary=binary)
        _lib.call("simpfem_policy_batch", ctypes.byref(o), states, n, results, _lib.stream_ptr())
        self.last_xs = xs
        return [native_row(results[k]) for k in range(n)]

    def run_many(self, densities, *, binary: bool = False, on_result=None) -> list:
        """Run the policy on every state; returns the result rows in input order.
        ``on_result(k, worker, row)`` runs on the worker's thread and stream right
        after state k finishes (e.g. to copy ``worker.last_x`` to the host)."""
        torch = _lib.require_cuda()
        n = len(densities)
        rows: list = [None] * n
        errors: list = []
        caller = torch.cuda.current_stream()
        for s in self.streams:
            s.wait_stream(caller)  # inputs prepared on the caller's stream are visible

        def work(i: int) -> None:
            try:
                with torch.cuda.stream(self.streams[i]):
                    for k in range(i, n, self.width):
                        rows[k] = self.workers[i].run(densities[k], binary=binary)
                        if on_result is not None:
                            on_result(k, self.workers[i], rows[k])
            except BaseException as e:  # re-raised on the calling thread
                errors.append(e)

        threads = [threading.Thread(target=work, args=(i,)) for i in range(min(self.width, n))]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        for s in self.streams:
            caller.wait_stream(s)
        if errors:
            raise errors[0]
        return rows
