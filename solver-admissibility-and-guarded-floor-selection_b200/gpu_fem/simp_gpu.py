"""The reference's SIMP loop entry (gpu_fem/simp_gpu.py) on this library.

``run_simp_surrogate_gpu(params, fixed, free, F, ndof, surrogate, router,
device="auto", param_controller=None, passive_mask=None, verbose=False,
progress_callback=None, solver_class=None, solver_kwargs=None) -> dict`` with
``TO3DParams`` (:55-77) runs the loop of simp_gpu.py:301-618 with the design
fields resident on the device:

* the solver is ``solver_class(edof=, row_idx=, col_idx=, KE_UNIT=, free=, F=,
  ndof=, E0=1, Emin=params.emin, backend=device, amg_ndof_threshold=,
  amg_rebuild_tol=, **solver_kwargs)`` (:357-381): ``SolverV4`` or a subclass,
  such as the trajectory driver's guarded floor policy;
* rho_f = H rho (simpfem_cone_filter, which takes the radius per call, so a
  controller's new radius only drops the solver's warm start, :411-416), and
  rho_phys its Heaviside projection (simpfem_heaviside) when ``use_heaviside``
  and beta > 1e-6 (:418-423);
* the solve, or with a surrogate attached, the router's choice between the
  solve and the surrogate's prediction (:425-454);
* the OC step of _oc_step_cupy (:212-294): simpfem_oc_update_projected with
  the projection, else simpfem_oc_update on H^T dc with volume weights H^T 1;
* the best-design gate (penal >= min_penal_for_best, grayness <
  max_gray_for_best, :476-486), the convergence test (change < tol, relative
  compliance change across the window < compliance_tol, iteration >= min_iter,
  :488-495), beta doubled every 20 iterations (:497-499), and the controller's
  action on a ``StepState``: penal clipped to [1, 5], rmin to [1.1, 4], move to
  [0.03, 0.4], beta to [1, 64], a restart from the best design; when the
  controller raises, the rest of its action is skipped, as in the reference
  (:501-535), with a RuntimeWarning here;
* per iteration one ``params_log`` row and one ``progress_callback`` state with
  the reference's keys in its order, the solver's ``last_*`` attributes (floor,
  trigger, probe read-outs, FP64 true residual) included (:537-590).

The returned ``rho_final`` / ``rho_best`` are numpy arrays, as the reference's
are; ``fixed`` is accepted for the signature (the solver takes the free DOFs).  Only 3D meshes (nelz > 0) and solver classes of the matrix-free GMG path
are on the accelerated solve; the reference's default ``GPUFEMSolver``
(assembled CSR) is not provided.

    python simp_gpu.py [--dims 200 100 50] [--iters 50] [--fine-smoother fp32]
                       [--restart 100] [--controller none|schedule] [--out run.json]

runs the loop on a cantilever of the given size with the in-loop guarded floor
policy (floors 1e-12 | 1e-3, 1e-2; probe 100, r50 at 50; tol 1e-6), the call
the trajectory driver makes, and prints the per-iteration record's summary.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import sys
import time
import warnings
from dataclasses import dataclass
from typing import Callable, Optional

import numpy as np

if __package__ in (None, ""):
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    __package__ = "gpu_fem"  # noqa: A001

from . import _lib  # noqa: E402
from .pub_simp_solver import KE_UNIT_3D, StepState, _build_sparse_indices, _edof_table_3d  # noqa: E402
from .simp_loop import OCUpdater, cone_filter, heaviside  # noqa: E402


@dataclass
class TO3DParams:
    """Topology optimisation parameters (simp_gpu.py:55-77)."""
    nelx: int = 24
    nely: int = 12
    nelz: int = 12
    volfrac: float = 0.3
    penal: float = 3.0
    emin: float = 1e-9
    rmin: float = 1.5
    move: float = 0.2
    max_iter: int = 100
    tol: float = 0.01
    compliance_tol: float = 5e-4
    compliance_window: int = 5
    min_iter: int = 30
    use_heaviside: bool = True
    beta_init: float = 1.0
    beta_max: float = 32.0
    eta: float = 0.5
    min_penal_for_best: float = 3.0
    max_gray_for_best: float = 0.25
    amg_ndof_threshold: int = 3000
    amg_rebuild_tol: float = 0.15


_DEVICE = "cuda"  # where the loop keeps its design fields


def _grayness(x) -> float:
    return float(4.0 * (x * (1.0 - x)).mean())


def _checkerboard(x, nx: int, ny: int, nz: int) -> float:
    """Standard deviation (population) of the 2x2x2 block means of the element
    field in (x, y, z) order, 0 for a mesh thinner than two elements."""
    if nx < 2 or ny < 2 or nz < 2:
        return 0.0
    R = x.view(nx, ny, nz)
    lo, hi = slice(None, -1, 2), slice(1, None, 2)
    blocks = sum(R[a, b, c] for a in (lo, hi) for b in (lo, hi) for c in (lo, hi)) / 8.0
    return float(blocks.std(correction=0))


def _solver_readouts(solver, emin: float) -> dict:
    """The solver's last_* attributes under the loop's column names."""
    g = lambda name, default: getattr(solver, name, default)  # noqa: E731
    return {
        "solver_true_rel_residual": float(g("last_true_rel_residual", math.nan)),
        "selected_rho_min": float(g("last_selected_rho_min", emin)),
        "policy_trigger": str(g("last_policy_trigger", "")),
        "policy_fallback_used": int(g("last_policy_fallback_used", 0)),
        "policy_attempted_rho_mins": str(g("last_policy_attempted_rho_mins", "")),
        "policy_probe_r50": float(g("last_policy_probe_r50", math.nan)),
        "policy_probe_r100": float(g("last_policy_probe_r100", math.nan)),
        "policy_probe_true_rel_residual": float(g("last_policy_probe_true_rel_residual", math.nan)),
    }


def _oc_step(oc, cache: dict, dims, rmin: float, rho, rho_f, dc, beta: float, eta: float, volfrac: float,
             move: float, projected: bool):
    """One OC update as _oc_step_cupy makes it (simp_gpu.py:212-294): with the
    projection simpfem_oc_update_projected, without it simpfem_oc_update on H^T dc
    with the volume weights H^T 1 (kept in ``cache`` for the current radius).
    Returns (rho_new, change)."""
    if projected:
        rho_new, change, _, _ = oc.projected(dims, rmin, rho, rho_f, dc, beta, eta, volfrac, move)
        return rho_new, change
    weights = cache.get(rmin)
    if weights is None:
        torch = _lib.require_cuda()
        weights = cone_filter(torch.ones(rho.numel(), dtype=torch.float64, device=_DEVICE), dims, rmin,
                              transpose=True)
        cache.clear()
        cache[rmin] = weights
    rho_new, change, _, _ = oc(rho, cone_filter(dc, dims, rmin, transpose=True), weights, volfrac, move)
    return rho_new, change


def run_simp_surrogate_gpu(params: TO3DParams, fixed, free, F, ndof: int, surrogate, router: Callable,
                           device: str = "auto", param_controller: Optional[Callable] = None,
                           passive_mask=None, verbose: bool = False, progress_callback: Optional[Callable] = None,
                           solver_class=None, solver_kwargs: Optional[dict] = None) -> dict:
    t_start = time.time()
    nx, ny, nz = int(params.nelx), int(params.nely), int(params.nelz)
    if nz <= 0:
        raise NotImplementedError("only 3D meshes (nelz > 0) are on the accelerated solve")
    if device == "cpu":
        raise NotImplementedError("the SIMP loop runs on the CUDA device only")
    if solver_class is None:
        raise NotImplementedError("the reference's default GPUFEMSolver (assembled CSR) is not provided; "
                                  "pass solver_class=SolverV4 or a subclass")
    torch = _lib.require_cuda()
    dims = (nx, ny, nz)
    n_elem = nx * ny * nz
    E0, Emin = 1.0, float(params.emin)
    extra = dict(solver_kwargs or {})
    edof = _edof_table_3d(nx, ny, nz)
    if extra.get("enable_matrix_free", False):
        row_idx = col_idx = np.empty(0, dtype=np.int32)
    else:
        row_idx, col_idx = _build_sparse_indices(edof)
    solver = solver_class(edof=edof, row_idx=row_idx, col_idx=col_idx, KE_UNIT=KE_UNIT_3D, free=free, F=F,
                          ndof=ndof, E0=E0, Emin=Emin, backend=device,
                          amg_ndof_threshold=params.amg_ndof_threshold, amg_rebuild_tol=params.amg_rebuild_tol,
                          **extra)

    dev = dict(dtype=torch.float64, device=_DEVICE)
    passive = None
    if passive_mask is not None:
        pm = torch.as_tensor(np.asarray(passive_mask), device=_DEVICE)
        passive = (pm == 1, pm == 2)

    def pin_passive(x):
        if passive is not None:
            x[passive[0]] = 1e-3
            x[passive[1]] = 1.0
        return x

    rho = pin_passive(torch.full((n_elem,), float(params.volfrac), **dev))
    penal, rmin, move = float(params.penal), float(params.rmin), float(params.move)
    beta, eta = float(params.beta_init), float(params.eta)
    prev_rmin = rmin
    oc = OCUpdater()
    vol_cache: dict = {}

    best_rho = rho.clone()
    best_compliance = math.inf
    best_iteration = 0
    best_is_valid = False
    best_grayness = _grayness(rho)
    compliance_hist: list = []
    params_log: list = []
    last_compliance = math.inf
    fem_calls = surrogate_calls = 0
    iteration = 0
    rho_phys = rho

    for iteration in range(1, int(params.max_iter) + 1):
        iter_t0 = time.time()
        if abs(rmin - prev_rmin) > 1e-6:
            solver.invalidate()
            prev_rmin = rmin

        rho_f = cone_filter(rho, dims, rmin)
        projected = bool(params.use_heaviside) and beta > 1e-6
        rho_phys = heaviside(rho_f, beta, eta) if projected else rho_f.clone()
        iter_ratio = iteration / params.max_iter

        use_fem = True
        if surrogate is not None:
            use_fem = router(iteration, surrogate.uncertainty, surrogate.is_ready, beta, rho=rho_phys,
                             compliance=last_compliance)
        dc_phys = None
        if not use_fem:
            dc_pred, _ = surrogate.predict(rho_phys, rho_f, penal, iter_ratio)
            if dc_pred is not None:
                dc_phys, compliance = dc_pred, last_compliance
                surrogate_calls += 1
        if dc_phys is None:
            compliance, dc_phys = solver.solve(rho_phys, penal)
            last_compliance = compliance
            fem_calls += 1
            if surrogate is not None:
                surrogate.update(rho_phys, rho_f, penal, iter_ratio, dc_phys)
        compliance = float(compliance)
        dc_dev = _lib.as_cuda(dc_phys, torch.float64)

        rho_new, change = _oc_step(oc, vol_cache, dims, rmin, rho, rho_f, dc_dev, beta, eta, params.volfrac, move,
                                   projected)
        rho_new = pin_passive(rho_new)

        gray_now = _grayness(rho_phys)
        if compliance < best_compliance and penal >= params.min_penal_for_best \
                and gray_now < params.max_gray_for_best:
            best_compliance, best_iteration, best_grayness = compliance, iteration, gray_now
            best_rho = rho_phys.clone()
            best_is_valid = True
        compliance_hist.append(compliance)

        window = compliance_hist[-params.compliance_window:]
        settled = (len(window) == params.compliance_window
                   and abs(window[-1] - window[0]) / max(abs(window[0]), 1e-10) < params.compliance_tol)
        converged = change < params.tol and settled and iteration >= params.min_iter

        if iteration % 20 == 0 and beta < params.beta_max:
            beta = min(beta * 2.0, params.beta_max)

        if param_controller is not None:
            try:
                rel1 = 0.0 if len(compliance_hist) < 2 else (
                    (compliance_hist[-1] - compliance_hist[-2]) / max(abs(compliance_hist[-2]), 1e-10))
                state = StepState(
                    iteration=iteration, compliance=compliance, best_compliance=best_compliance,
                    best_iteration=best_iteration, volume_fraction=float(rho_phys.sum()) / n_elem,
                    grayness=gray_now, best_grayness=best_grayness,
                    checkerboard=_checkerboard(rho_phys, nx, ny, nz), obj_slope=0.0, rel_change_1=rel1,
                    rel_change_5=0.0, stagnation_counter=0, penal=penal, rmin=rmin, move=move, beta=beta,
                    converged=converged, best_is_valid=best_is_valid, compliance_history=list(compliance_hist))
                action = param_controller(state, rho_new)
                if action:
                    if "penal" in action:
                        penal = float(np.clip(action["penal"], 1.0, 5.0))
                    if "rmin" in action:
                        rmin = float(np.clip(action["rmin"], 1.1, 4.0))
                    if "move" in action:
                        move = float(np.clip(action["move"], 0.03, 0.4))
                    if "beta" in action:
                        beta = float(np.clip(action["beta"], 1.0, 64.0))
                    if action.get("restart", False) and best_is_valid:
                        rho_new = best_rho.clone()
                        solver.invalidate()
            except Exception as exc:  # the reference keeps going and skips the rest of the action
                warnings.warn(f"SIMP parameter controller raised {exc!r} at iteration {iteration}; "
                              "the rest of its action is skipped", RuntimeWarning, stacklevel=2)

        readouts = _solver_readouts(solver, Emin)
        uncertainty = surrogate.uncertainty if surrogate is not None else 0.0
        volume = float(rho_phys.sum()) / n_elem
        params_log.append({
            "iter": iteration, "penal": penal, "rmin": rmin, "move": move, "beta": beta, "emin": Emin,
            "compliance": compliance, "grayness": gray_now, "used_surrogate": not use_fem,
            "surrogate_uncertainty": uncertainty, "cg_iters": int(getattr(solver, "last_cg_iters", -1)),
            **readouts, "change": float(change), "volume": volume, "iter_wall_sec": time.time() - iter_t0,
        })
        if verbose:
            src = "SUR" if not use_fem else "GPU"
            print(f"  [{src}] iter {iteration:3d}  C={compliance:8.4f}  gray={gray_now:.3f}  p={penal:.2f}  "
                  f"beta={beta:.1f}  chg={change:.4f}", flush=True)
        if progress_callback is not None:
            progress_callback({
                "iteration": iteration, "max_iter": params.max_iter, "compliance": compliance,
                "grayness": gray_now, "used_surrogate": not use_fem, "uncertainty": uncertainty, "beta": beta,
                "change": change, "penal": penal, "rmin": rmin, "move": move, "emin": Emin,
                "cg_iters": getattr(solver, "last_cg_iters", -1), **readouts,
            })
        rho = rho_new
        if converged:
            if verbose:
                print(f"  Converged at iteration {iteration}.", flush=True)
            break

    rho_final = best_rho if best_is_valid else rho_phys
    reported_final = compliance_hist[-1] if compliance_hist else math.inf
    if best_is_valid and reported_final > best_compliance * 2.0:
        reported_final = best_compliance
    total_calls = fem_calls + surrogate_calls
    return {
        "nelx": nx, "nely": ny, "nelz": nz,
        "n_iter": iteration,
        "final_compliance": reported_final,
        "best_compliance": best_compliance,
        "best_iteration": best_iteration,
        "final_grayness": _grayness(rho_final),
        "best_grayness": best_grayness,
        "best_is_valid": best_is_valid,
        "rho_final": rho_final.cpu().numpy(),
        "rho_best": best_rho.cpu().numpy(),
        "compliance_history": compliance_hist,
        "fem_calls": fem_calls,
        "surrogate_calls": surrogate_calls,
        "surrogate_used_fraction": surrogate_calls / max(total_calls, 1),
        "is_3d": True,
        "params_log": params_log,
        "wall_time_sec": time.time() - t_start,
        "gpu_backend": getattr(solver, "_backend", "cupy"),
    }


def main() -> None:
    ap = argparse.ArgumentParser(description="run_simp_surrogate_gpu with the in-loop guarded floor policy")
    ap.add_argument("--dims", type=int, nargs=3, default=[200, 100, 50])
    ap.add_argument("--iters", type=int, default=50)
    ap.add_argument("--penal", type=float, default=3.0)
    ap.add_argument("--fine-smoother", default="fp32", choices=["fp64", "fp32"])
    ap.add_argument("--smoother-type", default="chebyshev", choices=["chebyshev", "jacobi"])
    ap.add_argument("--levels", type=int, default=4)
    ap.add_argument("--restart", type=int, default=100)
    ap.add_argument("--maxiter", type=int, default=300)
    ap.add_argument("--heaviside", action="store_true", help="Heaviside projection (beta 1, doubled every 20)")
    ap.add_argument("--controller", default="none", choices=["none", "schedule"])
    ap.add_argument("--out", default=None)
    a = ap.parse_args()

    from .bc_generator import generate_bc
    from .floor_trajectory import GuardedAdaptiveFloorSolverV4
    from .local_agents import PureFEMRouter
    from .presets import cantilever_spec
    from .pub_baseline_controller import ScheduleOnlyController

    nx, ny, nz = a.dims
    spec = cantilever_spec(nx, ny, nz)
    bc = generate_bc(spec)
    params = TO3DParams(nelx=nx, nely=ny, nelz=nz, volfrac=spec.volfrac, penal=a.penal, emin=1e-12,
                        rmin=spec.rmin if spec.rmin is not None else 1.5, max_iter=a.iters, min_iter=a.iters,
                        use_heaviside=a.heaviside)
    kw = dict(grid_dims=(nx, ny, nz), enable_warm_start=True, enable_matrix_free=True, enable_fused_cuda=False,
              enable_matfree_gmg=True, matfree_gmg_levels=a.levels, gmg_fine_smoother=a.fine_smoother,
              gmg_fine_degree=2, gmg_outer_solver="fgmres", gmg_restart=a.restart, gmg_smoother_type=a.smoother_type,
              gmg_cycle_type="v", cg_tol=1e-6, cg_maxiter=a.maxiter, guarded_base_rho_min=1e-12,
              guarded_ladder=(1e-3, 1e-2), guarded_probe_iters=100, guarded_probe_r50=50)

    def show(st):
        print(f"iter {st['iteration']:3d}  C={st['compliance']:.6g}  gray={st['grayness']:.4f}  "
              f"floor={st['selected_rho_min']:.0e}  {st['policy_trigger']}  its={st['cg_iters']}  "
              f"r={st['solver_true_rel_residual']:.2e}", flush=True)

    torch = _lib.require_cuda()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    res = run_simp_surrogate_gpu(params, bc.fixed_dofs, bc.free_dofs, bc.F, bc.ndof, None, PureFEMRouter(),
                                 param_controller=ScheduleOnlyController() if a.controller == "schedule" else None,
                                 progress_callback=show, solver_class=GuardedAdaptiveFloorSolverV4,
                                 solver_kwargs=kw)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    log = res["params_log"]
    walls = [row["iter_wall_sec"] for row in log]
    its = [row["cg_iters"] for row in log]
    floors: dict = {}
    for row in log:
        key = f"{row['selected_rho_min']:.0e}"
        floors[key] = floors.get(key, 0) + 1
    summary = {
        "dims": [nx, ny, nz], "elements": nx * ny * nz, "iterations": res["n_iter"], "wall_s": wall,
        "first_iteration_s": walls[0] if walls else None,
        "median_iteration_s": float(np.median(walls[1:])) if len(walls) > 1 else None,
        "compliance_first_last": [log[0]["compliance"], log[-1]["compliance"]] if log else None,
        "outer_iterations_median": float(np.median(its)) if its else None,
        "outer_iterations_range": [min(its), max(its)] if its else None,
        "floor_counts": floors,
        "max_true_rel_residual": max(row["solver_true_rel_residual"] for row in log) if log else None,
        "fine_smoother": a.fine_smoother, "smoother_type": a.smoother_type, "restart": a.restart,
        "controller": a.controller, "heaviside": bool(a.heaviside),
    }
    print(json.dumps(summary))
    if a.out:
        with open(a.out, "w") as fh:
            json.dump({"summary": summary, "params_log": log}, fh, indent=1)


if __name__ == "__main__":
    main()
