"""SIMP topology optimisation around the guarded solve, on the GPU.

Each iteration follows the reference's GPU SIMP loop (gpu_fem/simp_gpu.py:
run_simp_surrogate_gpu :301-618, without surrogate or parameter controller)
with the floor policy in place of the plain solve:

1. rho_f = H rho, the row-normalised cone filter (simpfem_cone_filter), and
   rho_phys = rho_f, or with ``use_heaviside`` its Heaviside projection
   (simpfem_heaviside; :419-423), beta doubling every 20 iterations up to
   beta_max (:498-499);
2. one guarded solve of K(E) u = F with E = rho_min + (1 - rho_min) rho_phys^p,
   the floor chosen by the policy -- LearnedFloorPolicy (the floor proposer
   deciding at r50, the probe-and-ladder as fallback) or GuardedFloorPolicy --
   and every accepted answer checked by the FP64 recomputed true residual;
3. compliance c = F.u and dc = -p (1 - rho_min) rho_phys^(p-1) u_e^T KE u_e
   (simpfem_element_energy), as SolverV4 returns them (solver_v4.py:257-264);
4. the OC update of _oc_step_cupy (simp_gpu.py:212-294): without the projection,
   design sensitivities H^T dc, volume sensitivities 1 (:262-263), the multiplier
   bisection against sum(H rn) (simpfem_oc_update, volume weights H^T 1); with it,
   H^T (dc dh) and H^T dh and the bisection against the projected filtered volume
   (simpfem_oc_update_projected).

    python simp_loop.py [--dims 200 100 50] [--iters 50] [--policy learned|plain] [--out result.json]

The default problem is the 1M-element cantilever: volume fraction 0.3, filter
radius 1.5, move 0.2, SIMP p = 3, initial density 0.3 plus seeded N(0, 0.02)
noise, mixed-precision hierarchy, FGMRES restart 100, floors {1e-12 | 1e-3, 1e-2}.
"""

from __future__ import annotations

import argparse
import ctypes
import json
import os
import sys
import time
from typing import Callable, Optional

import numpy as np

if __package__ in (None, ""):
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    __package__ = "gpu_fem"  # noqa: A001

from . import _lib  # noqa: E402


def cone_filter(x, dims, rmin: float, transpose: bool = False):
    """H x (or H^T x) for the row-normalised cone filter on the element grid."""
    torch = _lib.require_cuda()
    xx = _lib.as_cuda(x, torch.float64)
    y = torch.empty_like(xx)
    _lib.call("simpfem_cone_filter", int(dims[0]), int(dims[1]), int(dims[2]), float(rmin), int(bool(transpose)),
              _lib.ptr(xx), _lib.ptr(y), _lib.stream_ptr())
    return y


class OCUpdater:
    """The OC multiplier bisection with a preallocated device workspace."""

    def __init__(self):
        torch = _lib.require_cuda()
        nbytes = int(_lib.lib().simpfem_oc_work_bytes())
        self._work = torch.empty((nbytes + 7) // 8, dtype=torch.float64, device="cuda")
        self._nbytes = nbytes

    def __call__(self, rho, dc_design, vol_weights, volfrac: float, move: float, dv_design=None):
        """Returns (rho_new, change, multiplier, bisection steps).  ``vol_weights``
        = H^T 1 (so sum(vol_weights * rn) = sum(H rn)); ``dv_design`` the volume
        sensitivities, None for ones as the reference has them without a projection."""
        torch = _lib.require_cuda()
        r = _lib.as_cuda(rho, torch.float64)
        dc = _lib.as_cuda(dc_design, torch.float64)
        vw = _lib.as_cuda(vol_weights, torch.float64)
        dv = _lib.as_cuda(dv_design, torch.float64) if dv_design is not None else None
        out = torch.empty_like(r)
        ch, lm, st = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        _lib.call("simpfem_oc_update", int(r.numel()), _lib.ptr(r), _lib.ptr(dc),
                  _lib.ptr(dv) if dv is not None else None, _lib.ptr(vw), float(volfrac), float(move), _lib.ptr(out),
                  _lib.ptr(self._work), self._nbytes, ctypes.byref(ch), ctypes.byref(lm), ctypes.byref(st),
                  _lib.stream_ptr())
        return out, float(ch.value), float(lm.value), int(st.value)

    def projected(self, dims, rmin: float, rho, rho_f, dc_phys, beta: float, eta: float, volfrac: float,
                  move: float):
        """The OC step with the Heaviside projection (simpfem_oc_update_projected):
        returns (rho_new, change, multiplier, bisection steps)."""
        torch = _lib.require_cuda()
        r = _lib.as_cuda(rho, torch.float64)
        rf = _lib.as_cuda(rho_f, torch.float64)
        dc = _lib.as_cuda(dc_phys, torch.float64)
        nbytes = int(_lib.lib().simpfem_oc_projected_work_bytes(int(r.numel())))
        if getattr(self, "_pwork", None) is None or self._pwork.numel() * 8 < nbytes:
            self._pwork = torch.empty((nbytes + 7) // 8, dtype=torch.float64, device="cuda")
        out = torch.empty_like(r)
        ch, lm, st = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        _lib.call("simpfem_oc_update_projected", int(dims[0]), int(dims[1]), int(dims[2]), float(rmin), _lib.ptr(r),
                  _lib.ptr(rf), _lib.ptr(dc), float(beta), float(eta), float(volfrac), float(move), _lib.ptr(out),
                  _lib.ptr(self._pwork), self._pwork.numel() * 8, ctypes.byref(ch), ctypes.byref(lm),
                  ctypes.byref(st), _lib.stream_ptr())
        return out, float(ch.value), float(lm.value), int(st.value)


def heaviside(x, beta: float, eta: float, derivative: bool = False):
    """The Heaviside projection of x (or its derivative) on the device."""
    torch = _lib.require_cuda()
    xx = _lib.as_cuda(x, torch.float64)
    y = torch.empty_like(xx)
    _lib.call("simpfem_heaviside", int(xx.numel()), _lib.ptr(xx), float(beta), float(eta),
              None if derivative else _lib.ptr(y), _lib.ptr(y) if derivative else None, _lib.stream_ptr())
    return y


def run_simp_guarded(dims=(200, 100, 50), *, volfrac: float = 0.3, rmin: float = 1.5, move: float = 0.2,
                     penal: float = 3.0, max_iter: int = 50, seed: int = 0, noise: float = 0.02,
                     policy: str = "learned", restart: int = 100, maxiter: int = 300,
                     cycle_precision: str = "fp32", raised_rho_mins=(1e-3, 1e-2),
                     use_heaviside: bool = False, beta_init: float = 1.0, beta_max: float = 32.0, eta: float = 0.5,
                     callback: Optional[Callable] = None) -> dict:
    torch = _lib.require_cuda()
    from .floor_proposer import FloorProposerNet, LearnedFloorPolicy
    from .paper4 import PLAIN_JACOBI_STACK
    from .policy import GuardedFloorPolicy
    from .presets import cantilever_spec
    from .solver_v4 import element_energy

    nx, ny, nz = (int(d) for d in dims)
    n = nx * ny * nz
    spec = cantilever_spec(nx, ny, nz)
    stack = dict(PLAIN_JACOBI_STACK, fine_smoother="fp32" if cycle_precision == "fp32" else "fp64")
    kw = dict(penal=penal, tol=1e-6, restart=restart, maxiter=maxiter, probe_iters=100, probe_r50=50,
              raised_rho_mins=tuple(raised_rho_mins), stack=stack, cycle_precision=cycle_precision)
    if policy == "learned":
        pol = LearnedFloorPolicy(spec, proposer=FloorProposerNet.load(max_batch=1), dims=(nx, ny, nz), **kw)
    elif policy == "plain":
        pol = GuardedFloorPolicy(spec, **kw)
    else:
        raise ValueError("policy must be 'learned' or 'plain'")
    oc = OCUpdater()
    rng = np.random.default_rng(seed)
    rho = torch.as_tensor(np.clip(volfrac + noise * rng.standard_normal(n), 1e-3, 1.0), device="cuda")
    # H^T 1: weights that turn sum(rn) into the filtered volume sum(H rn)
    vol_w = cone_filter(torch.ones(n, dtype=torch.float64, device="cuda"), dims, rmin, transpose=True)
    F = pol.F_free_gpu
    rows = []
    t_run = time.perf_counter()
    beta = float(beta_init)
    for it in range(1, max_iter + 1):
        stream = torch.cuda.current_stream()
        stream.synchronize()
        t0 = time.perf_counter()
        rho_f = cone_filter(rho, dims, rmin)
        projected = use_heaviside and beta > 1e-6
        rho_phys = heaviside(rho_f, beta, eta) if projected else rho_f
        r = pol.run(rho_phys)
        x = pol.last_x
        rho_min = float(r["recommended_rho_min"])
        compliance = float(torch.dot(F, x))
        ce = element_energy(pol.mf_op, x)
        dc_phys = -penal * (1.0 - rho_min) * rho_phys.clamp_min(0.0) ** (penal - 1.0) * ce
        if projected:
            rho_new, change, lm, steps = oc.projected(dims, rmin, rho, rho_f, dc_phys, beta, eta, volfrac, move)
        else:
            dc = cone_filter(dc_phys, dims, rmin, transpose=True)
            rho_new, change, lm, steps = oc(rho, dc, vol_w, volfrac, move)
        stream.synchronize()
        row = {
            "iter": it, "compliance": compliance, "volume": float(rho_phys.mean()), "change": change,
            "selected_rho_min": rho_min, "trigger": r["trigger"], "attempted_rho_mins": r["attempted_rho_mins"],
            "guarded": int(r["solve_converged"]), "true_rel_residual": float(r["solve_final_rel_residual"]),
            "outer_iterations": int(r["total_iters"]), "setups": int(r["n_setups"]),
            "stopped_at_r50": r.get("stopped_at_r50", ""),
            "policy_time_s": float(r.get("policy_time_s", r.get("recorded_policy_time_s", float("nan")))),
            "oc_multiplier": lm, "oc_steps": steps, "beta": beta if projected else 0.0,
            "iter_wall_s": time.perf_counter() - t0,
        }
        rows.append(row)
        if callback is not None:
            callback(row)
        rho = rho_new
        # the projection's continuation (simp_gpu.py:498-499): beta doubles every 20 iterations
        if use_heaviside and it % 20 == 0 and beta < beta_max:
            beta = min(beta * 2.0, beta_max)
    torch.cuda.synchronize()
    return {
        "dims": [nx, ny, nz], "elements": n, "volfrac": volfrac, "rmin": rmin, "move": move, "penal": penal,
        "policy": policy, "restart": restart, "cycle_precision": cycle_precision, "iterations": rows,
        "compliance_history": [r["compliance"] for r in rows],
        "use_heaviside": bool(use_heaviside), "beta_init": beta_init, "beta_max": beta_max, "eta": eta,
        "all_guarded": all(r["guarded"] for r in rows), "wall_s": time.perf_counter() - t_run,
        "rho": rho, "rho_phys": (heaviside(cone_filter(rho, dims, rmin), beta, eta)
                                 if use_heaviside and beta > 1e-6 else cone_filter(rho, dims, rmin)),
    }


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--dims", type=int, nargs=3, default=[200, 100, 50])
    ap.add_argument("--iters", type=int, default=50)
    ap.add_argument("--policy", default="learned", choices=["learned", "plain"])
    ap.add_argument("--restart", type=int, default=100)
    ap.add_argument("--heaviside", action="store_true", help="Heaviside projection, beta 1 -> 32 (x2 every 20)")
    ap.add_argument("--out", default=None)
    a = ap.parse_args()

    def show(row):
        print(f"iter {row['iter']:3d}  c={row['compliance']:.6g}  vol={row['volume']:.4f}  change={row['change']:.3f}  "
              f"floor={row['selected_rho_min']:.0e}  its={row['outer_iterations']}  "
              f"guarded={row['guarded']}  {row['iter_wall_s'] * 1e3:.1f} ms", flush=True)

    res = run_simp_guarded(tuple(a.dims), max_iter=a.iters, policy=a.policy, restart=a.restart,
                           use_heaviside=a.heaviside, callback=show)
    res.pop("rho")
    res.pop("rho_phys")
    print(json.dumps({k: v for k, v in res.items() if k != "iterations"}))
    if a.out:
        with open(a.out, "w") as fh:
            json.dump(res, fh, indent=1)


if __name__ == "__main__":
    main()
