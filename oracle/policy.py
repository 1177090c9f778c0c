"""Restatement of the guarded floor policy of
experiments/phase5/run_gmg_floor_detector_prospective.py (:77-90 _classify,
:220-261 solve_at_floor, :263-354 probe, severity jump, ladder and fallback)."""

from __future__ import annotations

import numpy as np

from .solver import fgmres


def classify(r50, r100, high=1e-2, plateau=1e-4, ratio=0.6):
    if r50 >= high:
        return True, "high_r50"
    if r100 >= plateau and r100 / max(r50, 1e-300) >= ratio:
        return True, "plateau"
    return False, "keep"


def run_state(op, gmg, F, rho_of_floor, *, baseline=1e-12, raised=(1e-3,), penal=4.5, tol=1e-6,
              probe_iters=100, probe_r50=50, maxiter=300, restart=300, thresholds=(1e-2, 1e-4, 0.6),
              severity_r50=0.0, severity_floor=1e-2):
    """rho_of_floor(rho_min) -> element density used in E = rho_min + (1 - rho_min) rho^penal."""
    bn = float(np.linalg.norm(F))

    def solve(rho_min, mi, hist):
        E = rho_min + (1.0 - rho_min) * rho_of_floor(rho_min) ** penal
        gmg.setup(E)
        x, it, rep = fgmres(lambda v: op.matvec(v, E), F, gmg.apply, tol=tol, maxiter=mi, restart=restart, history=hist)
        final = float(np.linalg.norm(F - op.matvec(x, E)) / bn)
        return it, rep, final <= tol, final, x

    ph = []
    solve(baseline, probe_iters, ph)
    r50 = ph[min(probe_r50, len(ph) - 1)]
    r100 = ph[min(probe_iters, len(ph) - 1)]
    raise_floor, trigger = classify(r50, r100, *thresholds)
    sev = raise_floor and severity_r50 > 0.0 and r50 >= severity_r50
    if raise_floor and sev:
        ladder = [v for v in raised if v >= severity_floor] or [severity_floor]
    else:
        ladder = list(raised) if raise_floor else [baseline]
    attempted, sel = [], None

    def seq(floors):
        nonlocal sel
        for f in floors:
            if f in attempted:
                continue
            attempted.append(f)
            it, rep, conv, final, x = solve(f, maxiter, [])
            sel = dict(rho_min=f, iters=it, reported=rep, converged=conv, final=final, x=x)
            if conv:
                break

    seq(ladder)
    fallback = False
    if not (sel and sel["converged"]) and not raise_floor:
        fallback = True
        seq(list(raised))
    return dict(r50=r50, r100=r100, trigger=trigger, raise_floor=raise_floor, fallback=fallback,
                attempted=";".join(f"{v:.0e}" for v in attempted), selected=sel, probe_history=ph)
