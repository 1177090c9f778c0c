"""Golden log of the reference's SIMP loop control flow.

Run from the repository root where the reference source tree is readable
(its root given by SIMPFEM_REFERENCE_ROOT):

    python tests/golden/make_simp_control_golden.py

Calls the reference's own gpu_fem.simp_gpu.run_simp_surrogate_gpu (through the
numpy ``cupy`` stand-in of ``_refshim.py``) with its schedule-only controller
and the stand-ins of simp_control_fakes.py in place of the numeric steps (its
_build_density_filter, _heaviside and _oc_step_cupy are replaced by the same
host code the package's test uses; the solver is the closed-form stand-in) on
16x8x6 elements, in the two scenarios of simp_control_fakes.SCENARIOS:
"controlled" (72 iterations, projection on, schedule-only controller, a passive
mask, a surrogate on every fourth iteration) and "plain" (the unprojected OC
step until the convergence test stops the loop).  Writes simp_control_16x8x6.json:
per scenario the params_log rows (without wall times), the result's scalars,
rho_final and the stand-in solver's sequence of solves and invalidations.
"""

from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import _refshim  # noqa: E402
import simp_control_fakes as fakes  # noqa: E402

SCALARS = ("n_iter", "final_compliance", "best_compliance", "best_iteration", "final_grayness", "best_grayness",
           "best_is_valid", "fem_calls", "surrogate_calls", "surrogate_used_fraction", "gpu_backend")


def main() -> None:
    _refshim.install()
    sg = _refshim.load("simp_gpu")
    controllers = _refshim.load("pub_baseline_controller")
    sg._build_density_filter = fakes.build_density_filter
    sg._heaviside = fakes.project
    sg._oc_step_cupy = (lambda rho, rho_f, dc, beta, eta, volfrac, move, H, H_T, n, use_heaviside:
                        fakes.oc_step(rho, rho_f, dc, beta, eta, volfrac, move, H, use_heaviside and beta > 1e-6))
    fixed, free, F, ndof = fakes.problem()
    out = {}
    for name, sc in fakes.SCENARIOS.items():
        fakes.EVENTS.clear()
        res = sg.run_simp_surrogate_gpu(
            sg.TO3DParams(**sc["params"]), fixed, free, F, ndof, fakes.EchoSurrogate() if sc["surrogate"] else None,
            fakes.router, device="auto",
            param_controller=controllers.ScheduleOnlyController() if sc["controller"] else None,
            passive_mask=fakes.passive_mask() if sc["passive"] else None, solver_class=fakes.FakeSolver,
            solver_kwargs=dict(fakes.SOLVER_KWARGS))
        log = [{k: v for k, v in row.items() if k != "iter_wall_sec"} for row in res["params_log"]]
        out[name] = {
            "params_log": log,
            "scalars": {k: (v.item() if hasattr(v, "item") else v) for k, v in res.items() if k in SCALARS},
            "rho_final": np.asarray(res["rho_final"], dtype=np.float64).tolist(),
            "events": [e if isinstance(e, str) else list(e) for e in fakes.EVENTS],
        }
        print(name, out[name]["scalars"], sum(e == "invalidate" for e in fakes.EVENTS), "invalidations",
              "last change", log[-1]["change"])
    with open(os.path.join(HERE, "simp_control_16x8x6.json"), "w") as f:
        json.dump(out, f, separators=(",", ":"))


if __name__ == "__main__":
    main()
