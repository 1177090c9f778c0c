"""Golden data for the branches of the SIMP loop entry (run_simp_surrogate_gpu)
that the trajectory driver does not reach.

Run from the repository root where the reference source tree is readable
(its root given by SIMPFEM_REFERENCE_ROOT):

    python tests/golden/make_simp_entry_golden.py

Calls the reference's own gpu_fem.simp_gpu.run_simp_surrogate_gpu (through the
numpy ``cupy`` stand-in of ``_refshim.py``) on the cantilever_3d preset
(24x12x6) with SolverV4 (three levels, FP64 Chebyshev smoothing, FGMRES restart
300, maxiter 150, tol 1e-6, Emin 1e-9), no projection (the unprojected OC step),
12 iterations, no parameter controller, and

* a passive mask: elements with x index 20-23, y 4-7 held solid (2), elements
  with x index 8-11, y 0-3, z 0-2 held void (1);
* ``EchoSurrogate`` with ``EveryThirdRouter``: iterations 3, 6, 9 and 12 take
  the surrogate's prediction, which is the sensitivity of the last solve.

Once as given and once with the load vector scaled entry by entry by
(1 + 1e-12 xi), xi standard normal from numpy's default_rng(0).  Writes
simp_entry_cantilever_3d.npz: per run the per-iteration compliance, change,
volume, grayness, outer iterations and surrogate flags, and rho_final.
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import _refshim  # noqa: E402

ITERS = 12
PERT = 1e-12
KW = dict(enable_warm_start=True, enable_matrix_free=True, enable_fused_cuda=False, enable_matfree_gmg=True,
          matfree_gmg_levels=3, gmg_fine_smoother="fp64", gmg_fine_degree=2, gmg_outer_solver="fgmres",
          gmg_restart=300,
          gmg_smoother_type="chebyshev", gmg_cycle_type="v", cg_tol=1e-6, cg_maxiter=150, enable_profiling=False)


def passive_mask(nx: int, ny: int, nz: int) -> np.ndarray:
    """Element passivity in the (x, y, z) element order: 2 solid, 1 void, 0 free."""
    m = np.zeros((nx, ny, nz), dtype=np.int32)
    m[20:24, 4:8, :] = 2
    m[8:12, 0:4, 0:3] = 1
    return m.ravel()


class EchoSurrogate:
    """Predicts the sensitivity of the last solve; ready after the first one."""

    uncertainty = 0.0

    def __init__(self):
        self._dc = None

    @property
    def is_ready(self) -> bool:
        return self._dc is not None

    def update(self, rho_phys, rho_f, penal, iter_ratio, dc_phys):
        self._dc = dc_phys.clone() if hasattr(dc_phys, "clone") else np.array(dc_phys, copy=True)

    def predict(self, rho_phys, rho_f, penal, iter_ratio):
        return self._dc, 0.0


class EveryThirdRouter:
    """A solve unless the iteration is a multiple of three."""

    def __call__(self, iteration, uncertainty, surrogate_ready, beta=1.0, **kwargs):
        return iteration % 3 != 0


def main() -> None:
    _refshim.install()
    sg = _refshim.load("simp_gpu")
    s4 = _refshim.load("solver_v4")
    presets = _refshim.load("presets")
    bcg = _refshim.load("bc_generator")
    spec = presets.get_preset("cantilever_3d")
    nx, ny, nz = spec.nelx, spec.nely, spec.nelz
    out = {}
    for run in ("base", "pert"):
        bc = bcg.generate_bc(spec)
        F = bc.F * (1.0 + PERT * np.random.default_rng(0).standard_normal(bc.F.shape)) if run == "pert" else bc.F
        params = sg.TO3DParams(nelx=nx, nely=ny, nelz=nz, volfrac=spec.volfrac, penal=3.0, emin=1e-9, rmin=1.5,
                               max_iter=ITERS, min_iter=ITERS, use_heaviside=False)
        res = sg.run_simp_surrogate_gpu(params, bc.fixed_dofs.astype(np.int32), bc.free_dofs.astype(np.int32), F,
                                        bc.ndof, EchoSurrogate(), EveryThirdRouter(), device="auto",
                                        passive_mask=passive_mask(nx, ny, nz), solver_class=s4.SolverV4,
                                        solver_kwargs=dict(KW, grid_dims=(nx, ny, nz)))
        log = res["params_log"]
        for key in ("compliance", "change", "volume", "grayness"):
            out[f"{run}_{key}"] = np.array([row[key] for row in log], dtype=np.float64)
        out[f"{run}_cg_iters"] = np.array([row["cg_iters"] for row in log], dtype=np.int64)
        out[f"{run}_used_surrogate"] = np.array([row["used_surrogate"] for row in log], dtype=bool)
        out[f"{run}_rho_final"] = np.asarray(res["rho_final"], dtype=np.float64)
        for key in ("fem_calls", "surrogate_calls", "best_iteration", "n_iter"):
            out[f"{run}_{key}"] = np.int64(res[key])
        out[f"{run}_best_is_valid"] = np.bool_(res["best_is_valid"])
    np.savez_compressed(os.path.join(HERE, "simp_entry_cantilever_3d.npz"), **out)
    print({k: v for k, v in out.items() if v.ndim == 0})
    print("compliance", out["base_compliance"], "\nused_surrogate", out["base_used_surrogate"])


if __name__ == "__main__":
    main()
