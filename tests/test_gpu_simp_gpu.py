"""The SIMP loop entry (gpu_fem.simp_gpu.run_simp_surrogate_gpu) on the GPU
against the reference trajectory driver's own runs, and against the reference's
own entry on the branches that driver does not reach (unprojected OC step,
passive mask, surrogate and router hooks, plain SolverV4).

The call is the one run_simp_floor_trajectory.py makes (_run_case, :277-352,
with _solver_kwargs, :244-275): cantilever_3d (24x12x6), SIMP penal 4.5 at the
start, schedule-only controller, FEM-only router, three-level hierarchy, FP64
smoothing, FGMRES restart 300, maxiter 150, tol 1e-6.  Golden rows come from
the unchanged reference driver (tests/golden/make_trajectory_driver_golden.py):

* guarded (GuardedAdaptiveFloorSolverV4, probe 30 / r50 15, floors 1e-12 |
  1e-3, 1e-2), 45 iterations: on every iteration the same continuation
  parameters, trigger, selected floor, attempted floors and fallback flag, the
  FP64 true residual at or below 1e-6, outer iteration counts at most one
  further apart than the reference's own run under a 1e-12 load perturbation
  is at that iteration (at least 2; the perturbation moves a warm-started
  solve of the raised-floor phase by up to 3) and within 1% over the
  trajectory, and compliance and grayness inside 100 times the
  running maximum of that run's relative deviation, floored at 1e-9 (a SIMP
  trajectory carries each solve's round-off into the next design); the same
  best iteration, validity and iteration count, and rho_final inside the same
  envelope;
* fixed floor 1e-3 (SolverV4), 20 iterations: the same checks without the
  policy columns, against its own perturbed run.
"""

import csv
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
ENVELOPE, FLOOR = 100.0, 1e-9


def _rows(name):
    with open(os.path.join(GOLDEN, f"trajectory_{name}.csv"), newline="") as f:
        return list(csv.DictReader(f))


def _run(policy: str, iters: int, rho_min: float):
    from gpu_fem.bc_generator import generate_bc
    from gpu_fem.floor_trajectory import GuardedAdaptiveFloorSolverV4
    from gpu_fem.local_agents import PureFEMRouter
    from gpu_fem.presets import get_preset
    from gpu_fem.pub_baseline_controller import ScheduleOnlyController
    from gpu_fem.simp_gpu import TO3DParams, run_simp_surrogate_gpu
    from gpu_fem.solver_v4 import SolverV4

    spec = get_preset("cantilever_3d")
    bc = generate_bc(spec)
    params = TO3DParams(nelx=spec.nelx, nely=spec.nely, nelz=spec.nelz, volfrac=spec.volfrac, penal=4.5,
                        emin=rho_min, rmin=spec.rmin if spec.rmin is not None else 1.5, max_iter=iters, tol=0.01,
                        min_iter=min(20, iters))
    kw = dict(grid_dims=(spec.nelx, spec.nely, spec.nelz), enable_warm_start=True, enable_matrix_free=True,
              enable_fused_cuda=False, enable_matfree_gmg=True, matfree_gmg_levels=3, gmg_fine_smoother="fp64",
              gmg_fine_degree=2, gmg_outer_solver="fgmres", gmg_restart=300, gmg_smoother_type="chebyshev",
              gmg_cycle_type="v", cg_tol=1e-6, cg_maxiter=150, enable_profiling=True)
    if policy == "guarded_adaptive":
        kw.update(guarded_base_rho_min=1e-12, guarded_ladder=(1e-3, 1e-2), guarded_probe_iters=30,
                  guarded_probe_r50=15, guarded_high_residual_threshold=1e-2,
                  guarded_plateau_residual_threshold=1e-4, guarded_plateau_ratio_threshold=0.6)
    states = []
    result = run_simp_surrogate_gpu(
        params=params, fixed=bc.fixed_dofs.astype(np.int32), free=bc.free_dofs.astype(np.int32), F=bc.F,
        ndof=bc.ndof, surrogate=None, router=PureFEMRouter(), device="auto",
        param_controller=ScheduleOnlyController(), verbose=False, progress_callback=states.append,
        solver_class=GuardedAdaptiveFloorSolverV4 if policy == "guarded_adaptive" else SolverV4,
        solver_kwargs=kw)
    return result, states


def _envelope(run):
    base, pert = _rows(f"{run}_iters"), _rows(f"{run}_pert_iters")
    env = {}
    for key in ("compliance", "grayness"):
        a = np.array([float(r[key]) for r in base])
        b = np.array([float(r[key]) for r in pert])
        env[key] = np.maximum(FLOOR, ENVELOPE * np.maximum.accumulate(np.abs(a - b) / np.abs(a)))
    env["iters"] = [max(2, 1 + abs(int(r["cg_iters"]) - int(p["cg_iters"]))) for r, p in zip(base, pert)]
    g = np.load(os.path.join(GOLDEN, "trajectory_driver_cantilever_3d.npz"))
    env["rho"] = max(FLOOR, ENVELOPE * float(np.linalg.norm(g[f"{run}_pert_rho_final"] - g[f"{run}_rho_final"])
                                             / np.linalg.norm(g[f"{run}_rho_final"])))
    return env


def _check(states, ref, env, policy_columns: bool):
    assert len(states) == len(ref)
    for k, (s, r) in enumerate(zip(states, ref)):
        it = r["iteration"]
        assert s["iteration"] == int(it)
        for key in ("penal", "beta", "rmin", "move", "emin"):
            assert s[key] == float(r[key]), (it, key, s[key], r[key])
        if policy_columns:
            for key in ("policy_trigger", "policy_attempted_rho_mins"):
                assert s[key] == r[key], (it, key, s[key], r[key])
            assert s["selected_rho_min"] == float(r["selected_rho_min"]), it
            assert s["policy_fallback_used"] == int(r["policy_fallback_used"]), it
        assert s["solver_true_rel_residual"] <= 1e-6, it
        e = min(k, len(env["compliance"]) - 1)
        assert abs(int(s["cg_iters"]) - int(r["cg_iters"])) <= env["iters"][e], (it, s["cg_iters"], r["cg_iters"])
        for key in ("compliance", "grayness"):
            dev = abs(s[key] - float(r[key])) / abs(float(r[key]))
            assert dev <= env[key][e], (it, key, dev, env[key][e])
    total, total_ref = sum(int(s["cg_iters"]) for s in states), sum(int(r["cg_iters"]) for r in ref)
    assert abs(total - total_ref) <= 0.01 * total_ref, (total, total_ref)


def test_guarded_trajectory_matches_reference(cuda):
    result, states = _run("guarded_adaptive", 45, 1e-12)
    ref = _rows("guarded_iters")
    env = _envelope("guarded")
    _check(states, ref, env, policy_columns=True)
    summary = _rows("guarded_summary")[0]
    assert result["n_iter"] == int(summary["iters_completed"])
    assert result["best_iteration"] == int(summary["best_iteration"])
    assert result["best_is_valid"] == (summary["best_is_valid"] == "True")
    assert result["fem_calls"] == int(summary["fem_calls"]) and result["surrogate_calls"] == 0
    assert abs(result["best_compliance"] - float(summary["best_compliance"])) \
        <= env["compliance"][-1] * float(summary["best_compliance"])
    g = np.load(os.path.join(GOLDEN, "trajectory_driver_cantilever_3d.npz"))
    ref_rho = g["guarded_rho_final"]
    assert isinstance(result["rho_final"], np.ndarray) and result["rho_final"].shape == ref_rho.shape
    assert np.linalg.norm(result["rho_final"] - ref_rho) <= env["rho"] * np.linalg.norm(ref_rho)
    assert [row["iter"] for row in result["params_log"]] == list(range(1, 46))
    assert list(result["params_log"][0])[:6] == ["iter", "penal", "rmin", "move", "beta", "emin"]


def test_fixed_floor_trajectory_matches_reference(cuda):
    result, states = _run("fixed_floor", 20, 1e-3)
    env = _envelope("fixed")
    _check(states, _rows("fixed_iters"), env, policy_columns=False)
    summary = _rows("fixed_summary")[0]
    assert result["n_iter"] == int(summary["iters_completed"])
    assert result["best_is_valid"] == (summary["best_is_valid"] == "True")
    ref_rho = np.load(os.path.join(GOLDEN, "trajectory_driver_cantilever_3d.npz"))["fixed_rho_final"]
    assert np.linalg.norm(result["rho_final"] - ref_rho) <= env["rho"] * np.linalg.norm(ref_rho)


def _entry_passive_mask(nx, ny, nz):
    """The passive mask of make_simp_entry_golden.py: 2 solid, 1 void."""
    m = np.zeros((nx, ny, nz), dtype=np.int32)
    m[20:24, 4:8, :] = 2
    m[8:12, 0:4, 0:3] = 1
    return m.ravel()


class _EchoSurrogate:
    """The generator's surrogate: predicts the sensitivity of the last solve."""

    uncertainty = 0.0

    def __init__(self):
        self._dc = None

    @property
    def is_ready(self):
        return self._dc is not None

    def update(self, rho_phys, rho_f, penal, iter_ratio, dc_phys):
        self._dc = dc_phys.clone() if hasattr(dc_phys, "clone") else np.array(dc_phys, copy=True)

    def predict(self, rho_phys, rho_f, penal, iter_ratio):
        return self._dc, 0.0


def _every_third_router(iteration, uncertainty, surrogate_ready, beta=1.0, **kwargs):
    return iteration % 3 != 0


def run_entry_branches():
    """The unprojected OC step, a passive mask and the surrogate / router hooks
    through run_simp_surrogate_gpu with plain SolverV4, as the golden generator
    calls the reference's."""
    from gpu_fem.bc_generator import generate_bc
    from gpu_fem.presets import get_preset
    from gpu_fem.simp_gpu import TO3DParams, run_simp_surrogate_gpu
    from gpu_fem.solver_v4 import SolverV4

    spec = get_preset("cantilever_3d")
    nx, ny, nz = spec.nelx, spec.nely, spec.nelz
    bc = generate_bc(spec)
    params = TO3DParams(nelx=nx, nely=ny, nelz=nz, volfrac=spec.volfrac, penal=3.0, emin=1e-9, rmin=1.5,
                        max_iter=12, min_iter=12, use_heaviside=False)
    kw = dict(grid_dims=(nx, ny, nz), enable_warm_start=True, enable_matrix_free=True, enable_fused_cuda=False,
              enable_matfree_gmg=True, matfree_gmg_levels=3, gmg_fine_smoother="fp64", gmg_fine_degree=2,
              gmg_outer_solver="fgmres", gmg_restart=300, gmg_smoother_type="chebyshev", gmg_cycle_type="v",
              cg_tol=1e-6, cg_maxiter=150, enable_profiling=False)
    return run_simp_surrogate_gpu(params, bc.fixed_dofs.astype(np.int32), bc.free_dofs.astype(np.int32), bc.F,
                                  bc.ndof, _EchoSurrogate(), _every_third_router, device="auto",
                                  passive_mask=_entry_passive_mask(nx, ny, nz), solver_class=SolverV4,
                                  solver_kwargs=kw)


def test_entry_branches_match_reference(cuda):
    """tests/golden/simp_entry_cantilever_3d.npz (make_simp_entry_golden.py):
    the reference's own run_simp_surrogate_gpu with the unprojected OC step, a
    passive mask, and a surrogate taking iterations 3, 6, 9, 12.  The same
    surrogate flags, solve and surrogate counts, outer iteration counts within
    2, every solve's FP64 true residual at or below 1e-6, and compliance,
    change, volume, grayness and rho_final (the last filtered design: no design
    passes the best-design gate in 12 iterations) inside
    100 times the reference's own deviation under a 1e-12 load perturbation,
    floored at 1e-9."""
    g = np.load(os.path.join(GOLDEN, "simp_entry_cantilever_3d.npz"))
    res = run_entry_branches()
    log = res["params_log"]
    assert len(log) == int(g["base_n_iter"]) == res["n_iter"]
    assert [row["used_surrogate"] for row in log] == list(g["base_used_surrogate"])
    assert res["fem_calls"] == int(g["base_fem_calls"]) and res["surrogate_calls"] == int(g["base_surrogate_calls"])
    assert res["best_is_valid"] == bool(g["base_best_is_valid"])
    for k, row in enumerate(log):
        assert abs(row["cg_iters"] - int(g["base_cg_iters"][k])) <= 2, (k, row["cg_iters"], g["base_cg_iters"][k])
        assert row["solver_true_rel_residual"] <= 1e-6, k
    for key in ("compliance", "change", "volume", "grayness"):
        a, b = g[f"base_{key}"], g[f"pert_{key}"]
        env = np.maximum(FLOOR, ENVELOPE * np.maximum.accumulate(np.abs(a - b) / np.abs(a)))
        got = np.array([row[key] for row in log])
        dev = np.abs(got - a) / np.abs(a)
        assert np.all(dev <= env), (key, dev, env)
    ref, pert = g["base_rho_final"], g["pert_rho_final"]
    env = max(FLOOR, ENVELOPE * float(np.linalg.norm(pert - ref) / np.linalg.norm(ref)))
    assert np.linalg.norm(res["rho_final"] - ref) <= env * np.linalg.norm(ref)
