"""The drop-in tree (solver-admissibility-and-guarded-floor-selection_b200/drop_in)
that lets the reference's phase-5 drivers run unchanged against this library.

The drivers load experiments/paper4/run_experiments_e1_e10.py two directories
above themselves (run_gmg_floor_detector_prospective.py:18-24), put <root>/src
first on sys.path and import gpu_fem and cupy from there.  Checked here without
a GPU: the runner stand-in hands out this library's _build_components, and the
cupy stand-in has the surface those drivers use.  With SIMPFEM_REFERENCE_ROOT
set to a reference checkout, each of the four detector drivers and the SIMP
trajectory driver is also placed, unchanged, in a copy of the drop-in tree and
its own loader and imports are run: they must resolve to this library."""

import json
import os
import shutil
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROP = os.path.join(REPO, "solver-admissibility-and-guarded-floor-selection_b200", "drop_in")
PKG = os.path.realpath(os.path.join(REPO, "solver-admissibility-and-guarded-floor-selection_b200", "gpu_fem"))


def _run(code: str) -> dict:
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    return json.loads(out.stdout.strip().splitlines()[-1])


def test_runner_stand_in_hands_out_this_library():
    code = f"""
import importlib.util, json, os
spec = importlib.util.spec_from_file_location(
    "paper4_runner", {os.path.join(DROP, "experiments", "paper4", "run_experiments_e1_e10.py")!r})
m = importlib.util.module_from_spec(spec)
spec.loader.exec_module(m)
import gpu_fem.paper4 as p4
print(json.dumps({{"same": m._build_components is p4._build_components,
                   "pkg": os.path.realpath(os.path.dirname(p4.__file__))}}))
"""
    r = _run(code)
    assert r["same"] and r["pkg"] == PKG


def test_cupy_stand_in_surface():
    code = f"""
import json, sys
sys.path.insert(0, {os.path.join(DROP, "src")!r})
import cupy as cp
names = ["float64", "float32", "asarray", "zeros", "dot", "asnumpy"]
ok = all(hasattr(cp, n) for n in names)
ok = ok and callable(cp.linalg.norm) and callable(cp.cuda.Stream.null.synchronize)
ok = ok and callable(cp.cuda.runtime.memGetInfo)
ok = ok and callable(cp.get_default_memory_pool().used_bytes) and callable(cp.get_default_memory_pool().total_bytes)
ok = ok and cp.get_default_pinned_memory_pool().n_free_blocks() == 0
import torch
one = torch.ones(2, dtype=torch.float64)
ok = ok and float(cp.dot(one, one).get()) == 2.0 and float(cp.dot(one, one)) == 2.0
print(json.dumps({{"ok": ok, "file": cp.__file__}}))
"""
    r = _run(code)
    assert r["ok"] and r["file"].startswith(os.path.join(DROP, "src", "cupy"))


DRIVERS = ["run_gmg_floor_detector_prospective.py", "run_gmg_floor_detector_density_field.py",
           "run_gmg_fixed_floor_controls.py", "run_gmg_floor_rule_check.py"]


@pytest.mark.skipif(not os.environ.get("SIMPFEM_REFERENCE_ROOT"), reason="needs a reference checkout")
@pytest.mark.parametrize("driver", DRIVERS)
def test_unchanged_reference_driver_resolves_here(tmp_path, driver):
    src = os.path.join(os.environ["SIMPFEM_REFERENCE_ROOT"], "experiments", "phase5", driver)
    (tmp_path / "experiments" / "phase5").mkdir(parents=True)
    shutil.copyfile(src, tmp_path / "experiments" / "phase5" / driver)
    os.symlink(os.path.join(DROP, "experiments", "paper4"), tmp_path / "experiments" / "paper4")
    os.symlink(os.path.join(DROP, "src"), tmp_path / "src")
    code = f"""
import importlib.util, json, os
spec = importlib.util.spec_from_file_location("drv", {str(tmp_path / "experiments" / "phase5" / driver)!r})
d = importlib.util.module_from_spec(spec)
spec.loader.exec_module(d)
runner = d._load_paper4_runner()
import cupy, gpu_fem.multigrid_v4 as mg, gpu_fem.paper4 as p4
print(json.dumps({{"same": runner._build_components is p4._build_components,
                   "fgmres": os.path.realpath(mg.__file__),
                   "cupy": os.path.realpath(cupy.__file__)}}))
"""
    r = _run(code)
    assert r["same"]
    assert r["fgmres"] == os.path.join(PKG, "multigrid_v4.py")
    assert r["cupy"] == os.path.realpath(os.path.join(DROP, "src", "cupy", "__init__.py"))


@pytest.mark.skipif(not os.environ.get("SIMPFEM_REFERENCE_ROOT"), reason="needs a reference checkout")
def test_unchanged_trajectory_driver_resolves_here(tmp_path):
    """run_simp_floor_trajectory.py imports the SIMP loop, the solver, the router
    and the controller from gpu_fem (:34-39) and subclasses SolverV4 (:65)."""
    driver = "run_simp_floor_trajectory.py"
    src = os.path.join(os.environ["SIMPFEM_REFERENCE_ROOT"], "experiments", "phase5", driver)
    (tmp_path / "experiments" / "phase5").mkdir(parents=True)
    shutil.copyfile(src, tmp_path / "experiments" / "phase5" / driver)
    os.symlink(os.path.join(DROP, "src"), tmp_path / "src")
    code = f"""
import importlib.util, json, os
spec = importlib.util.spec_from_file_location("drv", {str(tmp_path / "experiments" / "phase5" / driver)!r})
d = importlib.util.module_from_spec(spec)
spec.loader.exec_module(d)
import gpu_fem.simp_gpu as sg, gpu_fem.solver_v4 as s4, gpu_fem.local_agents as la, gpu_fem.pub_baseline_controller as pc
print(json.dumps({{"loop": d.run_simp_surrogate_gpu is sg.run_simp_surrogate_gpu and d.TO3DParams is sg.TO3DParams,
                   "solver": issubclass(d.GuardedAdaptiveFloorSolverV4, s4.SolverV4),
                   "agents": d.PureFEMRouter is la.PureFEMRouter and d.ScheduleOnlyController is pc.ScheduleOnlyController,
                   "pkg": os.path.realpath(os.path.dirname(sg.__file__))}}))
"""
    r = _run(code)
    assert r["loop"] and r["solver"] and r["agents"]
    assert r["pkg"] == PKG


def _csv(path):
    import csv

    with open(path, newline="") as f:
        return list(csv.DictReader(f))


@pytest.mark.skipif(not os.environ.get("SIMPFEM_REFERENCE_ROOT"), reason="needs a reference checkout")
def test_unchanged_direct_solve_drivers_match_reference(tmp_path):
    """run_direct_floor_atlas.py, run_direct_floor_conditioning.py and
    compare_reduced_floor_perturbation.py assemble K from the paper-4 runner's
    KE_UNIT_3D, _edof_table_3d and _build_sparse_indices and solve it with scipy on
    the host, so they run here without a GPU.  Unchanged, over the drop-in tree,
    against their run over the reference's own package
    (tests/golden/make_direct_floor_golden.py): the same rows, flags and counts; the
    matrix diagonal to 1e-14 (the two element matrices differ in the last bits);
    lambda_max to 1e-12; the solution norm, lambda_min and kappa within ten times the
    row's own kappa * eps (at least 1e-8), the round-off a solve at that
    conditioning carries; direct residuals below 1e-10; for the floor comparison,
    compliances to 1e-8, the solution change against the 1e-12 solve within ten
    times that solve's kappa * eps, and the raised solution's residual under the
    1e-12 operator to 1e-6 (round-off level, below 1e-10, on the 1e-12 rows)."""
    args = ["--preset", "cantilever_3d", "--probabilities", "0.2,0.35", "--rho-min-values", "1e-12,1e-6,1e-3",
            "--seeds", "3", "--out-dir", str(tmp_path / "out")]
    (tmp_path / "experiments" / "phase5").mkdir(parents=True)
    os.symlink(os.path.join(DROP, "experiments", "paper4"), tmp_path / "experiments" / "paper4")
    os.symlink(os.path.join(DROP, "src"), tmp_path / "src")
    for driver in ("run_direct_floor_atlas.py", "run_direct_floor_conditioning.py",
                   "compare_reduced_floor_perturbation.py"):
        src = os.path.join(os.environ["SIMPFEM_REFERENCE_ROOT"], "experiments", "phase5", driver)
        shutil.copyfile(src, tmp_path / "experiments" / "phase5" / driver)
        out = subprocess.run([sys.executable, str(tmp_path / "experiments" / "phase5" / driver)] + args,
                             capture_output=True, text=True, timeout=900)
        assert out.returncode == 0, out.stderr[-2000:]
    golden = os.path.join(REPO, "tests", "golden")
    cond = _csv(os.path.join(golden, "direct_floor_conditioning_cantilever_3d.csv"))
    kappa_eps = {(r["solid_probability"], r["rho_min"]): float(r["kappa_times_eps"]) for r in cond}

    def close(a, b, rel, where):
        a, b = float(a), float(b)
        assert abs(a - b) <= rel * abs(b), (where, a, b, rel)

    for mine, ref in (("direct_floor_atlas.csv", "direct_floor_atlas_cantilever_3d.csv"),
                      ("direct_floor_conditioning.csv", "direct_floor_conditioning_cantilever_3d.csv")):
        got, exp = _csv(tmp_path / "out" / mine), _csv(os.path.join(golden, ref))
        assert len(got) == len(exp) and list(got[0]) == list(exp[0])
        for g, r in zip(got, exp):
            key = (r["solid_probability"], r["rho_min"])
            loose = max(1e-8, 10.0 * kappa_eps[key])
            for k in ("preset", "seed", "solid_probability", "rho_min", "penal", "tol", "converged", "n_free", "nnz"):
                if k in r:
                    assert g[k] == r[k], (mine, key, k)
            for k in ("diag_min", "diag_max", "diag_ratio"):
                if k in r:
                    close(g[k], r[k], 1e-14, (mine, key, k))
            if "lambda_max" in r:
                close(g["lambda_max"], r["lambda_max"], 1e-12, (mine, key))
            for k in ("x_norm", "lambda_min", "kappa"):
                if k in r:
                    close(g[k], r[k], loose, (mine, key, k))
            assert float(g["rel_residual"]) <= 1e-10 and float(r["rel_residual"]) <= 1e-10
    crit = _csv(tmp_path / "out" / "direct_floor_critical.csv")
    exp = _csv(os.path.join(golden, "direct_floor_critical_cantilever_3d.csv"))
    assert [{k: v for k, v in r.items() if not k.startswith("critical_rel") and k != "critical_x_norm"} for r in crit] \
        == [{k: v for k, v in r.items() if not k.startswith("critical_rel") and k != "critical_x_norm"} for r in exp]
    got = _csv(tmp_path / "out" / "reduced_floor_perturbation_summary.csv")
    exp = _csv(os.path.join(golden, "reduced_floor_perturbation_cantilever_3d.csv"))
    assert len(got) == len(exp) and list(got[0]) == list(exp[0])
    for g, r in zip(got, exp):
        key = (r["solid_probability"], r["rho_min"])
        ref_noise = 10.0 * kappa_eps[(r["solid_probability"], "1e-12")]
        for k in ("preset", "seed", "solid_probability", "n_elem", "n_free", "rho_min", "reference_rho_min", "penal",
                  "solid_count", "solid_fraction"):
            assert g[k] == r[k], (key, k)
        for k in ("compliance", "reference_compliance"):
            close(g[k], r[k], 1e-8, key)
        assert abs(float(g["rel_compliance_change"]) - float(r["rel_compliance_change"])) <= 1e-8, key
        assert abs(float(g["rel_u_error"]) - float(r["rel_u_error"])) <= ref_noise, key
        for k in ("direct_rel_residual", "reference_direct_rel_residual"):
            assert float(g[k]) <= 1e-10 and float(r[k]) <= 1e-10, (key, k)
        k = "raised_solution_residual_under_reference_operator"
        if float(r[k]) <= 1e-10:
            assert float(g[k]) <= 1e-10, key
        else:
            close(g[k], r[k], 1e-6, key)


@pytest.mark.skipif(not os.environ.get("SIMPFEM_REFERENCE_ROOT"), reason="needs a reference checkout")
def test_unchanged_direct_solve_drivers_reproduce_published_tables(tmp_path):
    """The two direct-solve drivers, unchanged over the drop-in tree at the arguments
    of the reference's published tables (tests/golden/published_direct_floor_*_seed19.csv,
    from its data/analysis_tables; make_published_direct_floor.py): the atlas at its
    defaults (seed 19, six solid probabilities, floors 1e-12 to 1e-3) gives the same
    critical floor for every probability, with the solution norm there within 1e-5;
    the conditioning sweep at seed 19 (48 rows, floors 1e-12 to 1e-2) the same
    converged flag on every row, lambda_max to 1e-12 and lambda_min within the row's
    own kappa * eps (at least 1e-8).  Residuals at these conditionings are round-off
    and are compared through the flags."""
    (tmp_path / "experiments" / "phase5").mkdir(parents=True)
    os.symlink(os.path.join(DROP, "experiments", "paper4"), tmp_path / "experiments" / "paper4")
    os.symlink(os.path.join(DROP, "src"), tmp_path / "src")
    runs = {"run_direct_floor_atlas.py": [], "run_direct_floor_conditioning.py": ["--seeds", "19"]}
    for driver, extra in runs.items():
        shutil.copyfile(os.path.join(os.environ["SIMPFEM_REFERENCE_ROOT"], "experiments", "phase5", driver),
                        tmp_path / "experiments" / "phase5" / driver)
        out = subprocess.run([sys.executable, str(tmp_path / "experiments" / "phase5" / driver), *extra,
                              "--out-dir", str(tmp_path / "out")], capture_output=True, text=True, timeout=1200)
        assert out.returncode == 0, out.stderr[-2000:]
    golden = os.path.join(REPO, "tests", "golden")
    got = _csv(tmp_path / "out" / "direct_floor_critical.csv")
    exp = _csv(os.path.join(golden, "published_direct_floor_critical_seed19.csv"))
    assert len(got) == len(exp) == 6 and list(got[0]) == list(exp[0])
    for g, r in zip(got, exp):
        for k in ("preset", "seed", "solid_probability", "critical_rho_min", "all_failed"):
            assert g[k] == r[k], (r["solid_probability"], k, g[k], r[k])
        x, y = float(g["critical_x_norm"]), float(r["critical_x_norm"])
        assert abs(x - y) <= 1e-5 * y, (r["solid_probability"], x, y)
    got = _csv(tmp_path / "out" / "direct_floor_conditioning.csv")
    exp = _csv(os.path.join(golden, "published_direct_floor_conditioning_seed19.csv"))
    assert len(got) == len(exp) == 48 and list(got[0]) == list(exp[0])
    for g, r in zip(got, exp):
        key = (r["solid_probability"], r["rho_min"])
        for k in ("preset", "seed", "solid_probability", "rho_min", "penal", "converged", "n_free"):
            assert g[k] == r[k], (key, k, g[k], r[k])
        lmax, lmax_ref = float(g["lambda_max"]), float(r["lambda_max"])
        assert abs(lmax - lmax_ref) <= 1e-12 * lmax_ref, key
        lmin, lmin_ref = float(g["lambda_min"]), float(r["lambda_min"])
        assert abs(lmin - lmin_ref) <= max(1e-8, float(r["kappa_times_eps"])) * lmin_ref, (key, lmin, lmin_ref)
