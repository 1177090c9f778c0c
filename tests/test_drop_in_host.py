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
