"""A solve driven the way the reference's phase-5 drivers drive it, through the
drop-in tree: the runner stand-in loaded by path, ``import cupy`` and
``gpu_fem`` from its src directory, the moduli built with cupy calls, the
hierarchy set up and FGMRES run, the true residual taken with cupy.linalg.norm
(run_gmg_floor_detector_prospective.py:178-248 make the same calls).  Run in a
child process so that its cupy stand-in stays out of this one."""

import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROP = os.path.join(REPO, "solver-admissibility-and-guarded-floor-selection_b200", "drop_in")


def test_solve_through_drop_in(cuda):
    code = f"""
import importlib.util, json, sys
import numpy as np
root = {DROP!r}
sys.path.insert(0, root + "/src")
spec = importlib.util.spec_from_file_location("paper4_runner", root + "/experiments/paper4/run_experiments_e1_e10.py")
paper4 = importlib.util.module_from_spec(spec)
spec.loader.exec_module(paper4)
import cupy as cp
from gpu_fem.multigrid_v4 import _cupy_fgmres
spec_, bc, free, free_gpu, edof_gpu, F_free_gpu, mf_op, gmg = paper4._build_components(
    "cantilever_3d", fine_smoother="fp64", smoother_type="jacobi")
n_e = spec_.nelx * spec_.nely * spec_.nelz
rho = (np.random.default_rng(3).random(n_e) >= 0.35).astype(np.float64)
b_norm = float(cp.linalg.norm(F_free_gpu))
E_e = 1e-3 + (1.0 - 1e-3) * cp.asarray(rho, dtype=cp.float64) ** 3.0
cp.cuda.Stream.null.synchronize()
gmg.setup(E_e)
x, iters, conv = _cupy_fgmres(lambda v: mf_op.matvec(v, E_e), F_free_gpu, gmg.apply, tol=1e-6, maxiter=200,
                              restart=100)
cp.cuda.Stream.null.synchronize()
rel = float(cp.linalg.norm(F_free_gpu - mf_op.matvec(x, E_e)) / b_norm)
compliance = float(cp.dot(F_free_gpu, x).get())
direct = float((F_free_gpu * x).sum())
free_b, total_b = cp.cuda.runtime.memGetInfo()
used = cp.get_default_memory_pool().used_bytes()
print(json.dumps({{"iters": int(iters), "conv": bool(conv), "rel": rel, "mem_ok": 0 < free_b <= total_b,
                   "used": used, "cupy": cp.__file__, "compliance": compliance, "direct": direct}}))
"""
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=900)
    assert out.returncode == 0, out.stderr[-3000:]
    r = json.loads(out.stdout.strip().splitlines()[-1])
    assert r["conv"] and 0 < r["iters"] <= 200
    assert r["rel"] <= 1e-6
    assert r["mem_ok"] and r["used"] > 0
    assert r["cupy"].startswith(os.path.join(DROP, "src", "cupy"))
    assert r["compliance"] > 0 and abs(r["compliance"] - r["direct"]) <= 1e-12 * r["direct"]
