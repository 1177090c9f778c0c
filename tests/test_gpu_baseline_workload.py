"""The CUDA path on the benchmark workload's own states, against the reference.

tests/golden/baseline_policy_<grid>.npz (make_baseline_golden.py) hold the
reference's own guarded policy run (its MatrixFreeKff, GalerkinMatFreeGMG and
_cupy_fgmres, unmodified) on filtered void-probability states -- void with
probability (0.2, 0.35, 0.5)[seed % 3], cone filter r = 1.5, E = rho_min +
(1 - rho_min) rho^3, damped-Jacobi 4-level V-cycle, FGMRES restart 300, tol
1e-6, 100-iteration probe, ladder {1e-3, 1e-2} -- with every state of a grid
solved in seed order through one hierarchy: seeds 0-5 on 80 x 40 x 20 and
seeds 0-1 on the measured 160 x 80 x 40 grid.

FP64 mode (the reference's arithmetic; the probe is re-solved at a kept
floor, as the reference driver does): trigger, attempted and selected floors,
fallback and convergence flags and iteration counts identical; the probe's
residual history within 1e-6 relative; compliance F.x and the displacement
sample within max(1e-7, 100 x the reference's own deviation under a 1e-14
perturbation of E).

Mixed mode (FP32 V-cycle with BF16 coarse stencils, FP64 Krylov and guard):
the same decisions, every answer through the FP64 guard, and its error
against the reference's FP64 answer within 1e-5 (compliance) and 1e-4
(displacement); the measured errors are printed.
"""

import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
GRIDS = {"80x40x20": ("cantilever_gpu_medium", (80, 40, 20)),
         "160x80x40": ("cantilever_gpu_xlarge", (160, 80, 40))}


def _load(grid):
    path = os.path.join(HERE, f"baseline_policy_{grid}.npz")
    if not os.path.exists(path):
        pytest.skip(f"no fixture for {grid}")
    g = np.load(path)
    return (json.loads(str(g["meta"])), json.loads(str(g["rows"])), json.loads(str(g["pert_rows"])),
            json.loads(str(g["probe_history"])), g["x_sample"], g["pert_x_sample"])


def _policy(preset, precision):
    from gpu_fem.paper4 import PLAIN_JACOBI_STACK
    from gpu_fem.policy import GuardedFloorPolicy

    stack = dict(PLAIN_JACOBI_STACK, fine_smoother="fp64" if precision == "fp64" else "fp32")
    return GuardedFloorPolicy(preset, penal=3.0, tol=1e-6, restart=300, maxiter=300, probe_iters=100, probe_r50=50,
                              raised_rho_mins=(1e-3, 1e-2), stack=stack, cycle_precision=precision,
                              reuse_probe=False)


def _run(grid, precision):
    import torch

    from gpu_fem.pub_simp_solver import _build_density_filter

    meta, rows, pert, hist, xs_ref, xs_pert = _load(grid)
    preset, (nx, ny, nz) = GRIDS[grid]
    n = nx * ny * nz
    H = _build_density_filter(nx, ny, meta["rmin"], nz)
    pol = _policy(preset, precision)
    F = pol.F_free_gpu
    out = []
    for k, ref in enumerate(rows):
        seed = ref["seed"]
        p = meta["probs"][seed % len(meta["probs"])]
        rho = H @ (np.random.default_rng(seed).random(n) >= p).astype(np.float64)
        row = pol.run(torch.as_tensor(rho, device="cuda"))
        x = pol.last_x
        xs = x[:: meta["stride"]].cpu().numpy()
        c = float(torch.dot(F, x))
        dev_c = abs(pert[k]["compliance"] - ref["compliance"]) / ref["compliance"]
        dev_x = np.linalg.norm(xs_pert[k] - xs_ref[k]) / np.linalg.norm(xs_ref[k])
        out.append(dict(ref=ref, row=row, hist=hist[k], c_err=abs(c - ref["compliance"]) / ref["compliance"],
                        x_err=float(np.linalg.norm(xs - xs_ref[k]) / np.linalg.norm(xs_ref[k])), dev_c=dev_c,
                        dev_x=dev_x))
    return out


def _same_decisions(o, iters: bool):
    ref, row = o["ref"], o["row"]
    assert row["trigger"] == ref["trigger"], (row["trigger"], ref)
    assert row["attempted_rho_mins"] == ref["attempted"], (row["attempted_rho_mins"], ref)
    assert row["recommended_rho_min"] == ref["rho_min"]
    assert bool(row["post_solve_fallback_triggered"]) == ref["fallback"]
    assert bool(row["solve_converged"]) == ref["converged"] and row["solve_final_rel_residual"] <= 1e-6
    if iters:
        assert row["solve_iters"] == ref["iters"] and row["probe_iters"] == ref["probe_iters"], (row, ref)


@pytest.mark.parametrize("grid", list(GRIDS))
def test_fp64_policy_matches_reference(cuda, grid):
    for k, o in enumerate(_run(grid, "fp64")):
        _same_decisions(o, iters=True)
        m = min(20, len(o["hist"]))
        np.testing.assert_allclose(o["row"]["probe_history"][:m], o["hist"][:m], rtol=1e-6)
        assert o["c_err"] <= max(1e-7, 100 * o["dev_c"]), (grid, k, o["c_err"], o["dev_c"])
        assert o["x_err"] <= max(1e-7, 100 * o["dev_x"]), (grid, k, o["x_err"], o["dev_x"])
        print(f"{grid} seed {o['ref']['seed']} fp64: compliance rel err {o['c_err']:.2e}, x rel err {o['x_err']:.2e}")


@pytest.mark.parametrize("grid", list(GRIDS))
def test_mixed_policy_error_against_reference(cuda, grid):
    for k, o in enumerate(_run(grid, "fp32")):
        _same_decisions(o, iters=False)
        assert o["c_err"] <= 1e-5 and o["x_err"] <= 1e-4, (grid, k, o["c_err"], o["x_err"])
        print(f"{grid} seed {o['ref']['seed']} mixed: compliance rel err {o['c_err']:.2e}, x rel err {o['x_err']:.2e}")
