"""The mixed-precision guarded solve against the FP64 one on the same states:
cantilever 40x20x20 and 80x40x20 (the 64k case), void probability
{0.2, 0.35, 0.5} by seed, cone filter 1.5, SIMP p = 3, floors 1e-12 | 1e-3,
1e-2, plain stack, FGMRES restart 300.  Trigger, selected floor and
convergence flag identical; both answers pass the FP64 guard; the mixed
displacement within 1e-4 and compliance within 1e-5 of the FP64 ones (each
solve stops at true relative residual 1e-6, so they differ by the two
solves' own errors, not by the mixed cycle's rounding)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dims", [(40, 20, 20), (80, 40, 20)])
def test_mixed_matches_fp64_decisions(cuda, dims):
    torch = cuda
    from gpu_fem.paper4 import PLAIN_JACOBI_STACK
    from gpu_fem.policy import GuardedFloorPolicy
    from gpu_fem.presets import cantilever_spec
    from gpu_fem.pub_simp_solver import _build_density_filter

    n = int(np.prod(dims))
    H = _build_density_filter(dims[0], dims[1], 1.5, dims[2])
    kw = dict(penal=3.0, tol=1e-6, restart=300, maxiter=300, probe_iters=100, probe_r50=50,
              raised_rho_mins=(1e-3, 1e-2))
    pols = {
        "fp64": GuardedFloorPolicy(cantilever_spec(*dims), stack=PLAIN_JACOBI_STACK, **kw),
        "mixed": GuardedFloorPolicy(cantilever_spec(*dims), stack=dict(PLAIN_JACOBI_STACK, fine_smoother="fp32"),
                                    cycle_precision="fp32", **kw),
    }
    F = pols["fp64"].F_free_gpu
    for seed in range(6):
        p = (0.2, 0.35, 0.5)[seed % 3]
        dens = torch.as_tensor(np.asarray(H @ (np.random.default_rng(seed).random(n) >= p).astype(np.float64)),
                               device="cuda")
        out = {}
        for name, pol in pols.items():
            r = pol.run(dens)
            out[name] = (r, pol.last_x.clone())
        (r64, x64), (rm, xm) = out["fp64"], out["mixed"]
        for key in ("trigger", "recommended_rho_min", "solve_converged"):
            assert rm[key] == r64[key], (seed, key, rm[key], r64[key])
        assert rm["solve_converged"] == 1 and rm["solve_final_rel_residual"] <= 1e-6
        assert float(torch.linalg.norm(xm - x64) / torch.linalg.norm(x64)) <= 1e-4, seed
        c64, cm = float(torch.dot(F, x64)), float(torch.dot(F, xm))
        assert abs(cm - c64) <= 1e-5 * abs(c64), seed
