"""Several states in flight on one GPU (gpu_fem.policy.BatchedFloorPolicy).

The batched form runs ``width`` independent policies on their own streams and
host threads; state k goes to worker k mod width.  It must give exactly the
rows that the same workers give when they take their states one after another
on a single stream (the computation of each worker is unchanged, only
interleaved with the others on the device), and every accepted answer must pass
the FP64 recomputed-residual guard.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KEYS = ("trigger", "recommended_rho_min", "attempted_rho_mins", "solve_converged", "solve_iters",
        "probe_iters", "total_iters")


def _states(n_elem, seeds):
    out = []
    for s in seeds:
        p = (0.2, 0.35, 0.5)[s % 3]
        out.append((np.random.default_rng(s).random(n_elem) >= p).astype(np.float64))
    return out


def test_batched_matches_sequential_workers(cuda):
    torch = cuda
    from gpu_fem.paper4 import PLAIN_JACOBI_STACK
    from gpu_fem.policy import BatchedFloorPolicy, GuardedFloorPolicy

    kw = dict(penal=3.0, tol=1e-6, probe_iters=60, probe_r50=30, maxiter=120, raised_rho_mins=(1e-3, 1e-2),
              stack=dict(PLAIN_JACOBI_STACK, fine_smoother="fp32"), cycle_precision="fp32")
    width = 3
    bp = BatchedFloorPolicy(width, "cantilever_3d", **kw)
    spec = bp.workers[0].spec
    dens = _states(spec.nelx * spec.nely * spec.nelz, range(7))
    xs = {}
    rows = bp.run_many([torch.as_tensor(d, device="cuda") for d in dens],
                       on_result=lambda k, w, r: xs.__setitem__(k, w.last_x.clone()))
    torch.cuda.synchronize()
    seq = [GuardedFloorPolicy("cantilever_3d", **kw) for _ in range(width)]
    for k, d in enumerate(dens):
        ref = seq[k % width].run(torch.as_tensor(d, device="cuda"))
        for key in KEYS:
            assert rows[k][key] == ref[key], (k, key, rows[k][key], ref[key])
        assert rows[k]["solve_final_rel_residual"] == ref["solve_final_rel_residual"]
        assert torch.equal(xs[k], seq[k % width].last_x)
        assert rows[k]["solve_converged"] == 1 and rows[k]["solve_final_rel_residual"] <= 1e-6


def test_batched_width_validation(cuda):
    from gpu_fem.policy import BatchedFloorPolicy

    with pytest.raises(ValueError):
        BatchedFloorPolicy(0, "cantilever_3d")
