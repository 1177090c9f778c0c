"""The captured V/W-cycle (use_graphs, CUDA graph replayed after the second
cycle of each setup) against direct launches: the same kernels with the same
arguments, so every FGMRES history, iterate and preconditioner output is
bitwise identical -- FP64 canonical stack (inner Krylov and root-local
correction around the captured cycle), FP64 W-cycle with line search and
enrichment, and the mixed FP32 cycle -- across setups that change the sweep
counts (the high-contrast schedule, which changes the graph's topology) and
back.  The replay counter shows the graphs ran."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STACKS = {
    "canonical": dict(fine_smoother="fp64", coarse_correction_policy="residual_line_search",
                      root_local_correction_mode="node_block_inner_fgmres", root_local_correction_inner_steps=20,
                      root_local_correction_inner_restart=20, inner_krylov_steps=10, inner_krylov_restart=10),
    "wcycle_enrich": dict(fine_smoother="fp64", cycle_type="w", coarse_correction_policy="residual_line_search",
                          root_enrichment_mode="void_gap_second"),
    "mixed": dict(fine_smoother="fp32", cycle_precision="fp32"),
}


@pytest.mark.parametrize("stack", sorted(STACKS))
def test_graph_replay_is_bitwise_identical(cuda, stack):
    import torch

    from gpu_fem.multigrid_v4 import GalerkinMatFreeGMG, _cupy_fgmres
    from gpu_fem.paper4 import _build_components
    from gpu_fem.presets import cantilever_spec
    from gpu_fem.pub_simp_solver import KE_UNIT_3D

    dims = (48, 24, 12)
    n = int(np.prod(dims))
    rng = np.random.default_rng(11)
    fields = [1e-3 + (1 - 1e-3) * (rng.random(n) > 0.35),       # high contrast: 4 fine sweeps
              0.2 + 0.8 * rng.random(n),                       # mild: 2 fine sweeps
              1e-9 + (1 - 1e-9) * (rng.random(n) > 0.5)]       # high contrast again
    out = {}
    for graphs in (True, False):
        spec, _, free, free_gpu, _, F, mf, _ = _build_components(cantilever_spec(*dims), n_levels=4)
        gmg = GalerkinMatFreeGMG(mf_op=mf, free=free, free_gpu=free_gpu, nelx=dims[0], nely=dims[1],
                                 nelz=dims[2], KE_UNIT=KE_UNIT_3D, n_levels=4, use_graphs=graphs, **STACKS[stack])
        runs = []
        for E in fields:
            E = torch.as_tensor(E, device="cuda")
            gmg.setup(E)
            hist = []
            x, it, conv = _cupy_fgmres(lambda v: mf.matvec(v, E), F, gmg.apply, tol=1e-8, maxiter=40, restart=30,
                                       history=hist)
            z1 = gmg.apply(F)
            z2 = gmg.apply(F)
            z3 = gmg.apply(F)
            runs.append((x.clone(), it, conv, list(hist), z1.clone(), z2.clone(), z3.clone()))
        out[graphs] = (runs, gmg._get_props().cycle_graph_replays)
    (with_g, replays), (without, none) = out[True], out[False]
    assert none == 0 and replays > 0
    for a, b in zip(with_g, without):
        assert a[1] == b[1] and a[2] == b[2] and a[3] == b[3]
        for u, v in zip(a[:1] + a[4:], b[:1] + b[4:]):
            assert torch.equal(u, v)
