"""GalerkinMatFreeGMG.cycle_trace on the device (csrc/trace.cu through
simpfem_gmg_cycle_trace) against the reference's own traces
(tests/golden/cycle_trace_cant24.json, to which the oracle is pinned): every
visit and every field of 20 traces -- V and W cycles, line search, both
enrichment families, both root-local corrections, FP32 coarse levels -- in
the FP64 cycle, to 1e-9 relative (1e-6 with FP32 levels).  In the FP32 cycle
the traced V-cycle's answer is the preconditioner's, and a trace leaves the
hierarchy's apply unchanged."""

import json
import os

import numpy as np
import pytest

from test_gpu_parity import _components
from test_oracle_cycle_trace import assert_trace_close

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "cycle_trace_cant24.json")
with open(GOLDEN) as _fh:
    _TRACES = json.load(_fh)["traces"]


@pytest.mark.parametrize("key", sorted(_TRACES))
def test_device_trace_matches_reference(cuda, ref, key):
    case = _TRACES[key]
    _, gmg, _ = _components("cant24", case["stack"], n_levels=case.get("n_levels", 3))
    gmg.setup(cuda.as_tensor(ref[f"cant24/E_{key.split('/')[1]}"], device="cuda"))
    got = gmg.cycle_trace(cuda.as_tensor(ref["cant24/rhs"], device="cuda")).to_dict()
    rtol = 1e-6 if key.startswith("level_fp32") else 1e-9
    assert_trace_close(got, case["trace"], rtol, key)


def test_trace_cycle_type_override(cuda, ref):
    _, gmg, _ = _components("cant24", {})
    gmg.setup(cuda.as_tensor(ref["cant24/E_mid"], device="cuda"))
    rhs = cuda.as_tensor(ref["cant24/rhs"], device="cuda")
    assert_trace_close(gmg.cycle_trace(rhs, cycle_type="w").to_dict(), _TRACES["wcycle/mid"]["trace"], 1e-9, "w")
    with pytest.raises(ValueError, match="cycle_type"):
        gmg.cycle_trace(rhs, cycle_type="x")


@pytest.mark.parametrize("cycle", ["v", "w"])
def test_fp32_cycle_trace_four_levels(cuda, cycle):
    import torch

    from gpu_fem.paper4 import _build_components
    from gpu_fem.presets import cantilever_spec

    spec, _, _, _, _, F, _, gmg = _build_components(cantilever_spec(48, 24, 12), n_levels=4, cycle_type=cycle,
                                                     cycle_precision="fp32")
    nel = spec.nelx * spec.nely * spec.nelz
    rng = np.random.default_rng(3)
    E = torch.as_tensor(1e-3 + (1 - 1e-3) * (rng.random(nel) > 0.3), device="cuda")
    gmg.setup(E)
    z0 = gmg.apply(F)
    tr = gmg.cycle_trace(F)
    z1 = gmg.apply(F)
    assert torch.equal(z0, z1)  # the trace leaves the hierarchy as it was
    levels = [v.level for v in tr.visits]
    if cycle == "v":
        assert levels == [0, 1, 2, 3]
        # same kernels in the same order as apply: the same answer
        assert tr.output_norm == pytest.approx(float(torch.linalg.norm(z0)), rel=1e-12)
        assert tr.rz == pytest.approx(float(torch.dot(F, z0)), rel=1e-12)
    else:
        assert len(levels) == 15 and levels[:4] == [0, 1, 2, 3]
        # the W-cycle trace forms its second residual as res - A c (the cycle as rhs - A x)
        assert tr.output_norm == pytest.approx(float(torch.linalg.norm(z0)), rel=1e-4)
        scale = float(torch.linalg.norm(F)) * float(torch.linalg.norm(z0))
        assert abs(tr.rz - float(torch.dot(F, z0))) <= 1e-4 * scale
    assert [v.visit_id for v in tr.visits] == list(range(len(levels)))
    assert tr.visits[-1].is_coarsest and tr.visits[-1].coarsest_mode == "dense"
    assert all(np.isfinite(v.postsmooth_residual_norm) for v in tr.visits)
    assert tr.pd == (tr.rz > 0.0)
    assert tr.rhs_norm == pytest.approx(float(torch.linalg.norm(F)), rel=1e-12)


with open(GOLDEN) as _fh:
    _DIAG = json.load(_fh)["diagnostics"]


@pytest.mark.parametrize("key", sorted(_DIAG))
def test_device_probe_quality_and_kappa_match_reference(cuda, ref, key):
    """probe_quality (multigrid_v4.py:1348-1360) and the 30-step Lanczos
    estimate_kappa_eff (:1057-1117) of the device hierarchy against the
    reference's values on the same start vector."""
    case = _DIAG[key]
    _, gmg, _ = _components("cant24", case["stack"])
    gmg.setup(cuda.as_tensor(ref[f"cant24/E_{key.split('/')[1]}"], device="cuda"))
    pq = gmg.probe_quality(cuda.as_tensor(ref["cant24/rhs"], device="cuda"))
    want = case["probe_quality"]
    assert pq["finite"] == want["finite"] and pq["pd"] == want["pd"]
    rtol = 1e-6 if key.startswith("level_fp32") else 1e-9
    for k in ("z_norm", "jacobi_norm", "z_over_jacobi"):
        assert pq[k] == pytest.approx(want[k], rel=rtol), k
    # Lanczos amplifies the FP32 levels' rounding (FP32 vs FP64 levels differ by 3e-5 here)
    ktol = 1e-5 if key.startswith("level_fp32") else 1e-7
    assert gmg.estimate_kappa_eff(30) == pytest.approx(case["kappa_eff_30"], rel=ktol)
    assert gmg.kappa_eff == pytest.approx(case["kappa_eff_30"], rel=ktol)


@pytest.mark.parametrize("dims", [(24, 12, 6), (20, 10, 10)])
def test_fp32_coarsest_solve(cuda, dims):
    """The mixed cycle's coarsest solve (FP32 copies of L^-1 and L^-T, FP64
    accumulation; float4 rows when the coarsest size is a multiple of 4, as
    for 24x12x6 with 144 unknowns, scalar rows otherwise, as for 20x10x10 with
    135) against the FP64 cycle's, both with FP32 level operators on a uniform
    field: the coarsest visit sees the same right-hand side to 1e-5, returns
    the same correction to 1e-4, and leaves a relative residual below 1e-3
    (measured with the FP32 level operator)."""
    import torch

    from gpu_fem.paper4 import _build_components
    from gpu_fem.presets import cantilever_spec

    got = {}
    for prec in ("fp64", "fp32"):
        spec, _, _, _, _, F, _, gmg = _build_components(cantilever_spec(*dims), n_levels=3, cycle_precision=prec,
                                                         fine_smoother="fp32", level_precisions=["fp32"] * 3)
        gmg.setup(torch.ones(spec.nelx * spec.nely * spec.nelz, dtype=torch.float64, device="cuda"))
        got[prec] = [v for v in gmg.cycle_trace(F).visits if v.is_coarsest][0]
    a, b = got["fp32"], got["fp64"]
    assert a.rhs_norm == pytest.approx(b.rhs_norm, rel=1e-5)
    assert a.coarse_correction_norm == pytest.approx(b.coarse_correction_norm, rel=1e-4)
    assert a.postsmooth_residual_ratio <= 1e-3 and b.postsmooth_residual_ratio <= 1e-6
