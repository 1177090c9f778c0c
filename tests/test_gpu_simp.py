"""The SIMP loop around the guarded solve (gpu_fem.simp_loop, csrc/simp.cu)
against the oracle.

* the cone filter H x and H^T x against the oracle's sparse filter matrix
  (to 1e-13 of the largest entry; radii 1.2, 1.5, 2.5, ragged grids);
* the OC update against the reference's own _oc_step_cupy outputs
  (tests/golden/oc_reference.npz) and against its bisection restated in
  oracle/simp.py, which evaluates every candidate's volume as sum(H rn) through
  the sparse matrix (the kernel uses sum_j (H^T 1)_j rn_j): same step count,
  multiplier and new densities to the final bisection bracket (1e-8);
* the first loop iteration's compliance and sensitivities against a direct
  sparse solve (1e-6 and 1e-5 relative: the solve stops at true residual 1e-6);
* a short loop: every solve guarded, the volume held at the target by the OC
  step, the compliance falling from its first value.
"""

import numpy as np
import pytest

from oracle import simp as osimp
from oracle import solver as osol

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dims,rmin", [((13, 7, 5), 1.5), ((24, 12, 6), 1.2), ((9, 11, 6), 2.5), ((40, 20, 20), 1.5)])
def test_cone_filter_matches_oracle(cuda, dims, rmin):
    from gpu_fem.simp_loop import cone_filter

    H = osol.density_filter(*dims, rmin)
    x = np.random.default_rng(int(10 * rmin) + sum(dims)).random(int(np.prod(dims)))
    xd = cuda.as_tensor(x, device="cuda")
    for t, ref in ((False, H @ x), (True, H.T @ x)):
        got = cone_filter(xd, dims, rmin, transpose=t).cpu().numpy()
        assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max(), t


@pytest.mark.parametrize("case", [0, 1, 2])
def test_oc_update_matches_reference_outputs(cuda, case):
    """The device OC update on the inputs of the reference's own _oc_step_cupy
    runs (tests/golden/oc_reference.npz): new densities to 1e-8 (the last
    bisection bracket), the same change."""
    import os

    from gpu_fem.simp_loop import OCUpdater, cone_filter

    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "oc_reference.npz"))
    rmin, volfrac, move = (float(v) for v in g[f"c{case}/params"])
    dims = (24, 12, 6)
    n = int(np.prod(dims))
    dc = cone_filter(cuda.as_tensor(g[f"c{case}/dc_phys"], device="cuda"), dims, rmin, transpose=True)
    vol_w = cone_filter(cuda.ones(n, dtype=cuda.float64, device="cuda"), dims, rmin, transpose=True)
    rn, change, _, _ = OCUpdater()(cuda.as_tensor(g[f"c{case}/rho"], device="cuda"), dc, vol_w, volfrac, move)
    np.testing.assert_allclose(rn.cpu().numpy(), g[f"c{case}/rn"], rtol=0, atol=1e-8)
    assert change == pytest.approx(float(g[f"c{case}/change"][0]), abs=1e-8)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_oc_update_matches_reference_bisection(cuda, seed):
    from gpu_fem.simp_loop import OCUpdater, cone_filter

    dims, rmin = (24, 12, 6), 1.5
    n = int(np.prod(dims))
    rng = np.random.default_rng(seed)
    rho = np.clip(0.3 + 0.2 * rng.standard_normal(n), 1e-3, 1.0)
    dc_phys = -np.exp(rng.standard_normal(n))
    H = osol.density_filter(*dims, rmin)
    ref_rn, ref_change, ref_lm, ref_steps = osimp.oc_update(rho, dc_phys, H, 0.3, 0.2)
    dc = cone_filter(cuda.as_tensor(dc_phys, device="cuda"), dims, rmin, transpose=True)
    vol_w = cone_filter(cuda.ones(n, dtype=cuda.float64, device="cuda"), dims, rmin, transpose=True)
    rn, change, lm, steps = OCUpdater()(cuda.as_tensor(rho, device="cuda"), dc, vol_w, 0.3, 0.2)
    # the bracket halves every step, so the step count is fixed; the last steps
    # compare volumes within round-off of the target, where the two (equal)
    # volume formulas may round apart: the multiplier agrees to the final
    # bracket width (1e-9)
    assert steps == ref_steps
    assert lm == pytest.approx(ref_lm, rel=1e-8)
    np.testing.assert_allclose(rn.cpu().numpy(), ref_rn, rtol=0, atol=1e-8)
    assert change == pytest.approx(ref_change, abs=1e-8)
    # the update meets the volume target to the bisection's precision
    assert abs(float((H @ rn.cpu().numpy()).sum()) / n - 0.3) < 1e-6


def test_first_iteration_matches_direct_solve(cuda):
    from gpu_fem.simp_loop import run_simp_guarded

    dims = (24, 12, 6)
    seen = {}
    res = run_simp_guarded(dims, max_iter=1, policy="plain", restart=100, seed=3,
                           callback=lambda row: seen.update(row))
    n = int(np.prod(dims))
    rho0 = np.clip(0.3 + 0.02 * np.random.default_rng(3).standard_normal(n), 1e-3, 1.0)
    H = osol.density_filter(*dims, 1.5)
    rho_phys = H @ rho0
    free, F = osol.cantilever_bc(*dims)
    c, dc, _ = osimp.compliance_and_sensitivity(*dims, rho_phys, free, F, 3.0, seen["selected_rho_min"])
    assert res["all_guarded"]
    assert res["compliance_history"][0] == pytest.approx(c, rel=1e-6)
    ref_rn, _, _, _ = osimp.oc_update(rho0, dc, H, 0.3, 0.2)
    # the sensitivities differ at the solve's tolerance; the update follows them closely
    assert np.abs(res["rho"].cpu().numpy() - ref_rn).max() < 1e-4


@pytest.mark.parametrize("policy", ["plain", "learned"])
def test_short_loop_is_guarded_and_descends(cuda, policy):
    from gpu_fem.simp_loop import run_simp_guarded

    res = run_simp_guarded((24, 12, 6), max_iter=8, policy=policy, restart=100, seed=0)
    rows = res["iterations"]
    assert res["all_guarded"]
    assert all(r["true_rel_residual"] <= 1e-6 for r in rows)
    assert all(abs(r["volume"] - 0.3) < 1e-3 for r in rows[1:])
    assert rows[-1]["compliance"] < rows[0]["compliance"]


@pytest.mark.parametrize("case", [0, 1, 2, 3])
def test_projected_oc_update_matches_reference_outputs(cuda, case):
    """With the Heaviside projection (beta 1, 4, 16, 32; the reference's default
    loop projects): the device projection and its derivative against the
    reference's _heaviside / _heaviside_deriv (1e-14 / 1e-13 relative), and the
    device OC step against the reference's own _oc_step_cupy with use_heaviside
    (new densities to 1e-8, the last bisection bracket; the same change)."""
    import os

    from gpu_fem.simp_loop import OCUpdater, cone_filter, heaviside

    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "oc_reference.npz"))
    rmin, volfrac, move, beta, eta = (float(v) for v in g[f"h{case}/params"])
    dims = (24, 12, 6)
    rho = cuda.as_tensor(g[f"h{case}/rho"], device="cuda")
    rho_f = cone_filter(rho, dims, rmin)
    p = heaviside(rho_f, beta, eta).cpu().numpy()
    dp = heaviside(rho_f, beta, eta, derivative=True).cpu().numpy()
    assert np.abs(p - g[f"h{case}/proj"]).max() <= 1e-14
    assert np.abs(dp - g[f"h{case}/dproj"]).max() <= 1e-13 * np.abs(g[f"h{case}/dproj"]).max()
    dc = cuda.as_tensor(g[f"h{case}/dc_phys"], device="cuda")
    rn, change, lm, steps = OCUpdater().projected(dims, rmin, rho, rho_f, dc, beta, eta, volfrac, move)
    np.testing.assert_allclose(rn.cpu().numpy(), g[f"h{case}/rn"], rtol=0, atol=1e-8)
    assert change == pytest.approx(float(g[f"h{case}/change"][0]), abs=1e-8)
    # and against the oracle's restatement: the same bisection
    H = osol.density_filter(*dims, rmin)
    rn_o, _, lm_o, steps_o = osimp.oc_update_projected(g[f"h{case}/rho"], H @ g[f"h{case}/rho"],
                                                       g[f"h{case}/dc_phys"], H, volfrac, move, beta, eta)
    assert steps == steps_o and abs(lm - lm_o) <= 1e-9


def test_projected_loop_doubles_beta_and_stays_guarded(cuda):
    """A 22-iteration loop with the projection: beta 1 through iteration 20, 2
    after it (the reference's continuation), every solve guarded, and while beta
    stays at 1 the projected volume at the target (the OC step enforces it for
    the beta it is given, so the first iteration after a doubling moves it)."""
    from gpu_fem.simp_loop import run_simp_guarded

    res = run_simp_guarded((24, 12, 6), max_iter=22, policy="plain", restart=100, seed=0, use_heaviside=True)
    rows = res["iterations"]
    assert res["all_guarded"] and all(r["true_rel_residual"] <= 1e-6 for r in rows)
    assert [r["beta"] for r in rows] == [1.0] * 20 + [2.0] * 2
    vols = [r["volume"] for r in rows]
    assert all(abs(v - 0.3) < 2e-3 for v in vols[1:20]), vols
    assert rows[19]["compliance"] < rows[0]["compliance"]
