"""The oracle's OC update (oracle/simp.py) pinned to the reference's own
``_oc_step_cupy`` (simp_gpu.py:212-294, no Heaviside projection) run on three
seeded cases through the numpy stand-in (tests/golden/make_oc_golden.py):
new densities to 1e-14, the same change.  Without the projection the
reference's volume sensitivities are ones, not H^T 1 (which moves the
densities by up to 0.035 on the first case)."""

import os

import numpy as np
import pytest

from oracle import simp as osimp
from oracle import solver as osol

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "oc_reference.npz")


@pytest.mark.parametrize("case", [0, 1, 2])
def test_oc_update_matches_reference(case):
    g = np.load(GOLDEN)
    rmin, volfrac, move = g[f"c{case}/params"]
    H = osol.density_filter(24, 12, 6, rmin)
    rn, change, lm, steps = osimp.oc_update(g[f"c{case}/rho"], g[f"c{case}/dc_phys"], H, volfrac, move)
    np.testing.assert_allclose(rn, g[f"c{case}/rn"], rtol=0, atol=1e-14)
    assert change == pytest.approx(float(g[f"c{case}/change"][0]), abs=1e-14)
    assert 1 <= steps <= 100 and lm > 0


@pytest.mark.parametrize("case", [0, 1, 2, 3])
def test_projected_oc_update_matches_reference(case):
    """With the Heaviside projection (beta 1, 4, 16, 32): the update, the change,
    the projection and its derivative of the reference's own functions."""
    g = np.load(GOLDEN)
    rmin, volfrac, move, beta, eta = g[f"h{case}/params"]
    H = osol.density_filter(24, 12, 6, rmin)
    rho = g[f"h{case}/rho"]
    rho_f = H @ rho
    np.testing.assert_allclose(osimp.heaviside(rho_f, beta, eta), g[f"h{case}/proj"], rtol=0, atol=1e-14)
    np.testing.assert_allclose(osimp.heaviside_deriv(rho_f, beta, eta), g[f"h{case}/dproj"], rtol=1e-13,
                               atol=1e-13)
    rn, change, lm, steps = osimp.oc_update_projected(rho, rho_f, g[f"h{case}/dc_phys"], H, volfrac, move, beta, eta)
    np.testing.assert_allclose(rn, g[f"h{case}/rn"], rtol=0, atol=1e-14)
    assert change == pytest.approx(float(g[f"h{case}/change"][0]), abs=1e-14)
    assert 1 <= steps <= 100
