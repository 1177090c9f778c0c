"""The cone density filter -- this package's _build_density_filter and the
oracle's restatement, which the device filter kernel is tested against -- pinned
to the reference's own _build_density_filter (tests/golden/filter_reference.npz,
make_filter_golden.py) at radii 1.2, 1.5, 2.5 and 3.5 on ragged grids."""

import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "filter_reference.npz")
_KEYS = sorted(np.load(GOLDEN).files)


@pytest.mark.parametrize("key", _KEYS)
def test_filters_match_reference(key):
    from gpu_fem.pub_simp_solver import _build_density_filter
    from oracle import solver as osol

    ref = np.load(GOLDEN)[key]
    dims, r = key.split("_r")
    nx, ny, nz = (int(v) for v in dims.split("x"))
    r = float(r)
    assert np.abs(_build_density_filter(nx, ny, r, nz).toarray() - ref).max() <= 1e-15
    assert np.abs(osol.density_filter(nx, ny, nz, r).toarray() - ref).max() <= 1e-15
