"""Every 3-D reference preset (tests/golden/presets_bc.json,
made by make_presets_golden.py from the reference's own presets and
generate_bc): the same names, grids, domains and volume fractions; up to
600,000 elements bit-identical free-DOF lists and load vectors from this
package's presets and generate_bc, above it the same supports and loads."""

import hashlib
import json
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "presets_bc.json")
with open(GOLDEN) as _fh:
    _REF = json.load(_fh)


@pytest.mark.parametrize("name", sorted(_REF))
def test_preset_boundary_conditions_match_reference(name):
    from gpu_fem import presets
    from gpu_fem.bc_generator import generate_bc

    ref = _REF[name]
    spec = presets.get_preset(name)
    assert [spec.nelx, spec.nely, spec.nelz] == ref["grid"]
    assert [spec.Lx, spec.Ly, spec.Lz] == ref["domain"] and spec.volfrac == ref["volfrac"]
    if "supports" in ref:  # above 600,000 elements: the specification only
        assert repr(spec.supports) == ref["supports"] and repr(spec.loads) == ref["loads"]
        return
    bc = generate_bc(spec)
    free = np.asarray(bc.free_dofs, dtype=np.int64)
    F = np.asarray(bc.F, dtype=np.float64)
    nz = np.nonzero(F)[0]
    assert free.size == ref["n_free"]
    assert hashlib.sha256(free.tobytes()).hexdigest() == ref["free_sha256"]
    assert nz.size == ref["load_nnz"] and float(F.sum()) == pytest.approx(ref["load_sum"], abs=1e-12)
    assert hashlib.sha256(nz.astype(np.int64).tobytes() + F[nz].tobytes()).hexdigest() == ref["load_sha256"]


def test_every_small_reference_preset_exists_here():
    from gpu_fem import presets

    assert set(_REF) <= set(presets.list_presets())


@pytest.mark.parametrize("name", ["cantilever_3d", "cantilever_gpu_medium", "cantilever_gpu_large",
                                  "cantilever_gpu_xlarge"])
def test_oracle_cantilever_bc_matches_reference(name):
    """The oracle's closed-form cantilever BCs (used by the oracle-side tests)
    against the reference's generate_bc digests."""
    from oracle import solver as osol

    ref = _REF[name]
    free, F = osol.cantilever_bc(*ref["grid"], *ref["domain"])
    free = np.asarray(free, dtype=np.int64)
    nz = np.nonzero(F)[0]
    assert free.size == ref["n_free"]
    assert hashlib.sha256(free.tobytes()).hexdigest() == ref["free_sha256"]
    assert hashlib.sha256(nz.astype(np.int64).tobytes() + F[nz].tobytes()).hexdigest() == ref["load_sha256"]
