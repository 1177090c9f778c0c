"""Golden boundary conditions of the reference presets.

Run from the repository root where the reference source tree is readable
(its root given by SIMPFEM_REFERENCE_ROOT):

    python tests/golden/make_presets_golden.py

For each preset of the reference's ``gpu_fem.presets.ALL_PRESETS`` (presets.py)
with at most 600,000 elements, the reference's own ``generate_bc``
(bc_generator.py:381-447) runs on the host through the numpy stand-in
(``_refshim.py``); ``presets_bc.json`` keeps the grid, the domain, the volume
fraction, the number of free DOFs and SHA-256 digests of the free-DOF list and
of the non-zero load entries (indices and values), with the load's count and sum.
Larger 3-D presets keep their specification (grid, domain, volume fraction,
supports and loads as the reference's dataclasses print them).
"""

from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import _refshim  # noqa: E402

MAX_ELEMENTS = 600_000


def record(spec, bc) -> dict:
    free = np.asarray(bc.free_dofs, dtype=np.int64)
    F = np.asarray(bc.F, dtype=np.float64)
    nz = np.nonzero(F)[0]
    return {
        "grid": [int(spec.nelx), int(spec.nely), int(spec.nelz)],
        "domain": [float(spec.Lx), float(spec.Ly), float(spec.Lz)],
        "volfrac": float(spec.volfrac),
        "n_free": int(free.size),
        "free_sha256": hashlib.sha256(free.tobytes()).hexdigest(),
        "load_nnz": int(nz.size),
        "load_sum": float(F.sum()),
        "load_sha256": hashlib.sha256(nz.astype(np.int64).tobytes() + F[nz].tobytes()).hexdigest(),
    }


def main() -> None:
    presets = _refshim.load("presets")
    bcg = _refshim.load("bc_generator")
    out = {}
    for name in sorted(presets.ALL_PRESETS):
        spec = presets.ALL_PRESETS[name]
        if spec.nelz < 1:
            continue
        if spec.nelx * spec.nely * spec.nelz > MAX_ELEMENTS:
            # larger presets: the specification only (their BCs come from the same generator)
            out[name] = {"grid": [int(spec.nelx), int(spec.nely), int(spec.nelz)],
                         "domain": [float(spec.Lx), float(spec.Ly), float(spec.Lz)], "volfrac": float(spec.volfrac),
                         "supports": repr(spec.supports), "loads": repr(spec.loads)}
            continue
        out[name] = record(spec, bcg.generate_bc(spec))
    with open(os.path.join(HERE, "presets_bc.json"), "w") as fh:
        json.dump(out, fh, indent=0, sort_keys=True)
    print(f"wrote presets_bc.json: {len(out)} presets")


if __name__ == "__main__":
    main()
