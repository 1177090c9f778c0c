"""Golden cone density filters from the reference's own ``_build_density_filter``.

Run from the repository root where the reference source tree is readable
(its root given by SIMPFEM_REFERENCE_ROOT):

    python tests/golden/make_filter_golden.py

pub_simp_solver.py:90-117 runs on the host through the numpy stand-in
(``_refshim.py``) for radii 1.2, 2.5 and 3.5 on small ragged grids;
``filter_reference.npz`` keeps each filter as a dense matrix.
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import _refshim  # noqa: E402

CASES = (((6, 4, 3), 1.2), ((5, 7, 3), 2.5), ((7, 5, 4), 3.5), ((9, 3, 2), 1.5))


def main() -> None:
    pss = _refshim.load("pub_simp_solver")
    out = {}
    for (nx, ny, nz), r in CASES:
        out[f"{nx}x{ny}x{nz}_r{r}"] = np.asarray(pss._build_density_filter(nx, ny, r, nz).toarray())
    np.savez_compressed(os.path.join(HERE, "filter_reference.npz"), **out)
    print("wrote filter_reference.npz")


if __name__ == "__main__":
    main()
