"""Stand-in for the reference's experiments/paper4/run_experiments_e1_e10.py.

The reference's phase-5 drivers (run_gmg_floor_detector_prospective.py:18-24 and
the same loader in the density-field, fixed-floor and rule-check drivers) load
this file by path, two directories above their own, and call its
``_build_components`` (run_experiments_e1_e10.py:128-179).  Here it hands them
this library's factory (``gpu_fem.paper4``): the same keyword arguments and the
same 8-tuple, over torch CUDA tensors, with every kernel from libsimpfem.so.
The other helpers of the reference runner that the drivers reach are exported
alongside, among them the host-side mesh data the direct-solve drivers
(run_direct_floor_atlas.py, run_direct_floor_conditioning.py,
compare_reduced_floor_perturbation.py) assemble their sparse matrices from:
``KE_UNIT_3D``, ``_edof_table_3d`` and ``_build_sparse_indices``.
"""

from __future__ import annotations

import os
import sys

_SRC = os.path.join(os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))), "src")
if _SRC not in sys.path:
    sys.path.insert(0, _SRC)

from gpu_fem.paper4 import (  # noqa: E402,F401
    CANONICAL_STACK,
    PLAIN_JACOBI_STACK,
    _build_components,
    _E_e,
    _E_e_heterogeneous,
    _fgmres,
    _pcg,
)
from gpu_fem.pub_simp_solver import KE_UNIT_3D, _build_sparse_indices, _edof_table_3d  # noqa: E402,F401
