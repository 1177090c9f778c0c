"""Golden OC updates from the reference's own ``_oc_step_cupy``.

Run from the repository root where the reference source tree is readable
(its root given by SIMPFEM_REFERENCE_ROOT):

    python tests/golden/make_oc_golden.py

``gpu_fem.simp_gpu._oc_step_cupy`` (simp_gpu.py:212-294) runs unmodified on the
host through the numpy-backed ``cupy`` stand-in (``_refshim.py``) without the
Heaviside projection, on seeded densities and sensitivities of a 24 x 12 x 6
grid with the reference's own cone filter (``_build_density_filter``, radius
1.5 and 2.5), and with the projection (beta 1, 4, 16, 32; eta 0.5) together with
the reference's ``_heaviside`` / ``_heaviside_deriv`` of the filtered field; the
inputs and outputs go to ``oc_reference.npz``.
"""

from __future__ import annotations

import os
import sys

import numpy as np
import scipy.sparse as sp

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import _refshim  # noqa: E402

DIMS = (24, 12, 6)


def main() -> None:
    sg = _refshim.load("simp_gpu")
    pss = _refshim.load("pub_simp_solver")
    n = int(np.prod(DIMS))
    out = {}
    for case, (seed, rmin, volfrac, move) in enumerate(((0, 1.5, 0.3, 0.2), (1, 2.5, 0.4, 0.1), (2, 1.5, 0.5, 0.2))):
        rng = np.random.default_rng(seed)
        rho = np.clip(volfrac + 0.2 * rng.standard_normal(n), 1e-3, 1.0)
        dc_phys = -np.exp(rng.standard_normal(n))
        H = sp.csr_matrix(pss._build_density_filter(DIMS[0], DIMS[1], rmin, DIMS[2]))
        rn, change = sg._oc_step_cupy(rho, H @ rho, dc_phys, 0.0, 0.5, volfrac, move, H, H.T.tocsr(), n, False)
        for k, v in (("rho", rho), ("dc_phys", dc_phys), ("rn", rn), ("change", np.array([change])),
                     ("params", np.array([rmin, volfrac, move]))):
            out[f"c{case}/{k}"] = np.asarray(v)
    # with the Heaviside projection (the reference's default, use_heaviside=True,
    # beta doubling from 1 to 32, eta = 0.5): the update of _oc_step_cupy, and the
    # projection and its derivative (pub_simp_solver.py:245-253) on the filtered field
    for case, (seed, rmin, volfrac, move, beta) in enumerate(((3, 1.5, 0.3, 0.2, 1.0), (4, 2.5, 0.4, 0.1, 4.0),
                                                              (5, 1.5, 0.5, 0.2, 16.0), (6, 1.5, 0.3, 0.2, 32.0))):
        rng = np.random.default_rng(seed)
        rho = np.clip(volfrac + 0.2 * rng.standard_normal(n), 1e-3, 1.0)
        dc_phys = -np.exp(rng.standard_normal(n))
        H = sp.csr_matrix(pss._build_density_filter(DIMS[0], DIMS[1], rmin, DIMS[2]))
        rho_f = H @ rho
        rn, change = sg._oc_step_cupy(rho, rho_f, dc_phys, beta, 0.5, volfrac, move, H, H.T.tocsr(), n, True)
        for k, v in (("rho", rho), ("dc_phys", dc_phys), ("rn", rn), ("change", np.array([change])),
                     ("params", np.array([rmin, volfrac, move, beta, 0.5])),
                     ("proj", pss._heaviside(rho_f, beta, 0.5)), ("dproj", pss._heaviside_deriv(rho_f, beta, 0.5))):
            out[f"h{case}/{k}"] = np.asarray(v)
    np.savez_compressed(os.path.join(HERE, "oc_reference.npz"), **out)
    print("wrote oc_reference.npz")


if __name__ == "__main__":
    main()
