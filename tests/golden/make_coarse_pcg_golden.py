"""Reference fixtures of the iterative coarsest solve (fixed-count Jacobi PCG).

    SIMPFEM_REFERENCE_ROOT=<reference checkout> python tests/golden/make_coarse_pcg_golden.py

GalerkinMatFreeGMG factors its coarsest operator when it has at most
``dense_chol_max`` free DOFs and otherwise solves it with ``_fixed_pcg_coarse``
(solver_v2.py:781-810): ``coarse_pcg_iters`` Jacobi-PCG iterations, at least
200 when the field is high-contrast (multigrid_v4.py:1302-1339, :1919-1927).
The 1M-element workload (coarsest 25 x 12 x 6, 6,825 free DOFs) takes that
path.  Here ``dense_chol_max=0`` selects it on small cantilevers -- 24 x 12 x 6
(preset cantilever_3d) and 40 x 20 x 10 -- with three levels, through the
reference's own unmodified objects run on the host by ``_refshim``:

* one preconditioner apply of a seeded vector for the damped-Jacobi and the
  Chebyshev V-cycle, on a high-contrast Bernoulli field (1e-12 floor, penal
  4.5: 200 coarse iterations) and a smooth field (80 iterations);
  each also with E multiplied by (1 + 1e-14 N(0, 1)), the reference's own
  round-off envelope;
* one FGMRES solve (restart 300, tol 1e-6) on the high-contrast field with the
  Jacobi V-cycle, and the same with E multiplied by (1 + 1e-14 N(0, 1)) to
  record the reference's own round-off envelope.

Output: coarse_pcg_reference.npz.
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import _refshim  # noqa: E402

STACKS = {"jacobi": dict(smoother_type="jacobi"), "cheb": dict()}


def _fields(n: int):
    rng = np.random.default_rng(17)
    solid = (rng.random(n) < 0.4).astype(np.float64)
    smooth = 0.3 + 0.7 * rng.random(n)
    return {"hi": 1e-12 + (1 - 1e-12) * solid ** 4.5, "lo": 1e-3 + (1 - 1e-3) * smooth ** 3.0}


def _build(spec, stack):
    bcg = _refshim.load("bc_generator")
    sv2 = _refshim.load("solver_v2")
    mg = _refshim.load("multigrid_v4")
    pss = _refshim.load("pub_simp_solver")
    bc = bcg.generate_bc(spec)
    free = bc.free_dofs.astype(np.int32)
    edof = pss._edof_table_3d(spec.nelx, spec.nely, spec.nelz).astype(np.int32)
    mf = sv2.MatrixFreeKff(edof, pss.KE_UNIT_3D, free, len(free), bc.ndof)
    gmg = mg.GalerkinMatFreeGMG(mf_op=mf, free=free, free_gpu=free, nelx=spec.nelx, nely=spec.nely,
                                nelz=spec.nelz, KE_UNIT=pss.KE_UNIT_3D, n_levels=3, fine_smoother="fp64",
                                dense_chol_max=0, **stack)
    return bc, free, mf, gmg


def main() -> None:
    ps = _refshim.load("problem_spec")
    presets = _refshim.load("presets")
    mg = _refshim.load("multigrid_v4")
    cases = {
        "cant24": presets.get_preset("cantilever_3d"),
        "cant40": ps.ProblemSpec(Lx=2.0, Ly=1.0, Lz=0.5, nelx=40, nely=20, nelz=10, volfrac=0.3,
                                 supports=[ps.EdgeSupport(edge="left", constraint="fixed")],
                                 loads=[ps.PointLoad(x=2.0, y=0.5, z=0.25, fy=-1.0)]),
    }
    out = {}
    for name, spec in cases.items():
        n = spec.nelx * spec.nely * spec.nelz
        fields = _fields(n)
        pre = f"{name}/"
        out[pre + "dims"] = np.array([spec.nelx, spec.nely, spec.nelz])
        for sname, stack in STACKS.items():
            for tag, E in fields.items():
                bc, free, mf, gmg = _build(spec, stack)
                gmg.setup(E)
                assert gmg._coarse_chol_mode == "iterative"
                rhs = np.random.default_rng(23).standard_normal(len(free))
                out[pre + f"rhs"] = rhs
                out[pre + f"E_{tag}"] = E
                out[pre + f"apply_{sname}_{tag}"] = gmg.apply(rhs)
                out[pre + f"lam_{sname}_{tag}"] = np.array(gmg.lambda_max_per_level)
                out[pre + f"high_{sname}_{tag}"] = np.array([int(gmg.is_high_contrast)])
                # the same apply with E perturbed by 1e-14 relative (the reference's own
                # round-off sensitivity: an unconverged fixed-count PCG amplifies it)
                _, _, _, gp = _build(spec, stack)
                gp.setup(E * (1.0 + 1e-14 * np.random.default_rng(5).standard_normal(E.size)))
                out[pre + f"apply_pert_{sname}_{tag}"] = gp.apply(rhs)
                print(name, sname, tag, "coarse n", gmg._K_gpu[2].shape[0], "high", gmg.is_high_contrast, flush=True)
        for variant in ("", "_pert"):
            bc, free, mf, gmg = _build(spec, STACKS["jacobi"])
            E = fields["hi"]
            if variant:
                E = E * (1.0 + 1e-14 * np.random.default_rng(5).standard_normal(E.size))
            gmg.setup(E)
            F = bc.F[free].astype(np.float64)
            hist = []
            x, it, conv = mg._cupy_fgmres(lambda v: mf.matvec(v, E), F, gmg.apply, tol=1e-6, maxiter=300,
                                          restart=300, history=hist)
            out[pre + f"solve{variant}_x"] = x
            out[pre + f"solve{variant}_hist"] = np.array(hist)
            out[pre + f"solve{variant}_info"] = np.array([it, int(conv), float(F @ x)])
            print(name, "solve", variant, it, conv, float(F @ x), flush=True)
    np.savez_compressed(os.path.join(HERE, "coarse_pcg_reference.npz"), **out)


if __name__ == "__main__":
    main()
