"""The CPU oracle (oracle/) pinned against the reference's own outputs
(tests/golden/reference_small.npz, made by tests/golden/make_golden.py)."""

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import solver as S
from oracle.gmg import GMG

CASES = {"cant24": (24, 12, 6), "odd13": (13, 7, 5), "bridge30": (30, 10, 5)}
STACKS = {
    "plain_jacobi": dict(smoother_type="jacobi"),
    "plain_cheb": dict(),
    "line_search": dict(coarse_correction_policy="residual_line_search"),
    "wcycle": dict(cycle_type="w"),
    "nb_line_search": dict(root_local_correction_mode="node_block_line_search"),
    "enrich": dict(coarse_correction_policy="residual_line_search", root_enrichment_mode="weighted_gap_second"),
    "enrich_void": dict(root_enrichment_mode="void_residual_second"),
    "level_fp32": dict(level_precisions=["fp64", "fp32", "fp32"]),
    "fine_fp32": dict(fine_smoother="fp32"),
    "canonical": dict(coarse_correction_policy="residual_line_search",
                      root_local_correction_mode="node_block_inner_fgmres",
                      root_local_correction_inner_steps=20, root_local_correction_inner_restart=20,
                      inner_krylov_steps=10, inner_krylov_restart=10),
}


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


def _op(ref, name):
    return S.Operator(*CASES[name], ref[f"{name}/free"])


def test_element_data(ref):
    assert np.abs(S.KE - ref["KE_UNIT_3D"]).max() <= 1e-15
    assert np.array_equal(S.edof_table(3, 2, 2), ref["edof_3x2x2"])
    for s in range(2):
        for t in range(2):
            for u in range(2):
                assert np.abs(S.local_prolongation(s, t, u) - ref[f"Ploc_{s}{t}{u}"]).max() == 0.0
    for key, (nf, nc) in {"Pscalar_644": ((6, 4, 4), (3, 2, 2)), "Pscalar_753": ((7, 5, 3), (3, 2, 1)),
                          "Pscalar_132": ((1, 3, 2), (1, 1, 1))}.items():
        assert np.abs(S.scalar_prolongation(*nf, *nc).toarray() - ref[key]).max() == 0.0
    assert np.abs(S.density_filter(6, 4, 3, 1.5).toarray() - ref["filter_643_r15"]).max() <= 1e-15


@pytest.mark.parametrize("name", ["cant24", "odd13"])
def test_cantilever_bc(ref, name):
    free, F = S.cantilever_bc(*CASES[name])
    assert np.array_equal(free, ref[f"{name}/free"])
    assert np.abs(F - ref[f"{name}/F"]).max() == 0.0


@pytest.mark.parametrize("name", list(CASES))
def test_operator_and_levels(ref, name):
    op = _op(ref, name)
    u = ref[f"{name}/u"]
    for tag in ("hi", "mid", "lo"):
        E = ref[f"{name}/E_{tag}"]
        assert _rel(op.matvec(u, E), ref[f"{name}/Ku_{tag}"]) <= 1e-14
        assert _rel(op.matvec(u.astype(np.float32), E.astype(np.float32)), ref[f"{name}/Ku32_{tag}"]) <= 1e-6
        assert _rel(op.diagonal(E), ref[f"{name}/diag_{tag}"]) <= 1e-15
    g = GMG(op, n_levels=3, fine_smoother="fp64")
    for lv in range(3):
        assert np.array_equal(g.free[lv], ref[f"{name}/free_l{lv}"])
    for lv in range(2):
        P = g.P[lv].tocoo()
        ij, v = ref[f"{name}/P_l{lv}_ij"], ref[f"{name}/P_l{lv}_v"]
        Pref = sp.coo_matrix((v, (ij[0], ij[1])), shape=P.shape).toarray()
        assert np.abs(P.toarray() - Pref).max() == 0.0
    for tag in ("hi", "mid", "lo"):
        g.setup(ref[f"{name}/E_{tag}"])
        np.testing.assert_allclose(g.lams, ref[f"{name}/lam_{tag}"], rtol=1e-11)
        assert abs(g.omega - ref[f"{name}/omega_{tag}"][0]) <= 1e-13 * g.omega
        a = ref[f"{name}/adapt_{tag}"]
        assert (int(g.high), g.deg_adapt, g.c_adapt) == (int(a[1]), int(a[2]), int(a[3]))
        if tag == "hi":
            for lv in (1, 2):
                ij, v = ref[f"{name}/K_l{lv}_ij"], ref[f"{name}/K_l{lv}_v"]
                Kref = sp.coo_matrix((v, (ij[0], ij[1])), shape=g.K[lv].shape).toarray()
                assert np.abs(g.K[lv].toarray() - Kref).max() <= 1e-13 * np.abs(Kref).max()


@pytest.mark.parametrize("name", ["cant24", "odd13"])
@pytest.mark.parametrize("stack", list(STACKS))
def test_preconditioner_apply(ref, name, stack):
    op = _op(ref, name)
    for tag in ("hi", "mid"):
        g = GMG(op, n_levels=3, **dict(dict(fine_smoother="fp64"), **STACKS[stack]))
        g.setup(ref[f"{name}/E_{tag}"])
        z = g.apply(ref[f"{name}/rhs"])
        tol = 1e-5 if stack in ("level_fp32", "fine_fp32") else 1e-10
        assert _rel(z, ref[f"{name}/apply_{stack}_{tag}"]) <= tol


def test_node_block_jacobi(ref):
    for name in CASES:
        op = _op(ref, name)
        E = ref[f"{name}/E_hi"]
        nb = S.NodeBlockJacobi(op)
        nb.update(E, op.diagonal(E))
        assert _rel(nb.apply(ref[f"{name}/rhs"]), ref[f"{name}/nbj_hi"]) <= 1e-12


@pytest.mark.parametrize("name", ["cant24", "odd13"])
def test_full_solve_plain(ref, name):
    op = _op(ref, name)
    F = ref[f"{name}/F"][ref[f"{name}/free"]]
    g = GMG(op, n_levels=3, fine_smoother="fp64")
    E = ref[f"{name}/E_hi"]
    g.setup(E)
    hist = []
    x, it, conv = S.fgmres(lambda v: op.matvec(v, E), F, g.apply, tol=1e-6, maxiter=300, restart=300, history=hist)
    info = ref[f"{name}/fgmres_plain_cheb_info"]
    assert (it, int(conv)) == (int(info[0]), int(info[1]))
    np.testing.assert_allclose(hist[:20], ref[f"{name}/fgmres_plain_cheb_hist"][:20], rtol=1e-9)
    assert abs(F @ x - info[2]) <= 1e-10 * abs(info[2])


def test_restart_rule_and_pcg(ref):
    name = "cant24"
    op = _op(ref, name)
    F = ref[f"{name}/F"][ref[f"{name}/free"]]
    g = GMG(op, n_levels=3, fine_smoother="fp64")
    E = ref[f"{name}/E_mid"]
    g.setup(E)
    hist = []
    x, it, conv = S.fgmres(lambda v: op.matvec(v, E), F, g.apply, tol=1e-9, maxiter=12, restart=5, history=hist)
    info = ref[f"{name}/fgmres_restart5_info"]
    assert (it, int(conv)) == (int(info[0]), int(info[1]))
    np.testing.assert_allclose(hist, ref[f"{name}/fgmres_restart5_hist"], rtol=1e-10)
    hist = []
    S.pcg(lambda v: op.matvec(v, E), F, g.apply, tol=1e-6, maxiter=200, history=hist)
    np.testing.assert_allclose(hist[:10], ref[f"{name}/pcg_plain_hist"][:10], rtol=1e-9)


def test_fused_matvec_restatement_matches_operator():
    """The oracle's FusedMatvec arithmetic (float32 casts of u, KE, E) equals the
    FP64 operator on an all-free mesh to float32 rounding, and its BF16 variant
    only by bfloat16 rounding."""
    from oracle import solver as s

    dims = (6, 4, 3)
    nd = 3 * 7 * 5 * 4
    rng = np.random.default_rng(0)
    u = rng.standard_normal(nd)
    E = rng.random(6 * 4 * 3) + 0.1
    a = s.Operator(*dims, np.arange(nd)).matvec(u, E)
    b = s.fused_matvec_full(*dims, u, E, s.ke_unit_3d(), "fp32")
    c = s.fused_matvec_full(*dims, u, E, s.ke_unit_3d(), "bf16")
    assert np.abs(a - b).max() <= 1e-6 * np.abs(a).max()
    assert 1e-5 < np.abs(a - c).max() / np.abs(a).max() < 3e-2
