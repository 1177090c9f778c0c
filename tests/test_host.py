"""Host-side checks that need no GPU: the C-ABI library loads and exports every
entry point include/simpfem.h declares; the Python layer's boundary inputs
(KE, edof, presets, BCs) match the reference; argument validation raises the
reference's errors; the policy's classification rule."""

import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    with open(os.path.join(ROOT, "include", "simpfem.h")) as f:
        text = f.read()
    return sorted(set(re.findall(r"\b(simpfem_[A-Za-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from gpu_fem import _lib

    lib = _lib.load()
    declared = _declared()
    assert declared, "no declarations found"
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) == set(_lib.exported_symbols())
    assert lib.simpfem_version() >= 10000


def test_element_data_and_bcs(ref):
    from gpu_fem import presets
    from gpu_fem.bc_generator import generate_bc
    from gpu_fem.pub_simp_solver import KE_UNIT_3D, _build_density_filter, _edof_table_3d

    assert np.abs(KE_UNIT_3D - ref["KE_UNIT_3D"]).max() <= 1e-15
    assert np.array_equal(_edof_table_3d(3, 2, 2), ref["edof_3x2x2"])
    assert np.abs(_build_density_filter(6, 4, 1.5, 3).toarray() - ref["filter_643_r15"]).max() <= 1e-15
    for name, spec in (("cant24", presets.get_preset("cantilever_3d")), ("bridge30", presets.get_preset("bridge_3d")),
                       ("odd13", presets.cantilever_spec(13, 7, 5))):
        bc = generate_bc(spec)
        assert np.array_equal(bc.free_dofs, ref[f"{name}/free"])
        assert np.abs(bc.F - ref[f"{name}/F"]).max() == 0.0
    with pytest.raises(KeyError):
        presets.get_preset("no_such_preset")


def test_grid_from_edof():
    from gpu_fem._native import grid_from_edof
    from gpu_fem.pub_simp_solver import _edof_table_3d

    assert grid_from_edof(_edof_table_3d(7, 3, 5)) == (7, 3, 5)
    bad = _edof_table_3d(4, 3, 2).copy()
    bad[5, 0] += 3
    with pytest.raises(ValueError):
        grid_from_edof(bad)


@pytest.mark.parametrize("kw,msg", [
    (dict(smoother_type="sor"), "smoother_type must be"),
    (dict(cycle_type="f"), "cycle_type must be"),
    (dict(coarse_correction_policy="x"), "coarse_correction_policy must be"),
    (dict(coarse_correction_acceptance_ratio=0.0), "coarse_correction_acceptance_ratio must be positive"),
    (dict(root_enrichment_mode="x"), "root_enrichment_mode must be"),
    (dict(root_enrichment_weight_floor=0.0), "root_enrichment_weight_floor must lie"),
    (dict(root_local_correction_mode="x"), "root_local_correction_mode must be"),
    (dict(root_local_correction_inner_steps=0), "root_local_correction_inner_steps must be positive"),
    (dict(inner_krylov_steps=-1), "inner_krylov_steps must be non-negative"),
    (dict(inner_krylov_restart=0), "inner_krylov_restart must be positive"),
])
def test_gmg_option_validation(kw, msg):
    from gpu_fem.multigrid_v4 import GalerkinMatFreeGMG

    with pytest.raises(ValueError, match=msg):
        GalerkinMatFreeGMG(mf_op=None, free=np.arange(3), free_gpu=None, nelx=2, nely=2, nelz=2, KE_UNIT=None, **kw)


def test_classify_rule():
    from gpu_fem.policy import _classify

    th = dict(high_residual_threshold=1e-2, plateau_residual_threshold=1e-4, plateau_ratio_threshold=0.6)
    assert _classify(2e-2, 1e-6, **th) == (True, "high_r50")
    assert _classify(5e-4, 4e-4, **th) == (True, "plateau")
    assert _classify(5e-4, 1e-4 * 0.5, **th) == (False, "keep")
    assert _classify(1e-3, 5e-4, **th) == (False, "keep")   # ratio 0.5 < 0.6


def test_ops_refuse_without_gpu():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from gpu_fem import _lib

    with pytest.raises(RuntimeError, match="no CPU fallback"):
        _lib.require_cuda()


def test_abi_rejects_bad_arguments_before_touching_the_device():
    """Entry points added for the SIMP loop and the cycle trace check their
    arguments first: status SIMPFEM_EINVAL (1) and a message, no CUDA call."""
    import ctypes

    from gpu_fem import _lib

    lib = _lib.load()
    fake = ctypes.c_void_p(16)  # never dereferenced: every call below fails validation first
    nv = ctypes.c_int()

    def status(name, *args):
        st = getattr(lib, name)(*args)
        return st, (lib.simpfem_last_error() or b"").decode()

    st, msg = status("simpfem_gmg_cycle_trace", None, None, 0, None, 0, ctypes.byref(nv), None, None)
    assert st == 1 and "cycle_trace" in msg
    st, msg = status("simpfem_gmg_cycle_trace", fake, fake, 5, None, 0, ctypes.byref(nv), fake, None)
    assert st == 1 and "cycle_type" in msg
    st, msg = status("simpfem_oc_update", 0, fake, fake, None, fake, 0.3, 0.2, fake, fake, 1 << 20, None, None,
                     None, None)
    assert st == 1 and "oc_update" in msg
    st, msg = status("simpfem_oc_update", 8, fake, fake, None, None, 0.3, 0.2, fake, fake, 1 << 20, None, None,
                     None, None)
    assert st == 1 and "oc_update" in msg  # the volume weights H^T 1 are required
    st, msg = status("simpfem_cone_filter", 4, 4, 4, 0.5, 0, fake, ctypes.c_void_p(32), None)
    assert st == 1 and "rmin" in msg
    st, msg = status("simpfem_cone_filter", 4, 4, 4, 1.5, 0, fake, fake, None)
    assert st == 1 and "cone_filter" in msg


def test_every_entry_point_rejects_null_arguments_before_touching_the_device():
    """Every status-returning entry point of include/simpfem.h checks its handles,
    pointers and sizes before any CUDA call: with null arguments it returns
    SIMPFEM_EINVAL (1) and a message naming the call; the destroy functions take
    a null handle as a no-op (SIMPFEM_OK)."""
    import ctypes

    from gpu_fem import _lib

    lib = _lib.load()
    out = ctypes.c_void_p()
    o = ctypes.byref(out)
    N = None
    cases = {
        "simpfem_gmg_time_smoother_step": ((N, 0, 0, N, N), "time_smoother_step"),
        "simpfem_gmg_time_operator": ((N, 0, N, N), "time_operator"),
        "simpfem_mesh_create": ((0, 0, 0, N, 0, N, o), "mesh_create"),
        "simpfem_mesh_info": ((N, N, N, N), "null mesh"),
        "simpfem_mesh_tune": ((N, N), "null mesh"),
        "simpfem_matvec": ((N, 0, N, N, N, N), "simpfem_matvec"),
        "simpfem_matvec_full": ((N, 0, N, N, N, N), "simpfem_matvec_full"),
        "simpfem_extract_diagonal": ((N, N, N, N), "extract_diagonal"),
        "simpfem_node_blocks": ((N, N, N, N, N), "node_blocks"),
        "simpfem_node_block_apply": ((N, N, N, N, N), "node_block_apply"),
        "simpfem_element_energy": ((N, N, N, N), "element_energy"),
        "simpfem_true_residual": ((N, N, N, N, N, N), "true_residual"),
        "simpfem_true_residual_noalloc": ((N, N, N, N, N, N, N), "true_residual_noalloc"),
        "simpfem_gmg_create": ((N, N, o), "gmg_create"),
        "simpfem_gmg_setup": ((N, N, N, N), "gmg_setup"),
        "simpfem_gmg_apply": ((N, N, N, N), "gmg_apply"),
        "simpfem_gmg_cycle_trace": ((N, N, 0, N, 0, N, N, N), "cycle_trace"),
        "simpfem_gmg_props_get": ((N, N), "props_get"),
        "simpfem_gmg_reset_lambda_cache": ((N,), "null gmg"),
        "simpfem_gmg_fine_E": ((N, N), "null argument"),
        "simpfem_fgmres": ((N, N, N, N, 1e-6, 1, 1, N, 0, N, N, N, N), "simpfem_fgmres"),
        "simpfem_fgmres_checked": ((N, N, N, N, 1e-6, 1, 1, N, 0, N, N, N, 0, 0, N, N, N, N), "simpfem_fgmres"),
        "simpfem_pcg": ((N, N, N, N, 1e-6, 1, N, 0, N, N, N, N), "simpfem_pcg"),
        "simpfem_fgmres_op": ((0, N, N, N, N, N, N, 1e-6, 1, 1, N, 0, N, N, N, N), "simpfem_fgmres_op"),
        "simpfem_pcg_op": ((0, N, N, N, N, N, N, 1e-6, 1, N, 0, N, N, N, N), "simpfem_pcg_op"),
        "simpfem_dense_cholesky_inverse": ((-1, N, N, N, N), "dense_cholesky_inverse"),
        "simpfem_policy_run": ((N, N, N, N, N, N, N), "simpfem_policy"),
        "simpfem_policy_batch": ((N, N, 0, N, N), "simpfem_policy"),
        "simpfem_cone_filter": ((0, 0, 0, 1.5, 0, N, N, N), "cone_filter"),
        "simpfem_oc_update": ((0, N, N, N, N, 0.3, 0.2, N, N, 0, N, N, N, N), "oc_update"),
        "simpfem_heaviside": ((0, N, 1.0, 0.5, N, N, N), "heaviside"),
        "simpfem_oc_update_projected": ((0, 0, 0, 1.5, N, N, N, 4.0, 0.5, 0.3, 0.2, N, N, 0, N, N, N, N),
                                        "oc_update_projected"),
        "simpfem_cnn_create": ((0, o), "cnn_create"),
        "simpfem_cnn_set_params": ((N, N, 0), "cnn_set_params"),
        "simpfem_cnn_get_params": ((N, N, 0), "cnn_get_params"),
        "simpfem_cnn_pool16": ((0, 0, 0, N, N, N), "cnn_pool16"),
        "simpfem_cnn_forward": ((N, N, N, 0, N, N), "cnn_forward"),
        "simpfem_cnn_loss_grad": ((N, N, N, N, 0, N, N, N), "cnn_loss_grad"),
        "simpfem_cnn_adam_step": ((N, 0.0, 0.0, 0.0, 0.0, N), "cnn_adam_step"),
    }
    for name, (args, word) in cases.items():
        st = getattr(lib, name)(*args)
        msg = (lib.simpfem_last_error() or b"").decode()
        assert st == 1 and word in msg, (name, st, msg)
    for name in ("simpfem_mesh_destroy", "simpfem_gmg_destroy", "simpfem_cnn_destroy"):
        assert getattr(lib, name)(None) == 0, name
    status_entries = {n for n, (res, _) in _lib._SIGS.items() if res is ctypes.c_int} - {
        "simpfem_version", "simpfem_cnn_n_params", "simpfem_mesh_destroy", "simpfem_gmg_destroy",
        "simpfem_cnn_destroy"}
    assert status_entries == set(cases), sorted(status_entries ^ set(cases))
