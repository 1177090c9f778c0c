"""ctypes binding of libsimpfem.so (the C ABI declared in include/simpfem.h).

The library is built in-tree (``build_lib.py`` beside this package) and is the
only compute path: when it is missing or no CUDA device is present, every
operator raises instead of falling back to another implementation.
"""

from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsimpfem.so")

F64, F32, BF16 = 0, 1, 2
_STATUS = {1: "EINVAL", 2: "ECUDA", 5: "ENOTSETUP", 6: "ENONFINITE", 7: "ECALLBACK", 9: "EINTERNAL"}

_lock = threading.Lock()
_lib = None


class SimpfemError(RuntimeError):
    """A libsimpfem call returned a non-zero status."""

    def __init__(self, func: str, status: int, message: str):
        super().__init__(f"{func} failed ({_STATUS.get(status, status)}): {message}")
        self.status = status


class GmgOpts(ctypes.Structure):
    _fields_ = [
        ("n_levels", ctypes.c_int),
        ("coarse_smooth_iters", ctypes.c_int),
        ("fine_smoother", ctypes.c_int),
        ("fine_smoother_degree", ctypes.c_int),
        ("omega", ctypes.c_double),
        ("dense_chol_max", ctypes.c_int),
        ("coarse_pcg_iters", ctypes.c_int),
        ("smoother_type", ctypes.c_int),
        ("cheb_lower_frac", ctypes.c_double),
        ("level_prec", ctypes.c_int * 8),
        ("cycle_type", ctypes.c_int),
        ("coarse_correction_policy", ctypes.c_int),
        ("coarse_correction_acceptance_ratio", ctypes.c_double),
        ("coarse_correction_max_scale", ctypes.c_double),
        ("root_enrichment_mode", ctypes.c_int),
        ("root_enrichment_weight_floor", ctypes.c_double),
        ("root_enrichment_weight_power", ctypes.c_double),
        ("root_local_correction_mode", ctypes.c_int),
        ("root_local_correction_max_scale", ctypes.c_double),
        ("root_local_correction_inner_steps", ctypes.c_int),
        ("root_local_correction_inner_restart", ctypes.c_int),
        ("inner_krylov_steps", ctypes.c_int),
        ("inner_krylov_restart", ctypes.c_int),
        ("cycle_precision", ctypes.c_int),
        ("use_graphs", ctypes.c_int),
    ]


class GmgProps(ctypes.Structure):
    _fields_ = [
        ("n_levels", ctypes.c_int),
        ("n_free", ctypes.c_int64 * 8),
        ("dims", (ctypes.c_int * 3) * 8),
        ("lambda_max", ctypes.c_double * 8),
        ("omega_used", ctypes.c_double),
        ("contrast_ratio", ctypes.c_double),
        ("void_fraction", ctypes.c_double),
        ("is_high_contrast", ctypes.c_int),
        ("fine_degree_adapt", ctypes.c_int),
        ("coarse_iters_adapt", ctypes.c_int),
        ("level_prec", ctypes.c_int * 8),
        ("coarse_mode", ctypes.c_int),
        ("coarse_regularised", ctypes.c_int),
        ("lambda_reestimated", ctypes.c_int),
        ("nnz", ctypes.c_int64 * 8),
        ("cycle_graph_replays", ctypes.c_int64),
    ]


class PolicyOpts(ctypes.Structure):
    _fields_ = [
        ("penal", ctypes.c_double),
        ("binary", ctypes.c_int),
        ("tol", ctypes.c_double),
        ("restart", ctypes.c_int),
        ("maxiter", ctypes.c_int),
        ("probe_iters", ctypes.c_int),
        ("probe_r50", ctypes.c_int),
        ("baseline_rho_min", ctypes.c_double),
        ("n_raised", ctypes.c_int),
        ("raised_rho_mins", ctypes.c_double * 6),
        ("high_residual_threshold", ctypes.c_double),
        ("plateau_residual_threshold", ctypes.c_double),
        ("plateau_ratio_threshold", ctypes.c_double),
        ("reuse_probe", ctypes.c_int),
        ("proposer", ctypes.c_void_p),
        ("min_confidence", ctypes.c_double),
    ]


class PolicyResult(ctypes.Structure):
    _fields_ = [
        ("probe_r50", ctypes.c_double),
        ("probe_r100", ctypes.c_double),
        ("trigger", ctypes.c_int),
        ("raise_floor", ctypes.c_int),
        ("fallback", ctypes.c_int),
        ("proposal", ctypes.c_int),
        ("selected_rho_min", ctypes.c_double),
        ("converged", ctypes.c_int),
        ("reported_converged", ctypes.c_int),
        ("solve_iters", ctypes.c_int),
        ("probe_iters", ctypes.c_int),
        ("total_iters", ctypes.c_int),
        ("n_setups", ctypes.c_int),
        ("n_attempts", ctypes.c_int),
        ("reused_probe", ctypes.c_int),
        ("final_rel_residual", ctypes.c_double),
        ("attempted", ctypes.c_double * 8),
        ("seconds", ctypes.c_double),
    ]


class PolicyState(ctypes.Structure):
    _fields_ = [("g", ctypes.c_void_p), ("density", ctypes.c_void_p), ("b_free", ctypes.c_void_p),
                ("x_free", ctypes.c_void_p)]


_P = ctypes.c_void_p
_I = ctypes.c_int
_I64 = ctypes.c_int64
_D = ctypes.c_double
_SIGS = {
    "simpfem_last_error": (ctypes.c_char_p, []),
    "simpfem_version": (_I, []),
    "simpfem_launch_count": (_I64, []),
    "simpfem_device_alloc_count": (_I64, []),
    "simpfem_gmg_time_smoother_step": (_I, [_P, _I, _I, _P, _P]),
    "simpfem_gmg_time_operator": (_I, [_P, _I, _P, _P]),
    "simpfem_mesh_create": (_I, [_I, _I, _I, _P, _I64, _P, ctypes.POINTER(_P)]),
    "simpfem_mesh_destroy": (_I, [_P]),
    "simpfem_mesh_info": (_I, [_P, _P, _P, _P]),
    "simpfem_mesh_tune": (_I, [_P, _P]),
    "simpfem_matvec": (_I, [_P, _I, _P, _P, _P, _P]),
    "simpfem_matvec_full": (_I, [_P, _I, _P, _P, _P, _P]),
    "simpfem_extract_diagonal": (_I, [_P, _P, _P, _P]),
    "simpfem_node_blocks": (_I, [_P, _P, _P, _P, _P]),
    "simpfem_node_block_apply": (_I, [_P, _P, _P, _P, _P]),
    "simpfem_element_energy": (_I, [_P, _P, _P, _P]),
    "simpfem_true_residual": (_I, [_P, _P, _P, _P, _P, _P]),
    "simpfem_true_residual_noalloc": (_I, [_P, _P, _P, _P, _P, _P, _P]),
    "simpfem_gmg_default_opts": (None, [_P]),
    "simpfem_gmg_create": (_I, [_P, _P, ctypes.POINTER(_P)]),
    "simpfem_gmg_destroy": (_I, [_P]),
    "simpfem_gmg_setup": (_I, [_P, _P, _P, _P]),
    "simpfem_gmg_apply": (_I, [_P, _P, _P, _P]),
    "simpfem_gmg_cycle_trace": (_I, [_P, _P, _I, _P, _I, _P, _P, _P]),
    "simpfem_gmg_props_get": (_I, [_P, _P]),
    "simpfem_gmg_reset_lambda_cache": (_I, [_P]),
    "simpfem_gmg_fine_E": (_I, [_P, _P]),
    "simpfem_fgmres": (_I, [_P, _P, _P, _P, _D, _I, _I, _P, _I, _P, _P, _P, _P]),
    "simpfem_fgmres_checked": (_I, [_P, _P, _P, _P, _D, _I, _I, _P, _I, _P, _P, _P, _I, _I, _P, _P, _P, _P]),
    "simpfem_pcg": (_I, [_P, _P, _P, _P, _D, _I, _P, _I, _P, _P, _P, _P]),
    "simpfem_fgmres_op": (_I, [_I64, _P, _P, _P, _P, _P, _P, _D, _I, _I, _P, _I, _P, _P, _P, _P]),
    "simpfem_pcg_op": (_I, [_I64, _P, _P, _P, _P, _P, _P, _D, _I, _P, _I, _P, _P, _P, _P]),
    "simpfem_dense_cholesky_inverse": (_I, [_I, _P, _P, _P, _P]),
    "simpfem_policy_default_opts": (None, [_P]),
    "simpfem_policy_run": (_I, [_P, _P, _P, _P, _P, _P, _P]),
    "simpfem_policy_batch": (_I, [_P, _P, _I, _P, _P]),
    "simpfem_cone_filter": (_I, [_I, _I, _I, _D, _I, _P, _P, _P]),
    "simpfem_oc_work_bytes": (ctypes.c_size_t, []),
    "simpfem_oc_update": (_I, [_I64, _P, _P, _P, _P, _D, _D, _P, _P, ctypes.c_size_t, _P, _P, _P, _P]),
    "simpfem_heaviside": (_I, [_I64, _P, _D, _D, _P, _P, _P]),
    "simpfem_oc_projected_work_bytes": (ctypes.c_size_t, [_I64]),
    "simpfem_oc_update_projected": (_I, [_I, _I, _I, _D, _P, _P, _P, _D, _D, _D, _D, _P, _P, ctypes.c_size_t, _P, _P,
                                         _P, _P]),
    "simpfem_cnn_n_params": (_I, []),
    "simpfem_cnn_create": (_I, [_I, ctypes.POINTER(_P)]),
    "simpfem_cnn_destroy": (_I, [_P]),
    "simpfem_cnn_set_params": (_I, [_P, _P, _I]),
    "simpfem_cnn_get_params": (_I, [_P, _P, _I]),
    "simpfem_cnn_pool16": (_I, [_I, _I, _I, _P, _P, _P]),
    "simpfem_cnn_forward": (_I, [_P, _P, _P, _I, _P, _P]),
    "simpfem_cnn_loss_grad": (_I, [_P, _P, _P, _P, _I, _P, _P, _P]),
    "simpfem_cnn_adam_step": (_I, [_P, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, _P]),
}


def exported_symbols() -> list[str]:
    return sorted(_SIGS)


def load(path: str = LIB_PATH):
    """Load the shared library (no GPU needed) and bind every declared symbol."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(path):
            raise RuntimeError(
                f"libsimpfem.so not found at {path}; build it with "
                "python solver-admissibility-and-guarded-floor-selection_b200/build_lib.py"
            )
        lib = ctypes.CDLL(path)
        for name, (res, args) in _SIGS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def call(name: str, *args) -> None:
    lib = load()
    st = getattr(lib, name)(*args)
    if st != 0:
        msg = lib.simpfem_last_error()
        raise SimpfemError(name, st, msg.decode() if msg else "")


def lib():
    return load()


# ---------------------------------------------------------------- tensors
def torch_mod():
    import torch

    return torch


def require_cuda():
    torch = torch_mod()
    if not torch.cuda.is_available():
        raise RuntimeError("simpfem requires a CUDA device; no CPU fallback exists")
    load()
    return torch


def stream_ptr() -> int:
    torch = torch_mod()
    return int(torch.cuda.current_stream().cuda_stream)


def as_cuda(x, dtype):
    """torch CUDA tensor view of ``x`` (numpy / torch / sequence), contiguous."""
    torch = require_cuda()
    if isinstance(x, torch.Tensor):
        t = x
        if t.device.type != "cuda":
            t = t.to("cuda")
        if t.dtype != dtype:
            t = t.to(dtype)
        return t.contiguous()
    arr = np.asarray(x)
    return torch.as_tensor(arr, device="cuda").to(dtype).contiguous()


def ptr(t) -> int:
    return int(t.data_ptr())
