"""Galerkin matrix-free GMG and FGMRES with the reference's call signatures.

``GalerkinMatFreeGMG`` (gpu_fem/multigrid_v4.py:537-2024) keeps the reference's
constructor keywords, their ValueError validation (:600-700), ``setup`` /
``apply`` / ``apply_fine_operator`` / ``probe_quality`` / ``estimate_kappa_eff``
and the read-only properties (:772-837).  Everything below the Python surface --
hierarchy construction, the lambda_max cache, contrast adaptation, smoothers,
V/W-cycle, safeguarded corrections, inner Krylov wrappers, the coarsest
Cholesky -- runs in libsimpfem on the device.

``_cupy_fgmres`` (:416-534) dispatches to the library's device-resident FGMRES
when the preconditioner is a ``GalerkinMatFreeGMG.apply`` and the operator is
that hierarchy's fine operator (checked by applying both to one probe vector);
any other operator / preconditioner pair runs on the library's device Krylov
core (``simpfem_fgmres_op``) with the two callables applied through callbacks.
"""

from __future__ import annotations

import ctypes
import math
import os
from dataclasses import asdict, dataclass, field
from typing import Callable, Optional

import numpy as np

from . import _krylov, _lib
from ._native import to_numpy
from .solver_v2 import MatrixFreeKff, _native_gmg

_PREC = {"fp64": _lib.F64, "fp32": _lib.F32, "bf16": _lib.BF16}
# int check(void* ctx, int iters, const double* history, int history_len, double true_rel_residual)
_CHECK_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                             ctypes.c_int, ctypes.c_double)
_PREC_NAME = {v: k for k, v in _PREC.items()}
_ENRICH = {"none": 0, "weighted_residual_second": 1, "weighted_gap_second": 2, "void_residual_second": 3,
           "void_gap_second": 4}
_ROOT = {"none": 0, "node_block_line_search": 1, "node_block_inner_fgmres": 2}


@dataclass
class MultigridLevelStats:
    level: int
    kind: str
    n_elem: int
    n_free: int
    nnz: int
    estimated_vram_bytes: int


_CC_NOTES = ("", "degenerate_correction", "rejected_correction", "nonpositive_correction_scale",
             "clipped_correction_scale")
_RL_NOTES = ("", "degenerate_root_local_correction", "rejected_root_local_inner_fgmres", "root_local_inner_fgmres",
             "nonpositive_root_local_scale", "clipped_root_local_scale")
_COARSE_MODES = ("none", "dense", "iterative")


@dataclass
class MultigridCycleVisit:
    """One level visit of a traced cycle (multigrid_v4.py:39-78)."""

    visit_id: int
    level: int
    cycle_type: str
    is_coarsest: bool
    n_coarse_corrections: int
    rhs_norm: float
    jacobi_action_norm: float
    presmooth_solution_norm: float
    presmooth_residual_norm: float
    presmooth_residual_ratio: float
    restricted_rhs_norm: float
    restricted_rhs_ratio: float
    projector_norm: float
    coarse_space_gap_norm: float
    coarse_space_gap_ratio: float
    coarse_correction_norm: float
    prolongated_correction_norm: float
    correction_alignment: float
    corrected_residual_norm: float
    corrected_residual_vs_presmooth: float
    correction_scale_raw: Optional[float] = None
    correction_scale_applied: float = 1.0
    second_restricted_rhs_norm: Optional[float] = None
    second_coarse_correction_norm: Optional[float] = None
    second_prolongated_correction_norm: Optional[float] = None
    second_correction_alignment: Optional[float] = None
    second_correction_scale_raw: Optional[float] = None
    second_correction_scale_applied: Optional[float] = None
    second_corrected_residual_norm: Optional[float] = None
    second_corrected_residual_vs_corrected: Optional[float] = None
    postsmooth_solution_norm: float = 0.0
    postsmooth_residual_norm: float = 0.0
    postsmooth_residual_ratio: float = 0.0
    coarsest_mode: str = ""
    notes: str = ""

    def to_dict(self) -> dict:
        return asdict(self)


@dataclass
class MultigridCycleTrace:
    """A traced cycle and the root-local correction after it (multigrid_v4.py:80-113)."""

    cycle_type: str
    rhs_norm: float
    jacobi_action_norm: float
    output_norm: float
    z_over_jacobi: float
    rz: float
    pd: bool
    output_residual_norm: float
    output_residual_ratio: float
    contrast_ratio: float
    is_high_contrast: bool
    fine_degree_adapt: int
    coarse_iters_adapt: int
    coarse_correction_policy: str
    coarse_correction_acceptance_ratio: float
    coarse_correction_max_scale: float
    root_enrichment_mode: str
    root_enrichment_weight_floor: float
    root_enrichment_weight_power: float
    root_local_correction_mode: str
    root_local_correction_inner_steps: int
    root_local_correction_inner_restart: int
    root_local_correction_raw_scale: Optional[float]
    root_local_correction_applied_scale: float
    root_local_correction_residual_ratio: float
    inner_krylov_steps: int
    inner_krylov_restart: int
    visits: list = field(default_factory=list)

    def to_dict(self) -> dict:
        return asdict(self)


def _safe_ratio(num: float, den: float) -> float:
    """multigrid_v4.py:840-843."""
    if abs(den) <= 1e-300:
        return 0.0 if abs(num) <= 1e-300 else float("inf")
    return float(num / den)


def _opt(v) -> Optional[float]:
    return None if v is None or math.isnan(v) else float(v)


def trace_from_records(visits, summary, cycle_type: str, options: dict) -> MultigridCycleTrace:
    """Build the trace from the library's records (layout in include/simpfem.h,
    simpfem_gmg_cycle_trace): ratios, notes and None fields follow
    multigrid_v4.py:1362-1728.  ``options`` holds the hierarchy's constructor
    settings echoed by the trace (coarse_correction_policy, ...)."""
    out = []
    for r in np.asarray(visits, dtype=np.float64).reshape(-1, 32):
        coarsest = bool(r[2])
        rn, presn, crn1 = float(r[4]), float(r[7]), float(r[17])
        second = not coarsest and int(r[3]) == 2
        notes = []
        if not coarsest:
            notes.append(_CC_NOTES[int(r[27])])
            if second:
                notes.append(_CC_NOTES[int(r[28])])
            if r[29]:
                notes.append(f"root_enrichment:{options['root_enrichment_mode']}")
            if r[30]:
                notes.append("extra_fine_postsmooth")
        out.append(MultigridCycleVisit(
            visit_id=int(r[0]), level=int(r[1]), cycle_type=cycle_type, is_coarsest=coarsest,
            n_coarse_corrections=int(r[3]), rhs_norm=rn, jacobi_action_norm=float(r[5]),
            presmooth_solution_norm=float(r[6]), presmooth_residual_norm=presn,
            presmooth_residual_ratio=1.0 if coarsest else _safe_ratio(presn, rn),
            restricted_rhs_norm=float(r[8]), restricted_rhs_ratio=0.0 if coarsest else _safe_ratio(r[8], presn),
            projector_norm=float(r[9]), coarse_space_gap_norm=float(r[10]),
            coarse_space_gap_ratio=0.0 if coarsest else _safe_ratio(r[10], presn),
            coarse_correction_norm=float(r[11]), prolongated_correction_norm=float(r[12]),
            correction_alignment=float(r[13]), corrected_residual_norm=float(r[16]),
            corrected_residual_vs_presmooth=_safe_ratio(r[16], presn),
            correction_scale_raw=_opt(r[14]), correction_scale_applied=float(r[15]),
            second_restricted_rhs_norm=_opt(r[18]) if second else None,
            second_coarse_correction_norm=_opt(r[19]) if second else None,
            second_prolongated_correction_norm=_opt(r[20]) if second else None,
            second_correction_alignment=_opt(r[21]) if second else None,
            second_correction_scale_raw=_opt(r[22]) if second else None,
            second_correction_scale_applied=_opt(r[23]) if second else None,
            second_corrected_residual_norm=_opt(r[24]) if second else None,
            second_corrected_residual_vs_corrected=_safe_ratio(r[24], crn1) if second else None,
            postsmooth_solution_norm=float(r[25]), postsmooth_residual_norm=float(r[26]),
            postsmooth_residual_ratio=_safe_ratio(r[26], rn),
            coarsest_mode=_COARSE_MODES[int(r[31])] if coarsest else "",
            notes="|".join(n for n in notes if n),
        ))
    s = np.asarray(summary, dtype=np.float64)
    local_note = _RL_NOTES[int(s[8])]
    if local_note:
        root = next((v for v in out if v.level == 0 and not v.is_coarsest), None)
        if root is not None:
            root.notes = "|".join(n for n in (root.notes, local_note) if n)
    rz = float(s[3])
    return MultigridCycleTrace(
        cycle_type=cycle_type, rhs_norm=float(s[0]), jacobi_action_norm=float(s[1]), output_norm=float(s[2]),
        z_over_jacobi=_safe_ratio(s[2], s[1]), rz=rz, pd=bool(rz > 0.0), output_residual_norm=float(s[4]),
        output_residual_ratio=_safe_ratio(s[4], s[0]), contrast_ratio=float(s[9]), is_high_contrast=bool(s[10]),
        fine_degree_adapt=int(s[11]), coarse_iters_adapt=int(s[12]),
        coarse_correction_policy=options["coarse_correction_policy"],
        coarse_correction_acceptance_ratio=float(options["coarse_correction_acceptance_ratio"]),
        coarse_correction_max_scale=float(options["coarse_correction_max_scale"]),
        root_enrichment_mode=options["root_enrichment_mode"],
        root_enrichment_weight_floor=float(options["root_enrichment_weight_floor"]),
        root_enrichment_weight_power=float(options["root_enrichment_weight_power"]),
        root_local_correction_mode=options["root_local_correction_mode"],
        root_local_correction_inner_steps=int(options["root_local_correction_inner_steps"]),
        root_local_correction_inner_restart=int(options["root_local_correction_inner_restart"]),
        root_local_correction_raw_scale=_opt(s[6]), root_local_correction_applied_scale=float(s[7]),
        root_local_correction_residual_ratio=_safe_ratio(s[4], s[5]),
        inner_krylov_steps=int(options["inner_krylov_steps"]),
        inner_krylov_restart=int(options["inner_krylov_restart"]),
        visits=out,
    )


class GalerkinMatFreeGMG:
    def __init__(
        self,
        *,
        mf_op: MatrixFreeKff,
        free,
        free_gpu,
        nelx: int,
        nely: int,
        nelz: int,
        KE_UNIT,
        n_levels: int = 4,
        coarse_smooth_iters: int = 2,
        fine_smoother: str = "fp32",
        fine_smoother_degree: int = 2,
        omega: float = 0.5,
        fused_op=None,
        dense_chol_max: int = 5000,
        coarse_pcg_iters: int = 80,
        smoother_type: str = "chebyshev",
        cheb_lower_frac: float = 1.0 / 30.0,
        level_precisions: Optional[list] = None,
        cycle_type: str = "v",
        coarse_correction_policy: str = "none",
        coarse_correction_acceptance_ratio: float = 1.0,
        coarse_correction_max_scale: float = 1.0,
        root_enrichment_mode: str = "none",
        root_enrichment_weight_floor: float = 1e-6,
        root_enrichment_weight_power: float = 0.5,
        root_local_correction_mode: str = "none",
        root_local_correction_max_scale: float = 1.0,
        root_local_correction_inner_steps: int = 10,
        root_local_correction_inner_restart: Optional[int] = None,
        inner_krylov_steps: int = 0,
        inner_krylov_restart: Optional[int] = None,
        cycle_precision: str = "fp64",
        use_graphs: Optional[bool] = None,
    ) -> None:
        if smoother_type not in {"chebyshev", "jacobi"}:
            raise ValueError(f"smoother_type must be 'chebyshev' or 'jacobi'; got {smoother_type!r}")
        if cycle_type not in {"v", "w"}:
            raise ValueError(f"cycle_type must be 'v' or 'w'; got {cycle_type!r}")
        if coarse_correction_policy not in {"none", "residual_line_search"}:
            raise ValueError(
                "coarse_correction_policy must be 'none' or 'residual_line_search'; "
                f"got {coarse_correction_policy!r}"
            )
        if coarse_correction_acceptance_ratio <= 0.0:
            raise ValueError(
                "coarse_correction_acceptance_ratio must be positive; "
                f"got {coarse_correction_acceptance_ratio!r}"
            )
        if coarse_correction_max_scale <= 0.0:
            raise ValueError(f"coarse_correction_max_scale must be positive; got {coarse_correction_max_scale!r}")
        if root_enrichment_mode not in _ENRICH:
            raise ValueError(
                "root_enrichment_mode must be 'none', 'weighted_residual_second', "
                "'weighted_gap_second', 'void_residual_second', or 'void_gap_second'; "
                f"got {root_enrichment_mode!r}"
            )
        if not (0.0 < root_enrichment_weight_floor <= 1.0):
            raise ValueError(
                f"root_enrichment_weight_floor must lie in (0, 1]; got {root_enrichment_weight_floor!r}"
            )
        if root_enrichment_weight_power <= 0.0:
            raise ValueError(f"root_enrichment_weight_power must be positive; got {root_enrichment_weight_power!r}")
        if root_local_correction_mode not in _ROOT:
            raise ValueError(
                "root_local_correction_mode must be 'none', 'node_block_line_search', "
                "or 'node_block_inner_fgmres'; "
                f"got {root_local_correction_mode!r}"
            )
        if root_local_correction_max_scale <= 0.0:
            raise ValueError(
                f"root_local_correction_max_scale must be positive; got {root_local_correction_max_scale!r}"
            )
        if root_local_correction_inner_steps <= 0:
            raise ValueError(
                f"root_local_correction_inner_steps must be positive; got {root_local_correction_inner_steps!r}"
            )
        if root_local_correction_inner_restart is not None and root_local_correction_inner_restart <= 0:
            raise ValueError(
                "root_local_correction_inner_restart must be positive when provided; "
                f"got {root_local_correction_inner_restart!r}"
            )
        if inner_krylov_steps < 0:
            raise ValueError(f"inner_krylov_steps must be non-negative; got {inner_krylov_steps!r}")
        if inner_krylov_restart is not None and inner_krylov_restart <= 0:
            raise ValueError(f"inner_krylov_restart must be positive when provided; got {inner_krylov_restart!r}")
        if fine_smoother not in _PREC:
            raise ValueError(f"Unsupported fine smoother '{fine_smoother}'")
        if cycle_precision not in {"fp64", "fp32"}:
            raise ValueError(f"cycle_precision must be 'fp64' or 'fp32'; got {cycle_precision!r}")

        self._mf_op = mf_op
        self._free = np.asarray(to_numpy(free), dtype=np.int32)
        self._free_gpu = free_gpu
        self._fine_smoother = fine_smoother
        self._fine_degree = max(1, int(fine_smoother_degree))
        self._coarse_smooth_iters = max(1, int(coarse_smooth_iters))
        self._omega_max = float(omega)
        self._fused_op = fused_op
        self._n_levels = max(1, int(n_levels))
        self._smoother_type = smoother_type
        self._cycle_type = cycle_type
        self._coarse_correction_policy = coarse_correction_policy
        self._coarse_correction_acceptance_ratio = float(coarse_correction_acceptance_ratio)
        self._coarse_correction_max_scale = float(coarse_correction_max_scale)
        self._root_enrichment_mode = root_enrichment_mode
        self._root_enrichment_weight_floor = float(root_enrichment_weight_floor)
        self._root_enrichment_weight_power = float(root_enrichment_weight_power)
        self._root_local_correction_mode = root_local_correction_mode
        self._root_local_correction_max_scale = float(root_local_correction_max_scale)
        self._root_local_correction_inner_steps = int(root_local_correction_inner_steps)
        self._root_local_correction_inner_restart = (
            int(root_local_correction_inner_restart) if root_local_correction_inner_restart is not None
            else max(1, self._root_local_correction_inner_steps)
        )
        self._inner_krylov_steps = int(inner_krylov_steps)
        self._inner_krylov_restart = (
            int(inner_krylov_restart) if inner_krylov_restart is not None else max(1, self._inner_krylov_steps)
        )
        self._cycle_precision = cycle_precision
        self._level_prec_given = list(level_precisions) if level_precisions is not None else None
        self._kappa_eff = float("nan")
        self._is_setup = False

        o = _lib.GmgOpts()
        _lib.lib().simpfem_gmg_default_opts(ctypes.byref(o))
        o.n_levels = self._n_levels
        o.coarse_smooth_iters = int(coarse_smooth_iters)
        o.fine_smoother = _PREC[fine_smoother]
        o.fine_smoother_degree = int(fine_smoother_degree)
        o.omega = float(omega)
        o.dense_chol_max = int(dense_chol_max)
        o.coarse_pcg_iters = int(coarse_pcg_iters)
        o.smoother_type = 0 if smoother_type == "chebyshev" else 1
        o.cheb_lower_frac = float(cheb_lower_frac)
        for i in range(8):
            o.level_prec[i] = -1
        if self._level_prec_given is not None:
            for i, p in enumerate(self._level_prec_given[:8]):
                if p not in _PREC:
                    raise ValueError(f"unknown level precision {p!r}")
                o.level_prec[i] = _PREC[p]
            for i in range(len(self._level_prec_given), self._n_levels):
                o.level_prec[i] = _lib.F64
        o.cycle_type = 0 if cycle_type == "v" else 1
        o.coarse_correction_policy = 0 if coarse_correction_policy == "none" else 1
        o.coarse_correction_acceptance_ratio = float(coarse_correction_acceptance_ratio)
        o.coarse_correction_max_scale = float(coarse_correction_max_scale)
        o.root_enrichment_mode = _ENRICH[root_enrichment_mode]
        o.root_enrichment_weight_floor = float(root_enrichment_weight_floor)
        o.root_enrichment_weight_power = float(root_enrichment_weight_power)
        o.root_local_correction_mode = _ROOT[root_local_correction_mode]
        o.root_local_correction_max_scale = float(root_local_correction_max_scale)
        o.root_local_correction_inner_steps = int(root_local_correction_inner_steps)
        o.root_local_correction_inner_restart = self._root_local_correction_inner_restart
        o.inner_krylov_steps = int(inner_krylov_steps)
        o.inner_krylov_restart = self._inner_krylov_restart
        o.cycle_precision = _lib.F32 if cycle_precision == "fp32" else _lib.F64
        # the cycle body captured once per setup as a CUDA graph and replayed;
        # off unless asked for (use_graphs=True or SIMPFEM_USE_GRAPHS=1): with
        # several states in flight the per-setup capture costs more than the
        # replays save at these cycle counts
        if use_graphs is None:
            use_graphs = os.environ.get("SIMPFEM_USE_GRAPHS", "0") == "1"
        o.use_graphs = 1 if use_graphs else 0
        self._opts = o
        h = ctypes.c_void_p()
        _lib.call("simpfem_gmg_create", mf_op.mesh.handle, ctypes.byref(o), ctypes.byref(h))
        self._h = h
        self._E_ref = None
        self._props = None

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib._lib is not None:
            try:
                _lib._lib.simpfem_gmg_destroy(h)
            except Exception:  # pragma: no cover
                pass

    # ------------------------------------------------------------ properties
    def _get_props(self) -> _lib.GmgProps:
        p = _lib.GmgProps()
        _lib.call("simpfem_gmg_props_get", self._h, ctypes.byref(p))
        return p

    @property
    def level_stats(self) -> list:
        p = self._get_props()
        out = []
        for lv in range(p.n_levels):
            nx, ny, nz = p.dims[lv][0], p.dims[lv][1], p.dims[lv][2]
            kind = f"fine-matrixfree-{self._fine_smoother}" if lv == 0 else (
                "level1-galerkin" if lv == 1 else "galerkin-triple-product")
            out.append(MultigridLevelStats(lv, kind, nx * ny * nz, int(p.n_free[lv]), 0, 0))
        return out

    @property
    def omega_used(self) -> float:
        return float(self._get_props().omega_used)

    @property
    def lambda_max_estimate(self) -> float:
        return float(self._get_props().lambda_max[0])

    @property
    def lambda_max_per_level(self) -> list:
        p = self._get_props()
        return [float(p.lambda_max[i]) for i in range(p.n_levels)]

    @property
    def level_precisions(self) -> list:
        p = self._get_props()
        if p.level_prec[0] < 0:
            return []
        return [_PREC_NAME[p.level_prec[i]] for i in range(p.n_levels)]

    @property
    def contrast_ratio(self) -> float:
        return float(self._get_props().contrast_ratio)

    @property
    def is_high_contrast(self) -> bool:
        return bool(self._get_props().is_high_contrast)

    @property
    def kappa_eff(self) -> float:
        return self._kappa_eff

    @property
    def coarse_mode(self) -> str:
        return {0: "none", 1: "dense", 2: "iterative"}[self._get_props().coarse_mode]

    @property
    def adaptive_params(self) -> dict:
        p = self._get_props()
        return {
            "contrast_ratio": float(p.contrast_ratio),
            "is_high_contrast": bool(p.is_high_contrast),
            "fine_degree_base": self._fine_degree,
            "fine_degree_adapt": int(p.fine_degree_adapt),
            "coarse_iters_base": self._coarse_smooth_iters,
            "coarse_iters_adapt": int(p.coarse_iters_adapt),
            "coarse_correction_policy": self._coarse_correction_policy,
            "coarse_correction_acceptance_ratio": self._coarse_correction_acceptance_ratio,
            "coarse_correction_max_scale": self._coarse_correction_max_scale,
            "root_enrichment_mode": self._root_enrichment_mode,
            "root_enrichment_weight_floor": self._root_enrichment_weight_floor,
            "root_enrichment_weight_power": self._root_enrichment_weight_power,
            "root_local_correction_mode": self._root_local_correction_mode,
            "root_local_correction_max_scale": self._root_local_correction_max_scale,
            "root_local_correction_inner_steps": self._root_local_correction_inner_steps,
            "root_local_correction_inner_restart": self._root_local_correction_inner_restart,
            "inner_krylov_steps": self._inner_krylov_steps,
            "inner_krylov_restart": self._inner_krylov_restart,
        }

    def uses_bf16_smoother(self) -> bool:
        return self._fine_smoother == "bf16"

    def supports_spd_outer(self) -> bool:
        return (
            self._fine_smoother in {"fp64", "fp32"}
            and self._coarse_correction_policy == "none"
            and self._root_enrichment_mode == "none"
            and self._root_local_correction_mode == "none"
            and self._inner_krylov_steps == 0
        )

    # ------------------------------------------------------------ compute
    def setup(self, E_e_gpu, fine_diag=None) -> None:
        torch = _lib.require_cuda()
        E = _lib.as_cuda(E_e_gpu, torch.float64)
        d = _lib.as_cuda(fine_diag, torch.float64) if fine_diag is not None else None
        _lib.call("simpfem_gmg_setup", self._h, _lib.ptr(E), _lib.ptr(d) if d is not None else None,
                  _lib.stream_ptr())
        self._E_ref = E
        self._is_setup = True

    def reset_lambda_cache(self) -> None:
        """Forget the cached lambda_max estimates: the next setup re-estimates them."""
        _lib.call("simpfem_gmg_reset_lambda_cache", self._h)

    def apply(self, rhs):
        if not self._is_setup:
            raise RuntimeError("GalerkinMatFreeGMG.setup() must be called before apply().")
        if self._fine_smoother == "bf16" and self._fused_op is None:
            raise RuntimeError("BF16 fine smoothing requires enable_fused_cuda=True so the WMMA path exists.")
        torch = _lib.require_cuda()
        r = _lib.as_cuda(rhs, torch.float64)
        z = torch.empty_like(r)
        _lib.call("simpfem_gmg_apply", self._h, _lib.ptr(r), _lib.ptr(z), _lib.stream_ptr())
        return z

    def apply_fine_operator(self, v):
        return self._mf_op.matvec(v, self._E_ref)

    def apply_preconditioned_operator(self, v):
        return self.apply(self.apply_fine_operator(v))

    def probe_quality(self, rhs) -> dict:
        torch = _lib.require_cuda()
        rhs = _lib.as_cuda(rhs, torch.float64)
        z = self.apply(rhs)
        d = self._mf_op.extract_diagonal(self._E_ref)
        d = torch.where(torch.abs(d) > 1e-12, d, torch.ones_like(d))
        z_jac = (1.0 / d) * rhs
        zn = float(torch.linalg.norm(z))
        jn = float(torch.linalg.norm(z_jac))
        return {
            "finite": bool(torch.all(torch.isfinite(z))),
            "pd": float(torch.dot(rhs, z)) > 0.0,
            "z_norm": zn,
            "jacobi_norm": jn,
            "z_over_jacobi": zn / max(jn, 1e-30),
        }

    def cycle_trace(self, rhs, *, cycle_type: Optional[str] = None) -> MultigridCycleTrace:
        """Structured trace of one multigrid cycle on ``rhs`` (multigrid_v4.py:1362-1438):
        the norms of every level visit, measured on the device between the
        cycle's own kernels, then the root-local correction.  A diagnostic:
        the library synchronises at every norm; the solve path is unchanged."""
        if not self._is_setup:
            raise RuntimeError("GalerkinMatFreeGMG.setup() must be called before cycle_trace().")
        cycle = self._cycle_type if cycle_type is None else cycle_type
        if cycle not in {"v", "w"}:
            raise ValueError(f"cycle_type must be 'v' or 'w'; got {cycle!r}")
        torch = _lib.require_cuda()
        rhs64 = _lib.as_cuda(rhs, torch.float64)
        cap = 2 ** self._n_levels
        visits = np.full((cap, 32), np.nan)
        summary = np.full(16, np.nan)
        nv = ctypes.c_int()
        _lib.call("simpfem_gmg_cycle_trace", self._h, _lib.ptr(rhs64), 0 if cycle == "v" else 1,
                  visits.ctypes.data, cap, ctypes.byref(nv), summary.ctypes.data, _lib.stream_ptr())
        if nv.value > cap:
            raise RuntimeError(f"cycle_trace: {nv.value} visits exceed the record capacity {cap}")
        options = {
            "coarse_correction_policy": self._coarse_correction_policy,
            "coarse_correction_acceptance_ratio": self._coarse_correction_acceptance_ratio,
            "coarse_correction_max_scale": self._coarse_correction_max_scale,
            "root_enrichment_mode": self._root_enrichment_mode,
            "root_enrichment_weight_floor": self._root_enrichment_weight_floor,
            "root_enrichment_weight_power": self._root_enrichment_weight_power,
            "root_local_correction_mode": self._root_local_correction_mode,
            "root_local_correction_inner_steps": self._root_local_correction_inner_steps,
            "root_local_correction_inner_restart": self._root_local_correction_inner_restart,
            "inner_krylov_steps": self._inner_krylov_steps,
            "inner_krylov_restart": self._inner_krylov_restart,
        }
        return trace_from_records(visits[: nv.value], summary, cycle, options)

    def estimate_kappa_eff(self, n_iter: int = 30) -> float:
        """Lanczos estimate of kappa(M K) for a linear preconditioner
        (multigrid_v4.py:1057-1117)."""
        if not self._is_setup:
            raise RuntimeError("Call setup() before estimate_kappa_eff().")
        if (self._coarse_correction_policy != "none" or self._root_enrichment_mode != "none"
                or self._root_local_correction_mode != "none" or self._inner_krylov_steps > 0):
            raise RuntimeError(
                "estimate_kappa_eff requires a linear preconditioner; disable safeguarded "
                "coarse correction, root enrichment, root-local correction, and inner Krylov "
                "wrapping first."
            )
        torch = _lib.require_cuda()
        n = self._mf_op._n_free
        v = torch.as_tensor(np.random.RandomState(0).standard_normal(n), device="cuda")
        v = v / float(torch.linalg.norm(v))
        alpha = np.zeros(n_iter)
        beta = np.zeros(max(n_iter - 1, 0))
        v_prev = torch.zeros_like(v)
        for j in range(n_iter):
            w = self.apply(self.apply_fine_operator(v))
            a = float(torch.dot(v, w))
            alpha[j] = a
            w = w - a * v
            if j > 0:
                w = w - beta[j - 1] * v_prev
            if j < n_iter - 1:
                b = float(torch.linalg.norm(w))
                beta[j] = b
                if b < 1e-14:
                    alpha = alpha[: j + 1]
                    beta = beta[:j]
                    break
                v_prev = v
                v = w / b
        T = np.diag(alpha) + np.diag(beta, 1) + np.diag(beta, -1)
        eigs = np.linalg.eigvalsh(T)
        eigs = eigs[eigs > 0]
        self._kappa_eff = float("nan") if len(eigs) == 0 else float(eigs[-1] / max(eigs[0], 1e-300))
        return self._kappa_eff

    # ------------------------------------------------------------ native Krylov
    def _native_fgmres(self, b, x0, tol, maxiter, restart, history, check=None):
        """``check``: optional (iteration, fn) or (iteration, fn, True); fn runs once
        when the solve has completed that many iterations and is still running --
        fn(history_so_far), or with the third element fn(history_so_far,
        true_rel_residual) where true_rel_residual is the FP64 true relative
        residual of the iterate at that point -- and a true return ends the solve
        there (the result then reports not converged)."""
        torch = _lib.require_cuda()
        bb = _lib.as_cuda(b, torch.float64)
        x = torch.empty_like(bb)
        x0t = _lib.as_cuda(x0, torch.float64) if x0 is not None else None
        cap = int(maxiter) + int(maxiter) // max(int(restart), 1) + 4
        hist = np.zeros(cap, dtype=np.float64)
        hlen, it, conv = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self.last_stopped = False
        if check is None:
            _lib.call("simpfem_fgmres", self._h, _lib.ptr(bb), _lib.ptr(x0t) if x0t is not None else None,
                      _lib.ptr(x), float(tol), int(maxiter), int(restart), hist.ctypes.data_as(ctypes.c_void_p), cap,
                      ctypes.byref(hlen), ctypes.byref(it), ctypes.byref(conv), _lib.stream_ptr())
        else:
            check_iter, fn = check[0], check[1]
            want_true = len(check) > 2 and bool(check[2])
            errors = []

            def trampoline(_ctx, _iters, hptr, hn, true_rel):
                try:
                    hist_now = [float(hptr[k]) for k in range(hn)]
                    return 1 if (fn(hist_now, float(true_rel)) if want_true else fn(hist_now)) else 0
                except BaseException as e:  # raised again once the call returns
                    errors.append(e)
                    return 0

            cb = _CHECK_FN(trampoline)
            stopped = ctypes.c_int()
            _lib.call("simpfem_fgmres_checked", self._h, _lib.ptr(bb), _lib.ptr(x0t) if x0t is not None else None,
                      _lib.ptr(x), float(tol), int(maxiter), int(restart), hist.ctypes.data_as(ctypes.c_void_p), cap,
                      ctypes.byref(hlen), ctypes.byref(it), ctypes.byref(conv), int(check_iter), int(want_true),
                      ctypes.cast(cb, ctypes.c_void_p), None, ctypes.byref(stopped), _lib.stream_ptr())
            if errors:
                raise errors[0]
            self.last_stopped = bool(stopped.value)
        if history is not None:
            history.extend(float(v) for v in hist[: min(hlen.value, cap)])
        return x, int(it.value), bool(conv.value)

    def _native_pcg(self, b, x0, tol, maxiter, history):
        torch = _lib.require_cuda()
        bb = _lib.as_cuda(b, torch.float64)
        x = torch.empty_like(bb)
        x0t = _lib.as_cuda(x0, torch.float64) if x0 is not None else None
        cap = int(maxiter) + 4
        hist = np.zeros(cap, dtype=np.float64)
        hlen, it, conv = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _lib.call("simpfem_pcg", self._h, _lib.ptr(bb), _lib.ptr(x0t) if x0t is not None else None, _lib.ptr(x),
                  float(tol), int(maxiter), hist.ctypes.data_as(ctypes.c_void_p), cap, ctypes.byref(hlen),
                  ctypes.byref(it), ctypes.byref(conv), _lib.stream_ptr())
        if history is not None:
            history.extend(float(v) for v in hist[: min(hlen.value, cap)])
        return x, int(it.value), bool(conv.value)


def _cupy_fgmres(A_op: Callable, b, M_op: Callable, x0=None, tol: float = 1e-6, maxiter: int = 200,
                 restart: int = 32, history=None):
    """Flexible restarted GMRES, right preconditioning, Givens rotations (multigrid_v4.py:416-534).

    A hierarchy's own fine operator and ``apply`` are solved entirely in the
    library; any other pair of callables runs on the library's device Krylov
    core with the two operators applied through callbacks."""
    gmg = _native_gmg(A_op, M_op)
    if gmg is not None:
        return gmg._native_fgmres(b, x0, tol, maxiter, restart, history)
    return _krylov.fgmres(A_op, b, M_op, x0=x0, tol=tol, maxiter=maxiter, restart=restart, history=history)
