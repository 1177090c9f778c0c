"""Restatement of GalerkinMatFreeGMG (gpu_fem/multigrid_v4.py:537-2024) on numpy/scipy."""

from __future__ import annotations

import math

import numpy as np
import scipy.linalg as sla
import scipy.sparse as sp

from .solver import (KE, NodeBlockJacobi, Operator, coarse_free_injection, fgmres, fine_lambda, fixed_pcg,
                     level1_galerkin, scalar_prolongation, sparse_lambda)


class GMG:
    def __init__(self, op: Operator, *, n_levels=4, coarse_smooth_iters=2, fine_smoother="fp32",
                 fine_smoother_degree=2, omega=0.5, dense_chol_max=5000, coarse_pcg_iters=80,
                 smoother_type="chebyshev", cheb_lower_frac=1.0 / 30.0, level_precisions=None, cycle_type="v",
                 coarse_correction_policy="none", coarse_correction_acceptance_ratio=1.0,
                 coarse_correction_max_scale=1.0, root_enrichment_mode="none", root_enrichment_weight_floor=1e-6,
                 root_enrichment_weight_power=0.5, root_local_correction_mode="none",
                 root_local_correction_max_scale=1.0, root_local_correction_inner_steps=10,
                 root_local_correction_inner_restart=None, inner_krylov_steps=0, inner_krylov_restart=None):
        # constructor state, multigrid_v4.py:546-770
        self.op = op
        self.L = max(1, int(n_levels))
        self.fine = fine_smoother
        self.deg = max(1, int(fine_smoother_degree))
        self.c_iters = max(1, int(coarse_smooth_iters))
        self.omega_max = float(omega)
        self.chol_max = int(dense_chol_max)
        self.pcg_iters = int(coarse_pcg_iters)
        self.smoother = smoother_type
        self.lf = float(cheb_lower_frac)
        self.prec = list(level_precisions) if level_precisions is not None else None
        self.cycle = cycle_type
        self.cc = coarse_correction_policy
        self.cc_ratio = float(coarse_correction_acceptance_ratio)
        self.cc_max = float(coarse_correction_max_scale)
        self.enrich = root_enrichment_mode
        self.w_floor = float(root_enrichment_weight_floor)
        self.w_pow = float(root_enrichment_weight_power)
        self.rl = root_local_correction_mode
        self.rl_max = float(root_local_correction_max_scale)
        self.rl_steps = int(root_local_correction_inner_steps)
        self.rl_restart = int(root_local_correction_inner_restart) if root_local_correction_inner_restart else max(1, self.rl_steps)
        self.ik = int(inner_krylov_steps)
        self.ik_restart = int(inner_krylov_restart) if inner_krylov_restart else max(1, self.ik)
        self.lam_Emax = float("nan")
        self.lams = []
        dims = [op.dims]
        for _ in range(1, self.L):
            dims.append(tuple(max(1, d // 2) for d in dims[-1]))
        self.dims = dims
        self.free = [np.asarray(op.free)]
        self.P = []
        for lv in range(self.L - 1):
            fc = coarse_free_injection(*dims[lv], *dims[lv + 1], self.free[lv])
            Pv = sp.kron(scalar_prolongation(*dims[lv], *dims[lv + 1]), sp.eye(3), format="csr")
            self.P.append(Pv[self.free[lv]][:, fc].tocsr())
            self.free.append(fc)
        self.R = [P.T.tocsr() for P in self.P]
        self.nbj = None
        self.is_setup = False

    # ------------------------------------------------------------ setup (:1119-1341)
    def setup(self, E, fine_diag=None):
        self.E = np.asarray(E, dtype=np.float64)
        self.E32 = self.E.astype(np.float32)
        if self.prec is None:
            self.prec = ([self.fine] + (["fp32"] if self.L > 1 else [])) if self.fine == "bf16" else [self.fine]
        while len(self.prec) < self.L:
            self.prec.append("fp64")
        d0 = fine_diag if fine_diag is not None else self.op.diagonal(self.E)
        d0 = np.where(np.abs(d0) > 1e-12, d0, 1.0)
        self.dinv = [1.0 / d0] + [None] * (self.L - 1)
        if self.enrich != "none":
            w = np.clip(np.abs(d0) / max(float(np.max(np.abs(d0))), 1e-300), self.w_floor, 1.0)
            if abs(self.w_pow - 1.0) > 1e-12:
                w = w ** self.w_pow
            self.wenrich = w
        if self.rl != "none":
            if self.nbj is None:
                self.nbj = NodeBlockJacobi(self.op)
            self.nbj.update(self.E, d0)
        Emax = float(np.max(self.E))
        prev = self.lam_Emax
        reest = math.isnan(prev) or abs(Emax - prev) / max(abs(prev), 1e-12) > 0.10
        if reest:
            self.lam0 = fine_lambda(self.op, self.E, self.dinv[0])
            self.lam_Emax = Emax
        self.omega = min(self.omega_max, 0.9 * 2.0 / max(self.lam0, 1e-6))
        if len(self.lams) != self.L:
            self.lams = [float("nan")] * self.L
        self.lams[0] = self.lam0
        Emin = float(np.min(self.E))
        self.contrast = Emax / max(Emin, 1e-300)
        void = 1.0 - np.count_nonzero(self.E > Emax * 1e-8) / max(self.E.size, 1)
        if self.contrast > 1e5 or void > 0.8:
            self.c_adapt, self.deg_adapt, self.high = max(self.c_iters, 6), max(self.deg, 4), True
        elif self.contrast > 100 or void > 0.5:
            self.c_adapt, self.deg_adapt, self.high = max(self.c_iters, 4), max(self.deg, 3), True
        elif self.contrast > 10:
            self.c_adapt, self.deg_adapt, self.high = max(self.c_iters, 3), self.deg, False
        else:
            self.c_adapt, self.deg_adapt, self.high = self.c_iters, self.deg, False
        self.K = [None] * self.L
        for lv in range(1, self.L):
            if lv == 1:
                K = level1_galerkin(*self.dims[1], *self.dims[0], self.free[1], self.E)
            else:
                K = (self.R[lv - 1] @ (self.K[lv - 1] @ self.P[lv - 1])).tocsr()
            dg = K.diagonal()
            self.dinv[lv] = 1.0 / np.where(np.abs(dg) > 1e-12, dg, 1.0)
            self.K[lv] = K
            if reest or math.isnan(self.lams[lv]):
                self.lams[lv] = sparse_lambda(K, self.dinv[lv])
        self.coarse_mode = "none"
        if self.L > 1:
            Kc = self.K[-1]
            if Kc.shape[0] <= self.chol_max:
                A = Kc.toarray()
                try:
                    self.Lc = np.linalg.cholesky(A)
                    self.coarse_mode = "dense"
                except np.linalg.LinAlgError:
                    eps = max(float(A.diagonal().mean()) * 1e-8, 1e-14)
                    try:
                        self.Lc = np.linalg.cholesky(A + eps * np.eye(A.shape[0]))
                        self.coarse_mode = "dense"
                    except np.linalg.LinAlgError:
                        self.coarse_mode = "iterative"
            else:
                self.coarse_mode = "iterative"
        self.is_setup = True

    # ------------------------------------------------------------ operators
    def A0(self, v):
        return self.op.matvec(v, self.E)

    def Alv(self, lv, v):
        return self.A0(v) if lv == 0 else self.K[lv] @ v

    # ------------------------------------------------------------ smoothers (:1783-1906)
    @staticmethod
    def cheb(A, rhs, x, dinv, lm, lf, degree):
        lmin = lf * lm
        sigma = (lm + lmin) * 0.5
        delta = (lm - lmin) * 0.5
        r = rhs - A(x)
        z = dinv * r
        alpha = 2.0 / (lm + lmin)
        d = z
        x = x + alpha * d
        for _ in range(1, degree):
            r = rhs - A(x)
            z = dinv * r
            an = 1.0 / (sigma - (delta ** 2) * alpha * 0.25)
            d = an * (z + (delta ** 2) * alpha * 0.25 * d)
            x = x + d
            alpha = an
        return x

    def _low_matvec(self, prec):
        if prec == "fp32":
            return lambda v: self.op.matvec(v, self.E32)
        return lambda v: bf16_matvec(self.op, v, self.E32)

    def smooth_fine(self, x, rhs):
        prec = self.prec[0]
        lf = min(self.lf, 1.0 / 100.0) if self.high else self.lf
        if self.smoother == "chebyshev":
            if prec == "fp64":
                return self.cheb(self.A0, rhs, x.astype(np.float64, copy=True), self.dinv[0], self.lam0, lf,
                                 self.deg_adapt)
            x32, r32, d32 = x.astype(np.float32), rhs.astype(np.float32), self.dinv[0].astype(np.float32)
            return self.cheb(self._low_matvec(prec), r32, x32, d32, np.float32(self.lam0), np.float32(lf),
                             self.deg_adapt).astype(np.float64)
        if prec == "fp64":
            xc = x.astype(np.float64, copy=True)
            for _ in range(self.deg_adapt):
                xc = xc + self.omega * self.dinv[0] * (rhs - self.A0(xc))
            return xc
        x32, r32, d32 = x.astype(np.float32), rhs.astype(np.float32), self.dinv[0].astype(np.float32)
        A32 = self._low_matvec(prec)
        for _ in range(self.deg_adapt):
            x32 = x32 + self.omega * d32 * (r32 - A32(x32))
        return x32.astype(np.float64)

    def smooth_coarse(self, lv, x, rhs):
        lm = self.lams[lv] if np.isfinite(self.lams[lv]) else 1.0
        lf = min(self.lf, 1.0 / 100.0) if self.high else self.lf
        K = self.K[lv]
        if self.prec[lv] == "fp32":
            K32, d32 = K.astype(np.float32), self.dinv[lv].astype(np.float32)
            x32, r32 = x.astype(np.float32), rhs.astype(np.float32)
            if self.smoother == "chebyshev":
                x32 = self.cheb(lambda v: K32 @ v, r32, x32, d32, np.float32(lm), np.float32(lf), self.c_adapt)
            else:
                for _ in range(self.c_adapt):
                    x32 = x32 + self.omega * d32 * (r32 - K32 @ x32)
            return x32.astype(np.float64)
        if self.smoother == "chebyshev":
            return self.cheb(lambda v: K @ v, rhs, x, self.dinv[lv], lm, lf, self.c_adapt)
        for _ in range(self.c_adapt):
            x = x + self.omega * self.dinv[lv] * (rhs - K @ x)
        return x

    def solve_coarsest(self, rhs):
        if self.L == 1:
            return self.smooth_fine(np.zeros_like(rhs), rhs)
        if self.coarse_mode == "dense":
            y = sla.solve_triangular(self.Lc, rhs, lower=True)
            return sla.solve_triangular(self.Lc, y, lower=True, trans="T")
        iters = max(self.pcg_iters, 200) if self.high else self.pcg_iters
        return fixed_pcg(self.K[-1], rhs, self.dinv[-1], iters)

    # ------------------------------------------------------------ corrections (:867-1055)
    def correction(self, lv, x, res, c):
        """Returns (x, corrected residual)."""
        return self.correction_decision(lv, x, res, c)[:2]

    def correction_decision(self, lv, x, res, c):
        """(x, corrected residual, raw scale, applied scale, note) of the coarse
        correction (multigrid_v4.py:867-931); raw scale None is kept as None."""
        if self.cc == "none":
            return x + c, res - self.Alv(lv, c), 1.0, 1.0, ""
        cn, rn = float(np.linalg.norm(c)), float(np.linalg.norm(res))
        if cn <= 1e-300 or rn <= 1e-300:
            return x, res, 0.0, 0.0, "degenerate_correction"
        Ac = self.Alv(lv, c)
        den = float(np.dot(Ac, Ac))
        if den <= 1e-300:
            return x, res, 0.0, 0.0, "degenerate_correction"
        raw = float(np.dot(res, Ac) / den)
        s = min(self.cc_max, max(0.0, raw))
        trial = res - s * Ac
        if float(np.linalg.norm(trial)) > self.cc_ratio * rn:
            return x, res, raw, 0.0, "rejected_correction"
        note = ""
        if s <= 1e-12 and raw <= 0.0:
            note = "nonpositive_correction_scale"
        elif abs(s - raw) > 1e-12:
            note = "clipped_correction_scale"
        return x + s * c, trial, raw, s, note

    def enrichment_rhs(self, residual):
        w = self.wenrich
        vw = np.clip(1.0 - w, self.w_floor, 1.0)
        R0, P0 = self.R[0], self.P[0]
        if self.enrich == "weighted_residual_second":
            return R0 @ (w * residual)
        if self.enrich == "weighted_gap_second":
            return R0 @ (w * (residual - P0 @ (R0 @ residual)))
        if self.enrich == "void_residual_second":
            return R0 @ (vw * residual)
        return R0 @ (vw * (residual - P0 @ (R0 @ residual)))

    def root_local(self, x, residual):
        return self.root_local_decision(x, residual)[0]

    def root_local_decision(self, x, residual):
        """(x, residual, raw scale, applied scale, note) of the root-local
        correction (multigrid_v4.py:964-1055)."""
        if self.rl == "none":
            return x, residual, None, 0.0, ""
        if self.rl == "node_block_inner_fgmres":
            corr, _, _ = fgmres(self.A0, residual, self.nbj.apply, tol=0.0, maxiter=self.rl_steps,
                                restart=self.rl_restart)
            cn, rn = float(np.linalg.norm(corr)), float(np.linalg.norm(residual))
            if cn <= 1e-300 or rn <= 1e-300:
                return x, residual, 0.0, 0.0, "degenerate_root_local_correction"
            trial = residual - self.A0(corr)
            if float(np.linalg.norm(trial)) > rn:
                return x, residual, None, 0.0, "rejected_root_local_inner_fgmres"
            return x + corr, trial, None, 1.0, "root_local_inner_fgmres"
        corr = self.nbj.apply(residual)
        cn, rn = float(np.linalg.norm(corr)), float(np.linalg.norm(residual))
        if cn <= 1e-300 or rn <= 1e-300:
            return x, residual, 0.0, 0.0, "degenerate_root_local_correction"
        Ac = self.A0(corr)
        den = float(np.dot(Ac, Ac))
        if den <= 1e-300:
            return x, residual, 0.0, 0.0, "degenerate_root_local_correction"
        raw = float(np.dot(residual, Ac) / den)
        s = min(self.rl_max, max(0.0, raw))
        if s <= 1e-12:
            return x, residual, raw, 0.0, "nonpositive_root_local_scale"
        note = "clipped_root_local_scale" if abs(s - raw) > 1e-12 else ""
        return x + s * corr, residual - s * Ac, raw, s, note

    # ------------------------------------------------------------ cycles (:1929-2024)
    def vcycle(self, lv, rhs):
        if lv == self.L - 1:
            return self.solve_coarsest(rhs)
        x = self.smooth_fine(np.zeros_like(rhs), rhs) if lv == 0 else self.smooth_coarse(lv, np.zeros_like(rhs), rhs)
        res = rhs - self.Alv(lv, x)
        e = self.vcycle(lv + 1, self.R[lv] @ res)
        x, cres = self.correction(lv, x, res, self.P[lv] @ e)
        if lv == 0 and self.enrich != "none":
            e2 = self.vcycle(1, self.enrichment_rhs(cres))
            x, _ = self.correction(lv, x, cres, self.P[lv] @ e2)
        x = self.smooth_fine(x, rhs) if lv == 0 else self.smooth_coarse(lv, x, rhs)
        if lv == 0 and self.high:
            x = self.smooth_fine(x, rhs)
        return x

    def wcycle(self, lv, rhs):
        if lv == self.L - 1:
            return self.solve_coarsest(rhs)
        x = self.smooth_fine(np.zeros_like(rhs), rhs) if lv == 0 else self.smooth_coarse(lv, np.zeros_like(rhs), rhs)
        res = rhs - self.Alv(lv, x)
        e = self.wcycle(lv + 1, self.R[lv] @ res)
        if self.cc == "none":
            x = x + self.P[lv] @ e
            res2 = rhs - self.Alv(lv, x)
        else:
            x, res2 = self.correction(lv, x, res, self.P[lv] @ e)
        rc2 = self.enrichment_rhs(res2) if (lv == 0 and self.enrich != "none") else self.R[lv] @ res2
        e2 = self.wcycle(lv + 1, rc2)
        x, _ = self.correction(lv, x, res2, self.P[lv] @ e2)
        x = self.smooth_fine(x, rhs) if lv == 0 else self.smooth_coarse(lv, x, rhs)
        if lv == 0 and self.high:
            x = self.smooth_fine(x, rhs)
        return x

    def base_cycle(self, rhs):
        return self.wcycle(0, rhs) if self.cycle == "w" else self.vcycle(0, rhs)

    def apply(self, rhs):
        """multigrid_v4.py:1742-1767."""
        if not self.is_setup:
            raise RuntimeError("GalerkinMatFreeGMG.setup() must be called before apply().")
        rhs = np.asarray(rhs, dtype=np.float64)
        if self.ik > 0:
            x, _, _ = fgmres(self.A0, rhs, self.base_cycle, tol=0.0, maxiter=self.ik, restart=self.ik_restart)
        else:
            x = self.base_cycle(rhs)
        if self.rl != "none":
            x = self.root_local(x, rhs - self.A0(x))
        return x

    # ------------------------------------------------------------ diagnostics (:1057-1117, :1348-1360)
    def probe_quality(self, rhs) -> dict:
        """Preconditioner action against the Jacobi action on one right-hand side."""
        rhs = np.asarray(rhs, dtype=np.float64)
        z = self.apply(rhs)
        zn, jn = float(np.linalg.norm(z)), float(np.linalg.norm(self.dinv[0] * rhs))
        return {"finite": bool(np.all(np.isfinite(z))), "pd": float(rhs @ z) > 0.0, "z_norm": zn,
                "jacobi_norm": jn, "z_over_jacobi": zn / max(jn, 1e-30)}

    def estimate_kappa_eff(self, n_iter: int = 30) -> float:
        """lambda_max / lambda_min (positive Ritz values) of n_iter Lanczos steps on
        M K from numpy's RandomState(0) start vector."""
        if (self.cc != "none" or self.enrich != "none" or self.rl != "none" or self.ik > 0):
            raise RuntimeError("estimate_kappa_eff requires a linear preconditioner")
        n = len(self.free[0])
        v = np.random.RandomState(0).standard_normal(n)
        v /= np.linalg.norm(v)
        alpha, beta = np.zeros(n_iter), np.zeros(max(n_iter - 1, 0))
        v_prev = np.zeros(n)
        for j in range(n_iter):
            w = self.apply(self.A0(v))
            alpha[j] = float(v @ w)
            w = w - alpha[j] * v
            if j > 0:
                w = w - beta[j - 1] * v_prev
            if j < n_iter - 1:
                beta[j] = float(np.linalg.norm(w))
                if beta[j] < 1e-14:
                    alpha, beta = alpha[: j + 1], beta[:j]
                    break
                v_prev, v = v, w / beta[j]
        eigs = np.linalg.eigvalsh(np.diag(alpha) + np.diag(beta, 1) + np.diag(beta, -1))
        eigs = eigs[eigs > 0]
        return float("nan") if len(eigs) == 0 else float(eigs[-1] / max(eigs[0], 1e-300))

    # ------------------------------------------------------------ cycle trace (:1362-1728)
    def cycle_trace(self, rhs, cycle_type=None) -> dict:
        """One traced base cycle, then the root-local correction: the dictionary
        of MultigridCycleTrace.to_dict() (multigrid_v4.py:81-113, :1362-1438),
        visits in pre-order (visit_id).  The inner Krylov wrapper is not traced."""
        if not self.is_setup:
            raise RuntimeError("GalerkinMatFreeGMG.setup() must be called before cycle_trace().")
        cyc = self.cycle if cycle_type is None else cycle_type
        if cyc not in ("v", "w"):
            raise ValueError(f"cycle_type must be 'v' or 'w'; got {cyc!r}")
        rhs = np.asarray(rhs, dtype=np.float64)
        visits = []
        out = self._trace_level(0, rhs, visits, [0], cyc)
        pre = rhs - self.A0(out)
        out, res, lraw, lapp, lnote = self.root_local_decision(out, pre)
        visits.sort(key=lambda v: v["visit_id"])
        if lnote:
            root = next((v for v in visits if v["level"] == 0 and not v["is_coarsest"]), None)
            if root is not None:
                root["notes"] = _merge_notes(root["notes"], lnote)
        nrm = lambda v: float(np.linalg.norm(v))  # noqa: E731
        rn, jn, on, resn = nrm(rhs), nrm(self.dinv[0] * rhs), nrm(out), nrm(res)
        rz = float(np.dot(rhs, out))
        return {
            "cycle_type": cyc, "rhs_norm": rn, "jacobi_action_norm": jn, "output_norm": on,
            "z_over_jacobi": _safe_ratio(on, jn), "rz": rz, "pd": bool(rz > 0.0),
            "output_residual_norm": resn, "output_residual_ratio": _safe_ratio(resn, rn),
            "contrast_ratio": self.contrast, "is_high_contrast": self.high,
            "fine_degree_adapt": self.deg_adapt, "coarse_iters_adapt": self.c_adapt,
            "coarse_correction_policy": self.cc, "coarse_correction_acceptance_ratio": self.cc_ratio,
            "coarse_correction_max_scale": self.cc_max, "root_enrichment_mode": self.enrich,
            "root_enrichment_weight_floor": self.w_floor, "root_enrichment_weight_power": self.w_pow,
            "root_local_correction_mode": self.rl, "root_local_correction_inner_steps": self.rl_steps,
            "root_local_correction_inner_restart": self.rl_restart,
            "root_local_correction_raw_scale": lraw, "root_local_correction_applied_scale": lapp,
            "root_local_correction_residual_ratio": _safe_ratio(resn, nrm(pre)),
            "inner_krylov_steps": self.ik, "inner_krylov_restart": self.ik_restart,
            "visits": visits,
        }

    def _trace_level(self, lv, rhs, visits, counter, cyc):
        nrm = lambda v: float(np.linalg.norm(v))  # noqa: E731
        vid = counter[0]
        counter[0] += 1
        rn, jn = nrm(rhs), nrm(self.dinv[lv] * rhs)
        visit = {"visit_id": vid, "level": lv, "cycle_type": cyc, "rhs_norm": rn, "jacobi_action_norm": jn}
        if lv == self.L - 1:
            x = self.solve_coarsest(rhs)
            resn = nrm(rhs - self.Alv(lv, x))
            xn = nrm(x)
            visit.update(is_coarsest=True, n_coarse_corrections=0, presmooth_solution_norm=0.0,
                         presmooth_residual_norm=rn, presmooth_residual_ratio=1.0, restricted_rhs_norm=0.0,
                         restricted_rhs_ratio=0.0, projector_norm=0.0, coarse_space_gap_norm=0.0,
                         coarse_space_gap_ratio=0.0, coarse_correction_norm=xn, prolongated_correction_norm=xn,
                         correction_alignment=0.0, corrected_residual_norm=resn,
                         corrected_residual_vs_presmooth=_safe_ratio(resn, rn), correction_scale_raw=None,
                         correction_scale_applied=1.0, postsmooth_solution_norm=xn, postsmooth_residual_norm=resn,
                         postsmooth_residual_ratio=_safe_ratio(resn, rn), coarsest_mode=self.coarse_mode, notes="")
            visits.append(_visit_record(visit))
            return x
        smooth = (lambda x: self.smooth_fine(x, rhs)) if lv == 0 else (lambda x: self.smooth_coarse(lv, x, rhs))
        xs = smooth(np.zeros_like(rhs))
        res = rhs - self.Alv(lv, xs)
        presn = nrm(res)
        rc = self.R[lv] @ res
        proj = self.P[lv] @ rc
        e = self._trace_level(lv + 1, rc, visits, counter, cyc)
        Pe = self.P[lv] @ e
        align = _alignment(res, Pe)
        x, cres, raw, app, note1 = self.correction_decision(lv, xs, res, Pe)
        crn = nrm(cres)
        enrich = lv == 0 and self.enrich != "none"
        enrich_note = f"root_enrichment:{self.enrich}" if enrich else ""
        second, note2 = None, ""
        if cyc == "w" or enrich:
            rc2 = self.enrichment_rhs(cres) if enrich else self.R[lv] @ cres
            e2 = self._trace_level(lv + 1, rc2, visits, counter, cyc)
            Pe2 = self.P[lv] @ e2
            align2 = _alignment(cres, Pe2)
            x, cres2, raw2, app2, note2 = self.correction_decision(lv, x, cres, Pe2)
            cr2n = nrm(cres2)
            second = dict(second_restricted_rhs_norm=nrm(rc2), second_coarse_correction_norm=nrm(e2),
                          second_prolongated_correction_norm=nrm(Pe2), second_correction_alignment=align2,
                          second_correction_scale_raw=raw2, second_correction_scale_applied=app2,
                          second_corrected_residual_norm=cr2n,
                          second_corrected_residual_vs_corrected=_safe_ratio(cr2n, crn))
        # the V-cycle record reports the residual after its (enrichment) second
        # correction as corrected_residual_norm (multigrid_v4.py:1516-1563);
        # the W-cycle record keeps the first (:1670-1712)
        if second is not None and cyc == "v":
            crn = second["second_corrected_residual_norm"]
        extra = ""
        x = smooth(x)
        if lv == 0 and self.high:
            x = smooth(x)
            extra = "extra_fine_postsmooth"
        postn = nrm(rhs - self.Alv(lv, x))
        visit.update(is_coarsest=False, n_coarse_corrections=1 if second is None else 2,
                     presmooth_solution_norm=nrm(xs), presmooth_residual_norm=presn,
                     presmooth_residual_ratio=_safe_ratio(presn, rn), restricted_rhs_norm=nrm(rc),
                     restricted_rhs_ratio=_safe_ratio(nrm(rc), presn), projector_norm=nrm(proj),
                     coarse_space_gap_norm=nrm(res - proj), coarse_space_gap_ratio=_safe_ratio(nrm(res - proj), presn),
                     coarse_correction_norm=nrm(e), prolongated_correction_norm=nrm(Pe), correction_alignment=align,
                     correction_scale_raw=raw, correction_scale_applied=app, corrected_residual_norm=crn,
                     corrected_residual_vs_presmooth=_safe_ratio(crn, presn), postsmooth_solution_norm=nrm(x),
                     postsmooth_residual_norm=postn, postsmooth_residual_ratio=_safe_ratio(postn, rn),
                     coarsest_mode="",
                     notes=_merge_notes(note1, note2, enrich_note, extra))
        if second is not None:
            visit.update(second)
        visits.append(_visit_record(visit))
        return x


# MultigridCycleVisit fields in declaration order (multigrid_v4.py:39-74)
VISIT_FIELDS = (
    "visit_id", "level", "cycle_type", "is_coarsest", "n_coarse_corrections", "rhs_norm", "jacobi_action_norm",
    "presmooth_solution_norm", "presmooth_residual_norm", "presmooth_residual_ratio", "restricted_rhs_norm",
    "restricted_rhs_ratio", "projector_norm", "coarse_space_gap_norm", "coarse_space_gap_ratio",
    "coarse_correction_norm", "prolongated_correction_norm", "correction_alignment", "corrected_residual_norm",
    "corrected_residual_vs_presmooth", "correction_scale_raw", "correction_scale_applied",
    "second_restricted_rhs_norm", "second_coarse_correction_norm", "second_prolongated_correction_norm",
    "second_correction_alignment", "second_correction_scale_raw", "second_correction_scale_applied",
    "second_corrected_residual_norm", "second_corrected_residual_vs_corrected", "postsmooth_solution_norm",
    "postsmooth_residual_norm", "postsmooth_residual_ratio", "coarsest_mode", "notes",
)


def _visit_record(v: dict) -> dict:
    return {k: v.get(k) for k in VISIT_FIELDS}


def _safe_ratio(num: float, den: float) -> float:
    """multigrid_v4.py:840-843."""
    if abs(den) <= 1e-300:
        return 0.0 if abs(num) <= 1e-300 else float("inf")
    return float(num / den)


def _alignment(ref, corr) -> float:
    """Cosine of the angle between a residual and a correction (multigrid_v4.py:855-862)."""
    rn, cn = float(np.linalg.norm(ref)), float(np.linalg.norm(corr))
    if rn <= 1e-300 or cn <= 1e-300:
        return 0.0
    return float(np.dot(ref, corr) / (rn * cn))


def _merge_notes(*notes: str) -> str:
    return "|".join(n for n in notes if n)


def bf16_round(a32) -> np.ndarray:
    """Round float32 to bf16 (round to nearest even), returned as float32
    (the reference's packing, cuda_fused_matvec.py:323-337)."""
    bits = np.asarray(a32, dtype=np.float32).view(np.uint32).astype(np.uint64)
    rnd = 0x7FFF + ((bits >> 16) & 1)
    out = (((bits + rnd) >> 16) << 16).astype(np.uint32)
    return out.view(np.float32)


KE_F32 = KE.astype(np.float32)


def bf16_matvec(op: Operator, u32, E32):
    """FusedMatvec BF16 semantics (cuda_fused_matvec.py:112-246): bf16 u and KE,
    FP32 accumulation of KE @ u per element, times E in FP32, summed per DOF."""
    full = np.zeros(op.ndof, dtype=np.float32)
    full[op.free] = u32
    ue = bf16_round(full[op.edof])
    keb = bf16_round(KE_F32)
    f = (ue.astype(np.float64) @ keb.astype(np.float64)).astype(np.float32) * E32[:, None]
    y = np.bincount(op.edof.ravel(), weights=f.ravel().astype(np.float64), minlength=op.ndof).astype(np.float32)
    return y[op.free]
