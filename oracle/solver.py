"""numpy/scipy restatement of the reference's guarded-floor solve (test oracle).

Every function cites the reference routine it restates; all arithmetic is FP64
numpy / scipy except where the reference itself drops to FP32 (the fp32
smoothing paths), which are restated with numpy float32 scalars and arrays so
the rounding follows the same operations.
"""

from __future__ import annotations

import math

import numpy as np
import scipy.sparse as sp

# ----------------------------------------------------------------------------
# Element data -- gpu_fem/pub_simp_solver.py:157-213
_SIGNS = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                   [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], dtype=np.float64)


def ke_unit_3d(nu: float = 0.3, E: float = 1.0) -> np.ndarray:
    """Hex8 stiffness on [-1,1]^3 with 2x2x2 Gauss points (pub_simp_solver.py:157-183);
    the Jacobian is formed explicitly from the node coordinates."""
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    D = np.diag([lam + 2 * mu] * 3 + [mu] * 3)
    D[0, 1] = D[0, 2] = D[1, 0] = D[1, 2] = D[2, 0] = D[2, 1] = lam
    K = np.zeros((24, 24))
    gp = 1.0 / math.sqrt(3.0)
    for r, s, t in _SIGNS * gp:
        dN = 0.125 * np.stack([_SIGNS[:, 0] * (1 + s * _SIGNS[:, 1]) * (1 + t * _SIGNS[:, 2]),
                               _SIGNS[:, 1] * (1 + r * _SIGNS[:, 0]) * (1 + t * _SIGNS[:, 2]),
                               _SIGNS[:, 2] * (1 + r * _SIGNS[:, 0]) * (1 + s * _SIGNS[:, 1])], axis=1)
        J = dN.T @ _SIGNS
        G = dN @ np.linalg.inv(J).T
        B = np.zeros((6, 24))
        B[0, 0::3], B[1, 1::3], B[2, 2::3] = G[:, 0], G[:, 1], G[:, 2]
        B[3, 0::3], B[3, 1::3] = G[:, 1], G[:, 0]
        B[4, 1::3], B[4, 2::3] = G[:, 2], G[:, 1]
        B[5, 0::3], B[5, 2::3] = G[:, 2], G[:, 0]
        K += B.T @ D @ B * abs(np.linalg.det(J))
    return K


KE = ke_unit_3d()
_OFF = ((_SIGNS + 1) / 2).astype(np.int64)


def edof_table(nx: int, ny: int, nz: int) -> np.ndarray:
    """pub_simp_solver.py:196-207."""
    i, j, k = (a.ravel() for a in np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij"))
    nodes = np.stack([((i + o[0]) * (ny + 1) + j + o[1]) * (nz + 1) + k + o[2] for o in _OFF], axis=1)
    return (3 * nodes[:, :, None] + np.arange(3)).reshape(-1, 24)


def cantilever_bc(nx: int, ny: int, nz: int, Lx=2.0, Ly=1.0, Lz=0.5):
    """The cantilever presets' BCs through bc_generator.generate_bc
    (bc_generator.py:173-251, :381-447): x = 0 face clamped, unit -y load at the
    node nearest (Lx, Ly/2, Lz/2)."""
    ndof = 3 * (nx + 1) * (ny + 1) * (nz + 1)
    face = np.arange((ny + 1) * (nz + 1))
    fixed = np.sort(np.concatenate([3 * face, 3 * face + 1, 3 * face + 2]))
    free = np.setdiff1d(np.arange(ndof), fixed)
    I, J, K = (a.ravel() for a in np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij"))
    xyz = np.column_stack([I * (Lx / nx), J * (Ly / ny), K * (Lz / nz)])
    node = int(np.argmin(np.linalg.norm(xyz - np.array([Lx, Ly / 2, Lz / 2]), axis=1)))
    F = np.zeros(ndof)
    F[3 * node + 1] = -1.0
    F[fixed] = 0.0
    return free.astype(np.int32), F


def density_filter(nx: int, ny: int, nz: int, rmin: float) -> sp.csr_matrix:
    """Cone filter (pub_simp_solver.py:215-243) by direct neighbour enumeration."""
    i, j, k = (a.ravel().astype(np.float64) for a in np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij"))
    n = i.size
    rows, cols, vals = [], [], []
    r = int(math.floor(rmin))
    for dx in range(-r, r + 1):
        for dy in range(-r, r + 1):
            for dz in range(-r, r + 1):
                d = math.sqrt(dx * dx + dy * dy + dz * dz)
                if d > rmin - 1e-10 and (dx or dy or dz):
                    continue
                ii, jj, kk = i + dx, j + dy, k + dz
                ok = (ii >= 0) & (ii < nx) & (jj >= 0) & (jj < ny) & (kk >= 0) & (kk < nz)
                src = np.nonzero(ok)[0]
                dst = ((ii[ok] * ny + jj[ok]) * nz + kk[ok]).astype(np.int64)
                rows.append(src)
                cols.append(dst)
                vals.append(np.full(src.size, rmin - d))
    rows, cols, vals = np.concatenate(rows), np.concatenate(cols), np.concatenate(vals)
    Hs = np.bincount(rows, weights=vals, minlength=n)
    return sp.csr_matrix((vals / Hs[rows], (rows, cols)), shape=(n, n))


# ----------------------------------------------------------------------------
# Matrix-free operator -- solver_v2.py:1182-1251
class Operator:
    def __init__(self, nx, ny, nz, free):
        self.dims = (nx, ny, nz)
        self.edof = edof_table(nx, ny, nz)
        self.free = np.asarray(free)
        self.ndof = 3 * (nx + 1) * (ny + 1) * (nz + 1)

    def matvec(self, u, E):
        dt = u.dtype
        full = np.zeros(self.ndof, dtype=dt)
        full[self.free] = u
        ue = full[self.edof]
        KE_ = KE if dt == np.float64 else KE.astype(dt)
        f = (KE_ @ ue.T * E[None, :]).T
        y = np.bincount(self.edof.ravel(), weights=f.ravel(), minlength=self.ndof).astype(dt, copy=False)
        return y[self.free]

    def diagonal(self, E):
        w = E[:, None] * np.diag(KE)[None, :]
        return np.bincount(self.edof.ravel(), weights=w.ravel(), minlength=self.ndof)[self.free]


class NodeBlockJacobi:
    """solver_v2.py:1268-1451."""

    def __init__(self, op: Operator):
        self.op = op
        n_nodes = op.ndof // 3
        fm = np.zeros(op.ndof, bool)
        fm[op.free] = True
        nf = fm.reshape(n_nodes, 3)
        self.all_free = np.where(nf.all(1))[0]
        f2l = np.full(op.ndof, -1)
        f2l[op.free] = np.arange(op.free.size)
        self.af_local = f2l[3 * self.all_free[:, None] + np.arange(3)]
        part = np.where(nf.any(1) & ~nf.all(1))[0]
        self.part_local = np.array([f2l[3 * n + d] for n in part for d in range(3) if nf[n, d]], dtype=np.int64)
        self.node_of = op.edof[:, 0::3] // 3
        self.n_nodes = n_nodes

    def update(self, E, scalar_diag):
        B = np.zeros((self.n_nodes, 3, 3))
        for a in range(8):
            blk = KE[3 * a:3 * a + 3, 3 * a:3 * a + 3]
            for r in range(3):
                for c in range(3):
                    B[:, r, c] += np.bincount(self.node_of[:, a], weights=E * blk[r, c], minlength=self.n_nodes)
        self.Binv = np.linalg.inv(B[self.all_free])
        d = scalar_diag[self.part_local]
        self.pinv = 1.0 / np.where(np.abs(d) > 1e-12, d, 1.0)

    def apply(self, r):
        z = np.zeros(self.op.free.size)
        z[self.af_local] = np.einsum("nij,nj->ni", self.Binv, r[self.af_local])
        if self.part_local.size:
            z[self.part_local] = self.pinv * r[self.part_local]
        return z


# ----------------------------------------------------------------------------
# Transfers -- solver_v2.py:62-149, :716-763 ; multigrid_v4.py:192-216, :719-748
def scalar_prolongation(nxf, nyf, nzf, nxc, nyc, nzc) -> sp.csr_matrix:
    """Trilinear P, rows normalised to one; separable per axis."""
    def axis(nf, nc):
        rows, cols, vals = [], [], []
        for f in range(nf + 1):
            cand = [f // 2] if f % 2 == 0 else [(f - 1) // 2, (f + 1) // 2]
            cand = [c for c in cand if c <= nc]
            w = 1.0 if f % 2 == 0 else 0.5
            s = w * len(cand)
            for c in cand:
                rows.append(f)
                cols.append(c)
                vals.append(w / s)
        return sp.csr_matrix((vals, (rows, cols)), shape=(nf + 1, nc + 1))
    return sp.kron(sp.kron(axis(nxf, nxc), axis(nyf, nyc)), axis(nzf, nzc), format="csr")


def coarse_free_injection(nxf, nyf, nzf, nxc, nyc, nzc, free_f) -> np.ndarray:
    ndof_f = 3 * (nxf + 1) * (nyf + 1) * (nzf + 1)
    I, J, K = (a.ravel() for a in np.meshgrid(np.arange(nxc + 1), np.arange(nyc + 1), np.arange(nzc + 1), indexing="ij"))
    fn = 2 * I * (nyf + 1) * (nzf + 1) + 2 * J * (nzf + 1) + 2 * K
    mf = np.zeros(ndof_f, bool)
    mf[free_f] = True
    out = np.zeros(3 * fn.size, bool)
    for d in range(3):
        fd = 3 * fn + d
        ok = fd < ndof_f
        out[(3 * np.arange(fn.size) + d)[ok]] = mf[fd[ok]]
    return np.where(out)[0].astype(np.int32)


def local_prolongation(s, t, u) -> np.ndarray:
    P = np.zeros((8, 8))
    for fn in range(8):
        cc = (np.array([s, t, u]) + _OFF[fn]) / 2.0
        for cn in range(8):
            P[fn, cn] = np.prod([cc[d] if _OFF[cn][d] else 1.0 - cc[d] for d in range(3)])
    return P


def level1_galerkin(nxc, nyc, nzc, nxf, nyf, nzf, free_c, E_fine) -> sp.csr_matrix:
    """multigrid_v4.py:219-361: K1 = sum over coarse elements and sub-elements stu of
    E_fine[child] * P24^T KE P24, child indices clamped to the fine grid, free-free only."""
    edc = edof_table(nxc, nyc, nzc)
    ci, cj, ck = (a.ravel() for a in np.meshgrid(np.arange(nxc), np.arange(nyc), np.arange(nzc), indexing="ij"))
    ndof_c = 3 * (nxc + 1) * (nyc + 1) * (nzc + 1)
    Ke = np.zeros((edc.shape[0], 24, 24))
    for s in range(2):
        for t in range(2):
            for u in range(2):
                P24 = np.kron(local_prolongation(s, t, u), np.eye(3))
                Q = P24.T @ KE @ P24
                fi = np.minimum(2 * ci + s, nxf - 1)
                fj = np.minimum(2 * cj + t, nyf - 1)
                fk = np.minimum(2 * ck + u, nzf - 1)
                Ke += E_fine[(fi * nyf + fj) * nzf + fk][:, None, None] * Q[None]
    rows = np.repeat(edc, 24, axis=1).ravel()
    cols = np.tile(edc, (1, 24)).ravel()
    K = sp.csr_matrix((Ke.ravel(), (rows, cols)), shape=(ndof_c, ndof_c))
    return K[free_c][:, free_c].tocsr()


# ----------------------------------------------------------------------------
# Spectral estimates -- multigrid_v4.py:364-405
def fine_lambda(op, E, d_inv, n_iter=20):
    d = 1.0 / d_inv
    v = np.ones(d_inv.size)
    v /= np.sqrt(np.dot(v * d, v))
    lam = 1.0
    for _ in range(n_iter):
        Kv = op.matvec(v, E)
        lam = float(np.dot(v, Kv)) / max(float(np.dot(v * d, v)), 1e-300)
        Av = d_inv * Kv
        nrm = float(np.sqrt(np.dot(Av * d, Av)))
        if nrm <= 1e-300:
            break
        v = Av / nrm
    return lam


def sparse_lambda(K, d_inv, n_iter=10):
    v = np.ones(d_inv.size)
    v /= float(np.linalg.norm(v))
    lam = 1.0
    for _ in range(n_iter):
        Kv = K @ v
        Av = d_inv * Kv
        nrm = float(np.linalg.norm(Av))
        if nrm <= 1e-300:
            break
        lam = float(np.dot(v, Kv)) / max(float(np.dot(v, v / d_inv)), 1e-300)
        v = Av / nrm
    return max(lam, 1e-6)


# ----------------------------------------------------------------------------
# Krylov -- multigrid_v4.py:416-534 ; solver_v2.py:551-623, :781-810
def fgmres(A, b, M, x0=None, tol=1e-6, maxiter=200, restart=32, history=None):
    x = np.zeros_like(b) if x0 is None else x0.copy()
    bn = float(np.linalg.norm(b))
    if bn <= 1e-30:
        return x, 0, True
    total, converged = 0, False
    while total < maxiter:
        r = b - A(x)
        beta = float(np.linalg.norm(r))
        if history is not None:
            history.append(beta / bn)
        if beta / bn <= tol:
            converged = True
            break
        V, Z = [r / beta], []
        H = np.zeros((restart + 1, restart))
        cs, sn, g = np.zeros(restart), np.zeros(restart), np.zeros(restart + 1)
        g[0] = beta
        jf = 0
        for j in range(min(restart, maxiter - total)):
            Z.append(M(V[j]))
            w = A(Z[j])
            for i in range(j + 1):
                H[i, j] = float(np.dot(V[i], w))
                w = w - H[i, j] * V[i]
            h = float(np.linalg.norm(w))
            H[j + 1, j] = h
            if h > 1e-14:
                V.append(w / h)
            for i in range(j):
                a, c = H[i, j], H[i + 1, j]
                H[i, j], H[i + 1, j] = cs[i] * a + sn[i] * c, -sn[i] * a + cs[i] * c
            den = math.sqrt(H[j, j] ** 2 + H[j + 1, j] ** 2)
            cs[j], sn[j] = (1.0, 0.0) if den < 1e-300 else (H[j, j] / den, H[j + 1, j] / den)
            H[j, j] = cs[j] * H[j, j] + sn[j] * H[j + 1, j]
            H[j + 1, j] = 0.0
            g[j + 1], g[j] = -sn[j] * g[j], cs[j] * g[j]
            total += 1
            jf = j + 1
            if history is not None:
                history.append(abs(g[j + 1]) / bn)
            if abs(g[j + 1]) / bn <= tol or h <= 1e-14:
                converged = True
                break
        if jf:
            R = np.triu(H[:jf, :jf])
            try:
                y = np.linalg.solve(R, g[:jf].copy())
            except np.linalg.LinAlgError:
                y = np.linalg.lstsq(R, g[:jf].copy(), rcond=None)[0]
            for c, z in zip(y, Z):
                x = x + float(c) * z
        if converged:
            break
    return x, total, converged


def pcg(A, b, M, x0=None, tol=1e-5, maxiter=1000, history=None):
    x = np.zeros_like(b) if x0 is None else x0.copy()
    r = b - A(x)
    bsq = float(np.dot(b, b))
    tsq = tol ** 2 * bsq
    r0 = float(np.dot(r, r))
    if history is not None:
        history.append((r0 / bsq) ** 0.5 if bsq > 0 else 0.0)
    if r0 <= tsq:
        return x, 0, True
    z = M(r)
    p = z.copy()
    rz = float(np.dot(r, z))
    it, conv = 1, False
    for _ in range(maxiter - 1):
        Ap = A(p)
        alpha = rz / float(np.dot(p, Ap))
        x = x + alpha * p
        r = r - alpha * Ap
        rsq = float(np.dot(r, r))
        if history is not None:
            history.append((rsq / bsq) ** 0.5 if bsq > 0 else 0.0)
        if rsq <= tsq:
            conv = True
            break
        z = M(r)
        it += 1
        rzn = float(np.dot(r, z))
        p = z + (rzn / rz) * p
        rz = rzn
    return x, it, conv


def fixed_pcg(K, b, d_inv, n_iters):
    x = np.zeros_like(b)
    r = b.copy()
    z = d_inv * r
    p = z.copy()
    rz = r.dot(z)
    for _ in range(n_iters):
        Ap = K @ p
        alpha = rz / (p.dot(Ap) + 1e-300)
        x = x + alpha * p
        r = r - alpha * Ap
        z = d_inv * r
        rzn = r.dot(z)
        p = z + (rzn / (rz + 1e-300)) * p
        rz = rzn
    return x


def _bf16_round(x: np.ndarray) -> np.ndarray:
    """float32 -> bfloat16 (round to nearest, ties to even) -> float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    return ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32).view(np.float32)


def fused_matvec_full(nx: int, ny: int, nz: int, u_full: np.ndarray, E: np.ndarray, ke: np.ndarray,
                      dtype: str = "fp32") -> np.ndarray:
    """The reference's FusedMatvec arithmetic (gpu_fem/cuda_fused_matvec.py:41-88
    FP32, :112-246 BF16 WMMA, :343-416 wrapper): per element f_e = KE u_e with u and
    KE cast to float32 (and, for "bf16", rounded to bfloat16), times E_e (float32),
    scatter-added into every DOF of the full vector.  Evaluated in float64 here;
    the kernels accumulate in float32."""
    edof = edof_table(nx, ny, nz)
    u32 = np.asarray(u_full, dtype=np.float32)
    k32 = np.asarray(ke, dtype=np.float32)
    if dtype == "bf16":
        u32, k32 = _bf16_round(u32), _bf16_round(k32)
    elif dtype != "fp32":
        raise ValueError(dtype)
    U = u32.astype(np.float64)[edof]
    F = U @ k32.astype(np.float64).T
    F *= np.asarray(E, dtype=np.float32).astype(np.float64)[:, None]
    return np.bincount(edof.ravel(), weights=F.ravel(), minlength=u32.size)
