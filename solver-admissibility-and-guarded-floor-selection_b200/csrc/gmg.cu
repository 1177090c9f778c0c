// Host-side orchestration of the simpfem hot path: mesh state, the Galerkin
// multigrid hierarchy (setup, V/W-cycle, safeguarded corrections, inner Krylov
// wrappers) and the device-resident FGMRES / PCG drivers.
//
// Reference behaviour followed here (file:line in the reference project):
//   GalerkinMatFreeGMG.__init__ / setup      gpu_fem/multigrid_v4.py:546-770, :1119-1341
//   lambda_max cache and estimators          gpu_fem/multigrid_v4.py:1175-1188, :364-405
//   contrast-adaptive smoothing               gpu_fem/multigrid_v4.py:1190-1239
//   _chebyshev_steps / _smooth_fine / _coarse gpu_fem/multigrid_v4.py:1783-1906
//   _solve_coarsest / _vcycle / _wcycle       gpu_fem/multigrid_v4.py:1908-2024
//   corrections (line search, root-local)     gpu_fem/multigrid_v4.py:867-1055
//   apply / inner Krylov                      gpu_fem/multigrid_v4.py:1742-1767
//   _cupy_fgmres                              gpu_fem/multigrid_v4.py:416-534
//   _cupy_pcg / _fixed_pcg_coarse             gpu_fem/solver_v2.py:551-623, :781-810
// Every scalar decision of the reference's host-side Python (line-search scale,
// acceptance tests, Givens rotations, breakdown) runs in single-thread device
// kernels, so a preconditioner apply is a fixed kernel sequence with no host
// synchronisation.
#include <math.h>
#include <stdio.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <tuple>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "gmg_impl.h"

namespace simpfem {

static thread_local std::string g_err;
void set_error(const std::string& m) { g_err = m; }
const char* last_error() { return g_err.c_str(); }


// ----------------------------------------------------------------------------


static size_t dsize(DType t) { return t == F64 ? 8 : (t == F32 ? 4 : 2); }

// ----------------------------------------------------------------------------
// Local node order of the reference element (gpu_fem/pub_simp_solver.py:196-207):
// reference node a sits at offset kRefPos[a]; our corner index is q = dx*4+dy*2+dz.
static const int kRefPos[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                  {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
static int ref_of_corner(int q) {
  const int dx = q >> 2, dy = (q >> 1) & 1, dz = q & 1;
  for (int a = 0; a < 8; ++a)
    if (kRefPos[a][0] == dx && kRefPos[a][1] == dy && kRefPos[a][2] == dz) return a;
  return -1;
}

// Walsh-basis blocks of the unit stiffness (see fine.cu).
WhtBlocks make_wht_blocks(const double* ke, double* max_off) {
  double kem[24][24];
  for (int q = 0; q < 8; ++q)
    for (int c = 0; c < 3; ++c)
      for (int q2 = 0; q2 < 8; ++q2)
        for (int c2 = 0; c2 < 3; ++c2)
          kem[q * 3 + c][q2 * 3 + c2] = ke[(3 * ref_of_corner(q) + c) * 24 + 3 * ref_of_corner(q2) + c2];
  auto W = [](int s, int q) { return (__builtin_popcount(s & q) & 1) ? -1.0 : 1.0; };
  static double M[24][24];
  double mx = 0.0;
  for (int s = 0; s < 8; ++s)
    for (int c = 0; c < 3; ++c)
      for (int s2 = 0; s2 < 8; ++s2)
        for (int c2 = 0; c2 < 3; ++c2) {
          double acc = 0.0;
          for (int q = 0; q < 8; ++q)
            for (int q2 = 0; q2 < 8; ++q2) acc += W(s, q) * kem[q * 3 + c][q2 * 3 + c2] * W(s2, q2);
          M[s * 3 + c][s2 * 3 + c2] = acc / 64.0;
          mx = std::max(mx, fabs(acc / 64.0));
        }
  const int e[3] = {4, 2, 1};
  WhtBlocks wb;
  bool inblock[24][24] = {};
  for (int b = 0; b < 8; ++b)
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) {
        const int row = (b ^ e[r]) * 3 + r, col = (b ^ e[c]) * 3 + c;
        wb.b[b][r * 3 + c] = M[row][col];
        inblock[row][col] = true;
      }
  double off = 0.0;
  for (int i = 0; i < 24; ++i)
    for (int j = 0; j < 24; ++j)
      if (!inblock[i][j]) off = std::max(off, fabs(M[i][j]));
  *max_off = mx > 0 ? off / mx : 0.0;
  return wb;
}

// Q_stu = P24(stu)^T KE P24(stu) with the local trilinear prolongation of
// gpu_fem/multigrid_v4.py:192-216, returned in corner-major order
// Q[stu][(a*3+r)*24 + b*3+c] (a, b coarse-element corners).
std::vector<double> make_level1_Q(const double* ke) {
  std::vector<double> Q(8 * 576);
  for (int stu = 0; stu < 8; ++stu) {
    const int s = stu >> 2, t = (stu >> 1) & 1, u = stu & 1;
    double P[8][8];  // reference order: P[fine local node][coarse local node]
    for (int fn = 0; fn < 8; ++fn) {
      const double cc[3] = {(s + kRefPos[fn][0]) / 2.0, (t + kRefPos[fn][1]) / 2.0,
                            (u + kRefPos[fn][2]) / 2.0};
      for (int cn = 0; cn < 8; ++cn) {
        double w = 1.0;
        for (int d = 0; d < 3; ++d) w *= kRefPos[cn][d] == 0 ? (1.0 - cc[d]) : cc[d];
        P[fn][cn] = w;
      }
    }
    // Qref = P24^T KE P24, P24 = kron(P, I3)
    static double KP[24][24], Qr[24][24];
    for (int i = 0; i < 24; ++i)
      for (int j = 0; j < 24; ++j) {
        double acc = 0.0;
        const int cn = j / 3, c = j % 3;
        for (int fn = 0; fn < 8; ++fn) acc += ke[i * 24 + fn * 3 + c] * P[fn][cn];
        KP[i][j] = acc;
      }
    for (int i = 0; i < 24; ++i)
      for (int j = 0; j < 24; ++j) {
        double acc = 0.0;
        const int cn = i / 3, c = i % 3;
        for (int fn = 0; fn < 8; ++fn) acc += P[fn][cn] * KP[fn * 3 + c][j];
        Qr[i][j] = acc;
      }
    for (int a = 0; a < 8; ++a)
      for (int r = 0; r < 3; ++r)
        for (int b = 0; b < 8; ++b)
          for (int c = 0; c < 3; ++c)
            Q[(size_t)stu * 576 + (a * 3 + r) * 24 + b * 3 + c] =
                Qr[3 * ref_of_corner(a) + r][3 * ref_of_corner(b) + c];
  }
  return Q;
}

// 1-D row-normalised trilinear weights fine(nf elements) <- coarse(nc elements):
// w[3*f + (f - 2*c + 1)] (gpu_fem/solver_v2.py:62-149, separable per axis).
static std::vector<double> make_w1(int nf, int nc) {
  std::vector<double> w(3 * (nf + 1), 0.0);
  for (int f = 0; f <= nf; ++f) {
    double raw[3] = {0, 0, 0};
    double sum = 0.0;
    for (int d = 0; d < 3; ++d) {
      // d = f - 2c + 1  ->  c = (f + 1 - d) / 2
      const int num = f + 1 - d;
      if (num % 2 != 0) continue;
      const int c = num / 2;
      if (c < 0 || c > nc) continue;
      double v;
      if (f % 2 == 0)
        v = (c * 2 == f) ? 1.0 : 0.0;
      else
        v = 0.5;
      raw[d] = v;
      sum += v;
    }
    const double scale = sum > 1e-12 ? 1.0 / sum : 1.0;
    for (int d = 0; d < 3; ++d) w[3 * f + d] = raw[d] * scale;
  }
  return w;
}

// ----------------------------------------------------------------------------

SweepShape default_shape(const Grid& g, int maxt) {
  SweepShape s;
  const int full_k = g.nz + 2;
  if (full_k <= 64 && full_k * 2 <= maxt) {
    s.bk = full_k;
  } else {
    s.bk = 32;
  }
  s.bj = std::max(2, std::min(maxt / s.bk, g.ny + 2));
  s.cx = 8;
  return s;
}

void fine_apply(Mesh& m, DType t, Epi epi, const void* E, const void* u, const EpiArgs& ea,
                       cudaStream_t s) {
  const SweepShape& sh = m.sh[t == F64 ? 0 : 1];
  SF_CUDA(launch_fine(t, epi, m.g, sh, E, m.mask.as<uint8_t>(), u, ea, s));
}

// Tuner: time candidate sweep shapes on this mesh and keep the fastest.  The
// choice is cached per process by grid size and precision, so every mesh of a
// size runs the same kernels (identical results across handles, and handles
// tuned while other streams are busy cannot pick a different shape).
static std::mutex g_tune_mutex;
static std::map<std::tuple<int, int, int, int>, SweepShape> g_tuned;

void tune_mesh(Mesh& m, DType t, cudaStream_t s) {
  const int idx = t == F64 ? 0 : 1;
  if (m.tuned[idx]) return;
  std::lock_guard<std::mutex> lk(g_tune_mutex);
  const auto key = std::make_tuple(m.g.nx, m.g.ny, m.g.nz, idx);
  const auto hit = g_tuned.find(key);
  if (hit != g_tuned.end()) {
    m.sh[idx] = hit->second;
    m.tuned[idx] = true;
    return;
  }
  const int maxt = t == F64 ? 256 : 512;
  const size_t es = dsize(t == BF16 ? F32 : t);
  DevBuf E, u, y;
  E.alloc(es * std::max<int64_t>(1, m.g.ne()));
  u.alloc(es * m.g.ndof);
  y.alloc(es * m.g.ndof);
  SF_CUDA(launch_fill_hash(t == F64 ? F64 : F32, m.g.ndof, 7u, u.p, s));
  SF_CUDA(launch_fill(t == F64 ? F64 : F32, m.g.ne(), 1.0, E.p, nullptr, s));
  std::vector<SweepShape> cands;
  std::vector<int> bks;
  if (m.g.nz + 2 <= 64) bks.push_back(m.g.nz + 2);
  for (int bk : {16, 32, 64})
    if (bk < m.g.nz + 2) bks.push_back(bk);
  for (int bk : bks)
    for (int nt : {128, 256, maxt}) {
      const int bj = nt / bk;
      if (bj < 2 || bj * bk > maxt) continue;
      for (int cx : {4, 6, 8, 10, 12, 14, 16, 20}) {  // fine steps: the wave count depends on it
        SweepShape sh;
        sh.bj = bj;
        sh.bk = bk;
        sh.cx = cx;
        cands.push_back(sh);
        // FP32: also the one-element-per-thread sweep (twice the threads of the packed
        // sweep for the same tile) and the packed sweep with a register cap (more
        // resident blocks); on grids too small to fill the GPU either can hide more
        // latency than the packed sweep
        if (t == F32) {
          for (int v : {1, 2}) {
            sh.variant = v;
            cands.push_back(sh);
          }
        }
      }
    }
  cudaEvent_t e0, e1;
  SF_CUDA(cudaEventCreate(&e0));
  SF_CUDA(cudaEventCreate(&e1));
  float best = 1e30f;
  SweepShape best_sh = default_shape(m.g, maxt);
  // SIMPFEM_TUNE_VERBOSE=1 prints every candidate's time (stderr)
  const char* vb = getenv("SIMPFEM_TUNE_VERBOSE");
  const bool verbose = vb != nullptr && vb[0] != '\0' && vb[0] != '0';
  EpiArgs ea;
  ea.y = y.p;
  for (const SweepShape& sh : cands) {
    cudaError_t err = launch_fine(t, EPI_APPLY, m.g, sh, E.p, m.mask.as<uint8_t>(), u.p, ea, s);
    if (err != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    SF_CUDA(cudaEventRecord(e0, s));
    for (int r = 0; r < 3; ++r)
      SF_CUDA(launch_fine(t, EPI_APPLY, m.g, sh, E.p, m.mask.as<uint8_t>(), u.p, ea, s));
    SF_CUDA(cudaEventRecord(e1, s));
    SF_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    SF_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (verbose)
      fprintf(stderr, "[simpfem tune] %s %dx%dx%d bj=%d bk=%d cx=%d variant=%d: %.1f us\n",
              t == F64 ? "f64" : "f32", m.g.nx, m.g.ny, m.g.nz, sh.bj, sh.bk, sh.cx, sh.variant, ms * 1000.f / 3.f);
    if (ms < best) {
      best = ms;
      best_sh = sh;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  m.sh[idx] = best_sh;
  m.tuned[idx] = true;
  g_tuned[key] = best_sh;
}

// ----------------------------------------------------------------------------
// Device FGMRES workspace (one per FGMRES instance).

// ----------------------------------------------------------------------------


// ----------------------------------------------------------------------------
// Level construction (GalerkinMatFreeGMG.__init__): dims by max(1, n // 2), free
// DOFs by injection (gpu_fem/solver_v2.py:716-763, linear-index arithmetic kept).
static std::vector<uint8_t> injection_mask(const Grid& gf, const std::vector<uint8_t>& mf, const Grid& gc) {
  std::vector<uint8_t> mc(gc.ndof, 0);
  const int64_t nyf = gf.ny + 1, nzf = gf.nz + 1;
  for (int I = 0; I <= gc.nx; ++I)
    for (int J = 0; J <= gc.ny; ++J)
      for (int K = 0; K <= gc.nz; ++K) {
        const int64_t fine_node = 2LL * I * nyf * nzf + 2LL * J * nzf + 2LL * K;
        const int64_t cn = ((int64_t)I * (gc.ny + 1) + J) * (gc.nz + 1) + K;
        for (int d = 0; d < 3; ++d) {
          const int64_t fd = 3 * fine_node + d;
          if (fd < gf.ndof) mc[3 * cn + d] = mf[fd];
        }
      }
  return mc;
}

static void alloc_level_vectors(Gmg& G, Level& L, bool need_fp32_scratch) {
  const size_t vs = dsize(G.cyc) * L.g.ndof;
  for (int i = 0; i < 2; ++i) L.x[i].alloc(vs);
  L.res.alloc(vs);
  L.c.alloc(vs);
  L.Ac.alloc(vs);
  L.d.alloc(vs);
  L.rhs.alloc(vs);
  L.trial.alloc(vs);
  L.res2.alloc(vs);
  L.ptmp.alloc(vs);
  if (need_fp32_scratch) {
    for (int i = 0; i < 2; ++i) L.xs[i].alloc(4 * L.g.ndof);
    L.ds.alloc(4 * L.g.ndof);
    L.rhss.alloc(4 * L.g.ndof);
  }
}

Gmg* gmg_create(Mesh* m, const simpfem_gmg_opts& o) {
  auto G = std::make_unique<Gmg>();
  G->m = m;
  G->o = o;
  G->L = std::max(1, o.n_levels);
  if (G->L > 8) throw InvalidArg{"n_levels must be <= 8"};
  G->cyc = (o.cycle_precision == SIMPFEM_F32) ? F32 : F64;
  G->omega_used = o.omega;
  G->fine_deg = std::max(1, o.fine_smoother_degree);
  G->coarse_iters = o.coarse_smooth_iters;
  G->lv.resize(G->L);
  G->lv[0].g = m->g;
  G->lv[0].mask_h = m->mask_h;
  for (int l = 1; l < G->L; ++l) {
    const Grid& gf = G->lv[l - 1].g;
    G->lv[l].g = Grid::make(std::max(1, gf.nx / 2), std::max(1, gf.ny / 2), std::max(1, gf.nz / 2));
    G->lv[l].mask_h = injection_mask(gf, G->lv[l - 1].mask_h, G->lv[l].g);
  }
  for (int l = 0; l < G->L; ++l) {
    Level& L = G->lv[l];
    L.n_free = 0;
    for (uint8_t b : L.mask_h) L.n_free += b;
    L.mask.alloc(L.g.ndof);
    SF_CUDA(cudaMemcpy(L.mask.p, L.mask_h.data(), L.g.ndof, cudaMemcpyHostToDevice));
    if (l + 1 < G->L) {
      const Grid& gc = G->lv[l + 1].g;
      auto wx = make_w1(L.g.nx, gc.nx), wy = make_w1(L.g.ny, gc.ny), wz = make_w1(L.g.nz, gc.nz);
      L.wx.alloc(8 * wx.size());
      L.wy.alloc(8 * wy.size());
      L.wz.alloc(8 * wz.size());
      SF_CUDA(cudaMemcpy(L.wx.p, wx.data(), 8 * wx.size(), cudaMemcpyHostToDevice));
      SF_CUDA(cudaMemcpy(L.wy.p, wy.data(), 8 * wy.size(), cudaMemcpyHostToDevice));
      SF_CUDA(cudaMemcpy(L.wz.p, wz.data(), 8 * wz.size(), cudaMemcpyHostToDevice));
    }
    alloc_level_vectors(*G, L, G->cyc == F64);
    if (l >= 1) {
      L.K64.alloc(sizeof(double) * 243 * L.g.nn);
      L.dinv64.alloc(sizeof(double) * L.g.ndof);
      L.s64a.alloc(sizeof(double) * L.g.ndof);
      L.s64b.alloc(sizeof(double) * L.g.ndof);
      L.s64c.alloc(sizeof(double) * L.g.ndof);
    }
  }
  // coarsest compact index
  if (G->L > 1) {
    const Level& C = G->lv[G->L - 1];
    std::vector<int32_t> idx, didx(C.g.ndof, -1);
    for (int64_t d = 0; d < C.g.ndof; ++d)
      if (C.mask_h[d]) {
        didx[d] = (int32_t)idx.size();
        idx.push_back((int32_t)d);
      }
    G->nc = (int)idx.size();
    // the dense coarsest matrix's structural lower bandwidth: the widest reach
    // of the 27-point stencil in the compact (order-preserving) numbering; its
    // values can only be zero farther out, so the factorisation needs no scan
    {
      const int NY = C.g.ny + 1, NZ = C.g.nz + 1;
      int bw = 0;
      for (int64_t d = 0; d < C.g.ndof; ++d) {
        if (didx[d] < 0) continue;
        const int64_t node = d / 3;
        const int k = (int)(node % NZ), j = (int)((node / NZ) % NY), i = (int)(node / ((int64_t)NZ * NY));
        for (int o = 0; o < 27; ++o) {
          const int mi = i + o / 9 - 1, mj = j + (o / 3) % 3 - 1, mk = k + o % 3 - 1;
          if (mi < 0 || mj < 0 || mk < 0 || mi > C.g.nx || mj > C.g.ny || mk > C.g.nz) continue;
          const int64_t m = ((int64_t)mi * NY + mj) * NZ + mk;
          for (int c = 0; c < 3; ++c) {
            const int32_t q = didx[3 * m + c];
            if (q >= 0) bw = std::max(bw, didx[d] - q);
          }
        }
      }
      G->c_bw = bw;
    }
    G->c_idx.alloc(4 * std::max<size_t>(1, idx.size()));
    G->c_didx.alloc(4 * didx.size());
    if (!idx.empty()) SF_CUDA(cudaMemcpy(G->c_idx.p, idx.data(), 4 * idx.size(), cudaMemcpyHostToDevice));
    SF_CUDA(cudaMemcpy(G->c_didx.p, didx.data(), 4 * didx.size(), cudaMemcpyHostToDevice));
    G->cb.alloc(8 * std::max(1, G->nc));
    G->cx.alloc(8 * std::max(1, G->nc));
    G->ctmp.alloc(8 * std::max(1, G->nc));
    G->cinfo.alloc(16);
  }
  const int64_t n = m->g.ndof;
  G->Qdev.alloc(8 * m->Q.size());
  SF_CUDA(cudaMemcpy(G->Qdev.p, m->Q.data(), 8 * m->Q.size(), cudaMemcpyHostToDevice));
  G->E64.alloc(8 * std::max<int64_t>(1, m->g.ne()));
  G->E32.alloc(4 * std::max<int64_t>(1, m->g.ne()));
  G->diag0.alloc(8 * n);
  G->lv[0].dinv64.alloc(8 * n);
  G->lv[0].dinv32.alloc(4 * n);
  G->sc.alloc(8 * 32);
  G->rhs64.alloc(8 * n);
  G->out64.alloc(8 * n);
  G->tmp64a.alloc(8 * n);
  G->tmp64b.alloc(8 * n);
  G->tmp64c.alloc(8 * n);
  G->tmp64d.alloc(8 * n);
  if (G->cyc == F32) {
    G->cyc_in.alloc(4 * n);
    G->cyc_out.alloc(4 * n);
  }
  return G.release();
}

// ----------------------------------------------------------------------------
// Operator helpers
static const void* fine_E(Gmg& G, DType t) { return t == F64 ? G.E64.p : G.E32.p; }

// level operator in the vector dtype vt, coefficient storage chosen by prec
void level_op(Gmg& G, int l, DType vt, int precsel, Epi epi, const void* u, EpiArgs ea) {
  ea.guard = G.guard;
  if (l == 0) {
    DType ft = vt;
    if (vt == F32 && precsel == BF16) ft = BF16;
    fine_apply(*G.m, ft, epi, fine_E(G, vt), u, ea, G.st);
    return;
  }
  Level& L = G.lv[l];
  DType ct = F64;
  const void* coef = L.K64.p;
  if (vt == F32) {
    if (precsel == BF16 && L.K16.p) {
      // BF16 copy node-major by neighbour column, nine lanes per node
      SF_CUDA(launch_stencil_col_bf16(epi, L.g, L.K16.as<__nv_bfloat16>(), L.mask.as<uint8_t>(), (const float*)u,
                                      ea, G.st));
      return;
    } else {
      ct = F32;
      coef = L.K32.p;
    }
  }
  SF_CUDA(launch_stencil(vt, ct, epi, L.g, coef, L.mask.as<uint8_t>(), u, ea, G.st));
}

const void* level_dinv(Gmg& G, int l, DType t) {
  return t == F64 ? G.lv[l].dinv64.p : G.lv[l].dinv32.p;
}

static void dots(Gmg& G, DType t, int64_t n, const DotSet& ds, double* out, const int* guard) {
  SF_CUDA(launch_dots(t, n, ds, G.m->rw, out, guard, G.st));
}

// ----------------------------------------------------------------------------
// Smoothers
struct ChebCoefs {
  double alpha0;
  std::vector<double> s1, s2;
};

static ChebCoefs cheb_coefs(double lm, double lf, int degree, bool f32) {
  ChebCoefs c;
  c.s1.assign(std::max(degree, 1), 0.0);
  c.s2.assign(std::max(degree, 1), 0.0);
  if (f32) {
    const float lm32 = (float)lm, lf32 = (float)lf;
    const float lmin = lf32 * lm32;
    const float sigma = (lm32 + lmin) * 0.5f;
    const float delta = (lm32 - lmin) * 0.5f;
    float alpha = 2.0f / (lm32 + lmin);
    c.alpha0 = alpha;
    for (int k = 1; k < degree; ++k) {
      const float d2 = delta * delta;
      const float cc = d2 * alpha * 0.25f;
      const float an = 1.0f / (sigma - cc);
      c.s1[k] = an;
      c.s2[k] = cc;
      alpha = an;
    }
  } else {
    const double lmin = lf * lm;
    const double sigma = (lm + lmin) * 0.5;
    const double delta = (lm - lmin) * 0.5;
    double alpha = 2.0 / (lm + lmin);
    c.alpha0 = alpha;
    for (int k = 1; k < degree; ++k) {
      const double d2 = delta * delta;
      const double cc = d2 * alpha * 0.25;
      const double an = 1.0 / (sigma - cc);
      c.s1[k] = an;
      c.s2[k] = cc;
      alpha = an;
    }
  }
  return c;
}

// Runs `steps` smoothing steps of the level-l operator in dtype t.  x0 null =>
// zero initial guess.  xa / xb are the ping-pong buffers; returns the result buffer.
static void* run_smoother(Gmg& G, int l, DType t, int precsel, const void* rhs, const void* x0, void* xa,
                          void* xb, void* d, const void* dinv, double lm, double lf, int steps) {
  const int64_t n = G.lv[l].g.ndof;
  const bool f32 = (t == F32);
  void* cur = nullptr;
  void* nxt = xa;
  if (G.o.smoother_type == 0) {
    const ChebCoefs cc = cheb_coefs(lm, lf, steps, f32);
    for (int k = 0; k < steps; ++k) {
      EpiArgs ea;
      ea.b = rhs;
      ea.dinv = dinv;
      ea.d = d;
      if (k == 0) {
        if (x0 == nullptr) {
          SF_CUDA(launch_cheb_zero(t, n, cc.alpha0, dinv, rhs, d, nxt, G.guard, G.st));
        } else {
          ea.xo = nxt;
          ea.s1 = cc.alpha0;
          level_op(G, l, t, precsel, EPI_CHEB1, x0, ea);
        }
      } else {
        ea.xo = nxt;
        ea.s1 = cc.s1[k];
        ea.s2 = cc.s2[k];
        level_op(G, l, t, precsel, EPI_CHEB, cur, ea);
      }
      cur = nxt;
      nxt = (cur == xa) ? xb : xa;
    }
  } else {
    // damped Jacobi: x <- x + (omega * dinv) * (rhs - A x)
    const double om = f32 ? (double)(float)G.omega_used : G.omega_used;
    for (int k = 0; k < steps; ++k) {
      if (k == 0 && x0 == nullptr) {
        SF_CUDA(launch_jac_zero(t, n, om, dinv, rhs, nxt, G.guard, G.st));
      } else {
        EpiArgs ea;
        ea.b = rhs;
        ea.dinv = dinv;
        ea.xo = nxt;
        ea.s1 = om;
        level_op(G, l, t, precsel, EPI_JAC, k == 0 ? x0 : cur, ea);
      }
      cur = nxt;
      nxt = (cur == xa) ? xb : xa;
    }
  }
  return cur;
}

// smooth at level l; x_in null => zero initial guess; result in one of lv[l].x
void* smooth(Gmg& G, int l, const void* rhs, const void* x_in) {
  Level& L = G.lv[l];
  const int64_t n = L.g.ndof;
  double lm, lf = G.o.cheb_lower_frac;
  if (G.high) lf = std::min(G.o.cheb_lower_frac, 1.0 / 100.0);
  int steps;
  if (l == 0) {
    lm = G.lv[0].lam;
    steps = G.fine_deg;
  } else {
    lm = std::isfinite(L.lam) ? L.lam : 1.0;
    steps = G.coarse_iters;
  }
  const int p = G.prec[l];
  // output buffer that is not x_in
  void* xa = (x_in == L.x[0].p) ? L.x[1].p : L.x[0].p;
  void* xb = (x_in == L.x[0].p) ? L.x[0].p : L.x[1].p;
  if (G.cyc == F32) {
    return run_smoother(G, l, F32, p, rhs, x_in, xa, xb, L.d.p, level_dinv(G, l, F32), lm, lf, steps);
  }
  // reference mode: FP64 vectors; FP32 / BF16 smoothing on cast copies
  const bool low = (l == 0) ? (p == F32 || p == BF16) : (p == F32 && L.K32.p != nullptr);
  if (!low) {
    return run_smoother(G, l, F64, F64, rhs, x_in, xa, xb, L.d.p, level_dinv(G, l, F64), lm, lf, steps);
  }
  SF_CUDA(launch_convert(F64, F32, rhs, L.rhss.p, n, G.guard, G.st));
  const void* x0 = nullptr;
  if (x_in != nullptr) {
    SF_CUDA(launch_convert(F64, F32, x_in, L.xs[1].p, n, G.guard, G.st));
    x0 = L.xs[1].p;
  }
  void* r = run_smoother(G, l, F32, p, L.rhss.p, x0, L.xs[0].p, L.xs[1].p, L.ds.p,
                         level_dinv(G, l, F32), lm, lf, steps);
  SF_CUDA(launch_convert(F32, F64, r, xa, n, G.guard, G.st));
  return xa;
}

// ----------------------------------------------------------------------------
// Coarsest solve (dense via explicit Cholesky inverse factor, or fixed Jacobi-PCG)
static void fixed_pcg_coarse(Gmg& G, int l, const double* b, double* x);

void solve_coarsest(Gmg& G, const void* rhs, void* x) {
  const int l = G.L - 1;
  Level& L = G.lv[l];
  const int64_t n = L.g.ndof;
  if (G.L == 1) {
    void* r = smooth(G, 0, rhs, nullptr);
    if (r != x) SF_CUDA(launch_copy(G.cyc, n, r, x, G.guard, G.st));
    return;
  }
  const double* b64 = (const double*)rhs;
  double* x64 = (double*)x;
  if (G.cyc == F32) {
    SF_CUDA(launch_convert(F32, F64, rhs, G.tmp64a.p, n, G.guard, G.st));
    b64 = G.tmp64a.as<double>();
    x64 = G.tmp64b.as<double>();
  }
  if (G.coarse_mode == 1) {
    SF_CUDA(launch_gather_idx(G.nc, G.c_idx.as<int32_t>(), b64, G.cb.as<double>(), G.guard, G.st));
    if (G.cyc == F32 && G.LinvF.p)
      SF_CUDA(launch_coarsest_solve_f32(G.LinvF.as<float>(), G.LinvTF.as<float>(), G.nc, G.cb.as<double>(),
                                        G.ctmp.as<double>(), G.cx.as<double>(), G.guard, G.st));
    else
      SF_CUDA(launch_coarsest_solve(G.Linv.as<double>(), G.LinvT.as<double>(), G.nc, G.cb.as<double>(),
                                    G.ctmp.as<double>(), G.cx.as<double>(), G.guard, G.st));
    SF_CUDA(launch_fill(F64, n, 0.0, x64, G.guard, G.st));
    SF_CUDA(launch_scatter_idx(G.nc, G.c_idx.as<int32_t>(), G.cx.as<double>(), x64, G.guard, G.st));
  } else {
    fixed_pcg_coarse(G, l, b64, x64);
  }
  if (G.cyc == F32) SF_CUDA(launch_convert(F64, F32, x64, x, n, G.guard, G.st));
}

// ----------------------------------------------------------------------------
// Coarse correction at level l: x <- x + s c (line search) ; corrected residual
// in `res_out` when non-null.
void coarse_correction(Gmg& G, int l, void* x, const void* res, const void* c, void* res_out) {
  Level& L = G.lv[l];
  const int64_t n = L.g.ndof;
  const DType t = G.cyc;
  // the reference applies the correction operator in FP64 (the level's FP64 matrix)
  const int psel = (t == F32) ? G.prec[l] : F64;
  if (G.o.coarse_correction_policy == 0) {
    SF_CUDA(launch_axpby(t, n, 1.0, x, 1.0, c, x, G.guard, G.st));
    if (res_out) {
      EpiArgs ea;
      ea.y = L.Ac.p;
      level_op(G, l, t, psel, EPI_APPLY, c, ea);
      SF_CUDA(launch_axpby(t, n, 1.0, res, -1.0, L.Ac.p, res_out, G.guard, G.st));
    }
    return;
  }
  double* sc = G.sc.as<double>();
  DotSet d1;
  d1.a[0] = c; d1.b[0] = c;
  d1.a[1] = res; d1.b[1] = res;
  d1.nd = 2;
  dots(G, t, n, d1, sc + 0, G.guard);
  EpiArgs ea;
  ea.y = L.Ac.p;
  level_op(G, l, t, psel, EPI_APPLY, c, ea);
  DotSet d2;
  d2.a[0] = L.Ac.p; d2.b[0] = L.Ac.p;
  d2.a[1] = res; d2.b[1] = L.Ac.p;
  d2.nd = 2;
  dots(G, t, n, d2, sc + 2, G.guard);
  SF_CUDA(launch_scalar_op(OP_LS1, sc, 0.0, G.o.coarse_correction_max_scale, G.guard, G.st));
  SF_CUDA(launch_trial_residual(t, n, res, L.Ac.p, sc, 0, L.trial.p, G.m->rw, G.guard, G.st));
  SF_CUDA(launch_scalar_op(OP_LS2, sc, G.o.coarse_correction_acceptance_ratio, 0.0, G.guard, G.st));
  SF_CUDA(launch_select_axpy(t, n, x, c, sc, 0, G.guard, G.st));
  if (res_out) SF_CUDA(launch_select_vec(t, n, L.trial.p, res, sc, res_out, G.guard, G.st));
}

// root enrichment right-hand side at level 0 (multigrid_v4.py:938-962)
void enrichment_rhs(Gmg& G, const void* residual, void* rc_out) {
  Level& L0 = G.lv[0];
  Level& L1 = G.lv[1];
  const int64_t n = L0.g.ndof;
  const int mode = G.o.root_enrichment_mode;
  const int kmode = (mode == 1) ? 0 : (mode == 2) ? 2 : (mode == 3) ? 1 : 3;
  const double* r64 = (const double*)residual;
  if (G.cyc == F32) {
    SF_CUDA(launch_convert(F32, F64, residual, G.tmp64c.p, n, G.guard, G.st));
    r64 = G.tmp64c.as<double>();
  }
  const double* proj = nullptr;
  if (kmode >= 2) {
    // projector = P (R residual)
    SF_CUDA(launch_restrict(F64, L0.g, L1.g, L0.wx.as<double>(), L0.wy.as<double>(), L0.wz.as<double>(),
                            L1.mask.as<uint8_t>(), r64, G.tmp64a.p, G.guard, G.st));
    SF_CUDA(launch_prolong(F64, L0.g, L1.g, L0.wx.as<double>(), L0.wy.as<double>(), L0.wz.as<double>(),
                           L0.mask.as<uint8_t>(), G.tmp64a.p, G.tmp64b.p, G.guard, G.st));
    proj = G.tmp64b.as<double>();
  }
  SF_CUDA(launch_enrich_rhs(n, kmode, G.wenrich.as<double>(), G.o.root_enrichment_weight_floor, r64, proj,
                            L0.mask.as<uint8_t>(), G.tmp64a.as<double>(), G.guard, G.st));
  if (G.cyc == F32) {
    SF_CUDA(launch_convert(F64, F32, G.tmp64a.p, L0.ptmp.p, n, G.guard, G.st));
    SF_CUDA(launch_restrict(F32, L0.g, L1.g, L0.wx.as<double>(), L0.wy.as<double>(), L0.wz.as<double>(),
                            L1.mask.as<uint8_t>(), L0.ptmp.p, rc_out, G.guard, G.st));
  } else {
    SF_CUDA(launch_restrict(F64, L0.g, L1.g, L0.wx.as<double>(), L0.wy.as<double>(), L0.wz.as<double>(),
                            L1.mask.as<uint8_t>(), G.tmp64a.p, rc_out, G.guard, G.st));
  }
}

static void* cycle(Gmg& G, int l, const void* rhs);

// one coarse visit: restrict `res`, recurse, prolong into lv[l].c
static void coarse_visit(Gmg& G, int l, const void* res, bool restrict_given) {
  Level& L = G.lv[l];
  Level& C = G.lv[l + 1];
  const DType t = G.cyc;
  if (!restrict_given)
    SF_CUDA(launch_restrict(t, L.g, C.g, L.wx.as<double>(), L.wy.as<double>(), L.wz.as<double>(),
                            C.mask.as<uint8_t>(), res, C.rhs.p, G.guard, G.st));
  void* e = cycle(G, l + 1, C.rhs.p);
  SF_CUDA(launch_prolong(t, L.g, C.g, L.wx.as<double>(), L.wy.as<double>(), L.wz.as<double>(),
                         L.mask.as<uint8_t>(), e, L.c.p, G.guard, G.st));
}

// V-cycle (cycle_type 0) or W-cycle (1) at level l; returns the buffer with x.
static void* cycle(Gmg& G, int l, const void* rhs) {
  Level& L = G.lv[l];
  const int64_t n = L.g.ndof;
  const DType t = G.cyc;
  if (l == G.L - 1) {
    solve_coarsest(G, rhs, L.x[0].p);
    return L.x[0].p;
  }
  const int rsel = (t == F32) ? G.prec[l] : F64;  // residual operator precision
  void* x = smooth(G, l, rhs, nullptr);
  {
    EpiArgs ea;
    ea.y = L.res.p;
    ea.b = rhs;
    level_op(G, l, t, rsel, EPI_RESID, x, ea);
  }
  const bool enrich = (l == 0 && G.o.root_enrichment_mode != 0 && G.L > 1);
  if (G.o.cycle_type == 0) {
    coarse_visit(G, l, L.res.p, false);
    coarse_correction(G, l, x, L.res.p, L.c.p, enrich ? L.res2.p : nullptr);
    if (enrich) {
      enrichment_rhs(G, L.res2.p, G.lv[1].rhs.p);
      coarse_visit(G, l, nullptr, true);
      coarse_correction(G, l, x, L.res2.p, L.c.p, nullptr);
    }
  } else {
    coarse_visit(G, l, L.res.p, false);
    if (G.o.coarse_correction_policy == 0) {
      SF_CUDA(launch_axpby(t, n, 1.0, x, 1.0, L.c.p, x, G.guard, G.st));
      EpiArgs ea;
      ea.y = L.res2.p;
      ea.b = rhs;
      level_op(G, l, t, rsel, EPI_RESID, x, ea);
    } else {
      coarse_correction(G, l, x, L.res.p, L.c.p, L.res2.p);
    }
    if (enrich) {
      enrichment_rhs(G, L.res2.p, G.lv[1].rhs.p);
      coarse_visit(G, l, nullptr, true);
    } else {
      coarse_visit(G, l, L.res2.p, false);
    }
    coarse_correction(G, l, x, L.res2.p, L.c.p, nullptr);
  }
  x = smooth(G, l, rhs, x);
  if (l == 0 && G.high) x = smooth(G, l, rhs, x);
  return x;
}

// kernel nodes of a captured graph
static int kernel_nodes(cudaGraph_t graph) {
  size_t nn = 0;
  SF_CUDA(cudaGraphGetNodes(graph, nullptr, &nn));
  std::vector<cudaGraphNode_t> nodes(nn);
  if (nn) SF_CUDA(cudaGraphGetNodes(graph, nodes.data(), &nn));
  int k = 0;
  for (cudaGraphNode_t v : nodes) {
    cudaGraphNodeType t;
    SF_CUDA(cudaGraphNodeGetType(v, &t));
    if (t == cudaGraphNodeTypeKernel) ++k;
  }
  return k;
}

// The cycle body on the fixed cycle-dtype input `in` (cyc_in, or rhs64 in the
// FP64 cycle): run directly, or captured once per setup and guard pointer on a
// private stream and replayed on the hierarchy's stream (Gmg::CycleGraph).
// Replays run the identical kernels with identical arguments.
static void* run_cycle(Gmg& G, const void* in) {
  if (!G.o.use_graphs || G.graphs_off) return cycle(G, 0, in);
  Gmg::CycleGraph* cg = nullptr;
  for (Gmg::CycleGraph& c : G.graphs)
    if (c.guard == G.guard) cg = &c;
  if (!cg) {
    G.graphs.emplace_back();
    cg = &G.graphs.back();
    cg->guard = G.guard;
  }
  if (cg->epoch != G.setup_epoch) {
    cg->epoch = G.setup_epoch;
    cg->valid = false;
    cg->direct = 0;
  }
  if (cg->valid) {
    SF_CUDA(cudaGraphLaunch(cg->exec, G.st));
    SF_CUDA(sf_launched(cg->launches));
    ++G.graph_replays;
    return cg->out;
  }
  if (cg->direct++ == 0) return cycle(G, 0, in);  // first cycle after a setup: direct
  if (!G.cap_stream) SF_CUDA(cudaStreamCreateWithFlags(&G.cap_stream, cudaStreamNonBlocking));
  cudaStream_t user = G.st;
  cudaGraph_t graph = nullptr;
  void* out = nullptr;
  bool ok = cudaStreamBeginCapture(G.cap_stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
  if (ok) {
    G.st = G.cap_stream;
    try {
      out = cycle(G, 0, in);
    } catch (...) {  // the stream must leave capture mode before anything is reported
      ok = false;
    }
    G.st = user;
    ok = (cudaStreamEndCapture(G.cap_stream, &graph) == cudaSuccess) && ok && graph != nullptr;
  }
  int nk = 0;
  if (ok) {
    nk = kernel_nodes(graph);
    sf_launched(-nk);  // captured, not run
    if (cg->exec) {  // the previous setup's executable, when the topology is unchanged
      cudaGraphExecUpdateResultInfo info;
      if (cudaGraphExecUpdate(cg->exec, graph, &info) != cudaSuccess) {
        cudaGraphExecDestroy(cg->exec);
        cg->exec = nullptr;
      }
    }
    if (!cg->exec && cudaGraphInstantiate(&cg->exec, graph, 0) != cudaSuccess) {
      cg->exec = nullptr;
      ok = false;
    }
  }
  if (graph) cudaGraphDestroy(graph);
  cudaGetLastError();  // a refused capture leaves its error here; the cycle then runs directly
  if (!ok) {
    G.graphs_off = true;
    return cycle(G, 0, in);
  }
  cg->launches = nk;
  cg->out = out;
  cg->valid = true;
  SF_CUDA(cudaGraphLaunch(cg->exec, G.st));
  SF_CUDA(sf_launched(nk));
  ++G.graph_replays;
  return out;
}

// base cycle in FP64 (rhs -> out)
static void base_cycle(Gmg& G, const double* rhs, double* out) {
  const int64_t n = G.nfull();
  if (G.cyc == F32) {
    SF_CUDA(launch_convert(F64, F32, rhs, G.cyc_in.p, n, G.guard, G.st));
    void* r = run_cycle(G, G.cyc_in.p);
    SF_CUDA(launch_convert(F32, F64, r, out, n, G.guard, G.st));
  } else if (G.o.use_graphs && !G.graphs_off) {
    // a captured cycle reads a fixed input buffer
    SF_CUDA(launch_copy(F64, n, rhs, G.rhs64.p, G.guard, G.st));
    void* r = run_cycle(G, G.rhs64.p);
    SF_CUDA(launch_copy(F64, n, r, out, G.guard, G.st));
  } else {
    void* r = cycle(G, 0, rhs);
    SF_CUDA(launch_copy(F64, n, r, out, G.guard, G.st));
  }
}

// ----------------------------------------------------------------------------
// FGMRES (_cupy_fgmres) with the fine FP64 operator and preconditioner M.
// host_control: synchronise after each Givens update and stop early; otherwise
// the whole solve is a fixed kernel sequence whose skipped parts are gated by
// device flags.

static void fgmres(Gmg& G, KrylovWs& K, const double* b, double* x, bool x0_zero, double tol, int maxiter,
                   int restart, const PrecFn& M, const int* parent, bool host_control, double* hist_dev,
                   int hist_cap, const CheckHook* check = nullptr) {
  Mesh& m = *G.m;
  const int* saved_guard = G.guard;
  KrylovEnv E;
  E.n = G.nfull();
  E.st = G.st;
  E.rw = m.rw;
  E.A = [&G, &m](const double* u, double* y, const int* guard) {
    EpiArgs ea;
    ea.y = y;
    ea.guard = guard;
    fine_apply(m, F64, EPI_APPLY, G.E64.p, u, ea, G.st);
  };
  E.R = [&G, &m](const double* u, const double* rhs, double* r, const int* guard) {
    EpiArgs ea;
    ea.y = r;
    ea.b = rhs;
    ea.guard = guard;
    fine_apply(m, F64, EPI_RESID, G.E64.p, u, ea, G.st);
  };
  // the preconditioner may move the hierarchy's skip flag; the operator's
  // launches after it take theirs explicitly
  PrecFn Mg = [&G, &M, saved_guard](const double* in, double* out, const int* guard) {
    M(in, out, guard);
    G.guard = saved_guard;
  };
  fgmres_core(E, K, b, x, x0_zero, tol, maxiter, restart, Mg, parent, host_control, hist_dev, hist_cap, check);
  G.guard = saved_guard;
}

// ----------------------------------------------------------------------------
// root-local correction (multigrid_v4.py:964-1055)
void root_local(Gmg& G, const double* rhs, double* x) {
  Mesh& m = *G.m;
  const int64_t n = G.nfull();
  double* residual = G.tmp64a.as<double>();
  double* corr = G.tmp64b.as<double>();
  double* Ac = G.tmp64c.as<double>();
  double* sc = G.sc.as<double>() + 16;
  {
    EpiArgs ea;
    ea.y = residual;
    ea.b = rhs;
    ea.guard = G.guard;
    fine_apply(m, F64, EPI_RESID, G.E64.p, x, ea, G.st);
  }
  if (G.o.root_local_correction_mode == 2) {
    const int steps = G.o.root_local_correction_inner_steps;
    const int rst = G.o.root_local_correction_inner_restart > 0 ? G.o.root_local_correction_inner_restart
                                                                : std::max(1, steps);
    PrecFn bj = [&G](const double* in, double* out, const int* guard) {
      SF_CUDA(launch_node_block_apply(G.m->g, G.binv.as<double>(), in, out, guard, G.st));
    };
    fgmres(G, G.rl, residual, corr, true, 0.0, steps, rst, bj, G.guard, false, nullptr, 0);
    DotSet d1;
    d1.a[0] = corr; d1.b[0] = corr;
    d1.a[1] = residual; d1.b[1] = residual;
    d1.nd = 2;
    dots(G, F64, n, d1, sc + 0, G.guard);
    EpiArgs ea;
    ea.y = Ac;
    ea.guard = G.guard;
    fine_apply(m, F64, EPI_APPLY, G.E64.p, corr, ea, G.st);
    SF_CUDA(launch_trial_residual(F64, n, residual, Ac, sc, 1, nullptr, m.rw, G.guard, G.st));
    SF_CUDA(launch_scalar_op(OP_RLF, sc, 0.0, 0.0, G.guard, G.st));
    SF_CUDA(launch_select_axpy(F64, n, x, corr, sc, 1, G.guard, G.st));
  } else {
    SF_CUDA(launch_node_block_apply(m.g, G.binv.as<double>(), residual, corr, G.guard, G.st));
    DotSet d1;
    d1.a[0] = corr; d1.b[0] = corr;
    d1.a[1] = residual; d1.b[1] = residual;
    d1.nd = 2;
    dots(G, F64, n, d1, sc + 0, G.guard);
    EpiArgs ea;
    ea.y = Ac;
    ea.guard = G.guard;
    fine_apply(m, F64, EPI_APPLY, G.E64.p, corr, ea, G.st);
    DotSet d2;
    d2.a[0] = Ac; d2.b[0] = Ac;
    d2.a[1] = residual; d2.b[1] = Ac;
    d2.nd = 2;
    dots(G, F64, n, d2, sc + 2, G.guard);
    SF_CUDA(launch_scalar_op(OP_RLL, sc, 0.0, G.o.root_local_correction_max_scale, G.guard, G.st));
    SF_CUDA(launch_select_axpy(F64, n, x, corr, sc, 0, G.guard, G.st));
  }
}

// apply (multigrid_v4.py:1759-1767), full layout FP64 in/out
void apply_full(Gmg& G, const double* rhs, double* out, const int* guard) {
  G.guard = guard;
  if (G.o.inner_krylov_steps > 0) {
    const int rst = G.o.inner_krylov_restart > 0 ? G.o.inner_krylov_restart : std::max(1, G.o.inner_krylov_steps);
    PrecFn bc = [&G](const double* in, double* o, const int* g) {
      G.guard = g;
      base_cycle(G, in, o);
    };
    fgmres(G, G.ik, rhs, out, true, 0.0, G.o.inner_krylov_steps, rst, bc, guard, false, nullptr, 0);
    G.guard = guard;
  } else {
    base_cycle(G, rhs, out);
  }
  if (G.o.root_local_correction_mode != 0) root_local(G, rhs, out);
  G.guard = nullptr;
}

// ----------------------------------------------------------------------------
// Fixed-count Jacobi-PCG coarse solve (solver_v2.py:781-810), device scalars.
static void fixed_pcg_coarse(Gmg& G, int l, const double* b, double* x) {
  Level& L = G.lv[l];
  const int64_t n = L.g.ndof;
  int iters = G.o.coarse_pcg_iters;
  if (G.high) iters = std::max(iters, 200);
  double* r = G.pr.as<double>();
  double* z = G.pz.as<double>();
  double* p = G.pp.as<double>();
  double* Ap = G.pAp.as<double>();
  double* sc = G.sc.as<double>() + 24;  // [0]=rz [1]=pAp [2]=rz_new [3]=alpha [4]=beta
  const double* dinv = L.dinv64.as<double>();
  SF_CUDA(launch_fill(F64, n, 0.0, x, G.guard, G.st));
  SF_CUDA(launch_copy(F64, n, b, r, G.guard, G.st));
  SF_CUDA(launch_dmul(n, dinv, r, z, G.guard, G.st));
  SF_CUDA(launch_copy(F64, n, z, p, G.guard, G.st));
  DotSet d;
  d.a[0] = r; d.b[0] = z; d.nd = 1;
  dots(G, F64, n, d, sc + 0, G.guard);
  for (int it = 0; it < iters; ++it) {
    EpiArgs ea;
    ea.y = Ap;
    ea.guard = G.guard;
    SF_CUDA(launch_stencil(F64, F64, EPI_APPLY, L.g, L.K64.p, L.mask.as<uint8_t>(), p, ea, G.st));
    DotSet dp;
    dp.a[0] = p; dp.b[0] = Ap; dp.nd = 1;
    dots(G, F64, n, dp, sc + 1, G.guard);
    SF_CUDA(launch_pcg_scalar(0, sc, G.guard, G.st));
    SF_CUDA(launch_pcg_xr(n, x, r, z, p, Ap, dinv, sc, G.m->rw, G.guard, G.st));
    SF_CUDA(launch_pcg_scalar(1, sc, G.guard, G.st));
    SF_CUDA(launch_pcg_p(n, z, p, sc, G.guard, G.st));
  }
}

// ----------------------------------------------------------------------------
// setup (multigrid_v4.py:1119-1341)
struct PhaseTimer {
  Gmg& G;
  bool on;
  std::chrono::steady_clock::time_point t;
  explicit PhaseTimer(Gmg& g) : G(g), on(getenv("SIMPFEM_TIMING") != nullptr) {
    if (on) {
      cudaStreamSynchronize(G.st);
      t = std::chrono::steady_clock::now();
    }
  }
  void mark(const char* name) {
    if (!on) return;
    cudaStreamSynchronize(G.st);
    auto n = std::chrono::steady_clock::now();
    fprintf(stderr, "[simpfem setup] %-18s %8.3f ms\n", name,
            std::chrono::duration<double, std::milli>(n - t).count());
    t = n;
  }
};

static double sync_scalar(Gmg& G, const double* dev) {
  double h;
  SF_CUDA(cudaMemcpyAsync(&h, dev, sizeof(double), cudaMemcpyDeviceToHost, G.st));
  SF_CUDA(cudaStreamSynchronize(G.st));
  return h;
}

static void resolve_prec(Gmg& G) {
  if (G.prec_resolved) return;
  for (int l = 0; l < 8; ++l) G.prec[l] = -1;
  bool given = false;
  for (int l = 0; l < 8; ++l)
    if (G.o.level_prec[l] >= 0) given = true;
  if (given) {
    for (int l = 0; l < G.L; ++l) G.prec[l] = G.o.level_prec[l] >= 0 ? G.o.level_prec[l] : F64;
  } else if (G.o.fine_smoother == BF16) {
    G.prec[0] = BF16;
    if (G.L > 1) G.prec[1] = F32;
    for (int l = 2; l < G.L; ++l) G.prec[l] = F64;
  } else {
    G.prec[0] = G.o.fine_smoother;
    for (int l = 1; l < G.L; ++l) G.prec[l] = F64;
  }
  if (G.cyc == F32) {
    // mixed mode: FP32 fine smoothing (BF16 operands if requested), BF16-stored coarse stencils
    if (G.prec[0] != BF16) G.prec[0] = F32;
    for (int l = 1; l < G.L; ++l)
      if (G.prec[l] == F64 || G.prec[l] < 0) G.prec[l] = BF16;
  }
  G.prec_resolved = true;
}

static double fine_lambda(Gmg& G) {
  // _estimate_fine_lambda_max (multigrid_v4.py:364-386), 20 power iterations
  Mesh& m = *G.m;
  const int64_t n = G.nfull();
  const uint8_t* mask = m.mask.as<uint8_t>();
  double* v = G.tmp64a.as<double>();
  double* Kv = G.tmp64b.as<double>();
  double* Av = G.tmp64c.as<double>();
  double* d = G.tmp64d.as<double>();
  const double* dinv = G.lv[0].dinv64.as<double>();
  double* sc = m.dscal.as<double>();
  SF_CUDA(launch_vec_op(n, 0, dinv, nullptr, mask, 0.0, nullptr, d, G.st));  // d = 1 / dinv
  SF_CUDA(launch_vec_op(n, 4, v, nullptr, mask, 1.0, nullptr, v, G.st));     // v = ones
  DotSet ds;
  ds.a[0] = v; ds.b[0] = v; ds.c[0] = d; ds.mode[0] = 1; ds.nd = 1;
  dots(G, F64, n, ds, sc, nullptr);
  const double nrm0 = sqrt(sync_scalar(G, sc));
  SF_CUDA(launch_vec_op(n, 2, v, nullptr, nullptr, nrm0, nullptr, v, G.st));  // v /= sqrt(vDv)
  double lam = 1.0;
  for (int it = 0; it < 20; ++it) {
    EpiArgs ea;
    ea.y = Kv;
    fine_apply(m, F64, EPI_APPLY, G.E64.p, v, ea, G.st);
    DotSet d2;
    d2.a[0] = v; d2.b[0] = v; d2.c[0] = d; d2.mode[0] = 1;
    d2.a[1] = v; d2.b[1] = Kv;
    d2.nd = 2;
    dots(G, F64, n, d2, sc, nullptr);
    SF_CUDA(launch_vec_op(n, 3, Kv, dinv, nullptr, 0.0, nullptr, Av, G.st));  // Av = dinv * Kv
    DotSet d3;
    d3.a[0] = Av; d3.b[0] = Av; d3.c[0] = d; d3.mode[0] = 1; d3.nd = 1;
    dots(G, F64, n, d3, sc + 2, nullptr);
    double h[3];
    SF_CUDA(cudaMemcpyAsync(h, sc, 3 * sizeof(double), cudaMemcpyDeviceToHost, G.st));
    SF_CUDA(cudaStreamSynchronize(G.st));
    lam = h[1] / std::max(h[0], 1e-300);
    const double nrmD = sqrt(h[2]);
    if (nrmD <= 1e-300) break;
    SF_CUDA(launch_vec_op(n, 2, Av, nullptr, nullptr, nrmD, nullptr, v, G.st));
  }
  return lam;
}

static double sparse_lambda(Gmg& G, int l) {
  // _estimate_sparse_lambda_max (multigrid_v4.py:389-405), 10 iterations
  Level& L = G.lv[l];
  const int64_t n = L.g.ndof;
  double* v = L.s64a.as<double>();
  double* Kv = L.s64b.as<double>();
  double* Av = L.s64c.as<double>();
  const uint8_t* mask = L.mask.as<uint8_t>();
  const double* dinv = L.dinv64.as<double>();
  double* sc = G.m->dscal.as<double>();
  SF_CUDA(launch_fill(F64, n, 1.0, v, nullptr, G.st));
  SF_CUDA(launch_vec_op(n, 5, v, nullptr, mask, 0.0, nullptr, v, G.st));
  SF_CUDA(launch_vec_op(n, 2, v, nullptr, mask, sqrt((double)L.n_free), nullptr, v, G.st));
  double lam = 1.0;
  for (int it = 0; it < 10; ++it) {
    EpiArgs ea;
    ea.y = Kv;
    SF_CUDA(launch_stencil(F64, F64, EPI_APPLY, L.g, L.K64.p, mask, v, ea, G.st));
    SF_CUDA(launch_vec_op(n, 3, Kv, dinv, nullptr, 0.0, nullptr, Av, G.st));
    DotSet d;
    d.a[0] = v; d.b[0] = Kv;
    d.a[1] = Av; d.b[1] = Av;
    d.a[2] = v; d.b[2] = v; d.c[2] = dinv; d.mode[2] = 2;
    d.nd = 3;
    dots(G, F64, n, d, sc, nullptr);
    double h[3];
    SF_CUDA(cudaMemcpyAsync(h, sc, 3 * sizeof(double), cudaMemcpyDeviceToHost, G.st));
    SF_CUDA(cudaStreamSynchronize(G.st));
    const double nrm = sqrt(h[1]);
    if (nrm <= 1e-300) break;
    lam = h[0] / std::max(h[2], 1e-300);
    SF_CUDA(launch_vec_op(n, 2, Av, nullptr, nullptr, nrm, nullptr, v, G.st));
  }
  return std::max(lam, 1e-6);
}

static void setup_coarsest(Gmg& G) {
  const int l = G.L - 1;
  Level& L = G.lv[l];
  G.coarse_reg = false;
  const int n = G.nc;
  if (n <= G.o.dense_chol_max && n > 0) {
    const size_t nn = (size_t)n * n;
    G.Adense.alloc(8 * nn);
    // the FP64 cycle's L^{-1}; otherwise only the wide-band recursion's work array
    const bool band = band_tiles(G.c_bw) <= kBandMaxTiles && band_path_available();
    if (G.cyc != F32 || !band) G.Linv.alloc(8 * nn);
    G.cdinv.alloc(band_dinv_bytes(n));
    BandInvOut out;
    if (G.cyc == F32) {
      // the mixed cycle reads FP32 copies of both factors (FP64 accumulation)
      G.LinvF.alloc(4 * nn);
      G.LinvTF.alloc(4 * nn);
      out.L32 = G.LinvF.as<float>();
      out.LT32 = G.LinvTF.as<float>();
    } else {
      G.LinvT.alloc(8 * nn);
      out.L64 = G.Linv.as<double>();
      out.LT64 = G.LinvT.as<double>();
    }
    int* info = G.cinfo.as<int>();
    auto try_factor = [&](double eps) -> bool {
      SF_CUDA(launch_stencil_to_dense(L.g, L.K64.as<double>(), G.c_didx.as<int32_t>(), n, G.Adense.as<double>(),
                                      G.st));
      if (eps > 0) SF_CUDA(launch_add_diag(G.Adense.as<double>(), n, eps, G.st));
      SF_CUDA(chol_inverse(G.Adense.as<double>(), n, G.Linv.as<double>(), G.cdinv.as<double>(), out, info, G.st,
                           G.c_bw));
      int h = 0;
      SF_CUDA(cudaMemcpyAsync(&h, info, sizeof(int), cudaMemcpyDeviceToHost, G.st));
      SF_CUDA(cudaStreamSynchronize(G.st));
      return h == 0;
    };
    bool ok = try_factor(0.0);
    if (!ok) {
      // eps = max(mean(diag) * 1e-8, 1e-14) of the unregularised matrix
      SF_CUDA(launch_stencil_to_dense(L.g, L.K64.as<double>(), G.c_didx.as<int32_t>(), n, G.Adense.as<double>(),
                                      G.st));
      SF_CUDA(launch_diag_sum(G.Adense.as<double>(), n, G.m->dscal.as<double>(), G.st));
      const double mean = sync_scalar(G, G.m->dscal.as<double>()) / n;
      const double eps = std::max(mean * 1e-8, 1e-14);
      ok = try_factor(eps);
      if (ok) {
        G.coarse_reg = true;
        fprintf(stdout, "[GMG] coarsest matrix regularised (eps=%.2e): Cholesky OK\n", eps);
      } else {
        fprintf(stdout, "[GMG] WARNING: coarsest Cholesky failed even after regularisation "
                        "— using iterative coarse solve\n");
      }
    }
    if (ok) {
      G.coarse_mode = 1;
      return;
    }
  }
  G.coarse_mode = 2;
  const int64_t nd = L.g.ndof;
  G.pr.alloc(8 * nd);
  G.pz.alloc(8 * nd);
  G.pp.alloc(8 * nd);
  G.pAp.alloc(8 * nd);
}

void gmg_setup(Gmg& G, const double* E, const double* fine_diag_free) {
  ++G.setup_epoch;  // captured cycles hold the previous setup's launch arguments
  Mesh& m = *G.m;
  const int64_t n = m.g.ndof;
  const int64_t ne = m.g.ne();
  resolve_prec(G);
  PhaseTimer pt(G);
  if (!m.tuned[0]) tune_mesh(m, F64, G.st);
  if (!m.tuned[1]) tune_mesh(m, F32, G.st);
  pt.mark("tune");
  SF_CUDA(cudaMemcpyAsync(G.E64.p, E, 8 * ne, cudaMemcpyDeviceToDevice, G.st));
  SF_CUDA(launch_convert(F64, F32, G.E64.p, G.E32.p, ne, nullptr, G.st));
  // diag0 (full layout) and its inverse
  if (fine_diag_free != nullptr) {
    SF_CUDA(launch_fill(F64, n, 0.0, G.diag0.p, nullptr, G.st));
    SF_CUDA(launch_expand(F64, m.n_free, m.free_idx.as<int32_t>(), fine_diag_free, G.diag0.p, G.st));
  } else {
    SF_CUDA(launch_fine_diag(m.g, G.E64.as<double>(), m.mask.as<uint8_t>(), 0.0, G.diag0.as<double>(), G.st));
  }
  // where(|d| > 1e-12, d, 1) on free entries; dinv = 1 / diag0 (0 on constrained)
  SF_CUDA(launch_vec_op(n, 6, G.diag0.as<double>(), nullptr, m.mask.as<uint8_t>(), 0.0, nullptr,
                        G.diag0.as<double>(), G.st));
  SF_CUDA(launch_vec_op(n, 0, G.diag0.as<double>(), nullptr, m.mask.as<uint8_t>(), 0.0, nullptr,
                        G.lv[0].dinv64.as<double>(), G.st));
  SF_CUDA(launch_convert(F64, F32, G.lv[0].dinv64.p, G.lv[0].dinv32.p, n, nullptr, G.st));
  if (G.o.root_enrichment_mode != 0) {
    G.wenrich.alloc(8 * n);
    SF_CUDA(launch_minmax_count(n, G.diag0.as<double>(), 0.0, m.rw, m.dscal.as<double>(), G.st));
    SF_CUDA(launch_enrich_weights(n, G.diag0.as<double>(), m.mask.as<uint8_t>(), m.dscal.as<double>() + 1,
                                  G.o.root_enrichment_weight_floor, G.o.root_enrichment_weight_power,
                                  G.wenrich.as<double>(), G.st));
  }
  if (G.o.root_local_correction_mode != 0) {
    G.binv.alloc(8 * 9 * m.g.nn);
    SF_CUDA(launch_node_blocks(m.g, G.E64.as<double>(), m.mask.as<uint8_t>(), G.diag0.as<double>(),
                               G.binv.as<double>(), G.st));
  }
  pt.mark("diag/blocks");
  // lambda cache rule
  G.lam_calls += 1;
  SF_CUDA(launch_minmax_count(ne, G.E64.as<double>(), INFINITY, m.rw, m.dscal.as<double>(), G.st));
  double mm[3];
  SF_CUDA(cudaMemcpyAsync(mm, m.dscal.p, sizeof(mm), cudaMemcpyDeviceToHost, G.st));
  SF_CUDA(cudaStreamSynchronize(G.st));
  const double Emin = mm[0], Emax = mm[1];
  const double prev = G.lam_Emax;
  const bool reest = std::isnan(prev) || fabs(Emax - prev) / std::max(fabs(prev), 1e-12) > 0.10;
  G.lam_reest = reest;
  if (reest) {
    G.lv[0].lam = fine_lambda(G);
    G.lam_Emax = Emax;
  }
  G.omega_used = std::min(G.o.omega, 0.9 * 2.0 / std::max(G.lv[0].lam, 1e-6));
  pt.mark("lambda fine");
  // contrast classification
  G.contrast = Emax / std::max(Emin, 1e-300);
  SF_CUDA(launch_minmax_count(ne, G.E64.as<double>(), Emax * 1e-8, m.rw, m.dscal.as<double>(), G.st));
  SF_CUDA(cudaMemcpyAsync(mm, m.dscal.p, sizeof(mm), cudaMemcpyDeviceToHost, G.st));
  SF_CUDA(cudaStreamSynchronize(G.st));
  const double n_solid = mm[2];
  G.void_frac = 1.0 - n_solid / std::max<double>((double)ne, 1.0);
  const int bc = G.o.coarse_smooth_iters, bf = std::max(1, G.o.fine_smoother_degree);
  if (G.contrast > 1e5 || G.void_frac > 0.8) {
    G.coarse_iters = std::max(bc, 6);
    G.fine_deg = std::max(bf, 4);
    G.high = true;
  } else if (G.contrast > 100 || G.void_frac > 0.5) {
    G.coarse_iters = std::max(bc, 4);
    G.fine_deg = std::max(bf, 3);
    G.high = true;
  } else if (G.contrast > 10) {
    G.coarse_iters = std::max(bc, 3);
    G.fine_deg = bf;
    G.high = false;
  } else {
    G.coarse_iters = bc;
    G.fine_deg = bf;
    G.high = false;
  }
  // coarse operators
  for (int l = 1; l < G.L; ++l) {
    Level& L = G.lv[l];
    if (l == 1) {
      SF_CUDA(launch_level1_assemble(L.g, m.g, G.E64.as<double>(), G.Qdev.as<double>(), L.mask.as<uint8_t>(),
                                     L.K64.as<double>(), G.st));
    } else {
      Level& F = G.lv[l - 1];
      SF_CUDA(launch_rap(F.g, L.g, F.K64.as<double>(), L.mask.as<uint8_t>(), F.wx.as<double>(),
                         F.wy.as<double>(), F.wz.as<double>(), L.K64.as<double>(), G.st));
    }
    SF_CUDA(launch_stencil_diag(L.g, L.K64.as<double>(), L.mask.as<uint8_t>(), L.dinv64.as<double>(), G.st));
    pt.mark(l == 1 ? "level1 assemble" : "rap");
    if (reest || std::isnan(L.lam)) L.lam = sparse_lambda(G, l);
    pt.mark("lambda coarse");
    const int p = G.prec[l];
    const bool need32 = (p == F32) || (G.cyc == F32);
    if (need32) {
      L.K32.alloc(4 * 243 * L.g.nn);
      SF_CUDA(launch_convert(F64, F32, L.K64.p, L.K32.p, 243 * L.g.nn, nullptr, G.st));
      L.dinv32.alloc(4 * L.g.ndof);
      SF_CUDA(launch_convert(F64, F32, L.dinv64.p, L.dinv32.p, L.g.ndof, nullptr, G.st));
      if (G.cyc == F32 && L.xs[0].p == nullptr) {
        // nothing: mixed mode uses the cycle buffers directly
      }
    }
    if (G.cyc == F32 && p == BF16) {
      L.K16.alloc(2 * 288 * L.g.nn);  // node-major by neighbour column, 288 entries per node
      SF_CUDA(launch_stencil_colmajor_bf16(L.g.nn, L.K64.as<double>(), L.K16.as<__nv_bfloat16>(), G.st));
    }
  }
  pt.mark("precision copies");
  if (G.L > 1) setup_coarsest(G);
  pt.mark("coarsest");
  SF_CUDA(cudaStreamSynchronize(G.st));
  G.is_setup = true;
}

}  // namespace simpfem

namespace simpfem {

// Average duration of one smoothing step of `level` in the cycle precision (the
// kernel the V-cycle launches most), timed with CUDA events on the caller's stream.
float time_smoother_step(Gmg& G, int l, int reps) {
  Level& L = G.lv[l];
  const DType t = G.cyc;
  const int p = G.prec[l];
  DType vt = t;
  if (t == F64 && l == 0 && (p == F32 || p == BF16)) vt = F32;
  if (t == F64 && l > 0 && p == F32 && L.K32.p) vt = F32;
  void* x = vt == t ? L.x[0].p : L.xs[0].p;
  void* xo = vt == t ? L.x[1].p : L.xs[1].p;
  void* rhs = vt == t ? L.rhs.p : L.rhss.p;
  void* d = vt == t ? L.d.p : L.ds.p;
  const size_t es = vt == F64 ? 8 : 4;
  // non-constant inputs, so the timed step moves data like a real cycle does
  SF_CUDA(launch_fill_hash(vt, L.g.ndof, 11u, x, G.st));
  SF_CUDA(launch_fill_hash(vt, L.g.ndof, 12u, rhs, G.st));
  SF_CUDA(launch_fill_hash(vt, L.g.ndof, 13u, d, G.st));
  EpiArgs ea;
  ea.b = rhs;
  ea.dinv = level_dinv(G, l, vt);
  ea.d = d;
  ea.xo = xo;
  ea.s1 = 0.5;
  ea.s2 = 0.25;
  const Epi epi = G.o.smoother_type == 0 ? EPI_CHEB : EPI_JAC;
  const int psel = (vt == F32) ? p : F64;
  G.guard = nullptr;
  level_op(G, l, vt, psel, epi, x, ea);
  return time_cold([&]() { level_op(G, l, vt, psel, epi, x, ea); }, reps, G.st);
}

// Average device time of `launch` over `reps` runs, each from a cold L2: a
// 256 MB buffer (twice the L2) is overwritten with pseudo-random values (data
// the L2 cannot hold compressed) between runs, and only the launch itself is
// inside its event pair.
float time_cold(const std::function<void()>& launch, int reps, cudaStream_t st) {
  DevBuf flush;
  const int64_t flush_vals = int64_t(64) << 20;  // 64 Mi floats = 256 MB
  flush.alloc(sizeof(float) * flush_vals);
  std::vector<cudaEvent_t> ev(2 * reps);
  for (auto& e : ev) SF_CUDA(cudaEventCreate(&e));
  for (int r = 0; r < reps; ++r) {
    SF_CUDA(launch_fill_hash(F32, flush_vals, 0x9e3779b9u * (uint32_t)(r + 1), flush.p, st));
    SF_CUDA(cudaEventRecord(ev[2 * r], st));
    launch();
    SF_CUDA(cudaEventRecord(ev[2 * r + 1], st));
  }
  SF_CUDA(cudaEventSynchronize(ev.back()));
  float total = 0.f;
  for (int r = 0; r < reps; ++r) {
    float ms = 0.f;
    SF_CUDA(cudaEventElapsedTime(&ms, ev[2 * r], ev[2 * r + 1]));
    total += ms;
  }
  for (auto& e : ev) cudaEventDestroy(e);
  return total / reps;
}

// The FP64 fine operator product y = K(E) u of the outer FGMRES (and of the
// guard) on pseudo-random u, with the hierarchy's moduli of the last setup.
float time_fine_operator(Gmg& G, int reps) {
  const int64_t n = G.nfull();
  double* u = G.tmp64a.as<double>();
  double* y = G.tmp64b.as<double>();
  SF_CUDA(launch_fill_hash(F64, n, 21u, u, G.st));
  EpiArgs ea;
  ea.y = y;
  fine_apply(*G.m, F64, EPI_APPLY, G.E64.p, u, ea, G.st);
  return time_cold([&]() { fine_apply(*G.m, F64, EPI_APPLY, G.E64.p, u, ea, G.st); }, reps, G.st);
}

// Outer FGMRES: host-controlled (one synchronisation per iteration to read the
// device-side convergence flags), history written straight into mapped memory.
void run_outer_fgmres(Gmg& G, const double* b, double* x, bool x0_zero, double tol, int maxiter, int restart,
                      const PrecFn& M, double* hist_dev, int hist_cap, const CheckHook* check) {
  fgmres(G, G.outer, b, x, x0_zero, tol, maxiter, restart, M, nullptr, true, hist_dev, hist_cap, check);
  G.outer.sync_flags(G.st);
}

// _cupy_pcg (gpu_fem/solver_v2.py:551-623) with the hierarchy as preconditioner.
void run_pcg(Gmg& G, const double* b, double* x, double tol, int maxiter, std::vector<double>* hist, int* iters,
             int* conv) {
  Mesh& m = *G.m;
  const int64_t n = G.nfull();
  DevBuf rb, zb, pb, apb;
  rb.alloc(8 * n);
  zb.alloc(8 * n);
  pb.alloc(8 * n);
  apb.alloc(8 * n);
  KrylovEnv E;
  E.n = n;
  E.st = G.st;
  E.rw = m.rw;
  E.A = [&G, &m](const double* u, double* y, const int* guard) {
    EpiArgs ea;
    ea.y = y;
    ea.guard = guard;
    fine_apply(m, F64, EPI_APPLY, G.E64.p, u, ea, G.st);
  };
  E.R = [&G, &m](const double* u, const double* rhs, double* r, const int* guard) {
    EpiArgs ea;
    ea.y = r;
    ea.b = rhs;
    ea.guard = guard;
    fine_apply(m, F64, EPI_RESID, G.E64.p, u, ea, G.st);
  };
  PrecFn M = [&G](const double* in, double* out, const int*) { apply_full(G, in, out, nullptr); };
  pcg_core(E, M, b, x, tol, maxiter, rb.as<double>(), zb.as<double>(), pb.as<double>(), apb.as<double>(),
           m.dscal.as<double>() + 8, hist, iters, conv);
}

}  // namespace simpfem
