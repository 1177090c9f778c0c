// One multigrid cycle traced on the device: GalerkinMatFreeGMG.cycle_trace
// (gpu_fem/multigrid_v4.py:1362-1438), _trace_vcycle_level (:1440-1587) and
// _trace_wcycle_level (:1589-1728).
//
// The traced cycle runs the same building blocks as the production cycle
// (smooth, level_op, restrict / prolong, solve_coarsest, coarse_correction,
// enrichment_rhs, root_local), in the hierarchy's cycle dtype, and measures the
// reference's diagnostic norms between them with the deterministic device
// reductions.  Each norm is read back on the host as it is taken: the trace
// is a diagnostic, not a hot path.  Decisions of the line searches (raw and
// applied scale, acceptance) are read from the scalars the correction kernels
// leave behind, and turned into the reference's notes on the host.
#include <math.h>

#include <algorithm>
#include <vector>

#include "gmg_impl.h"

namespace simpfem {
namespace {

// visit record slots (kTraceVisitLen doubles; NaN where the reference has None)
enum VisitSlot {
  V_ID = 0, V_LEVEL, V_COARSEST, V_NCORR, V_RHS, V_JAC, V_PRE_SOL, V_PRE_RES, V_RESTR, V_PROJ, V_GAP, V_CC, V_PCC,
  V_ALIGN, V_RAW, V_APPLIED, V_CORR, V_CORR1, V_RESTR2, V_CC2, V_PCC2, V_ALIGN2, V_RAW2, V_APPLIED2, V_CORR2,
  V_POST_SOL, V_POST_RES, V_NOTE1, V_NOTE2, V_ENRICH, V_EXTRA, V_CMODE
};
static_assert(V_CMODE < kTraceVisitLen, "visit record too short");

// coarse-correction notes (multigrid_v4.py:867-931)
enum { NOTE_NONE = 0, NOTE_DEGENERATE = 1, NOTE_REJECTED = 2, NOTE_NONPOSITIVE = 3, NOTE_CLIPPED = 4 };
// root-local notes (:964-1055)
enum { RL_NONE = 0, RL_DEGENERATE = 1, RL_REJECTED_FGMRES = 2, RL_FGMRES = 3, RL_NONPOSITIVE = 4, RL_CLIPPED = 5 };

struct Tracer {
  Gmg& G;
  int cycle_type;
  std::vector<double>* rec;
  int counter = 0;
  DevBuf dd;  // dot results

  double fetch(const double* dev, int k, double* host) {
    SF_CUDA(cudaMemcpyAsync(host, dev, sizeof(double) * k, cudaMemcpyDeviceToHost, G.st));
    SF_CUDA(cudaStreamSynchronize(G.st));
    return host[0];
  }
  double dot(DType t, int64_t n, const void* a, const void* b, const void* c = nullptr, int mode = 0) {
    DotSet ds;
    ds.a[0] = a;
    ds.b[0] = b;
    ds.c[0] = c;
    ds.mode[0] = mode;
    ds.nd = 1;
    SF_CUDA(launch_dots(t, n, ds, G.m->rw, dd.as<double>(), nullptr, G.st));
    double h;
    return fetch(dd.as<double>(), 1, &h);
  }
  int64_t n_of(int l) const { return G.lv[l].g.ndof; }
  double norm(int l, const void* a) { return sqrt(std::max(dot(G.cyc, n_of(l), a, a), 0.0)); }
  // || D_l^{-1} r ||
  double jac_norm(int l, const void* r) {
    return sqrt(std::max(dot(G.cyc, n_of(l), r, r, level_dinv(G, l, G.cyc), 3), 0.0));
  }
  // cosine of the angle between a residual and a correction (:855-862)
  double alignment(int l, const void* r, const void* c, double rn, double cn) {
    if (rn <= 1e-300 || cn <= 1e-300) return 0.0;
    return dot(G.cyc, n_of(l), r, c) / (rn * cn);
  }
  // the decision of the coarse correction just applied, from G.sc[0..8]
  void decision(double* raw, double* applied, double* note) {
    if (G.o.coarse_correction_policy == 0) {
      *raw = 1.0;
      *applied = 1.0;
      *note = NOTE_NONE;
      return;
    }
    double sc[9];
    fetch(G.sc.as<double>(), 9, sc);
    if (sc[7] != 0.0) {
      *raw = 0.0;
      *applied = 0.0;
      *note = NOTE_DEGENERATE;
    } else if (sc[6] == 0.0) {
      *raw = sc[8];
      *applied = 0.0;
      *note = NOTE_REJECTED;
    } else {
      *raw = sc[8];
      *applied = sc[4];
      *note = (sc[4] <= 1e-12 && sc[8] <= 0.0) ? NOTE_NONPOSITIVE
              : fabs(sc[4] - sc[8]) > 1e-12    ? NOTE_CLIPPED
                                               : NOTE_NONE;
    }
  }
};

void restrict_to(Gmg& G, int l, const void* fine, void* coarse) {
  Level& L = G.lv[l];
  Level& C = G.lv[l + 1];
  SF_CUDA(launch_restrict(G.cyc, L.g, C.g, L.wx.as<double>(), L.wy.as<double>(), L.wz.as<double>(),
                          C.mask.as<uint8_t>(), fine, coarse, nullptr, G.st));
}

void prolong_to(Gmg& G, int l, const void* coarse, void* fine) {
  Level& L = G.lv[l];
  Level& C = G.lv[l + 1];
  SF_CUDA(launch_prolong(G.cyc, L.g, C.g, L.wx.as<double>(), L.wy.as<double>(), L.wz.as<double>(),
                         L.mask.as<uint8_t>(), coarse, fine, nullptr, G.st));
}

// residual rhs - K_l x into out, with the operator precision of the cycle's residual
void level_residual(Gmg& G, int l, const void* rhs, const void* x, void* out) {
  EpiArgs ea;
  ea.y = out;
  ea.b = rhs;
  level_op(G, l, G.cyc, G.cyc == F32 ? G.prec[l] : F64, EPI_RESID, x, ea);
}

void* trace_level(Tracer& T, int l, const void* rhs) {
  Gmg& G = T.G;
  Level& L = G.lv[l];
  double r[kTraceVisitLen];
  for (double& v : r) v = NAN;
  // the record slot is taken on entry: records come out in visit order
  const size_t slot = T.rec->size();
  T.rec->resize(slot + kTraceVisitLen, NAN);
  r[V_ID] = T.counter++;
  r[V_LEVEL] = l;
  const double rn = T.norm(l, rhs);
  r[V_RHS] = rn;
  r[V_JAC] = T.jac_norm(l, rhs);
  r[V_ENRICH] = 0.0;
  r[V_EXTRA] = 0.0;
  r[V_NOTE1] = NOTE_NONE;
  r[V_NOTE2] = -1.0;
  void* x;
  if (l == G.L - 1) {
    x = L.x[0].p;
    solve_coarsest(G, rhs, x);
    level_residual(G, l, rhs, x, L.res.p);
    const double xn = T.norm(l, x), resn = T.norm(l, L.res.p);
    r[V_COARSEST] = 1.0;
    r[V_NCORR] = 0.0;
    r[V_PRE_SOL] = 0.0;
    r[V_PRE_RES] = rn;
    r[V_RESTR] = r[V_PROJ] = r[V_GAP] = 0.0;
    r[V_CC] = r[V_PCC] = r[V_POST_SOL] = xn;
    r[V_ALIGN] = 0.0;
    r[V_APPLIED] = 1.0;
    r[V_CORR] = r[V_CORR1] = r[V_POST_RES] = resn;
    r[V_CMODE] = G.L == 1 ? 0.0 : (double)G.coarse_mode;
  } else {
    Level& C = G.lv[l + 1];
    const int64_t n = L.g.ndof;
    x = smooth(G, l, rhs, nullptr);
    level_residual(G, l, rhs, x, L.res.p);
    const double presn = T.norm(l, L.res.p);
    r[V_COARSEST] = 0.0;
    r[V_PRE_SOL] = T.norm(l, x);
    r[V_PRE_RES] = presn;
    restrict_to(G, l, L.res.p, C.rhs.p);
    r[V_RESTR] = T.norm(l + 1, C.rhs.p);
    prolong_to(G, l, C.rhs.p, L.c.p);
    r[V_PROJ] = T.norm(l, L.c.p);
    SF_CUDA(launch_axpby(G.cyc, n, 1.0, L.res.p, -1.0, L.c.p, L.res2.p, nullptr, G.st));
    r[V_GAP] = T.norm(l, L.res2.p);
    // level l+1 works in its own buffers, the coarse right-hand side C.rhs
    // included, so everything of level l above stays valid across the visit
    void* e = trace_level(T, l + 1, C.rhs.p);
    r[V_CC] = T.norm(l + 1, e);
    prolong_to(G, l, e, L.c.p);
    r[V_PCC] = T.norm(l, L.c.p);
    r[V_ALIGN] = T.alignment(l, L.res.p, L.c.p, presn, r[V_PCC]);
    coarse_correction(G, l, x, L.res.p, L.c.p, L.res2.p);
    T.decision(&r[V_RAW], &r[V_APPLIED], &r[V_NOTE1]);
    const double crn1 = T.norm(l, L.res2.p);
    r[V_CORR] = r[V_CORR1] = crn1;
    const bool enrich = l == 0 && G.o.root_enrichment_mode != 0;
    r[V_ENRICH] = enrich ? 1.0 : 0.0;
    r[V_NCORR] = 1.0;
    if (T.cycle_type == 1 || enrich) {
      if (enrich)
        enrichment_rhs(G, L.res2.p, C.rhs.p);
      else
        restrict_to(G, l, L.res2.p, C.rhs.p);
      r[V_RESTR2] = T.norm(l + 1, C.rhs.p);
      void* e2 = trace_level(T, l + 1, C.rhs.p);
      r[V_CC2] = T.norm(l + 1, e2);
      prolong_to(G, l, e2, L.c.p);
      r[V_PCC2] = T.norm(l, L.c.p);
      r[V_ALIGN2] = T.alignment(l, L.res2.p, L.c.p, crn1, r[V_PCC2]);
      coarse_correction(G, l, x, L.res2.p, L.c.p, L.res.p);
      T.decision(&r[V_RAW2], &r[V_APPLIED2], &r[V_NOTE2]);
      r[V_CORR2] = T.norm(l, L.res.p);
      r[V_NCORR] = 2.0;
      // the V-cycle record reports the residual after the enrichment correction
      // as its corrected residual (:1516-1563); the W-cycle record keeps the first
      if (T.cycle_type == 0) r[V_CORR] = r[V_CORR2];
    }
    x = smooth(G, l, rhs, x);
    if (l == 0 && G.high) {
      x = smooth(G, l, rhs, x);
      r[V_EXTRA] = 1.0;
    }
    level_residual(G, l, rhs, x, L.res2.p);
    r[V_POST_SOL] = T.norm(l, x);
    r[V_POST_RES] = T.norm(l, L.res2.p);
    r[V_CMODE] = -1.0;
  }
  std::copy(r, r + kTraceVisitLen, T.rec->begin() + slot);
  return x;
}

}  // namespace

void trace_cycle(Gmg& G, const double* rhs_full, int cycle_type, std::vector<double>* visits, double* summary) {
  G.guard = nullptr;
  Mesh& m = *G.m;
  const int64_t n = G.nfull();
  Tracer T{G, cycle_type, visits};
  T.dd.alloc(8 * sizeof(double));
  visits->clear();
  const void* rhs_c = rhs_full;
  if (G.cyc == F32) {
    SF_CUDA(launch_convert(F64, F32, rhs_full, G.cyc_in.p, n, nullptr, G.st));
    rhs_c = G.cyc_in.p;
  }
  void* xc = trace_level(T, 0, rhs_c);
  // the cycle's answer in FP64 (out64), its FP64 residual (rhs64)
  double* x = G.out64.as<double>();
  double* res = G.rhs64.as<double>();
  if (G.cyc == F32)
    SF_CUDA(launch_convert(F32, F64, xc, x, n, nullptr, G.st));
  else
    SF_CUDA(launch_copy(F64, n, xc, x, nullptr, G.st));
  auto residual = [&]() {
    EpiArgs ea;
    ea.y = res;
    ea.b = rhs_full;
    fine_apply(m, F64, EPI_RESID, G.E64.p, x, ea, G.st);
  };
  auto norm64 = [&](const double* v) { return sqrt(std::max(T.dot(F64, n, v, v), 0.0)); };
  residual();
  const double pre = norm64(res);
  double raw = NAN, applied = 0.0, note = RL_NONE;
  const int mode = G.o.root_local_correction_mode;
  if (mode != 0) {
    root_local(G, rhs_full, x);
    double sc[9];
    T.fetch(G.sc.as<double>() + 16, 9, sc);
    if (mode == 2) {  // node-block inner FGMRES
      if (sqrt(sc[0]) <= 1e-300 || sqrt(sc[1]) <= 1e-300) {
        raw = 0.0;
        note = RL_DEGENERATE;
      } else if (sc[6] == 0.0) {
        note = RL_REJECTED_FGMRES;
      } else {
        applied = 1.0;
        note = RL_FGMRES;
      }
    } else {  // node-block line search
      if (sc[7] != 0.0) {
        raw = 0.0;
        note = RL_DEGENERATE;
      } else if (sc[6] == 0.0) {
        raw = sc[8];
        note = RL_NONPOSITIVE;
      } else {
        raw = sc[8];
        applied = sc[4];
        note = fabs(sc[4] - sc[8]) > 1e-12 ? RL_CLIPPED : RL_NONE;
      }
    }
    residual();
  }
  for (int k = 0; k < kTraceSummaryLen; ++k) summary[k] = NAN;
  summary[0] = norm64(rhs_full);
  summary[1] = sqrt(std::max(T.dot(F64, n, rhs_full, rhs_full, G.lv[0].dinv64.p, 3), 0.0));
  summary[2] = norm64(x);
  summary[3] = T.dot(F64, n, rhs_full, x);
  summary[4] = norm64(res);
  summary[5] = pre;
  summary[6] = raw;
  summary[7] = applied;
  summary[8] = note;
  summary[9] = G.contrast;
  summary[10] = G.high ? 1.0 : 0.0;
  summary[11] = G.fine_deg;
  summary[12] = G.coarse_iters;
  summary[13] = (double)(visits->size() / kTraceVisitLen);
  summary[14] = G.L == 1 ? 0.0 : (double)G.coarse_mode;
}

}  // namespace simpfem
