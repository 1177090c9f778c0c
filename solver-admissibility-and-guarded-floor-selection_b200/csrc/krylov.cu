// Krylov drivers of the simpfem library, independent of the operator.
//
//   fgmres_core  restarted right-preconditioned FGMRES (_cupy_fgmres,
//                gpu_fem/multigrid_v4.py:416-534): modified Gram-Schmidt, Givens
//                rotations, history and lucky-breakdown rule, all on the device
//   pcg_core     preconditioned CG with the up-front convergence check
//                (_cupy_pcg, gpu_fem/solver_v2.py:551-623)
//
// The hierarchy's solves (gmg.cu) run these with the fused fine operator.  The
// two entry points at the end run them with operators the caller supplies as
// host callbacks that enqueue their work on the solve's stream: the reference's
// _cupy_fgmres / _cupy_pcg accept any pair of callables, and this is how such a
// pair is solved by the same device Arnoldi, rotations and reductions.
#include <math.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <vector>

#include "gmg_impl.h"
#include "simpfem.h"

namespace simpfem {

static void kdots(const KrylovEnv& E, const DotSet& ds, double* out, const int* guard) {
  SF_CUDA(launch_dots(F64, E.n, ds, E.rw, out, guard, E.st));
}

void fgmres_core(const KrylovEnv& E, KrylovWs& K, const double* b, double* x, bool x0_zero, double tol,
                 int maxiter, int restart, const PrecFn& M, const int* parent, bool host_control, double* hist_dev,
                 int hist_cap, const CheckHook* check) {
  const int64_t n = E.n;
  cudaStream_t st = E.st;
  K.ensure(n, restart);
  KrylovDev& kd = K.kd;
  const int ld = restart + 1;
  {
    DotSet ds;
    ds.a[0] = b;
    ds.b[0] = b;
    ds.nd = 1;
    kdots(E, ds, kd.sc + SC_BNORM2, parent);
  }
  SF_CUDA(launch_krylov_init(kd, parent, st));
  if (x0_zero) SF_CUDA(launch_fill(F64, n, 0.0, x, K.dflag(F_NOTDONE), st));
  const int ncycles = (maxiter + restart - 1) / std::max(restart, 1);
  bool stopped = false;
  for (int c = 0; c < ncycles && !stopped; ++c) {
    if (host_control) {
      K.sync_flags(st);
      if (K.hflags()[F_DONE]) break;
    }
    const int* nd = K.dflag(F_NOTDONE);
    if (c == 0 && x0_zero) {
      SF_CUDA(launch_copy(F64, n, b, K.r.p, nd, st));
    } else {
      E.R(x, b, K.r.as<double>(), nd);
    }
    {
      DotSet ds;
      ds.a[0] = K.r.p;
      ds.b[0] = K.r.p;
      ds.nd = 1;
      kdots(E, ds, kd.sc + SC_BETA2, nd);
    }
    SF_CUDA(launch_krylov_restart(kd, tol, hist_dev, hist_cap, st));
    const int* cyc = K.dflag(F_CYC);
    SF_CUDA(launch_scale_vec(n, K.r.as<double>(), kd.sc + SC_BETA, K.Vj(0), cyc, st));
    const int inner = std::min(restart, maxiter - c * restart);
    for (int j = 0; j < inner; ++j) {
      M(K.Vj(j), K.Zj(j), cyc);
      E.A(K.Zj(j), K.w.as<double>(), cyc);
      double* Hc = kd.H + (size_t)j * ld;
      SF_CUDA(launch_mgs_first(n, K.Vj(0), K.w.as<double>(), E.rw, Hc, cyc, st));
      for (int i = 0; i <= j; ++i) {
        const bool last = (i == j);
        SF_CUDA(launch_mgs_step(n, K.Vj(i), last ? nullptr : K.Vj(i + 1), K.w.as<double>(), Hc + i, E.rw,
                                last ? kd.sc + SC_HSQ : Hc + i + 1, cyc, st));
      }
      SF_CUDA(launch_givens(kd, j, tol, hist_dev, hist_cap, st));
      SF_CUDA(launch_scale_vec(n, K.w.as<double>(), kd.sc + SC_HNORM, K.Vj(j + 1), cyc, st));
      if (host_control) {
        K.sync_flags(st);
        if (!K.hflags()[F_CYC]) break;
        // the caller's check at a fixed iteration count (the solve is still running):
        // it sees the residual history so far and may end the solve here; the
        // iterate after these columns is then formed as at the end of a cycle
        if (check && check->fn && K.hflags()[F_TOTAL] == check->iter && hist_dev) {
          double true_rel = NAN;
          if (check->true_residual) {
            // the iterate after these columns, formed in the free restart-residual
            // vector (the back-solve writes only y), and its FP64 true residual in w
            SF_CUDA(launch_backsolve(kd, st));
            SF_CUDA(launch_copy(F64, n, x, K.r.p, nullptr, st));
            SF_CUDA(launch_update_x(n, K.r.as<double>(), (double* const*)K.Zptr.p, kd.y, kd.flags, st));
            E.R(K.r.as<double>(), b, K.w.as<double>(), nullptr);
            DotSet ds;
            ds.a[0] = K.w.p;
            ds.b[0] = K.w.p;
            ds.nd = 1;
            kdots(E, ds, kd.sc + 8, nullptr);
            double sc[9];
            SF_CUDA(cudaMemcpyAsync(sc, kd.sc, sizeof(sc), cudaMemcpyDeviceToHost, st));
            SF_CUDA(cudaStreamSynchronize(st));
            true_rel = sc[SC_BNORM] > 0.0 ? sqrt(sc[8]) / sc[SC_BNORM] : 0.0;
          }
          const int hn = std::min(K.hflags()[F_HISTN], hist_cap);
          check->buf.resize(hn);
          SF_CUDA(cudaMemcpyAsync(check->buf.data(), hist_dev, sizeof(double) * hn, cudaMemcpyDeviceToHost, st));
          SF_CUDA(cudaStreamSynchronize(st));
          if (check->fn(check->ctx, check->iter, check->buf.data(), hn, true_rel)) {
            stopped = true;
            check->stopped = true;
            break;
          }
        }
      }
    }
    SF_CUDA(launch_backsolve(kd, st));
    SF_CUDA(launch_update_x(n, x, (double* const*)K.Zptr.p, kd.y, kd.flags, st));
  }
}

void pcg_core(const KrylovEnv& E, const PrecFn& M, const double* b, double* x, double tol, int maxiter, double* r,
              double* z, double* p, double* Ap, double* sc, std::vector<double>* hist, int* iters, int* conv) {
  const int64_t n = E.n;
  cudaStream_t st = E.st;
  auto rd = [&](int k) {
    std::vector<double> h(k);
    SF_CUDA(cudaMemcpyAsync(h.data(), sc, sizeof(double) * k, cudaMemcpyDeviceToHost, st));
    SF_CUDA(cudaStreamSynchronize(st));
    return h;
  };
  E.R(x, b, r, nullptr);
  DotSet d0;
  d0.a[0] = b; d0.b[0] = b;
  d0.a[1] = r; d0.b[1] = r;
  d0.nd = 2;
  kdots(E, d0, sc, nullptr);
  auto h0 = rd(2);
  const double bsq = h0[0];
  const double tol_sq = tol * tol * bsq;
  hist->push_back(bsq > 0 ? sqrt(h0[1] / bsq) : 0.0);
  *iters = 0;
  *conv = 0;
  if (h0[1] <= tol_sq) {
    *conv = 1;
    return;
  }
  M(r, z, nullptr);
  SF_CUDA(launch_copy(F64, n, z, p, nullptr, st));
  DotSet d1;
  d1.a[0] = r; d1.b[0] = z; d1.nd = 1;
  kdots(E, d1, sc, nullptr);
  double rz = rd(1)[0];
  int it = 1;
  for (int k = 0; k < maxiter - 1; ++k) {
    E.A(p, Ap, nullptr);
    DotSet d2;
    d2.a[0] = p; d2.b[0] = Ap; d2.nd = 1;
    kdots(E, d2, sc, nullptr);
    const double pAp = rd(1)[0];
    const double alpha = rz / pAp;
    SF_CUDA(launch_axpby(F64, n, 1.0, x, alpha, p, x, nullptr, st));
    SF_CUDA(launch_axpby(F64, n, 1.0, r, -alpha, Ap, r, nullptr, st));
    DotSet d3;
    d3.a[0] = r; d3.b[0] = r; d3.nd = 1;
    kdots(E, d3, sc, nullptr);
    const double rsq = rd(1)[0];
    hist->push_back(bsq > 0 ? sqrt(rsq / bsq) : 0.0);
    if (rsq <= tol_sq) {
      *conv = 1;
      break;
    }
    M(r, z, nullptr);
    it += 1;
    DotSet d4;
    d4.a[0] = r; d4.b[0] = z; d4.nd = 1;
    kdots(E, d4, sc, nullptr);
    const double rzn = rd(1)[0];
    const double beta = rzn / rz;
    SF_CUDA(launch_axpby(F64, n, 1.0, z, beta, p, p, nullptr, st));
    rz = rzn;
  }
  *iters = it;
}

// ----------------------------------------------------------------------------
// Work buffers of the callback-operator solves: one set per host thread and
// device, grown on demand (these entry points serve the reference's generic
// Krylov signatures, not the hot path).
struct OpWork {
  DevBuf part, ticket, sc, hist, tmp, r, z, p, Ap;
  KrylovWs K;
  RedWork rw{};
  int64_t n = 0;
  void ensure(int64_t n_, int hist_cap) {
    if (!part.p) {
      part.alloc(sizeof(double) * 4 * kRedBlocksHost);
      ticket.alloc(sizeof(unsigned) * 4);
      SF_CUDA(cudaMemset(ticket.p, 0, sizeof(unsigned) * 4));
      sc.alloc(sizeof(double) * 8);
      rw.partials = part.as<double>();
      rw.ticket = ticket.as<unsigned>();
    }
    if (n_ != n) {
      tmp.alloc(8 * std::max<int64_t>(n_, 1));
      r.alloc(8 * std::max<int64_t>(n_, 1));
      z.alloc(8 * std::max<int64_t>(n_, 1));
      p.alloc(8 * std::max<int64_t>(n_, 1));
      Ap.alloc(8 * std::max<int64_t>(n_, 1));
      n = n_;
    }
    hist.alloc(sizeof(double) * std::max(hist_cap, 1));
  }
};

static OpWork& op_work() {
  thread_local std::map<int, std::unique_ptr<OpWork>> per_device;
  int dev = 0;
  SF_CUDA(cudaGetDevice(&dev));
  auto& w = per_device[dev];
  if (!w) w.reset(new OpWork());
  return *w;
}

struct CallbackFailure {};

static KrylovEnv callback_env(OpWork& W, int64_t n, simpfem_apply_fn A, void* ctx, cudaStream_t st) {
  KrylovEnv E;
  E.n = n;
  E.st = st;
  E.rw = W.rw;
  E.A = [A, ctx, st](const double* x, double* y, const int*) {
    if (A(ctx, x, y, (void*)st) != 0) throw CallbackFailure{};
  };
  double* tmp = W.tmp.as<double>();
  E.R = [A, ctx, st, n, tmp](const double* x, const double* b, double* r, const int*) {
    if (A(ctx, x, tmp, (void*)st) != 0) throw CallbackFailure{};
    SF_CUDA(launch_axpby(F64, n, 1.0, b, -1.0, tmp, r, nullptr, st));
  };
  return E;
}

static PrecFn callback_prec(simpfem_apply_fn M, void* ctx, cudaStream_t st) {
  return [M, ctx, st](const double* in, double* out, const int*) {
    if (M(ctx, in, out, (void*)st) != 0) throw CallbackFailure{};
  };
}

}  // namespace simpfem

using namespace simpfem;

#define SF_OP_BEGIN try {
#define SF_OP_END                                                               \
  }                                                                             \
  catch (const CallbackFailure&) {                                              \
    set_error("an operator callback reported a failure");                      \
    return SIMPFEM_ECALLBACK;                                                   \
  }                                                                             \
  catch (const CudaFailure&) {                                                  \
    return SIMPFEM_ECUDA;                                                       \
  }                                                                             \
  catch (const InvalidArg& e) {                                                 \
    set_error(e.msg);                                                           \
    return SIMPFEM_EINVAL;                                                      \
  }                                                                             \
  catch (const std::exception& e) {                                             \
    set_error(e.what());                                                        \
    return SIMPFEM_EINTERNAL;                                                   \
  }                                                                             \
  return SIMPFEM_OK;

extern "C" {

int simpfem_fgmres_op(int64_t n, simpfem_apply_fn A, simpfem_apply_fn M, void* ctx, const double* b,
                      const double* x0, double* x, double tol, int maxiter, int restart, double* history_host,
                      int history_cap, int* history_len, int* iters, int* converged, void* stream) {
  SF_OP_BEGIN
  if (n < 1 || !A || !M || !b || !x) throw InvalidArg{"simpfem_fgmres_op: null argument or empty system"};
  if (restart < 1 || restart > 1000 || maxiter < 0) throw InvalidArg{"simpfem_fgmres_op: restart must be in [1, 1000]"};
  cudaStream_t st = (cudaStream_t)stream;
  const int cap = maxiter + maxiter / std::max(restart, 1) + 4;
  OpWork& W = op_work();
  W.ensure(n, cap);
  // the zero start is written here: the core skips its own fill when b is zero
  if (x0 == nullptr)
    SF_CUDA(launch_fill(F64, n, 0.0, x, nullptr, st));
  else if (x0 != x)
    SF_CUDA(cudaMemcpyAsync(x, x0, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  KrylovEnv E = callback_env(W, n, A, ctx, st);
  fgmres_core(E, W.K, b, x, x0 == nullptr, tol, maxiter, restart, callback_prec(M, ctx, st), nullptr, true,
              W.hist.as<double>(), cap, nullptr);
  W.K.sync_flags(st);
  const int* f = W.K.hflags();
  const int hn = f[F_HISTN];
  if (history_len) *history_len = hn;
  if (history_host) {
    const int k = std::min(std::min(hn, history_cap), cap);
    if (k > 0) SF_CUDA(cudaMemcpyAsync(history_host, W.hist.p, sizeof(double) * k, cudaMemcpyDeviceToHost, st));
  }
  SF_CUDA(cudaStreamSynchronize(st));
  if (iters) *iters = f[F_TOTAL];
  if (converged) *converged = f[F_CONV];
  SF_OP_END
}

int simpfem_pcg_op(int64_t n, simpfem_apply_fn A, simpfem_apply_fn M, void* ctx, const double* b, const double* x0,
                   double* x, double tol, int maxiter, double* history_host, int history_cap, int* history_len,
                   int* iters, int* converged, void* stream) {
  SF_OP_BEGIN
  if (n < 1 || !A || !M || !b || !x) throw InvalidArg{"simpfem_pcg_op: null argument or empty system"};
  if (maxiter < 0) throw InvalidArg{"simpfem_pcg_op: maxiter must be >= 0"};
  cudaStream_t st = (cudaStream_t)stream;
  OpWork& W = op_work();
  W.ensure(n, 1);
  if (x0) {
    if (x0 != x) SF_CUDA(cudaMemcpyAsync(x, x0, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  } else {
    SF_CUDA(launch_fill(F64, n, 0.0, x, nullptr, st));
  }
  KrylovEnv E = callback_env(W, n, A, ctx, st);
  std::vector<double> hist;
  int it = 0, conv = 0;
  pcg_core(E, callback_prec(M, ctx, st), b, x, tol, maxiter, W.r.as<double>(), W.z.as<double>(),
           W.p.as<double>(), W.Ap.as<double>(), W.sc.as<double>(), &hist, &it, &conv);
  if (history_len) *history_len = (int)hist.size();
  if (history_host)
    std::memcpy(history_host, hist.data(), sizeof(double) * std::min<size_t>(hist.size(), (size_t)history_cap));
  if (iters) *iters = it;
  if (converged) *converged = conv;
  SF_OP_END
}

}  // extern "C"
