// The guarded floor policy in the library: per state (simpfem_policy_run) and for
// a batch of states of any mix of meshes solved together (simpfem_policy_batch).
//
// Reference behaviour followed (file:line in the reference project):
//   solve_at_floor (moduli, setup, FGMRES, guard)  experiments/phase5/run_gmg_floor_detector_prospective.py:220-261
//   probe r50 / r100 read-out                       :263-270
//   _classify                                        :77-90
//   floor sequence, post-solve fallback              :313-354
// The decision at r50 with a proposer network is the learned floor policy of
// this project (no reference counterpart).
//
// Everything between two states runs here: the moduli kernel, the hierarchy
// setup, the device FGMRES and the FP64 guard, with the host reading only the
// convergence flags once per iteration; a batch runs one host thread and one
// stream per hierarchy, so there is no interpreter between the steps.
#include <math.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"
#include "gmg_impl.h"
#include "simpfem.h"

namespace simpfem {
namespace {

// E = rho_min + (1 - rho_min) * r^penal with r = rho (for a solid mask: 1 at solid
// elements, rho_min at void ones), each operation rounded once as the host tensor expression does; the
// exponents 2 and 3 are evaluated as products and 0.5 as a square root, which is
// how the tensor library evaluates them, so both paths give identical moduli.
__global__ void moduli_kernel(int64_t n, const double* __restrict__ rho, double rho_min, double one_minus,
                              double penal, int pmode, int binary, double* __restrict__ E) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double r = rho[i];
  if (binary) r = (r != 0.0) ? 1.0 : rho_min;
  double t;
  if (pmode == 2)
    t = __dmul_rn(r, r);
  else if (pmode == 3)
    t = __dmul_rn(__dmul_rn(r, r), r);
  else if (pmode == 1)
    t = sqrt(r);
  else
    t = pow(r, penal);
  E[i] = __dadd_rn(rho_min, __dmul_rn(t, one_minus));
}

void launch_moduli(int64_t n, const double* rho, double rho_min, double penal, int binary, double* E,
                   cudaStream_t st) {
  const int pmode = penal == 2.0 ? 2 : (penal == 3.0 ? 3 : (penal == 0.5 ? 1 : 0));
  moduli_kernel<<<div_up(n, 256), 256, 0, st>>>(n, rho, rho_min, 1.0 - rho_min, penal, pmode, binary, E);
  SF_CUDA(sf_launched(1));
}

struct Attempt {
  double rho_min = NAN;
  int iters = 0;
  bool reported = false;  // FGMRES reported convergence
  bool converged = false; // the FP64 guard passed
  double final = NAN;
};

// The state a worker keeps between its attempts.
struct Worker {
  simpfem_gmg* g = nullptr;
  cudaStream_t st = nullptr;
  DevBuf E, xprobe, pooled, feats, prob;
  simpfem_cnn* cnn = nullptr;
  bool own_cnn = false;
  std::vector<int> states;
  int status = SIMPFEM_OK;
  std::string error;
  ~Worker() {
    if (own_cnn && cnn) simpfem_cnn_destroy(cnn);
  }
};

// One solve at rho_min from a zero start: moduli, setup, FGMRES, guard.  The
// iterate stays in the hierarchy's full-layout x buffer.
Attempt attempt(Worker& W, const simpfem_policy_opts& o, const double* density, double rho_min, int maxiter,
                std::vector<double>* hist, const CheckHook* hook) {
  Gmg& G = *W.g->impl;
  Mesh& m = *G.m;
  const int64_t n = m.g.ndof;
  G.st = W.st;
  launch_moduli(m.g.ne(), density, rho_min, o.penal, o.binary, W.E.as<double>(), W.st);
  gmg_setup(G, W.E.as<double>(), nullptr);
  const int cap = maxiter + maxiter / std::max(o.restart, 1) + 4;
  G.hist_pin.alloc(sizeof(double) * cap);
  G.hist_dev.alloc(sizeof(double) * cap);
  SF_CUDA(cudaMemsetAsync(W.g->xfull.p, 0, 8 * n, W.st));
  PrecFn M = [&G](const double* in, double* out, const int* guard) { apply_full(G, in, out, guard); };
  double* b = W.g->bfull.as<double>();
  double* x = W.g->xfull.as<double>();
  run_outer_fgmres(G, b, x, true, o.tol, maxiter, o.restart, M, G.hist_dev.as<double>(), cap, hook);
  Attempt a;
  a.rho_min = rho_min;
  const int* f = G.outer.hflags();
  a.iters = f[F_TOTAL];
  a.reported = f[F_CONV] != 0;
  if (hist) {
    const int hn = std::min(f[F_HISTN], cap);
    hist->resize(hn);
    SF_CUDA(cudaMemcpyAsync(hist->data(), G.hist_dev.p, sizeof(double) * hn, cudaMemcpyDeviceToHost, W.st));
  }
  // the recomputed FP64 guard ||b - K(E) x|| / ||b||
  EpiArgs ea;
  ea.y = G.tmp64a.p;
  ea.b = b;
  fine_apply(m, F64, EPI_RESID, G.E64.p, x, ea, W.st);
  DotSet ds;
  ds.a[0] = G.tmp64a.p;
  ds.b[0] = G.tmp64a.p;
  ds.a[1] = b;
  ds.b[1] = b;
  ds.nd = 2;
  SF_CUDA(launch_dots(F64, n, ds, m.rw, m.dscal.as<double>(), nullptr, W.st));
  double h[2];
  SF_CUDA(cudaMemcpyAsync(h, m.dscal.p, sizeof(h), cudaMemcpyDeviceToHost, W.st));
  SF_CUDA(cudaStreamSynchronize(W.st));
  a.final = h[1] > 0.0 ? sqrt(h[0]) / sqrt(h[1]) : 0.0;
  a.converged = a.final <= o.tol;
  return a;
}

int classify(double r50, double r100, const simpfem_policy_opts& o, bool* raise) {
  if (r50 >= o.high_residual_threshold) {
    *raise = true;
    return SIMPFEM_TRIGGER_HIGH_R50;
  }
  const double ratio = r100 / std::max(r50, 1e-300);
  if (r100 >= o.plateau_residual_threshold && ratio >= o.plateau_ratio_threshold) {
    *raise = true;
    return SIMPFEM_TRIGGER_PLATEAU;
  }
  *raise = false;
  return SIMPFEM_TRIGGER_KEEP;
}

double history_at(const std::vector<double>& h, int k) {
  return h.empty() ? INFINITY : h[std::min<size_t>((size_t)std::max(k, 0), h.size() - 1)];
}

// The proposer's decision at the probe's r50 point.
struct Decision {
  Worker* W = nullptr;
  const simpfem_policy_opts* o = nullptr;
  int proposed = -1;
  int stop = 0;  // 0 none, SIMPFEM_TRIGGER_LEARNED or SIMPFEM_TRIGGER_HIGH_RESIDUAL
};

int decide_at_r50(void* ctx, int, const double* hist, int hn, double) {
  Decision& d = *static_cast<Decision*>(ctx);
  const simpfem_policy_opts& o = *d.o;
  Worker& W = *d.W;
  const int k50 = o.probe_r50;
  const double r50 = hn > 0 ? hist[std::min(k50, hn - 1)] : INFINITY;
  int hit = k50;
  for (int k = 0; k <= std::min(k50, hn - 1); ++k)
    if (hist[k] <= o.high_residual_threshold) {
      hit = k;
      break;
    }
  const float feats[2] = {(float)(log10(std::max(r50, 1e-16)) / 4.0), (float)((double)hit / (double)k50)};
  SF_CUDA(cudaMemcpyAsync(W.feats.p, feats, sizeof(feats), cudaMemcpyHostToDevice, W.st));
  if (simpfem_cnn_forward(W.cnn, W.pooled.as<float>(), W.feats.as<float>(), 1, W.prob.as<float>(), W.st) != 0)
    throw std::runtime_error(std::string("floor proposer: ") + simpfem_last_error());
  float p[3];
  SF_CUDA(cudaMemcpyAsync(p, W.prob.p, sizeof(p), cudaMemcpyDeviceToHost, W.st));
  SF_CUDA(cudaStreamSynchronize(W.st));
  const int best = (int)(std::max_element(p, p + 3) - p);
  d.proposed = (double)p[best] >= o.min_confidence ? best : 0;
  d.stop = r50 >= o.high_residual_threshold ? SIMPFEM_TRIGGER_HIGH_RESIDUAL
                                            : (d.proposed >= 1 ? SIMPFEM_TRIGGER_LEARNED : 0);
  return d.stop != 0;
}

void run_state(Worker& W, const simpfem_policy_opts& o, const double* density, const double* b_free, double* x_free,
               simpfem_policy_result* out) {
  const auto t0 = std::chrono::steady_clock::now();
  Gmg& G = *W.g->impl;
  Mesh& m = *G.m;
  const int64_t n = m.g.ndof;
  W.E.alloc(8 * std::max<int64_t>(1, m.g.ne()));
  W.g->bfull.alloc(8 * n);
  W.g->xfull.alloc(8 * n);
  G.tmp64a.alloc(8 * n);
  SF_CUDA(cudaMemsetAsync(W.g->bfull.p, 0, 8 * n, W.st));
  SF_CUDA(launch_expand(F64, m.n_free, m.free_idx.as<int32_t>(), b_free, W.g->bfull.p, W.st));
  std::vector<double> rungs{o.baseline_rho_min};
  for (int k = 0; k < o.n_raised; ++k) rungs.push_back(o.raised_rho_mins[k]);

  Decision dec;
  dec.W = &W;
  dec.o = &o;
  CheckHook hook;
  const bool learned = W.cnn != nullptr;
  if (learned) {
    W.pooled.alloc(sizeof(float) * 4096);
    W.feats.alloc(sizeof(float) * 2);
    W.prob.alloc(sizeof(float) * 3);
    if (simpfem_cnn_pool16(m.g.nx, m.g.ny, m.g.nz, density, W.pooled.as<float>(), W.st) != 0)
      throw std::runtime_error(std::string("floor proposer: ") + simpfem_last_error());
    hook.iter = o.probe_r50;
    hook.fn = decide_at_r50;
    hook.ctx = &dec;
  }
  std::vector<double> probe_hist;
  const Attempt probe = attempt(W, o, density, o.baseline_rho_min, o.probe_iters, &probe_hist,
                                learned ? &hook : nullptr);
  const bool can_reuse = o.reuse_probe && probe.reported;
  if (can_reuse) {
    W.xprobe.alloc(8 * n);
    SF_CUDA(cudaMemcpyAsync(W.xprobe.p, W.g->xfull.p, 8 * n, cudaMemcpyDeviceToDevice, W.st));
  }
  const double r50 = history_at(probe_hist, o.probe_r50);
  double r100 = NAN;
  bool raise = false;
  int trigger;
  std::vector<int> seq;  // rung indices in attempt order
  std::vector<int> fallback_seq;
  std::vector<int> raised;
  for (int k = 1; k < (int)rungs.size(); ++k) raised.push_back(k);
  if (dec.stop != 0) {
    raise = true;
    trigger = dec.stop;
    const int start = std::max(1, dec.proposed);
    for (int k : raised)
      if (k >= start) seq.push_back(k);
    for (int k : raised)
      if (k < start) seq.push_back(k);
    if (dec.stop == SIMPFEM_TRIGGER_LEARNED) seq.push_back(0);
  } else {
    r100 = history_at(probe_hist, o.probe_iters);
    trigger = classify(r50, r100, o, &raise);
    if (raise) {
      seq = raised;
    } else if (learned) {
      seq.push_back(0);
      seq.insert(seq.end(), raised.begin(), raised.end());
    } else {
      seq.push_back(0);
      fallback_seq = raised;  // the reference's post-solve fallback after a failed keep
    }
  }
  std::vector<double> attempted;
  Attempt sel;
  bool have = false, sel_is_probe = false;
  int total = probe.iters, setups = 1;
  auto run_seq = [&](const std::vector<int>& s) {
    for (int k : s) {
      const double rm = rungs[k];
      if (std::find(attempted.begin(), attempted.end(), rm) != attempted.end()) continue;
      attempted.push_back(rm);
      if (can_reuse && rm == probe.rho_min) {
        sel = probe;
        sel_is_probe = true;
      } else {
        sel = attempt(W, o, density, rm, o.maxiter, nullptr, nullptr);
        sel_is_probe = false;
        total += sel.iters;
        setups += 1;
      }
      have = true;
      if (sel.converged) break;
    }
  };
  run_seq(seq);
  bool fell_back = false;
  if (!(have && sel.converged) && !fallback_seq.empty()) {
    fell_back = true;
    run_seq(fallback_seq);
  }
  if (x_free) {
    const double* xs = sel_is_probe ? W.xprobe.as<double>() : W.g->xfull.as<double>();
    SF_CUDA(launch_compress(F64, m.n_free, m.free_idx.as<int32_t>(), xs, x_free, W.st));
  }
  SF_CUDA(cudaStreamSynchronize(W.st));
  simpfem_policy_result r;
  std::memset(&r, 0, sizeof(r));
  r.probe_r50 = r50;
  r.probe_r100 = r100;
  r.trigger = trigger;
  r.raise_floor = raise ? 1 : 0;
  r.fallback = fell_back ? 1 : 0;
  r.proposal = learned ? dec.proposed : -1;
  r.selected_rho_min = have ? sel.rho_min : NAN;
  r.converged = have && sel.converged ? 1 : 0;
  r.reported_converged = have && sel.reported ? 1 : 0;
  r.solve_iters = have ? sel.iters : o.maxiter;
  r.probe_iters = probe.iters;
  r.total_iters = total;
  r.n_setups = setups;
  r.n_attempts = (int)std::min<size_t>(attempted.size(), 8);
  for (int k = 0; k < r.n_attempts; ++k) r.attempted[k] = attempted[k];
  r.reused_probe = sel_is_probe ? 1 : 0;
  r.final_rel_residual = have ? sel.final : NAN;
  r.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  *out = r;
}

void check_opts(const simpfem_policy_opts* o) {
  if (!o) throw InvalidArg{"simpfem_policy: null options"};
  if (o->restart < 1 || o->restart > 1000 || o->maxiter < 1 || o->probe_iters < 1 || o->probe_r50 < 1)
    throw InvalidArg{"simpfem_policy: restart must be in [1, 1000] and the iteration counts positive"};
  if (o->n_raised < 0 || o->n_raised > 6) throw InvalidArg{"simpfem_policy: n_raised must be in [0, 6]"};
  if (o->proposer && o->n_raised != 2)
    throw InvalidArg{"simpfem_policy: the floor proposer is trained on a baseline and two raised rungs"};
  if (!(o->tol > 0.0)) throw InvalidArg{"simpfem_policy: tol must be positive"};
}

}  // namespace
}  // namespace simpfem

using namespace simpfem;

#define SF_POLICY_BEGIN try {
#define SF_POLICY_END                                                           \
  }                                                                             \
  catch (const CudaFailure&) {                                                  \
    return SIMPFEM_ECUDA;                                                       \
  }                                                                             \
  catch (const InvalidArg& e) {                                                 \
    set_error(e.msg);                                                           \
    return SIMPFEM_EINVAL;                                                      \
  }                                                                             \
  catch (const NotSetup& e) {                                                   \
    set_error(e.msg);                                                           \
    return SIMPFEM_ENOTSETUP;                                                   \
  }                                                                             \
  catch (const std::exception& e) {                                             \
    set_error(e.what());                                                        \
    return SIMPFEM_EINTERNAL;                                                   \
  }                                                                             \
  return SIMPFEM_OK;

extern "C" {

void simpfem_policy_default_opts(simpfem_policy_opts* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->penal = 3.0;
  o->binary = 0;
  o->tol = 1e-6;
  o->restart = 300;
  o->maxiter = 300;
  o->probe_iters = 100;
  o->probe_r50 = 50;
  o->baseline_rho_min = 1e-12;
  o->n_raised = 2;
  o->raised_rho_mins[0] = 1e-3;
  o->raised_rho_mins[1] = 1e-2;
  o->high_residual_threshold = 1e-2;
  o->plateau_residual_threshold = 1e-4;
  o->plateau_ratio_threshold = 0.6;
  o->reuse_probe = 1;
  o->proposer = nullptr;
  o->min_confidence = 0.5;
}

int simpfem_policy_run(simpfem_gmg* g, const simpfem_policy_opts* o, const double* density, const double* b_free,
                       double* x_free, simpfem_policy_result* result, void* stream) {
  SF_POLICY_BEGIN
  check_opts(o);
  if (!g || !density || !b_free || !result) throw InvalidArg{"simpfem_policy_run: null argument"};
  Worker W;
  W.g = g;
  W.st = (cudaStream_t)stream;
  W.cnn = o->proposer;
  run_state(W, *o, density, b_free, x_free, result);
  SF_POLICY_END
}

int simpfem_policy_batch(const simpfem_policy_opts* o, const simpfem_policy_state* states, int n_states,
                         simpfem_policy_result* results, void* stream) {
  SF_POLICY_BEGIN
  check_opts(o);
  if (n_states < 0 || (n_states > 0 && (!states || !results))) throw InvalidArg{"simpfem_policy_batch: null argument"};
  // workers: the distinct hierarchies, in order of first appearance
  std::vector<std::unique_ptr<Worker>> workers;
  std::map<simpfem_gmg*, Worker*> by_g;
  std::map<simpfem_mesh*, simpfem_gmg*> mesh_owner;
  for (int s = 0; s < n_states; ++s) {
    const simpfem_policy_state& st = states[s];
    if (!st.g || !st.density || !st.b_free) throw InvalidArg{"simpfem_policy_batch: state with a null field"};
    auto it = by_g.find(st.g);
    if (it == by_g.end()) {
      auto mo = mesh_owner.find(st.g->mesh);
      if (mo != mesh_owner.end() && mo->second != st.g)
        throw InvalidArg{"simpfem_policy_batch: two hierarchies share one mesh handle"};
      mesh_owner[st.g->mesh] = st.g;
      workers.emplace_back(new Worker());
      workers.back()->g = st.g;
      it = by_g.emplace(st.g, workers.back().get()).first;
    }
    it->second->states.push_back(s);
  }
  if (workers.empty()) return SIMPFEM_OK;
  int dev = 0;
  SF_CUDA(cudaGetDevice(&dev));
  cudaStream_t caller = (cudaStream_t)stream;
  // every mesh picks its sweep shapes now, before the workers share the GPU
  for (auto& w : workers) {
    Mesh& m = *w->g->impl->m;
    if (!m.tuned[0]) tune_mesh(m, F64, caller);
    if (!m.tuned[1]) tune_mesh(m, F32, caller);
  }
  std::vector<float> theta;
  if (o->proposer) {
    theta.resize(simpfem_cnn_n_params());
    if (simpfem_cnn_get_params(o->proposer, theta.data(), (int)theta.size()) != 0)
      throw std::runtime_error(std::string("floor proposer: ") + simpfem_last_error());
  }
  cudaEvent_t start;
  SF_CUDA(cudaEventCreateWithFlags(&start, cudaEventDisableTiming));
  SF_CUDA(cudaEventRecord(start, caller));
  for (auto& w : workers) {
    SF_CUDA(cudaStreamCreateWithFlags(&w->st, cudaStreamNonBlocking));
    SF_CUDA(cudaStreamWaitEvent(w->st, start, 0));
    if (o->proposer) {
      // a network handle's workspaces serve one stream at a time: one copy per worker
      if (simpfem_cnn_create(1, &w->cnn) != 0 ||
          simpfem_cnn_set_params(w->cnn, theta.data(), (int)theta.size()) != 0)
        throw std::runtime_error(std::string("floor proposer: ") + simpfem_last_error());
      w->own_cnn = true;
    }
  }
  std::vector<std::thread> threads;
  for (auto& wp : workers) {
    Worker* w = wp.get();
    threads.emplace_back([w, o, states, results, dev]() {
      try {
        SF_CUDA(cudaSetDevice(dev));
        for (int s : w->states)
          run_state(*w, *o, states[s].density, states[s].b_free, states[s].x_free, &results[s]);
      } catch (const CudaFailure&) {
        w->status = SIMPFEM_ECUDA;
        w->error = last_error();
      } catch (const InvalidArg& e) {
        w->status = SIMPFEM_EINVAL;
        w->error = e.msg;
      } catch (const NotSetup& e) {
        w->status = SIMPFEM_ENOTSETUP;
        w->error = e.msg;
      } catch (const std::exception& e) {
        w->status = SIMPFEM_EINTERNAL;
        w->error = e.what();
      }
    });
  }
  for (auto& t : threads) t.join();
  int status = SIMPFEM_OK;
  std::string msg;
  for (auto& w : workers) {
    cudaEvent_t done;
    if (cudaEventCreateWithFlags(&done, cudaEventDisableTiming) == cudaSuccess) {
      cudaEventRecord(done, w->st);
      cudaStreamWaitEvent(caller, done, 0);
      cudaEventDestroy(done);
    }
    if (w->status != SIMPFEM_OK && status == SIMPFEM_OK) {
      status = w->status;
      msg = w->error;
    }
  }
  for (auto& w : workers) {
    // the hierarchy's stream field points at the worker stream, which goes away
    cudaStreamSynchronize(w->st);
    w->g->impl->st = caller;
    cudaStreamDestroy(w->st);
  }
  cudaEventDestroy(start);
  if (status != SIMPFEM_OK) {
    set_error("simpfem_policy_batch: " + msg);
    return status;
  }
  SF_POLICY_END
}

}  // extern "C"
