// extern "C" boundary of libsimpfem (declarations in include/simpfem.h).
//
// Every entry point converts C++ failures into a status code and a message
// (simpfem_last_error); no exception crosses the ABI.
#include <math.h>
#include <stdio.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "gmg_impl.h"
#include "simpfem.h"

using namespace simpfem;

#include <atomic>
static std::atomic<int64_t> g_launches{0};
static std::atomic<int64_t> g_device_allocs{0};
namespace simpfem {
void sf_count_device_alloc() { g_device_allocs.fetch_add(1, std::memory_order_relaxed); }
cudaError_t sf_launched(int k) {
  g_launches.fetch_add(k, std::memory_order_relaxed);
  return cudaGetLastError();
}
int64_t sf_launch_count() { return g_launches.load(); }
}  // namespace simpfem


#define SF_API_BEGIN try {
#define SF_API_END                                                              \
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

static cudaStream_t S(void* s) { return (cudaStream_t)s; }

// The element stiffness lives in the constant bank of each device (the sweep
// kernels read its Walsh blocks from there), so all meshes alive on a device
// share one.  A mesh whose stiffness differs from that of the meshes alive on
// its device is refused; once none is left, the next mesh installs its own.
namespace {
struct ResidentKE {
  double ke[576];
  int live = 0;
  bool installed = false;
};
std::mutex g_ke_mutex;
std::map<int, ResidentKE> g_ke;
}  // namespace

static void acquire_element_constants(int device, const double* ke, const WhtBlocks& wb) {
  std::lock_guard<std::mutex> lk(g_ke_mutex);
  ResidentKE& r = g_ke[device];
  const bool same = r.installed && std::memcmp(r.ke, ke, sizeof(r.ke)) == 0;
  if (!same && r.live > 0)
    throw InvalidArg{"simpfem_mesh_create: the element stiffness differs from the one of the " +
                     std::to_string(r.live) + " mesh(es) alive on this device; destroy them first"};
  if (!same) {
    set_fine_constants(ke, wb);
    std::memcpy(r.ke, ke, sizeof(r.ke));
    r.installed = true;
  }
  r.live += 1;
}

static void release_element_constants(int device) {
  std::lock_guard<std::mutex> lk(g_ke_mutex);
  auto it = g_ke.find(device);
  if (it != g_ke.end() && it->second.live > 0) it->second.live -= 1;
}

extern "C" {

const char* simpfem_last_error(void) { return last_error(); }
int simpfem_version(void) { return 10000; }

int64_t simpfem_launch_count(void) { return sf_launch_count(); }
int64_t simpfem_device_alloc_count(void) { return g_device_allocs.load(); }

int simpfem_gmg_time_smoother_step(simpfem_gmg* g, int level, int reps, float* avg_ms, void* stream) {
  SF_API_BEGIN
  if (!g || !avg_ms || reps < 1) throw InvalidArg{"simpfem_gmg_time_smoother_step: invalid argument"};
  Gmg& G = *g->impl;
  if (!G.is_setup) throw NotSetup{"GalerkinMatFreeGMG.setup() must be called before apply()."};
  if (level < 0 || level >= G.L - 1) throw InvalidArg{"simpfem_gmg_time_smoother_step: level out of range"};
  G.st = S(stream);
  *avg_ms = time_smoother_step(G, level, reps);
  SF_API_END
}

int simpfem_gmg_time_operator(simpfem_gmg* g, int reps, float* avg_ms, void* stream) {
  SF_API_BEGIN
  if (!g || !avg_ms || reps < 1) throw InvalidArg{"simpfem_gmg_time_operator: invalid argument"};
  Gmg& G = *g->impl;
  if (!G.is_setup) throw NotSetup{"GalerkinMatFreeGMG.setup() must be called before apply()."};
  G.st = S(stream);
  *avg_ms = time_fine_operator(G, reps);
  SF_API_END
}

int simpfem_mesh_create(int nelx, int nely, int nelz, const int32_t* free_dofs_host, int64_t n_free,
                        const double* ke_unit_host, simpfem_mesh** out) {
  SF_API_BEGIN
  if (out == nullptr || nelx < 1 || nely < 1 || nelz < 1 || ke_unit_host == nullptr ||
      (n_free > 0 && free_dofs_host == nullptr))
    throw InvalidArg{"simpfem_mesh_create: invalid argument"};
  auto* h = new simpfem_mesh();
  Mesh& m = h->impl;
  m.g = Grid::make(nelx, nely, nelz);
  m.n_free = n_free;
  m.free_h.assign(free_dofs_host, free_dofs_host + n_free);
  m.mask_h.assign(m.g.ndof, 0);
  for (int64_t i = 0; i < n_free; ++i) {
    const int32_t d = m.free_h[i];
    if (d < 0 || d >= m.g.ndof || (i > 0 && d <= m.free_h[i - 1])) {
      delete h;
      throw InvalidArg{"simpfem_mesh_create: free DOFs must be ascending and inside the mesh"};
    }
    m.mask_h[d] = 1;
  }
  std::memcpy(m.ke, ke_unit_host, sizeof(m.ke));
  double off = 0.0;
  m.wb = make_wht_blocks(m.ke, &off);
  if (off > 1e-9) {
    delete h;
    throw InvalidArg{"simpfem_mesh_create: element stiffness lacks the unit-cube reflection symmetry"};
  }
  m.Q = make_level1_Q(m.ke);
  SF_CUDA(cudaGetDevice(&m.device));
  try {
    acquire_element_constants(m.device, m.ke, m.wb);
  } catch (...) {
    delete h;
    throw;
  }
  m.free_idx.alloc(4 * std::max<int64_t>(1, n_free));
  if (n_free > 0) SF_CUDA(cudaMemcpy(m.free_idx.p, m.free_h.data(), 4 * n_free, cudaMemcpyHostToDevice));
  m.mask.alloc(m.g.ndof);
  SF_CUDA(cudaMemcpy(m.mask.p, m.mask_h.data(), m.g.ndof, cudaMemcpyHostToDevice));
  m.init_red();
  m.sh[0] = default_shape(m.g, 256);
  m.sh[1] = default_shape(m.g, 512);
  *out = h;
  SF_API_END
}

int simpfem_mesh_destroy(simpfem_mesh* m) {
  SF_API_BEGIN
  if (m) release_element_constants(m->impl.device);
  delete m;
  SF_API_END
}

int simpfem_mesh_info(const simpfem_mesh* m, int64_t* ndof, int64_t* n_free, int64_t* n_elem) {
  SF_API_BEGIN
  if (!m) throw InvalidArg{"null mesh"};
  if (ndof) *ndof = m->impl.g.ndof;
  if (n_free) *n_free = m->impl.n_free;
  if (n_elem) *n_elem = m->impl.g.ne();
  SF_API_END
}

int simpfem_mesh_tune(simpfem_mesh* m, void* stream) {
  SF_API_BEGIN
  if (!m) throw InvalidArg{"null mesh"};
  tune_mesh(m->impl, F64, S(stream));
  tune_mesh(m->impl, F32, S(stream));
  SF_API_END
}

static DType api_dtype(int dt) {
  if (dt == SIMPFEM_F64) return F64;
  if (dt == SIMPFEM_F32) return F32;
  if (dt == SIMPFEM_BF16) return BF16;
  throw InvalidArg{"unknown dtype"};
}

int simpfem_matvec(simpfem_mesh* mh, int dtype, const void* E, const void* u_free, void* y_free,
                   void* stream) {
  SF_API_BEGIN
  if (!mh || !E || !u_free || !y_free) throw InvalidArg{"simpfem_matvec: null argument"};
  Mesh& m = mh->impl;
  const DType t = api_dtype(dtype);
  if (t == BF16) throw InvalidArg{"simpfem_matvec: dtype must be F64 or F32"};
  const size_t es = t == F64 ? 8 : 4;
  m.ufull.alloc(8 * m.g.ndof);
  m.yfull.alloc(8 * m.g.ndof);
  SF_CUDA(cudaMemsetAsync(m.ufull.p, 0, es * m.g.ndof, S(stream)));
  SF_CUDA(launch_expand(t, m.n_free, m.free_idx.as<int32_t>(), u_free, m.ufull.p, S(stream)));
  EpiArgs ea;
  ea.y = m.yfull.p;
  fine_apply(m, t, EPI_APPLY, E, m.ufull.p, ea, S(stream));
  SF_CUDA(launch_compress(t, m.n_free, m.free_idx.as<int32_t>(), m.yfull.p, y_free, S(stream)));
  SF_API_END
}

int simpfem_matvec_full(simpfem_mesh* mh, int dtype, const void* E, const void* u_full, void* y_full,
                        void* stream) {
  SF_API_BEGIN
  if (!mh || !E || !u_full || !y_full) throw InvalidArg{"simpfem_matvec_full: null argument"};
  Mesh& m = mh->impl;
  const DType t = api_dtype(dtype);
  EpiArgs ea;
  ea.y = y_full;
  fine_apply(m, t, EPI_APPLY, E, u_full, ea, S(stream));
  SF_API_END
}

int simpfem_extract_diagonal(simpfem_mesh* mh, const double* E, double* diag_free, void* stream) {
  SF_API_BEGIN
  if (!mh || !E || !diag_free) throw InvalidArg{"simpfem_extract_diagonal: null argument"};
  Mesh& m = mh->impl;
  m.yfull.alloc(8 * m.g.ndof);
  SF_CUDA(launch_fine_diag(m.g, E, m.mask.as<uint8_t>(), 0.0, m.yfull.as<double>(), S(stream)));
  SF_CUDA(launch_compress(F64, m.n_free, m.free_idx.as<int32_t>(), m.yfull.p, diag_free, S(stream)));
  SF_API_END
}

int simpfem_node_blocks(simpfem_mesh* mh, const double* E, const double* scalar_diag_free, double* blocks,
                        void* stream) {
  SF_API_BEGIN
  if (!mh || !E || !blocks) throw InvalidArg{"simpfem_node_blocks: null argument"};
  Mesh& m = mh->impl;
  const double* dfull = nullptr;
  if (scalar_diag_free) {
    m.ufull.alloc(8 * m.g.ndof);
    SF_CUDA(cudaMemsetAsync(m.ufull.p, 0, 8 * m.g.ndof, S(stream)));
    SF_CUDA(launch_expand(F64, m.n_free, m.free_idx.as<int32_t>(), scalar_diag_free, m.ufull.p, S(stream)));
    dfull = m.ufull.as<double>();
  }
  SF_CUDA(launch_node_blocks(m.g, E, m.mask.as<uint8_t>(), dfull, blocks, S(stream)));
  SF_API_END
}

int simpfem_node_block_apply(simpfem_mesh* mh, const double* blocks, const double* r_free, double* z_free,
                             void* stream) {
  SF_API_BEGIN
  if (!mh || !blocks || !r_free || !z_free) throw InvalidArg{"simpfem_node_block_apply: null argument"};
  Mesh& m = mh->impl;
  m.ufull.alloc(8 * m.g.ndof);
  m.yfull.alloc(8 * m.g.ndof);
  SF_CUDA(cudaMemsetAsync(m.ufull.p, 0, 8 * m.g.ndof, S(stream)));
  SF_CUDA(launch_expand(F64, m.n_free, m.free_idx.as<int32_t>(), r_free, m.ufull.p, S(stream)));
  SF_CUDA(launch_node_block_apply(m.g, blocks, m.ufull.as<double>(), m.yfull.as<double>(), nullptr, S(stream)));
  SF_CUDA(launch_compress(F64, m.n_free, m.free_idx.as<int32_t>(), m.yfull.p, z_free, S(stream)));
  SF_API_END
}

int simpfem_element_energy(simpfem_mesh* mh, const double* u_free, double* ce, void* stream) {
  SF_API_BEGIN
  if (!mh || !u_free || !ce) throw InvalidArg{"simpfem_element_energy: null argument"};
  Mesh& m = mh->impl;
  m.ufull.alloc(8 * m.g.ndof);
  SF_CUDA(cudaMemsetAsync(m.ufull.p, 0, 8 * m.g.ndof, S(stream)));
  SF_CUDA(launch_expand(F64, m.n_free, m.free_idx.as<int32_t>(), u_free, m.ufull.p, S(stream)));
  SF_CUDA(launch_element_energy(m.g, m.ufull.as<double>(), ce, S(stream)));
  SF_API_END
}

int simpfem_true_residual(simpfem_mesh* mh, const double* E, const double* b_free, const double* x_free,
                          double* out_host, void* stream) {
  SF_API_BEGIN
  if (!mh || !E || !b_free || !x_free || !out_host) throw InvalidArg{"simpfem_true_residual: null argument"};
  Mesh& m = mh->impl;
  const int64_t n = m.g.ndof;
  m.ufull.alloc(8 * n);
  m.yfull.alloc(8 * n);
  m.scratch.alloc(8 * n);
  SF_CUDA(cudaMemsetAsync(m.ufull.p, 0, 8 * n, S(stream)));
  SF_CUDA(cudaMemsetAsync(m.scratch.p, 0, 8 * n, S(stream)));
  SF_CUDA(launch_expand(F64, m.n_free, m.free_idx.as<int32_t>(), x_free, m.ufull.p, S(stream)));
  SF_CUDA(launch_expand(F64, m.n_free, m.free_idx.as<int32_t>(), b_free, m.scratch.p, S(stream)));
  EpiArgs ea;
  ea.y = m.yfull.p;
  ea.b = m.scratch.p;
  fine_apply(m, F64, EPI_RESID, E, m.ufull.p, ea, S(stream));
  DotSet ds;
  ds.a[0] = m.yfull.p;
  ds.b[0] = m.yfull.p;
  ds.a[1] = m.scratch.p;
  ds.b[1] = m.scratch.p;
  ds.nd = 2;
  SF_CUDA(launch_dots(F64, n, ds, m.rw, m.dscal.as<double>(), nullptr, S(stream)));
  double h[2];
  SF_CUDA(cudaMemcpyAsync(h, m.dscal.p, sizeof(h), cudaMemcpyDeviceToHost, S(stream)));
  SF_CUDA(cudaStreamSynchronize(S(stream)));
  *out_host = sqrt(h[0]) / sqrt(h[1]);
  SF_API_END
}

void simpfem_gmg_default_opts(simpfem_gmg_opts* o) {
  std::memset(o, 0, sizeof(*o));
  o->n_levels = 4;
  o->coarse_smooth_iters = 2;
  o->fine_smoother = SIMPFEM_F32;
  o->fine_smoother_degree = 2;
  o->omega = 0.5;
  o->dense_chol_max = 5000;
  o->coarse_pcg_iters = 80;
  o->smoother_type = 0;
  o->cheb_lower_frac = 1.0 / 30.0;
  for (int i = 0; i < 8; ++i) o->level_prec[i] = -1;
  o->cycle_type = 0;
  o->coarse_correction_policy = 0;
  o->coarse_correction_acceptance_ratio = 1.0;
  o->coarse_correction_max_scale = 1.0;
  o->root_enrichment_mode = 0;
  o->root_enrichment_weight_floor = 1e-6;
  o->root_enrichment_weight_power = 0.5;
  o->root_local_correction_mode = 0;
  o->root_local_correction_max_scale = 1.0;
  o->root_local_correction_inner_steps = 10;
  o->root_local_correction_inner_restart = 0;
  o->inner_krylov_steps = 0;
  o->inner_krylov_restart = 0;
  o->cycle_precision = SIMPFEM_F64;
  o->use_graphs = 0;
}

int simpfem_gmg_create(simpfem_mesh* mh, const simpfem_gmg_opts* opts, simpfem_gmg** out) {
  SF_API_BEGIN
  if (!mh || !opts || !out) throw InvalidArg{"simpfem_gmg_create: null argument"};
  auto* h = new simpfem_gmg();
  h->mesh = mh;
  h->impl = gmg_create(&mh->impl, *opts);
  h->bfull.alloc(8 * mh->impl.g.ndof);
  h->xfull.alloc(8 * mh->impl.g.ndof);
  *out = h;
  SF_API_END
}

int simpfem_gmg_destroy(simpfem_gmg* g) {
  SF_API_BEGIN
  if (g) {
    delete g->impl;
    delete g;
  }
  SF_API_END
}

int simpfem_gmg_setup(simpfem_gmg* g, const double* E, const double* fine_diag_free, void* stream) {
  SF_API_BEGIN
  if (!g || !E) throw InvalidArg{"simpfem_gmg_setup: null argument"};
  g->impl->st = S(stream);
  gmg_setup(*g->impl, E, fine_diag_free);
  SF_API_END
}

int simpfem_gmg_apply(simpfem_gmg* g, const double* rhs_free, double* z_free, void* stream) {
  SF_API_BEGIN
  if (!g || !rhs_free || !z_free) throw InvalidArg{"simpfem_gmg_apply: null argument"};
  Gmg& G = *g->impl;
  if (!G.is_setup) throw NotSetup{"GalerkinMatFreeGMG.setup() must be called before apply()."};
  Mesh& m = *G.m;
  G.st = S(stream);
  const int64_t n = m.g.ndof;
  SF_CUDA(cudaMemsetAsync(g->bfull.p, 0, 8 * n, G.st));
  SF_CUDA(launch_expand(F64, m.n_free, m.free_idx.as<int32_t>(), rhs_free, g->bfull.p, G.st));
  apply_full(G, g->bfull.as<double>(), g->xfull.as<double>(), nullptr);
  SF_CUDA(launch_compress(F64, m.n_free, m.free_idx.as<int32_t>(), g->xfull.p, z_free, G.st));
  SF_API_END
}

int simpfem_gmg_cycle_trace(simpfem_gmg* g, const double* rhs_free, int cycle_type, double* visits, int max_visits,
                            int* n_visits, double* summary, void* stream) {
  SF_API_BEGIN
  if (!g || !rhs_free || !n_visits || !summary || max_visits < 0 || (max_visits > 0 && !visits))
    throw InvalidArg{"simpfem_gmg_cycle_trace: invalid argument"};
  if (cycle_type < -1 || cycle_type > 1) throw InvalidArg{"cycle_type must be 'v' or 'w'"};
  Gmg& G = *g->impl;
  if (!G.is_setup) throw NotSetup{"GalerkinMatFreeGMG.setup() must be called before cycle_trace()."};
  Mesh& m = *G.m;
  G.st = S(stream);
  SF_CUDA(cudaMemsetAsync(g->bfull.p, 0, 8 * m.g.ndof, G.st));
  SF_CUDA(launch_expand(F64, m.n_free, m.free_idx.as<int32_t>(), rhs_free, g->bfull.p, G.st));
  std::vector<double> rec;
  trace_cycle(G, g->bfull.as<double>(), cycle_type < 0 ? G.o.cycle_type : cycle_type, &rec, summary);
  const int nv = (int)(rec.size() / kTraceVisitLen);
  *n_visits = nv;
  std::copy(rec.begin(), rec.begin() + (size_t)std::min(nv, max_visits) * kTraceVisitLen, visits);
  SF_API_END
}

int simpfem_gmg_props_get(simpfem_gmg* g, simpfem_gmg_props* p) {
  SF_API_BEGIN
  if (!g || !p) throw InvalidArg{"simpfem_gmg_props_get: null argument"};
  Gmg& G = *g->impl;
  std::memset(p, 0, sizeof(*p));
  p->n_levels = G.L;
  for (int l = 0; l < G.L; ++l) {
    p->n_free[l] = G.lv[l].n_free;
    p->dims[l][0] = G.lv[l].g.nx;
    p->dims[l][1] = G.lv[l].g.ny;
    p->dims[l][2] = G.lv[l].g.nz;
    p->lambda_max[l] = G.lv[l].lam;
    p->level_prec[l] = G.prec_resolved ? G.prec[l] : -1;
  }
  p->omega_used = G.omega_used;
  p->contrast_ratio = G.contrast;
  p->void_fraction = G.void_frac;
  p->is_high_contrast = G.high ? 1 : 0;
  p->fine_degree_adapt = G.fine_deg;
  p->coarse_iters_adapt = G.coarse_iters;
  p->coarse_mode = G.coarse_mode;
  p->coarse_regularised = G.coarse_reg ? 1 : 0;
  p->lambda_reestimated = G.lam_reest ? 1 : 0;
  p->cycle_graph_replays = G.graph_replays;
  SF_API_END
}

int simpfem_gmg_reset_lambda_cache(simpfem_gmg* g) {
  SF_API_BEGIN
  if (!g) throw InvalidArg{"null gmg"};
  g->impl->lam_Emax = NAN;
  for (auto& L : g->impl->lv) L.lam = NAN;
  SF_API_END
}

int simpfem_gmg_fine_E(simpfem_gmg* g, const double** E_out) {
  SF_API_BEGIN
  if (!g || !E_out) throw InvalidArg{"null argument"};
  *E_out = g->impl->E64.as<double>();
  SF_API_END
}

int simpfem_fgmres_checked(simpfem_gmg* g, const double* b_free, const double* x0_free, double* x_free,
                           double tol, int maxiter, int restart, double* history_host, int history_cap,
                           int* history_len, int* iters, int* converged, int check_iter,
                           int check_true_residual,
                           int (*check_fn)(void* ctx, int iters, const double* history, int history_len,
                                           double true_rel_residual),
                           void* check_ctx, int* stopped, void* stream) {
  SF_API_BEGIN
  if (!g || !b_free || !x_free) throw InvalidArg{"simpfem_fgmres: null argument"};
  if (restart < 1 || restart > 1000 || maxiter < 0) throw InvalidArg{"simpfem_fgmres: restart must be in [1, 1000]"};
  Gmg& G = *g->impl;
  if (!G.is_setup) throw NotSetup{"GalerkinMatFreeGMG.setup() must be called before apply()."};
  Mesh& m = *G.m;
  G.st = S(stream);
  const int64_t n = m.g.ndof;
  SF_CUDA(cudaMemsetAsync(g->bfull.p, 0, 8 * n, G.st));
  SF_CUDA(launch_expand(F64, m.n_free, m.free_idx.as<int32_t>(), b_free, g->bfull.p, G.st));
  SF_CUDA(cudaMemsetAsync(g->xfull.p, 0, 8 * n, G.st));
  if (x0_free) SF_CUDA(launch_expand(F64, m.n_free, m.free_idx.as<int32_t>(), x0_free, g->xfull.p, G.st));
  const int cap = maxiter + maxiter / std::max(restart, 1) + 4;
  G.hist_pin.alloc(sizeof(double) * cap);
  G.hist_dev.alloc(sizeof(double) * cap);
  PrecFn M = [&G](const double* in, double* out, const int* guard) { apply_full(G, in, out, guard); };
  CheckHook hook;
  hook.iter = check_iter;
  hook.true_residual = check_true_residual ? 1 : 0;
  hook.fn = check_iter >= 1 ? check_fn : nullptr;
  hook.ctx = check_ctx;
  run_outer_fgmres(G, g->bfull.as<double>(), g->xfull.as<double>(), x0_free == nullptr, tol, maxiter, restart, M,
                   G.hist_dev.as<double>(), cap, &hook);
  if (stopped) *stopped = hook.stopped ? 1 : 0;
  SF_CUDA(cudaMemcpyAsync(G.hist_pin.h, G.hist_dev.p, sizeof(double) * cap, cudaMemcpyDeviceToHost, G.st));
  SF_CUDA(cudaStreamSynchronize(G.st));
  const int* f = G.outer.hflags();
  const int hn = f[F_HISTN];
  if (history_len) *history_len = hn;
  if (history_host) {
    const int k = std::min(std::min(hn, history_cap), cap);
    std::memcpy(history_host, G.hist_pin.h, sizeof(double) * k);
  }
  if (iters) *iters = f[F_TOTAL];
  if (converged) *converged = f[F_CONV];
  SF_CUDA(launch_compress(F64, m.n_free, m.free_idx.as<int32_t>(), g->xfull.p, x_free, G.st));
  SF_API_END
}

int simpfem_fgmres(simpfem_gmg* g, const double* b_free, const double* x0_free, double* x_free, double tol,
                   int maxiter, int restart, double* history_host, int history_cap, int* history_len, int* iters,
                   int* converged, void* stream) {
  return simpfem_fgmres_checked(g, b_free, x0_free, x_free, tol, maxiter, restart, history_host, history_cap,
                                history_len, iters, converged, -1, 0, nullptr, nullptr, nullptr, stream);
}

int simpfem_pcg(simpfem_gmg* g, const double* b_free, const double* x0_free, double* x_free, double tol,
                int maxiter, double* history_host, int history_cap, int* history_len, int* iters, int* converged,
                void* stream) {
  SF_API_BEGIN
  if (!g || !b_free || !x_free) throw InvalidArg{"simpfem_pcg: null argument"};
  Gmg& G = *g->impl;
  if (!G.is_setup) throw NotSetup{"GalerkinMatFreeGMG.setup() must be called before apply()."};
  Mesh& m = *G.m;
  G.st = S(stream);
  const int64_t n = m.g.ndof;
  SF_CUDA(cudaMemsetAsync(g->bfull.p, 0, 8 * n, G.st));
  SF_CUDA(launch_expand(F64, m.n_free, m.free_idx.as<int32_t>(), b_free, g->bfull.p, G.st));
  SF_CUDA(cudaMemsetAsync(g->xfull.p, 0, 8 * n, G.st));
  if (x0_free) SF_CUDA(launch_expand(F64, m.n_free, m.free_idx.as<int32_t>(), x0_free, g->xfull.p, G.st));
  std::vector<double> hist;
  int it = 0, conv = 0;
  run_pcg(G, g->bfull.as<double>(), g->xfull.as<double>(), tol, maxiter, &hist, &it, &conv);
  if (history_len) *history_len = (int)hist.size();
  if (history_host)
    std::memcpy(history_host, hist.data(), sizeof(double) * std::min<size_t>(hist.size(), (size_t)history_cap));
  if (iters) *iters = it;
  if (converged) *converged = conv;
  SF_CUDA(launch_compress(F64, m.n_free, m.free_idx.as<int32_t>(), g->xfull.p, x_free, G.st));
  SF_API_END
}

int simpfem_dense_cholesky_inverse(int n, double* A, double* Linv, int* info_host, void* stream) {
  SF_API_BEGIN
  if (n < 0 || (n > 0 && (!A || !Linv)) || !info_host)
    throw InvalidArg{"simpfem_dense_cholesky_inverse: bad argument"};
  DevBuf info, dinv;
  info.alloc(2 * sizeof(int));
  dinv.alloc(band_dinv_bytes(n));
  SF_CUDA(dense_chol_inverse(A, n, Linv, dinv.as<double>(), info.as<int>(), S(stream)));
  SF_CUDA(cudaMemcpyAsync(info_host, info.p, sizeof(int), cudaMemcpyDeviceToHost, S(stream)));
  SF_CUDA(cudaStreamSynchronize(S(stream)));
  SF_API_END
}

}  // extern "C"
