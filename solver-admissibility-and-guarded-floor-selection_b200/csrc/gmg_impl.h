// Host-side structures of the simpfem library shared by gmg.cu and capi.cu.
#pragma once

#include <math.h>

#include <cstring>
#include <functional>
#include <string>
#include <vector>

#include "internal.h"
#include "simpfem.h"

namespace simpfem {

struct NotSetup {
  std::string msg;
};

struct InvalidArg {
  std::string msg;
};

// Device allocations made by the library (instrumentation, simpfem_device_alloc_count).
void sf_count_device_alloc();

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), bytes(o.bytes) {
    o.p = nullptr;
    o.bytes = 0;
  }
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  void* alloc(size_t b) {
    if (b == 0) b = 16;
    if (b <= bytes && p) return p;
    release();
    SF_CUDA(cudaMalloc(&p, b));
    sf_count_device_alloc();
    bytes = b;
    return p;
  }
  template <class T>
  T* as() const { return (T*)p; }
};

struct PinnedBuf {
  void* h = nullptr;
  void* d = nullptr;
  size_t bytes = 0;
  PinnedBuf() = default;
  PinnedBuf(const PinnedBuf&) = delete;
  ~PinnedBuf() {
    if (h) cudaFreeHost(h);
  }
  void alloc(size_t b) {
    if (b <= bytes && h) return;
    if (h) cudaFreeHost(h);
    SF_CUDA(cudaHostAlloc(&h, b, cudaHostAllocMapped));
    SF_CUDA(cudaHostGetDevicePointer(&d, h, 0));
    std::memset(h, 0, b);
    bytes = b;
  }
};

struct Mesh {
  Grid g;
  int64_t n_free = 0;
  std::vector<int32_t> free_h;
  std::vector<uint8_t> mask_h;
  DevBuf free_idx, mask;
  double ke[576];
  WhtBlocks wb;
  std::vector<double> Q;
  SweepShape sh[2];
  bool tuned[2] = {false, false};
  DevBuf ufull, yfull, scratch;
  DevBuf red_part, red_ticket;
  RedWork rw{};
  DevBuf dscal;  // device scalars
  int device = 0;

  void init_red() {
    red_part.alloc(sizeof(double) * 4 * kRedBlocksHost);
    red_ticket.alloc(sizeof(unsigned) * 4);
    SF_CUDA(cudaMemset(red_ticket.p, 0, sizeof(unsigned) * 4));
    rw.partials = red_part.as<double>();
    rw.ticket = red_ticket.as<unsigned>();
    dscal.alloc(sizeof(double) * 64);
  }
};

struct KrylovWs {
  int restart = 0;
  int64_t n = 0;
  DevBuf V, Z, w, r, H, cs, sn, g, y, sc, Zptr;
  DevBuf flags_dev;     // device-side control flags (read by every guarded kernel)
  PinnedBuf flags_pin;  // host mirror, refreshed by sync_flags()
  KrylovDev kd;

  void ensure(int64_t n_, int restart_) {
    if (restart_ == restart && n_ == n && V.p) return;
    restart = restart_;
    n = n_;
    V.alloc(sizeof(double) * (size_t)(restart + 1) * n);
    Z.alloc(sizeof(double) * (size_t)restart * n);
    w.alloc(sizeof(double) * n);
    r.alloc(sizeof(double) * n);
    H.alloc(sizeof(double) * (size_t)(restart + 1) * restart);
    SF_CUDA(cudaMemset(H.p, 0, sizeof(double) * (size_t)(restart + 1) * restart));
    cs.alloc(sizeof(double) * restart);
    sn.alloc(sizeof(double) * restart);
    g.alloc(sizeof(double) * (restart + 1));
    y.alloc(sizeof(double) * restart);
    sc.alloc(sizeof(double) * 16);
    flags_dev.alloc(sizeof(int) * NFLAGS);
    SF_CUDA(cudaMemset(flags_dev.p, 0, sizeof(int) * NFLAGS));
    flags_pin.alloc(sizeof(int) * NFLAGS);
    std::vector<double*> zp(restart);
    for (int j = 0; j < restart; ++j) zp[j] = Z.as<double>() + (size_t)j * n;
    Zptr.alloc(sizeof(double*) * restart);
    SF_CUDA(cudaMemcpy(Zptr.p, zp.data(), sizeof(double*) * restart, cudaMemcpyHostToDevice));
    kd.H = H.as<double>();
    kd.cs = cs.as<double>();
    kd.sn = sn.as<double>();
    kd.g = g.as<double>();
    kd.y = y.as<double>();
    kd.sc = sc.as<double>();
    kd.flags = flags_dev.as<int>();
    kd.restart = restart;
  }
  double* Vj(int j) { return V.as<double>() + (size_t)j * n; }
  double* Zj(int j) { return Z.as<double>() + (size_t)j * n; }
  const int* hflags() const { return (const int*)flags_pin.h; }
  void sync_flags(cudaStream_t s) {
    SF_CUDA(cudaMemcpyAsync(flags_pin.h, flags_dev.p, sizeof(int) * NFLAGS, cudaMemcpyDeviceToHost, s));
    SF_CUDA(cudaStreamSynchronize(s));
  }
  const int* dflag(int f) const { return kd.flags + f; }
};

struct Level {
  Grid g;
  std::vector<uint8_t> mask_h;
  DevBuf mask;
  int64_t n_free = 0;
  // transfer weights between this level (fine side) and the next coarser one
  DevBuf wx, wy, wz;
  // coarse operator (levels >= 1)
  DevBuf K64, K32, K16;
  DevBuf s64a, s64b, s64c;  // FP64 scratch of the setup-time power iterations
  DevBuf dinv64, dinv32;
  double lam = NAN;
  // cycle vectors in the cycle dtype
  DevBuf x[2], res, c, Ac, d, rhs, trial, res2, ptmp;
  // FP32 smoothing scratch (reference mode with an fp32 level)
  DevBuf xs[2], ds, rhss;
};

struct Gmg {
  Mesh* m = nullptr;
  simpfem_gmg_opts o;
  int L = 1;
  std::vector<Level> lv;
  DType cyc = F64;  // cycle vector dtype
  int prec[8];      // resolved per-level smoother precision
  bool prec_resolved = false;

  DevBuf E64, E32, diag0, wenrich, binv, Qdev;
  bool is_setup = false;

  // lambda cache
  double lam_Emax = NAN;
  int lam_calls = 0;
  bool lam_reest = false;
  double omega_used;
  double contrast = NAN, void_frac = 0.0;
  bool high = false;
  int fine_deg = 2, coarse_iters = 2;

  // coarsest dense solve
  int coarse_mode = 0;
  bool coarse_reg = false;
  int nc = 0;
  int c_bw = -1;  // structural lower bandwidth of the dense coarsest matrix
  DevBuf c_idx, c_didx, Adense, Linv, LinvT, cb, cx, ctmp, cinfo;
  DevBuf LinvF, LinvTF;  // FP32 copies of Linv and LinvT read by the mixed cycle
  DevBuf cdinv;          // inverses of the diagonal tiles of the coarsest factor (scratch)
  // iterative coarse (fixed PCG) vectors
  DevBuf pr, pz, pp, pAp;

  DevBuf sc;         // scalar scratch of the corrections
  DevBuf rhs64, out64, tmp64a, tmp64b, tmp64c, tmp64d;  // apply-level FP64 vectors
  DevBuf cyc_in, cyc_out;  // mixed mode: FP32 copies at the cycle boundary
  KrylovWs ik, rl, outer;
  cudaStream_t st = nullptr;
  const int* guard = nullptr;

  // outer solve history (device) and its host copy
  DevBuf hist_dev;
  PinnedBuf hist_pin;

  // The V/W-cycle body captured as a CUDA graph (use_graphs): one per guard
  // pointer (the kernels' skip flag is a launch argument), valid for the setup
  // it was captured after -- every setup changes host-side launch arguments
  // (Chebyshev coefficients, sweep counts) and bumps setup_epoch.  The first
  // cycle after a setup runs directly, the second is captured (and replayed),
  // later ones are replayed.  A capture that fails turns graphs off for the
  // hierarchy.
  struct CycleGraph {
    const int* guard = nullptr;
    void* out = nullptr;  // level-0 buffer holding the cycle's answer
    cudaGraphExec_t exec = nullptr;
    int launches = 0;    // kernel nodes (launch accounting)
    uint64_t epoch = 0;  // setup the graph belongs to (0 = none)
    bool valid = false;  // exec holds this epoch's cycle
    int direct = 0;      // direct runs since that setup
  };
  std::vector<CycleGraph> graphs;
  uint64_t setup_epoch = 0;
  bool graphs_off = false;
  int64_t graph_replays = 0;
  cudaStream_t cap_stream = nullptr;  // private stream the cycle is captured on

  Gmg() = default;
  Gmg(const Gmg&) = delete;
  Gmg& operator=(const Gmg&) = delete;
  ~Gmg() {
    for (CycleGraph& c : graphs)
      if (c.exec) cudaGraphExecDestroy(c.exec);
    if (cap_stream) cudaStreamDestroy(cap_stream);
  }

  int64_t nfull() const { return m->g.ndof; }
};

using PrecFn = std::function<void(const double* in, double* out, const int* guard)>;

WhtBlocks make_wht_blocks(const double* ke, double* max_off);
std::vector<double> make_level1_Q(const double* ke);
SweepShape default_shape(const Grid& g, int maxt);
void fine_apply(Mesh& m, DType t, Epi epi, const void* E, const void* u, const EpiArgs& ea, cudaStream_t s);
void tune_mesh(Mesh& m, DType t, cudaStream_t s);
Gmg* gmg_create(Mesh* m, const simpfem_gmg_opts& o);
void gmg_setup(Gmg& G, const double* E, const double* fine_diag_free);
void apply_full(Gmg& G, const double* rhs, double* out, const int* guard);
// A host check called once, when the outer FGMRES has completed ``iter``
// iterations and is still running: fn(ctx, iter, history, history_len,
// true_rel) sees the relative-residual history so far (and, with
// true_residual set, ||b - A x_iter|| / ||b|| of the iterate formed at that
// point, else NaN) and returns nonzero to end the solve there.
struct CheckHook {
  int iter = -1;
  int true_residual = 0;
  int (*fn)(void* ctx, int iters, const double* history, int history_len, double true_rel) = nullptr;
  void* ctx = nullptr;
  mutable std::vector<double> buf;
  mutable bool stopped = false;
};
void run_outer_fgmres(Gmg& G, const double* b, double* x, bool x0_zero, double tol, int maxiter, int restart,
                      const PrecFn& M, double* hist_dev, int hist_cap, const CheckHook* check = nullptr);

// The operator side of a Krylov solve (krylov.cu): A computes y = A x and R the
// residual r = b - A x, both skipped on the device when *guard == 0 (guard may
// be null).  Vectors have n entries; reductions use rw on stream st.
struct KrylovEnv {
  int64_t n = 0;
  cudaStream_t st = nullptr;
  RedWork rw{};
  std::function<void(const double* x, double* y, const int* guard)> A;
  std::function<void(const double* x, const double* b, double* r, const int* guard)> R;
};
// Restarted right-preconditioned FGMRES with the Arnoldi basis, Hessenberg
// columns, Givens rotations and back-solve on the device (_cupy_fgmres,
// gpu_fem/multigrid_v4.py:416-534).  host_control: read the device flags after
// every Givens update and stop launching once the cycle has ended (one
// synchronisation per iteration); otherwise the whole solve is a fixed kernel
// sequence whose unneeded parts are skipped by device flags.
void fgmres_core(const KrylovEnv& E, KrylovWs& K, const double* b, double* x, bool x0_zero, double tol,
                 int maxiter, int restart, const PrecFn& M, const int* parent, bool host_control, double* hist_dev,
                 int hist_cap, const CheckHook* check);
// Preconditioned CG with the up-front convergence check (_cupy_pcg,
// gpu_fem/solver_v2.py:551-623); iters counts preconditioner applications.
// r, z, p, Ap: n-vectors of scratch; sc: 4 device doubles.
void pcg_core(const KrylovEnv& E, const PrecFn& M, const double* b, double* x, double tol, int maxiter, double* r,
              double* z, double* p, double* Ap, double* sc, std::vector<double>* hist, int* iters, int* conv);
float time_smoother_step(Gmg& G, int l, int reps);
float time_fine_operator(Gmg& G, int reps);
float time_cold(const std::function<void()>& launch, int reps, cudaStream_t st);
void run_pcg(Gmg& G, const double* b, double* x, double tol, int maxiter, std::vector<double>* hist, int* iters,
             int* conv);

// Building blocks of the cycle (vectors in the cycle dtype G.cyc, full layout of
// the level), shared by the cycle itself and the traced cycle.
// level operator: ea.y <- K_l u (EPI_APPLY) or ea.b - K_l u (EPI_RESID)
void level_op(Gmg& G, int l, DType vt, int precsel, Epi epi, const void* u, EpiArgs ea);
const void* level_dinv(Gmg& G, int l, DType t);
// smoothing sweeps on level l from x_in (nullptr = zero); returns the buffer holding x
void* smooth(Gmg& G, int l, const void* rhs, const void* x_in);
void solve_coarsest(Gmg& G, const void* rhs, void* x);
// x <- x + s c under the coarse-correction policy; the corrected residual in
// res_out when non-null; the decision scalars stay in G.sc[0..8]
void coarse_correction(Gmg& G, int l, void* x, const void* res, const void* c, void* res_out);
void enrichment_rhs(Gmg& G, const void* residual, void* rc_out);
// root-local correction of the FP64 full-layout x; decision scalars in G.sc[16..24]
void root_local(Gmg& G, const double* rhs, double* x);

// One cycle traced on the device (gpu_fem/multigrid_v4.py:1362-1728): records of
// kTraceVisitLen doubles per visit in pre-order, and a kTraceSummaryLen summary.
constexpr int kTraceVisitLen = 32;
constexpr int kTraceSummaryLen = 16;
void trace_cycle(Gmg& G, const double* rhs_full, int cycle_type, std::vector<double>* visits,
                 double* summary);

}  // namespace simpfem

// The C ABI's opaque handles (include/simpfem.h).
struct simpfem_mesh {
  simpfem::Mesh impl;
};
struct simpfem_gmg {
  simpfem::Gmg* impl = nullptr;
  simpfem_mesh* mesh = nullptr;
  simpfem::DevBuf bfull, xfull;
};

