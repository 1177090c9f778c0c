// Internal declarations shared by the simpfem CUDA sources.
//
// Data layout (every level, every vector): the reference's global DOF order,
// dof = 3 * node + component, node = (i * (ny + 1) + j) * (nz + 1) + k, with
// (i, j, k) the node's grid position and (nx, ny, nz) the element counts of the
// level.  Vectors inside the library are "full" (length 3 * n_nodes) and hold 0
// at constrained DOFs; the reference's compact free-DOF vectors only appear at
// the C-ABI boundary (expand / compress kernels).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <string>
#include <vector>

namespace simpfem {

enum DType { F64 = 0, F32 = 1, BF16 = 2 };

// Epilogues fused into the fine operator and the coarse stencil operator.
// Per owned DOF, with Ku the operator output and x the input value:
//   APPLY : y  = Ku
//   RESID : y  = b - Ku
//   CHEB1 : d  = dinv * (b - Ku);                  xo = x + s1 * d
//   CHEB  : d  = s1 * (dinv * (b - Ku) + s2 * d);  xo = x + d
//   JAC   : xo = x + (s1 * dinv) * (b - Ku)
// Constrained DOFs always receive 0 in every output.
enum Epi { EPI_APPLY = 0, EPI_RESID = 1, EPI_CHEB1 = 2, EPI_CHEB = 3, EPI_JAC = 4 };

struct EpiArgs {
  void* y = nullptr;
  const void* b = nullptr;
  const void* dinv = nullptr;
  void* d = nullptr;
  void* xo = nullptr;
  double s1 = 0.0, s2 = 0.0;
  const int* guard = nullptr;  // kernel body runs only when guard is null or *guard != 0
};

struct Grid {
  int nx = 0, ny = 0, nz = 0;  // elements
  int64_t nn = 0;              // nodes
  int64_t ndof = 0;
  __host__ __device__ int64_t ne() const { return (int64_t)nx * ny * nz; }
  static Grid make(int nx, int ny, int nz) {
    Grid g;
    g.nx = nx;
    g.ny = ny;
    g.nz = nz;
    g.nn = (int64_t)(nx + 1) * (ny + 1) * (nz + 1);
    g.ndof = 3 * g.nn;
    return g;
  }
};

// Tile shape of the fine-operator sweep kernel (chosen by the tuner).
struct SweepShape {
  int bj = 8;   // element columns along y per block (one of them is a halo column)
  int bk = 32;  // element columns along z per block (one halo column)
  int cx = 8;   // node planes along x per block
  int variant = 0;  // FP32 kernel, picked by the tuner like the tile: 0 = two elements per
                    // thread (packed FP32 pairs), 1 = one element per thread, 2 = two per
                    // thread compiled for two resident 256-thread blocks (a 128-register cap)
};

struct WhtBlocks {
  double b[8][9];  // 8 symmetry blocks (3x3 each) of the unit stiffness in the Walsh basis
};

// Workspace of the deterministic reductions (one per stream of work).
struct RedWork {
  double* partials;   // 4 * kRedBlocks doubles
  unsigned* ticket;   // zero-initialised counter
};

// Multi-dot: out[k] = sum_i term_k(i), double accumulation, fixed order.
//   mode 0: a*b ; mode 1: (a*c)*b ; mode 2: a*(b/c) where c != 0 ; mode 3: (a*c)*(b*c)
struct DotSet {
  const void* a[4] = {nullptr, nullptr, nullptr, nullptr};
  const void* b[4] = {nullptr, nullptr, nullptr, nullptr};
  const void* c[4] = {nullptr, nullptr, nullptr, nullptr};
  int mode[4] = {0, 0, 0, 0};
  int nd = 0;
};

// Device-resident Arnoldi / Givens state of one FGMRES instance.
enum KFlag {
  F_CYC = 0,      // current restart cycle active
  F_DONE = 1,     // solve finished
  F_CONV = 2,     // converged (incl. lucky breakdown)
  F_JF = 3,       // columns in the current cycle
  F_DID = 4,      // current cycle started (back-solve and update pending)
  F_TOTAL = 5,    // total iterations
  F_BREAK = 6,    // lucky breakdown seen
  F_NOTDONE = 7,  // 1 - done (guard for restart kernels)
  F_HISTN = 8,    // history entries written
  NFLAGS = 9
};
enum KScalar { SC_BNORM2 = 0, SC_BNORM = 1, SC_BETA2 = 2, SC_BETA = 3, SC_HSQ = 4, SC_HNORM = 5 };

struct KrylovDev {
  double* H = nullptr;   // (restart+1) x restart, column-major: H[j*(restart+1) + i]
  double* cs = nullptr;  // restart
  double* sn = nullptr;  // restart
  double* g = nullptr;   // restart+1
  double* y = nullptr;   // restart
  double* sc = nullptr;  // 16 scalars (KScalar)
  int* flags = nullptr;  // NFLAGS ints (KFlag); may live in mapped host memory
  int restart = 0;
};

enum ScalarOp { OP_LS1 = 0, OP_LS2 = 1, OP_RLF = 2, OP_RLL = 3 };

// ---------------------------------------------------------------- fine.cu
void set_fine_constants(const double* ke576, const WhtBlocks& wb);
cudaError_t launch_fine(DType t, Epi epi, const Grid& g, const SweepShape& sh, const void* E,
                        const uint8_t* mask, const void* u, const EpiArgs& ea, cudaStream_t s);
cudaError_t launch_fine_diag(const Grid& g, const double* E, const uint8_t* mask, double kd,
                             double* diag, cudaStream_t s);
cudaError_t launch_node_blocks(const Grid& g, const double* E, const uint8_t* mask,
                               const double* diag_full, double* binv, cudaStream_t s);
cudaError_t launch_node_block_apply(const Grid& g, const double* binv, const double* r, double* z,
                                    const int* guard, cudaStream_t s);
cudaError_t launch_element_energy(const Grid& g, const double* u_full, double* ce,
                                  cudaStream_t s);

// ------------------------------------------------------------- stencil.cu
// Coarse operators: 27-point 3x3-block stencils, coefficient c(o, r, q) of node n
// stored at coef[(o * 9 + r * 3 + q) * nn + n] (o = (dx+1)*9 + (dy+1)*3 + (dz+1)).
// BF16 copy of an FP64 structure-of-arrays stencil operator, node-major by
// neighbour column (288 entries per node), and the stencil application on it
// (FP32 vectors, nine lanes per node) used by the mixed cycle.
cudaError_t launch_stencil_colmajor_bf16(int64_t nn, const double* K64, __nv_bfloat16* out, cudaStream_t s);
cudaError_t launch_stencil_col_bf16(Epi epi, const Grid& g, const __nv_bfloat16* coefC, const uint8_t* mask,
                                    const float* u, const EpiArgs& ea, cudaStream_t s);
cudaError_t launch_stencil(DType vt, DType ct, Epi epi, const Grid& g, const void* coef,
                           const uint8_t* mask, const void* u, const EpiArgs& ea, cudaStream_t s);
cudaError_t launch_level1_assemble(const Grid& gc, const Grid& gf, const double* E_fine,
                                   const double* Q /*8*576*/, const uint8_t* mask_c, double* coef,
                                   cudaStream_t s);
cudaError_t launch_rap(const Grid& gf, const Grid& gc, const double* coef_f, const uint8_t* mask_c,
                       const double* wx, const double* wy, const double* wz, double* coef_c,
                       cudaStream_t s);
cudaError_t launch_stencil_diag(const Grid& g, const double* coef, const uint8_t* mask,
                                double* dinv, cudaStream_t s);
cudaError_t launch_restrict(DType t, const Grid& gf, const Grid& gc, const double* wx,
                            const double* wy, const double* wz, const uint8_t* mask_c,
                            const void* fine, void* coarse, const int* guard, cudaStream_t s);
cudaError_t launch_prolong(DType t, const Grid& gf, const Grid& gc, const double* wx,
                           const double* wy, const double* wz, const uint8_t* mask_f,
                           const void* coarse, void* fine, const int* guard, cudaStream_t s);
cudaError_t launch_stencil_to_dense(const Grid& g, const double* coef, const int32_t* dense_idx,
                                    int64_t n, double* A, cudaStream_t s);
cudaError_t launch_convert(DType from, DType to, const void* src, void* dst, int64_t n,
                           const int* guard, cudaStream_t s);

// -------------------------------------------------------------- linalg.cu
constexpr int kRedBlocksHost = 296;
cudaError_t launch_dots(DType t, int64_t n, const DotSet& ds, RedWork w, double* out,
                        const int* guard, cudaStream_t s);
cudaError_t launch_minmax_count(int64_t n, const double* E, double thr, RedWork w, double* out3,
                                cudaStream_t s);
cudaError_t launch_axpby(DType t, int64_t n, double alpha, const void* x, double beta,
                         const void* y, void* out, const int* guard, cudaStream_t s);
cudaError_t launch_fill(DType t, int64_t n, double v, void* out, const int* guard, cudaStream_t s);
cudaError_t launch_fill_hash(DType t, int64_t n, uint32_t seed, void* out, cudaStream_t s);
cudaError_t launch_copy(DType t, int64_t n, const void* src, void* dst, const int* guard,
                        cudaStream_t s);
cudaError_t launch_cheb_zero(DType t, int64_t n, double alpha, const void* dinv, const void* rhs,
                             void* d, void* x, const int* guard, cudaStream_t s);
cudaError_t launch_jac_zero(DType t, int64_t n, double omega, const void* dinv, const void* rhs,
                            void* x, const int* guard, cudaStream_t s);
cudaError_t launch_expand(DType t, int64_t n_free, const int32_t* free_idx, const void* src_free,
                          void* dst_full, cudaStream_t s);
cudaError_t launch_compress(DType t, int64_t n_free, const int32_t* free_idx,
                            const void* src_full, void* dst_free, cudaStream_t s);
cudaError_t launch_gather_idx(int64_t n, const int32_t* idx, const double* src, double* dst,
                              const int* guard, cudaStream_t s);
cudaError_t launch_scatter_idx(int64_t n, const int32_t* idx, const double* src, double* dst,
                               const int* guard, cudaStream_t s);
cudaError_t launch_vec_op(int64_t n, int op, const double* a, const double* b, const uint8_t* mask,
                          double s, const double* s_dev, double* out, cudaStream_t st);
cudaError_t launch_enrich_weights(int64_t n, const double* diag, const uint8_t* mask,
                                  const double* dmax_dev, double wfloor, double wpow, double* w,
                                  cudaStream_t s);
cudaError_t launch_enrich_rhs(int64_t n, int mode, const double* w, double wfloor, const double* r,
                              const double* p, const uint8_t* mask, double* out, const int* guard,
                              cudaStream_t s);

// Outputs of the factorisation: any of L^{-1} and L^{-T}, row-major n x n, in
// FP64 or FP32 (null: not written).  Entries on and below (L^{-1}) or on and
// above (L^{-T}) the diagonal are written; the other triangle is left as it is.
struct BandInvOut {
  double* L64 = nullptr;
  double* LT64 = nullptr;
  float* L32 = nullptr;
  float* LT32 = nullptr;
};
// The band path (bandchol.cu) takes matrices with ceil(bw / 32) <= kBandMaxTiles.
constexpr int kBandMaxTiles = 24;
int band_tiles(int bw);
bool band_path_available();  // the device can run the band path's 8-CTA cluster
size_t band_dinv_bytes(int n);  // scratch of the band path: the inverses of L's diagonal tiles
cudaError_t band_chol_inverse(double* A, int n, int bw, double* dinv, const BandInvOut& out, int* info,
                              cudaStream_t s);
// L^{-1} of the Cholesky factor of the SPD row-major A (destroyed) into the
// requested outputs.  The lower bandwidth bw of A is bw_known when that is >= 0
// (a structural bound: A is zero farther below the diagonal), else it is
// measured (one stream synchronisation); with ceil(bw / 32) <= kBandMaxTiles the band path writes
// the outputs directly, else the recursion in dense.cu factors into work64
// (n x n FP64) and the outputs are copied / transposed / converted from it.
// info_dev[0]: 0, or the 1-based index of the first non-positive pivot, or
// n + 1 when L^{-1} holds a non-finite entry; info_dev[1] is scratch.  dinv:
// band_dinv_bytes(n) of scratch.
cudaError_t chol_inverse(double* A, int n, double* work64, double* dinv, const BandInvOut& out, int* info_dev,
                         cudaStream_t s, int bw_known = -1);
// Linv <- L^{-1} (lower, zero upper): chol_inverse into a zeroed Linv.
cudaError_t dense_chol_inverse(double* A, int n, double* Linv, double* dinv, int* info_dev, cudaStream_t s);
cudaError_t launch_coarsest_solve(const double* Linv, const double* LinvT, int n, const double* b,
                                  double* tmp, double* x, const int* guard, cudaStream_t s);
// the same with FP32 copies of L^{-1} and L^{-T} (FP64 vectors and accumulation)
cudaError_t launch_coarsest_solve_f32(const float* Linv, const float* LinvT, int n, const double* b,
                                      double* tmp, double* x, const int* guard, cudaStream_t s);
cudaError_t launch_add_diag(double* A, int n, double eps, cudaStream_t s);
cudaError_t launch_diag_sum(const double* A, int n, double* out, cudaStream_t s);
cudaError_t launch_all_finite(const double* A, int64_t n, int* flag, cudaStream_t s);

cudaError_t launch_mgs_first(int64_t n, const double* v0, const double* w, RedWork rw, double* h0,
                             const int* guard, cudaStream_t s);
cudaError_t launch_mgs_step(int64_t n, const double* vi, const double* vnext, double* w,
                            const double* hi, RedWork rw, double* out, const int* guard,
                            cudaStream_t s);
cudaError_t launch_krylov_init(KrylovDev k, const int* parent, cudaStream_t s);
cudaError_t launch_krylov_restart(KrylovDev k, double tol, double* hist_host, int hist_cap,
                                  cudaStream_t s);
cudaError_t launch_givens(KrylovDev k, int j, double tol, double* hist_host, int hist_cap,
                          cudaStream_t s);
cudaError_t launch_scale_vec(int64_t n, const double* src, const double* denom_dev, double* dst,
                             const int* guard, cudaStream_t s);
cudaError_t launch_backsolve(KrylovDev k, cudaStream_t s);
cudaError_t launch_update_x(int64_t n, double* x, double* const* Z_dev, const double* y,
                            const int* flags, cudaStream_t s);
cudaError_t launch_scalar_op(int op, double* sc, double p0, double p1, const int* guard,
                             cudaStream_t s);
cudaError_t launch_select_axpy(DType t, int64_t n, void* x, const void* c, const double* sc,
                               int unit, const int* guard, cudaStream_t s);
cudaError_t launch_trial_residual(DType t, int64_t n, const void* r, const void* Ac, double* sc,
                                  int unit, void* trial, RedWork rw, const int* guard,
                                  cudaStream_t s);
cudaError_t launch_pcg_scalar(int which, double* sc, const int* guard, cudaStream_t s);
cudaError_t launch_pcg_xr(int64_t n, double* x, double* r, double* z, const double* p, const double* Ap,
                          const double* dinv, double* sc, RedWork rw, const int* guard, cudaStream_t s);
cudaError_t launch_pcg_p(int64_t n, const double* z, double* p, const double* sc, const int* guard,
                         cudaStream_t s);
cudaError_t launch_dmul(int64_t n, const double* dinv, const double* r, double* z, const int* guard,
                        cudaStream_t s);
cudaError_t launch_select_vec(DType t, int64_t n, const void* trial, const void* r,
                              const double* sc, void* out, const int* guard, cudaStream_t s);

// launch accounting: every launcher reports its kernel launches here
cudaError_t sf_launched(int k);

// Runs set() (a kernel attribute, say) the first time it is asked for the
// current device; `done` holds one bit per device.  Two host threads may both
// run it the first time -- harmless -- but none launches before its own call
// returned.
template <class F>
inline cudaError_t once_per_device(std::atomic<uint64_t>& done, F&& set) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const uint64_t bit = dev < 64 ? (uint64_t(1) << dev) : 0;
  if (bit != 0 && (done.load(std::memory_order_acquire) & bit) != 0) return cudaSuccess;
  e = set();
  if (e == cudaSuccess && bit != 0) done.fetch_or(bit, std::memory_order_release);
  return e;
}
int64_t sf_launch_count();

// error plumbing
void set_error(const std::string& msg);
const char* last_error();

#define SF_CUDA(call)                                                              \
  do {                                                                             \
    cudaError_t _e = (call);                                                       \
    if (_e != cudaSuccess) {                                                       \
      ::simpfem::set_error(std::string(#call) + ": " + cudaGetErrorString(_e));    \
      throw ::simpfem::CudaFailure(_e);                                            \
    }                                                                              \
  } while (0)

struct CudaFailure {
  cudaError_t err;
  explicit CudaFailure(cudaError_t e) : err(e) {}
};

}  // namespace simpfem
