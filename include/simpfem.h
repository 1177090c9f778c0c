/*
 * simpfem: B200-native guarded SIMP-floor linear-elasticity solve (C ABI).
 *
 * Every entry point returns 0 on success or a positive SIMPFEM_E* status; the
 * message of the last failure on the calling thread is simpfem_last_error().
 * Array arguments are device pointers unless the name ends in _host.  "free"
 * vectors are the reference's compact free-DOF vectors (length n_free, in the
 * order of the free-DOF list given to simpfem_mesh_create); "full" vectors have
 * one entry per global DOF (3 * n_nodes) and hold 0 at constrained DOFs.
 * Streams are cudaStream_t passed as void* (NULL = legacy default stream).  No
 * call allocates caller-visible memory; a handle keeps its own work buffers.
 * Element moduli E are indexed e = (i * nely + j) * nelz + k as in the
 * reference (gpu_fem/pub_simp_solver.py:196-207).
 */
#ifndef SIMPFEM_H
#define SIMPFEM_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#ifdef __cplusplus
extern "C" {
#endif

enum {
  SIMPFEM_OK = 0,
  SIMPFEM_EINVAL = 1,       /* bad argument */
  SIMPFEM_ECUDA = 2,        /* CUDA runtime failure */
  SIMPFEM_ENOTSETUP = 5,    /* apply before setup (reference raises RuntimeError) */
  SIMPFEM_ENONFINITE = 6,   /* non-finite input or result */
  SIMPFEM_ECALLBACK = 7,    /* a caller-supplied operator callback reported a failure */
  SIMPFEM_EINTERNAL = 9
};

enum { SIMPFEM_F64 = 0, SIMPFEM_F32 = 1, SIMPFEM_BF16 = 2 };

typedef struct simpfem_mesh simpfem_mesh;
typedef struct simpfem_gmg simpfem_gmg;

const char* simpfem_last_error(void);
int simpfem_version(void);
/* Number of CUDA kernels this library has launched in the process (no reference
 * counterpart: instrumentation for benchmarks). */
int64_t simpfem_launch_count(void);
/* Number of device allocations (cudaMalloc) this library has made in the process
 * (no reference counterpart: instrumentation, e.g. to check that an entry point
 * allocates nothing). */
int64_t simpfem_device_alloc_count(void);

/* Structured hex8 mesh of nelx*nely*nelz unit elements with the given free-DOF
 * list (ascending global DOF indices) and the 24x24 unit element stiffness in
 * the reference's local order.  Replaces the state MatrixFreeKff.__init__ keeps
 * (gpu_fem/solver_v2.py:1153-1176); the edof table is implicit. */
int simpfem_mesh_create(int nelx, int nely, int nelz, const int32_t* free_dofs_host,
                        int64_t n_free, const double* ke_unit_host, simpfem_mesh** out);
int simpfem_mesh_destroy(simpfem_mesh* m);
int simpfem_mesh_info(const simpfem_mesh* m, int64_t* ndof, int64_t* n_free, int64_t* n_elem);
/* Pick the sweep tile shape of the fine operator by timing candidates (the tuner);
 * runs on first use otherwise. */
int simpfem_mesh_tune(simpfem_mesh* m, void* stream);

/* y_free = K_ff(E) u_free; dtype SIMPFEM_F64 or SIMPFEM_F32 for E/u/y
 * (MatrixFreeKff.matvec, gpu_fem/solver_v2.py:1182-1222). */
int simpfem_matvec(simpfem_mesh* m, int dtype, const void* E, const void* u_free, void* y_free,
                   void* stream);
/* Full-layout operator (FusedMatvec.matvec_full, gpu_fem/cuda_fused_matvec.py:379-391):
 * dtype SIMPFEM_F32 or SIMPFEM_BF16 (bf16-rounded operands, FP32 accumulation), or F64. */
int simpfem_matvec_full(simpfem_mesh* m, int dtype, const void* E, const void* u_full,
                        void* y_full, void* stream);
/* diag(K_ff) (MatrixFreeKff.extract_diagonal, gpu_fem/solver_v2.py:1228-1251). */
int simpfem_extract_diagonal(simpfem_mesh* m, const double* E, double* diag_free, void* stream);
/* 3x3 node-block Jacobi: update with E and the scalar diagonal (free layout, may be
 * NULL), then apply z = M^{-1} r (NodeBlockJacobiMF.update/apply,
 * gpu_fem/solver_v2.py:1381-1451).  blocks: n_nodes * 9 doubles owned by the caller. */
int simpfem_node_blocks(simpfem_mesh* m, const double* E, const double* scalar_diag_free,
                        double* blocks, void* stream);
int simpfem_node_block_apply(simpfem_mesh* m, const double* blocks, const double* r_free,
                             double* z_free, void* stream);
/* u_e^T KE u_e per element from a free-layout displacement (SolverV4 sensitivity,
 * gpu_fem/solver_v4.py:257-264). */
int simpfem_element_energy(simpfem_mesh* m, const double* u_free, double* ce, void* stream);
/* ||b - K(E) x|| / ||b|| in FP64, written to *out_host (the recomputed true-residual
 * guard, experiments/phase5/run_gmg_floor_detector_prospective.py:246-247). */
int simpfem_true_residual(simpfem_mesh* m, const double* E, const double* b_free,
                          const double* x_free, double* out_host, void* stream);
/* The same guard for callers that must not allocate device memory (no counterpart
 * in the reference).  A host framework that owns all device memory through its own
 * pool may forbid a library's cudaMalloc/cudaFree (allocations escape its accounting,
 * cudaFree synchronises the device); simpfem_true_residual sizes work buffers in the
 * mesh handle on first use, this entry point allocates nothing.  Inputs are
 * full-layout vectors (3 * n_nodes); x_full must hold 0 at constrained DOFs (the
 * operator reads every entry, so a nonzero one adds its coupling K_fc x_c), while
 * entries of b_full at constrained DOFs are ignored.  r_full receives b - K(E) x
 * on the free DOFs and 0 elsewhere; *out_host = ||r|| / ||b|| over the free DOFs.  The reduction scratch is one fixed array of
 * about 64 KB compiled into the library and resident on every GPU that loads it; the
 * mesh may have at most 8,388,608 DOFs (SIMPFEM_EINVAL beyond).  All calls on a
 * device share that array, so calls that overlap on one GPU race: serialise them.
 * The first call on a device looks up the array's address with that device current;
 * make it before any stream capture. */
int simpfem_true_residual_noalloc(simpfem_mesh* m, const double* E, const double* b_full,
                                  const double* x_full, double* r_full, double* out_host,
                                  void* stream);

/* Options of the Galerkin GMG hierarchy: the keyword arguments of
 * GalerkinMatFreeGMG.__init__ (gpu_fem/multigrid_v4.py:546-580).  The caller
 * validates them (the Python layer raises the reference's ValueErrors). */
typedef struct simpfem_gmg_opts {
  int n_levels;                    /* 4 */
  int coarse_smooth_iters;         /* 2 */
  int fine_smoother;               /* SIMPFEM_F64 / F32 / BF16 ("fp64","fp32","bf16") */
  int fine_smoother_degree;        /* 2 */
  double omega;                    /* 0.5 */
  int dense_chol_max;              /* 5000 */
  int coarse_pcg_iters;            /* 80 */
  int smoother_type;               /* 0 chebyshev, 1 jacobi */
  double cheb_lower_frac;          /* 1/30 */
  int level_prec[8];               /* per level dtype; -1 = reference default schedule */
  int cycle_type;                  /* 0 V, 1 W */
  int coarse_correction_policy;    /* 0 none, 1 residual_line_search */
  double coarse_correction_acceptance_ratio; /* 1.0 */
  double coarse_correction_max_scale;        /* 1.0 */
  int root_enrichment_mode;        /* 0 none, 1 weighted_residual_second, 2 weighted_gap_second,
                                      3 void_residual_second, 4 void_gap_second */
  double root_enrichment_weight_floor;  /* 1e-6 */
  double root_enrichment_weight_power;  /* 0.5 */
  int root_local_correction_mode;  /* 0 none, 1 node_block_line_search, 2 node_block_inner_fgmres */
  double root_local_correction_max_scale; /* 1.0 */
  int root_local_correction_inner_steps;   /* 10 */
  int root_local_correction_inner_restart; /* steps when <= 0 */
  int inner_krylov_steps;          /* 0 */
  int inner_krylov_restart;        /* steps when <= 0 */
  int cycle_precision;             /* SIMPFEM_F64: the reference's FP64 cycle with per-level
                                      smoother precision; SIMPFEM_F32: mixed mode, the whole
                                      V-cycle in FP32 with BF16-stored coarse stencils
                                      (no reference counterpart) */
  int use_graphs;                  /* 1: the V/W-cycle body is captured as a CUDA graph on the
                                      second cycle after each setup (per skip-flag pointer) and
                                      replayed after that; identical kernels and arguments.
                                      0 (the C default): every kernel launched directly */
} simpfem_gmg_opts;

void simpfem_gmg_default_opts(simpfem_gmg_opts* o);

/* Read-only state after setup (GalerkinMatFreeGMG properties, multigrid_v4.py:772-837). */
typedef struct simpfem_gmg_props {
  int n_levels;
  int64_t n_free[8];
  int dims[8][3];
  double lambda_max[8];
  double omega_used;
  double contrast_ratio;
  double void_fraction;
  int is_high_contrast;
  int fine_degree_adapt;
  int coarse_iters_adapt;
  int level_prec[8];
  int coarse_mode;          /* 0 none, 1 dense Cholesky, 2 iterative (fixed Jacobi-PCG) */
  int coarse_regularised;   /* 1 if the eps-regularised retry was used */
  int lambda_reestimated;   /* 1 if the last setup re-estimated lambda_max */
  int64_t nnz[8];           /* structural nonzeros of the coarse operators (free-free) */
  int64_t cycle_graph_replays; /* cycles run by replaying a captured graph (use_graphs) */
} simpfem_gmg_props;

int simpfem_gmg_create(simpfem_mesh* m, const simpfem_gmg_opts* opts, simpfem_gmg** out);
int simpfem_gmg_destroy(simpfem_gmg* g);
/* GalerkinMatFreeGMG.setup (multigrid_v4.py:1119-1341); fine_diag_free may be NULL. */
int simpfem_gmg_setup(simpfem_gmg* g, const double* E, const double* fine_diag_free, void* stream);
/* z = M(rhs) (GalerkinMatFreeGMG.apply, multigrid_v4.py:1759-1767); FP64 free layout. */
int simpfem_gmg_apply(simpfem_gmg* g, const double* rhs_free, double* z_free, void* stream);
/* One base cycle traced on the device, then the root-local correction
 * (GalerkinMatFreeGMG.cycle_trace, multigrid_v4.py:1362-1728; the inner Krylov
 * wrapper is not traced).  rhs_free: device FP64 free layout.  cycle_type: 0 V,
 * 1 W, -1 the hierarchy's own.  visits / summary: HOST arrays.  Each visit is
 * SIMPFEM_TRACE_VISIT_LEN doubles in visit (pre-)order, NaN where the reference
 * records None:
 *   0 visit_id  1 level  2 is_coarsest  3 n_coarse_corrections  4 rhs_norm
 *   5 jacobi_action_norm  6 presmooth_solution_norm  7 presmooth_residual_norm
 *   8 restricted_rhs_norm  9 projector_norm  10 coarse_space_gap_norm
 *   11 coarse_correction_norm  12 prolongated_correction_norm  13 correction_alignment
 *   14 correction_scale_raw  15 correction_scale_applied  16 corrected_residual_norm
 *   17 residual norm after the first correction  18 second_restricted_rhs_norm
 *   19 second_coarse_correction_norm  20 second_prolongated_correction_norm
 *   21 second_correction_alignment  22 second_correction_scale_raw
 *   23 second_correction_scale_applied  24 second_corrected_residual_norm
 *   25 postsmooth_solution_norm  26 postsmooth_residual_norm
 *   27 first note, 28 second note (-1 none): 0 "", 1 degenerate_correction,
 *      2 rejected_correction, 3 nonpositive_correction_scale, 4 clipped_correction_scale
 *   29 root enrichment applied  30 extra fine post-smoothing
 *   31 coarsest mode (-1 not the coarsest, 0 none, 1 dense, 2 iterative)
 * summary (SIMPFEM_TRACE_SUMMARY_LEN doubles): 0 rhs_norm  1 jacobi_action_norm
 *   2 output_norm  3 rz  4 output_residual_norm  5 residual norm before the
 *   root-local correction  6 root-local raw scale  7 root-local applied scale
 *   8 root-local note (0 "", 1 degenerate_root_local_correction,
 *   2 rejected_root_local_inner_fgmres, 3 root_local_inner_fgmres,
 *   4 nonpositive_root_local_scale, 5 clipped_root_local_scale)  9 contrast ratio
 *   10 high contrast  11 fine degree  12 coarse sweeps  13 visits taken
 *   14 coarsest mode.  *n_visits = visits taken (records beyond max_visits are
 *   not written).  Synchronises the stream at every norm. */
#define SIMPFEM_TRACE_VISIT_LEN 32
#define SIMPFEM_TRACE_SUMMARY_LEN 16
int simpfem_gmg_cycle_trace(simpfem_gmg* g, const double* rhs_free, int cycle_type, double* visits,
                            int max_visits, int* n_visits, double* summary, void* stream);
int simpfem_gmg_props_get(simpfem_gmg* g, simpfem_gmg_props* out);
/* Average device time (ms) of one fused smoothing step of `level` (below the
 * coarsest) -- the operator kernel with the smoother's update fused into its
 * store, the kernel the cycle launches most -- over `reps` launches, each timed by
 * its own CUDA event pair on `stream` after 256 MB of pseudo-random values are
 * written (twice the L2, data it cannot hold compressed), on
 * pseudo-random input vectors; clobbers that level's cycle vectors (no reference
 * counterpart: instrumentation for the roofline report). */
int simpfem_gmg_time_smoother_step(simpfem_gmg* g, int level, int reps, float* avg_ms, void* stream);
/* Average device time (ms) of the FP64 fine operator product y = K(E) u -- the
 * product of every outer FGMRES iteration and of the guard -- with the moduli of
 * the last setup, timed like simpfem_gmg_time_smoother_step (cold L2, own event
 * pair per launch); clobbers the hierarchy's FP64 scratch vectors (no reference
 * counterpart: instrumentation for the roofline report). */
int simpfem_gmg_time_operator(simpfem_gmg* g, int reps, float* avg_ms, void* stream);
/* Forget the cached lambda_max estimates (the next setup re-estimates). */
int simpfem_gmg_reset_lambda_cache(simpfem_gmg* g);
/* Copy the fine-level operator of the last setup: E as FP64 (n_elem). */
int simpfem_gmg_fine_E(simpfem_gmg* g, const double** E_out);

/* FGMRES with the hierarchy as right preconditioner and the fine FP64 operator of
 * the last setup (_cupy_fgmres, multigrid_v4.py:416-534).  x0_free may be NULL.
 * history_host receives ||r||/||b|| entries with the reference's rule (start of each
 * restart, then after every iteration); *history_len may exceed history_cap, in which
 * case only history_cap entries are written. */
int simpfem_fgmres(simpfem_gmg* g, const double* b_free, const double* x0_free, double* x_free,
                   double tol, int maxiter, int restart, double* history_host, int history_cap,
                   int* history_len, int* iters, int* converged, void* stream);
/* simpfem_fgmres with a host check, no counterpart in the reference (the learned
 * floor policy decides at the probe's r50 point with it, and the checkpointed
 * guard -- the reference README's proposed extension -- reads the true residual
 * there): once the solve has completed check_iter iterations and is still
 * running, check_fn(check_ctx, check_iter, history, history_len, true_rel) is
 * called on the calling thread with the relative-residual history so far and,
 * when check_true_residual is nonzero, the FP64 true relative residual
 * ||b - A x|| / ||b|| of the iterate formed at that point (NaN otherwise; the
 * solve itself is not changed).  A nonzero return ends the solve there, with
 * x_free the iterate after check_iter iterations, *converged 0 and *stopped 1.
 * check_iter < 1 or check_fn NULL is simpfem_fgmres.  stopped may be NULL. */
int simpfem_fgmres_checked(simpfem_gmg* g, const double* b_free, const double* x0_free, double* x_free,
                           double tol, int maxiter, int restart, double* history_host, int history_cap,
                           int* history_len, int* iters, int* converged, int check_iter,
                           int check_true_residual,
                           int (*check_fn)(void* ctx, int iters, const double* history, int history_len,
                                           double true_rel_residual),
                           void* check_ctx, int* stopped, void* stream);
/* PCG with the hierarchy as preconditioner (_cupy_pcg, gpu_fem/solver_v2.py:551-623). */
int simpfem_pcg(simpfem_gmg* g, const double* b_free, const double* x0_free, double* x_free,
                double tol, int maxiter, double* history_host, int history_cap, int* history_len,
                int* iters, int* converged, void* stream);

/* Operator callback of the generic Krylov entry points: y = Op(x) for device
 * vectors of n doubles; the work is enqueued on `stream` (the solve's stream)
 * and the call returns 0, or nonzero to abort the solve (SIMPFEM_ECALLBACK). */
typedef int (*simpfem_apply_fn)(void* ctx, const double* x, double* y, void* stream);
/* FGMRES for any operator / preconditioner pair (_cupy_fgmres with callables that
 * are not a hierarchy's own fine operator and apply, gpu_fem/multigrid_v4.py:416-534):
 * the Arnoldi basis, Hessenberg, Givens rotations, back-solve and history rule of
 * simpfem_fgmres on the device, A and M applied through the callbacks (each gets
 * ctx).  b, x0 (may be NULL = zero start) and x are device vectors of n doubles;
 * the host reads the convergence flags once per iteration.  Work buffers are kept
 * per host thread and device. */
int simpfem_fgmres_op(int64_t n, simpfem_apply_fn A, simpfem_apply_fn M, void* ctx, const double* b,
                      const double* x0, double* x, double tol, int maxiter, int restart, double* history_host,
                      int history_cap, int* history_len, int* iters, int* converged, void* stream);
/* PCG for any operator / preconditioner pair (_cupy_pcg, gpu_fem/solver_v2.py:551-623):
 * the same recurrences and history as simpfem_pcg, A and M through the callbacks. */
int simpfem_pcg_op(int64_t n, simpfem_apply_fn A, simpfem_apply_fn M, void* ctx, const double* b, const double* x0,
                   double* x, double tol, int maxiter, double* history_host, int history_cap, int* history_len,
                   int* iters, int* converged, void* stream);

/* ---- guarded floor policy, per state and batched -------------------------------
 * The probe -> preserve/escalate -> floor ladder -> recomputed-true-residual guard of
 * experiments/phase5/run_gmg_floor_detector_prospective.py:220-354 (_classify :77-90),
 * run entirely in the library: per attempt E = rho_min + (1 - rho_min) rho^penal on
 * the device, simpfem_gmg_setup, FGMRES with the hierarchy, and the FP64 guard
 * ||b - K(E) x|| / ||b|| <= tol.  With a proposer network the decision at the
 * probe's r50 point follows the learned floor policy (no reference counterpart):
 * the probe stops there when r50 >= the high threshold (the plain rule raises the
 * floor whatever r100 shows) or when the network's most probable rung is raised
 * with probability >= min_confidence; the ladder then starts at that rung (skipped
 * rungs last, the baseline floor last after a network stop). */
enum { SIMPFEM_TRIGGER_KEEP = 0, SIMPFEM_TRIGGER_HIGH_R50 = 1, SIMPFEM_TRIGGER_PLATEAU = 2,
       SIMPFEM_TRIGGER_LEARNED = 3, SIMPFEM_TRIGGER_HIGH_RESIDUAL = 4 };
typedef struct simpfem_cnn simpfem_cnn;
typedef struct simpfem_policy_opts {
  double penal;                       /* 3.0 (the reference drivers default to 4.5) */
  int binary;                         /* 1: density is a solid mask, void elements take rho = rho_min */
  double tol;                         /* 1e-6 */
  int restart, maxiter;               /* 300, 300 */
  int probe_iters, probe_r50;         /* 100, 50 */
  double baseline_rho_min;            /* 1e-12 */
  int n_raised;                       /* 2 (at most 6) */
  double raised_rho_mins[6];          /* {1e-3, 1e-2} */
  double high_residual_threshold;     /* 1e-2 */
  double plateau_residual_threshold;  /* 1e-4 */
  double plateau_ratio_threshold;     /* 0.6 */
  int reuse_probe;                    /* 1: a probe that converged on its tolerance at the baseline floor is
                                         the answer at that floor; 0: re-solved, as the reference driver does */
  simpfem_cnn* proposer;              /* NULL: the plain probe-and-ladder; else the floor proposer
                                         (rungs baseline | raised[0], raised[1]) */
  double min_confidence;              /* 0.5 */
} simpfem_policy_opts;
void simpfem_policy_default_opts(simpfem_policy_opts* o);

typedef struct simpfem_policy_result {
  double probe_r50, probe_r100;       /* r100 NaN when the probe stopped at r50 */
  int trigger;                        /* SIMPFEM_TRIGGER_* */
  int raise_floor;                    /* the probe predicted a raised floor */
  int fallback;                       /* a kept floor failed the guard and the ladder ran */
  int proposal;                       /* rung proposed at r50 (-1 without a proposer or a check) */
  double selected_rho_min;            /* the accepted (or last attempted) floor */
  int converged;                      /* the selected attempt passed the FP64 guard */
  int reported_converged;             /* FGMRES reported convergence for it */
  int solve_iters, probe_iters, total_iters, n_setups, n_attempts, reused_probe;
  double final_rel_residual;          /* guard value of the selected attempt */
  double attempted[8];                /* floors in attempt order (n_attempts of them) */
  double seconds;                     /* host wall time of this state, attempts included */
} simpfem_policy_result;

/* One guarded solve of the state `density` (device, n_elem doubles) with right-hand
 * side b_free (device, n_free) on hierarchy g; x_free (device, n_free, may be NULL)
 * receives the selected attempt's solution.  Synchronises `stream` per iteration. */
int simpfem_policy_run(simpfem_gmg* g, const simpfem_policy_opts* o, const double* density, const double* b_free,
                       double* x_free, simpfem_policy_result* result, void* stream);

/* A batch of states, possibly of different meshes, solved together on one GPU
 * (replaces the per-state loop of run_gmg_floor_detector_prospective.py:191-226).
 * Each state names the hierarchy it is solved on; the hierarchies are the
 * workers: every worker runs its states in their order on its own stream from
 * its own host thread, all workers at once, so results depend only on the
 * assignment (each worker's lambda_max cache carries over between its states as
 * one driver hierarchy's does).  Distinct hierarchies must sit on distinct mesh
 * handles (a handle's scratch serves one stream at a time).  With a proposer,
 * each worker uses its own copy of the network.  The workers start after the
 * work already queued on `stream` and `stream` waits for all of them. */
typedef struct simpfem_policy_state {
  simpfem_gmg* g;
  const double* density;
  const double* b_free;
  double* x_free;                     /* may be NULL */
} simpfem_policy_state;
int simpfem_policy_batch(const simpfem_policy_opts* o, const simpfem_policy_state* states, int n_states,
                         simpfem_policy_result* results, void* stream);

/* Coarsest-level dense factorisation: Linv <- L^{-1}, L the lower Cholesky factor
 * of the SPD row-major n x n device matrix A (A is destroyed; Linv lower with zero
 * upper).  Replaces cp.linalg.cholesky and its finiteness check in
 * GalerkinMatFreeGMG.setup (gpu_fem/multigrid_v4.py:1308-1337); the coarse solve
 * (gpu_fem/multigrid_v4.py:1916-1917) then multiplies by L^{-1} and L^{-T}.
 * *info_host: 0 on success, else the 1-based index of the first non-positive or
 * non-finite pivot, or n + 1 when L^{-1} holds a non-finite entry.  The lower
 * bandwidth is measured from the data: up to 24 tiles of 32 (768) the band path
 * runs (one 8-CTA thread-block cluster for the factor, one launch for L^{-1}),
 * wider matrices take a recursive blocked factorisation. */
int simpfem_dense_cholesky_inverse(int n, double* A, double* Linv, int* info_host, void* stream);

/* ---- SIMP loop around the guarded solve ------------------------------------------
 * y = H x (transpose 0) or H^T x (transpose 1) for the row-normalised cone density
 * filter of radius rmin in [1, 3.5] on an nx x ny x nz element grid (weights
 * rmin - dist within distance < rmin, the element itself rmin; replaces
 * _build_density_filter's sparse matrix and its SpMVs, pub_simp_solver.py:90-117,
 * simp_gpu.py:212-294).  x and y are device arrays of nx*ny*nz doubles, x != y. */
int simpfem_cone_filter(int nx, int ny, int nz, double rmin, int transpose, const double* x, double* y,
                        void* stream);
/* Bytes of device workspace simpfem_oc_update needs (the caller allocates it). */
size_t simpfem_oc_work_bytes(void);
/* The optimality-criteria update of _oc_step_cupy (simp_gpu.py:212-294) without a
 * Heaviside projection: bisection on the multiplier over [0, 1e9] (at most 100
 * steps, until the bracket is below 1e-9) of
 * rn = clip(clip(rho sqrt(-min(dc,-1e-12) / (lm max(dv,1e-12))), rho -+ move), 1e-3, 1)
 * against sum(H rn) = volfrac n, evaluated as sum_j vol_w_j rn_j with vol_w = H^T 1.
 * dc: the design sensitivities H^T dc_phys; dv: the volume sensitivities, NULL for
 * ones (the reference's choice without a Heaviside projection, simp_gpu.py:262-263).
 * rho, dc, dv, vol_w, rho_new: device arrays of n doubles; work: device workspace of
 * at least simpfem_oc_work_bytes() bytes.  *change_host = max |rho_new - rho|,
 * *lambda_host the final multiplier, *steps_host the bisection steps (each may be
 * NULL).  Synchronises the stream once per bisection step. */
int simpfem_oc_update(int64_t n, const double* rho, const double* dc, const double* dv, const double* vol_w,
                      double volfrac, double move, double* rho_new, double* work, size_t work_bytes,
                      double* change_host, double* lambda_host, int* steps_host, void* stream);

/* Heaviside projection proj = (tanh(b eta) + tanh(b (x - eta))) / den and its
 * derivative dproj = b (1 - tanh(b (x - eta))^2) / den, den = tanh(b eta) +
 * tanh(b (1 - eta)) (_heaviside / _heaviside_deriv, pub_simp_solver.py:245-253);
 * x, proj, dproj: device arrays of n doubles (proj or dproj may be NULL); beta > 0. */
int simpfem_heaviside(int64_t n, const double* x, double beta, double eta, double* proj, double* dproj,
                      void* stream);
/* Bytes of device workspace simpfem_oc_update_projected needs for n elements. */
size_t simpfem_oc_projected_work_bytes(int64_t n);
/* The OC update with the Heaviside projection (_oc_step_cupy with use_heaviside and
 * beta > 1e-6, simp_gpu.py:245-290): dh = the projection's derivative at rho_f,
 * design sensitivities H^T (dc_phys dh) and H^T dh with the cone filter of radius
 * rmin on the nx x ny x nz grid, then the bisection (at most 100 steps, bracket
 * < 1e-9) of rn against the projected filtered volume
 * sum(tanh(b eta) + tanh(b (H rn - eta))) / den = volfrac n.  rho, rho_f, dc_phys,
 * rho_new: device arrays of nx ny nz doubles; work: at least
 * simpfem_oc_projected_work_bytes(n) bytes.  Synchronises the stream once per step. */
int simpfem_oc_update_projected(int nx, int ny, int nz, double rmin, const double* rho, const double* rho_f,
                                const double* dc_phys, double beta, double eta, double volfrac, double move,
                                double* rho_new, double* work, size_t work_bytes, double* change_host,
                                double* lambda_host, int* steps_host, void* stream);

/* ---- learned floor proposer (no counterpart in the reference) ------------------
 * A small 3D CNN over the density pooled to 16^3 plus two probe features, with a
 * 3-way softmax over the floor rungs {1e-12, 1e-3, 1e-2}: conv 1->16 (stride 1),
 * 16->16, 16->32, 32->32 (stride 2), 3x3x3, pad 1, ReLU; mean over the last 2^3;
 * dense 34 -> 3.  Weights are used as bfloat16, everything else float32.
 * Parameters (float32, simpfem_cnn_n_params() of them) in the order
 * W1 b1 W2 b2 W3 b3 W4 b4 Wfc bfc, conv weights [cout][cin][kz][ky][kx]. */
int simpfem_cnn_n_params(void);
/* Workspaces for batches of up to max_batch samples; parameters start at zero. */
int simpfem_cnn_create(int max_batch, simpfem_cnn** out);
int simpfem_cnn_destroy(simpfem_cnn* h);
/* Host parameter copies; set_params also resets the Adam moments and step count. */
int simpfem_cnn_set_params(simpfem_cnn* h, const float* host, int n);
int simpfem_cnn_get_params(simpfem_cnn* h, float* host, int n);
/* Average-pool one device density field (nx, ny, nz elements, element index
 * (i*ny + j)*nz + k, FP64) to the network input (16^3 float32, device); window i
 * along an axis of n elements covers [floor(i*n/16), ceil((i+1)*n/16)). */
int simpfem_cnn_pool16(int nx, int ny, int nz, const double* density, float* out, void* stream);
/* prob (N x 3, device) <- softmax of the network on x (N x 16^3, device) and
 * feats (N x 2, device); 1 <= N <= max_batch. */
int simpfem_cnn_forward(simpfem_cnn* h, const float* x, const float* feats, int N, float* prob, void* stream);
/* Mean cross-entropy against labels (N int32 in {0, 1, 2}, device) and its
 * gradient with respect to every parameter, kept on the device for adam_step;
 * grad_host (n_params) and loss_host (1) may be NULL, else they are filled and
 * the call synchronises the stream.  Reductions run in a fixed order. */
int simpfem_cnn_loss_grad(simpfem_cnn* h, const float* x, const float* feats, const int32_t* labels, int N,
                          float* grad_host, float* loss_host, void* stream);
/* One Adam update of the parameters with the last loss_grad gradient. */
int simpfem_cnn_adam_step(simpfem_cnn* h, float lr, float beta1, float beta2, float eps, void* stream);

#ifdef __cplusplus
}
#endif

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#endif /* SIMPFEM_H */
