// Band Cholesky and L^{-1} of the coarsest-level matrix in two launches.
//
// The coarsest matrix of the hierarchy is a 27-point stencil in lexicographic
// node order, so its lower bandwidth bw is small beside n (bw = 221 at
// n = 3,960 for the 160 x 80 x 40 cantilever).  The reference factors it with
// cp.linalg.cholesky and solves with two triangular solves per coarse
// correction (gpu_fem/multigrid_v4.py:1308-1337, :1916-1917); this library
// produces L^{-1} so that each coarse solve is two bandwidth-bound triangular
// matrix-vector products.  The work is ~n bw^2 flops for the factor and
// ~n^2 bw for the fill-in of L^{-1}; what limits it is the chain of n pivots,
// so the algorithm is laid out around that chain:
//
// 1. band_chol_kernel: one thread-block cluster (8 CTAs, distributed shared
//    memory) runs the tiled right-looking band Cholesky over 32 x 32 tiles,
//    with WB = ceil(bw / 32) tiles below the diagonal.  CTA 0 makes every
//    diagonal factor: step K, it forms L_{K+1,K} = A_{K+1,K} L_KK^{-T} on the
//    FP64 tensor cores (mma.sync m8n8k4) with its own L_KK^{-1}, subtracts
//    L_{K+1,K} L_{K+1,K}^T from A_{K+1,K+1}, factors it and inverts the factor
//    (one warp, pivot column broadcast through shared memory).  The seven other
//    CTAs copy L_KK^{-1} from CTA 0's distributed shared memory, form L_IK for
//    I = K+2..K+WB the same way and apply the rest of the trailing update
//    A_IJ -= L_IK L_JK^T, half a tile per warp on the tensor cores with
//    fragments loaded from L2.  Two cluster barriers a step.  The inverses of
//    the diagonal tiles are kept for step 2.
// 2. band_inverse_kernel: X = L^{-1} by 16-column blocks, independent of one
//    another: X_JJ = L_JJ^{-1}, X_IJ = -L_II^{-1} sum_{K=max(J,I-WB)}^{I-1} L_IK X_KJ,
//    the last WB tiles of the block kept in a power-of-two ring in shared
//    memory, the tiles of L and L_II^{-1} streamed through a cp.async ring, both products on the FP64 tensor
//    cores with four accumulator chains per warp.  Each CTA takes a long column
//    block and its mirror so that every CTA walks ~NB tile rows.  It writes any
//    of L^{-1} and L^{-T} in FP64 or FP32 directly (the mixed cycle reads only
//    the FP32 pair) and flags a non-finite entry as a failed factorisation, as
//    the recursive path does.
//
// A non-positive or non-finite pivot records its 1-based row in info (the
// first one in pivot order) and continues with pivot 1, as the recursive path
// in dense.cu does; the caller regularises and refactors.
#include <cooperative_groups.h>

#include <map>
#include <mutex>

#include "common.cuh"

namespace cg = cooperative_groups;

namespace simpfem {

namespace {

constexpr int TS = 32;           // tile size
constexpr int T33 = 33;          // row stride of a tile read one row per lane
constexpr int T36 = 36;          // row stride of a tile read as tensor-core fragments
constexpr int FT = 256;          // threads per CTA
constexpr int CL = 8;            // CTAs in the factorisation cluster
constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}
__device__ __forceinline__ void cluster_arrive() { asm volatile("barrier.cluster.arrive.aligned;\n" ::: "memory"); }
__device__ __forceinline__ void cluster_wait() { asm volatile("barrier.cluster.wait.aligned;\n" ::: "memory"); }

// tile (I, J) of the row-major n x n matrix into T[32][T33] through L2 (other
// CTAs of the cluster wrote it), all loads of a thread in flight together;
// entries outside the matrix read as the identity's
__device__ __forceinline__ void load_tile(const double* __restrict__ A, int n, int I, int J, double* T) {
  double v[TS * TS / FT];
#pragma unroll
  for (int u = 0; u < TS * TS / FT; ++u) {
    const int e = threadIdx.x + FT * u, r = e >> 5, c = e & 31, gr = TS * I + r, gc = TS * J + c;
    v[u] = (gr < n && gc < n) ? __ldcg(A + (int64_t)gr * n + gc) : (gr == gc ? 1.0 : 0.0);
  }
#pragma unroll
  for (int u = 0; u < TS * TS / FT; ++u) {
    const int e = threadIdx.x + FT * u;
    T[(e >> 5) * T33 + (e & 31)] = v[u];
  }
}
__device__ __forceinline__ void store_tile(double* __restrict__ A, int n, int I, int J, const double* T,
                                           bool lower) {
  for (int e = threadIdx.x; e < TS * TS; e += FT) {
    const int r = e >> 5, c = e & 31, gr = TS * I + r, gc = TS * J + c;
    if (gr < n && gc < n && (!lower || c <= r)) __stcg(A + (int64_t)gr * n + gc, T[r * T33 + c]);
  }
}

// Warp 0: Cholesky of the 32 x 32 tile in T and the inverse of the factor,
// pivot K, fully unrolled so that every register index is a constant.  Lane i
// holds row i of the tile (w) and column i of L^{-1} (x, formed right-looking
// from the same broadcast pivot column).  Only lane j+1's own update of its
// diagonal entry sits on the chain between two pivots; the other columns'
// updates fill the issue slots.  The dedicated factor CTA runs this every step,
// so its ~1,700 instructions stay in that SM's instruction cache.  Outputs: the
// factor in T (lower, zero upper), L^{-1} row-major in D (stride T36).
__device__ void potrf_inv_tile(double* T, double* col, double* D, int K, int n, int* info) {
  const int lane = threadIdx.x & 31, o = TS * K;
  double w[32], x[32];
#pragma unroll
  for (int c = 0; c < 32; ++c) {
    w[c] = T[lane * T33 + c];
    x[c] = c == lane ? 1.0 : 0.0;
  }
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    double d = __shfl_sync(FULL, w[j], j);
    if (!(d > 0.0) || !isfinite(d)) {
      d = 1.0;
      if (lane == 0 && o + j < n) atomicCAS(info, 0, o + j + 1);
    }
    const double rs = rsqrt(d);
    const double l = lane > j ? w[j] * rs : (lane == j ? d * rs : 0.0);  // column j of L
    T[lane * T33 + j] = l;
    double* cb = col + (j & 1) * 32;  // two buffers: one __syncwarp a pivot
    cb[lane] = lane > j ? l : 0.0;
    __syncwarp();
    const double lm = lane > j ? l : 0.0;
    const double xj = x[j] * rs;  // row j of L^{-1}: (row j so far) / L_jj
    D[j * T36 + lane] = xj;
    int cs = j + 1;
    if ((cs & 1) && cs < 32) {
      const double lc = cb[cs];
      w[cs] = fma(-lm, lc, w[cs]);
      x[cs] = fma(-xj, lc, x[cs]);
      ++cs;
    }
#pragma unroll
    for (int c = cs; c < 32; c += 2) {
      const double2 v = *reinterpret_cast<const double2*>(cb + c);
      w[c] = fma(-lm, v.x, w[c]);
      x[c] = fma(-xj, v.x, x[c]);
      w[c + 1] = fma(-lm, v.y, w[c + 1]);
      x[c + 1] = fma(-xj, v.y, x[c + 1]);
    }
  }
}

// L_IK = A_IK L_KK^{-T} = A_IK D^T on the tensor cores: warp w owns the 8 x 8
// blocks (w / 2, 2 (w % 2) + {0, 1}); A fragments straight from L2, D = L_KK^{-1}
// (stride T36) in this CTA's shared memory, all 24 fragment loads of a lane in
// flight together; two accumulator chains per block.  The result goes back to
// the global matrix and, for the next pivot's row, into Tq.  Called by every
// thread of the CTA.
__device__ void trsm_mma(double* __restrict__ A, int n, int I, int K, const double* D, double* Tq) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, g = lane >> 2, q = lane & 3;
  const int rl = 8 * (w >> 1) + g, ra = TS * I + rl;
  double af[8], bf[2][8];
#pragma unroll
  for (int ks = 0; ks < 8; ++ks) {
    af[ks] = ra < n ? __ldcg(A + (int64_t)ra * n + TS * K + 4 * ks + q) : 0.0;
#pragma unroll
    for (int b = 0; b < 2; ++b) bf[b][ks] = D[(8 * (2 * (w & 1) + b) + g) * T36 + 4 * ks + q];
  }
  double acc[2][2][2] = {};
#pragma unroll
  for (int ks = 0; ks < 8; ++ks)
#pragma unroll
    for (int b = 0; b < 2; ++b) dmma(acc[b][ks & 1][0], acc[b][ks & 1][1], af[ks], bf[b][ks]);
  // in place: warps w and w ^ 1 read the same rows of A_IK and write different
  // halves of them, so no warp writes before every warp has read
  __syncthreads();
#pragma unroll
  for (int b = 0; b < 2; ++b)
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const int c = 8 * (2 * (w & 1) + b) + 2 * q + e;
      const double v = acc[b][0][e] + acc[b][1][e];
      if (ra < n) __stcg(A + (int64_t)ra * n + TS * K + c, v);
      if (Tq) Tq[rl * T33 + c] = v;
    }
}

// C -= X X^T for 32 x 32 tiles in shared memory (stride T33) on the tensor
// cores: warp w owns the 8 x 8 blocks (w / 2, 2 (w % 2) + {0, 1}).
__device__ void syrk_smem(double* C, const double* X) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int r = 8 * (w >> 1) + (lane >> 2), q = lane & 3;
  double acc[2][2];
#pragma unroll
  for (int b = 0; b < 2; ++b) {
    const int c = 8 * (2 * (w & 1) + b) + 2 * q;
    acc[b][0] = C[r * T33 + c];
    acc[b][1] = C[r * T33 + c + 1];
  }
#pragma unroll
  for (int ks = 0; ks < 8; ++ks) {
    const double a = -X[r * T33 + 4 * ks + q];
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      const int yr = 8 * (2 * (w & 1) + b) + (lane >> 2);
      dmma(acc[b][0], acc[b][1], a, X[yr * T33 + 4 * ks + q]);
    }
  }
#pragma unroll
  for (int b = 0; b < 2; ++b) {  // each warp writes back only the entries it read
    const int c = 8 * (2 * (w & 1) + b) + 2 * q;
    C[r * T33 + c] = acc[b][0];
    C[r * T33 + c + 1] = acc[b][1];
  }
}

// One warp: rows 16 h .. 16 h + 15 of A_IJ -= L_IK L_JK^T in place in the
// global matrix on the tensor cores, the eight 8 x 8 output blocks as eight
// independent accumulator chains, all 64 fragment loads of a lane (from L2) in
// flight together.
__device__ void update_half_tile(double* __restrict__ A, int n, int I, int J, int K, int h) {
  const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
  double acc[2][4][2], af[2][8], bf[4][8];
#pragma unroll
  for (int rb = 0; rb < 2; ++rb) {
    const int r = TS * I + 16 * h + 8 * rb + g;
#pragma unroll
    for (int ks = 0; ks < 8; ++ks) af[rb][ks] = r < n ? -__ldcg(A + (int64_t)r * n + TS * K + 4 * ks + q) : 0.0;
#pragma unroll
    for (int cb = 0; cb < 4; ++cb)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int c = TS * J + 8 * cb + 2 * q + e;
        acc[rb][cb][e] = (r < n && c < n) ? __ldcg(A + (int64_t)r * n + c) : 0.0;
      }
  }
#pragma unroll
  for (int cb = 0; cb < 4; ++cb) {
    const int r = TS * J + 8 * cb + g;
#pragma unroll
    for (int ks = 0; ks < 8; ++ks) bf[cb][ks] = r < n ? __ldcg(A + (int64_t)r * n + TS * K + 4 * ks + q) : 0.0;
  }
#pragma unroll
  for (int ks = 0; ks < 8; ++ks)
#pragma unroll
    for (int rb = 0; rb < 2; ++rb)
#pragma unroll
      for (int cb = 0; cb < 4; ++cb) dmma(acc[rb][cb][0], acc[rb][cb][1], af[rb][ks], bf[cb][ks]);
#pragma unroll
  for (int rb = 0; rb < 2; ++rb) {
    const int r = TS * I + 16 * h + 8 * rb + g;
#pragma unroll
    for (int cb = 0; cb < 4; ++cb)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int c = TS * J + 8 * cb + 2 * q + e;
        if (r < n && c < n) __stcg(A + (int64_t)r * n + c, acc[rb][cb][e]);
      }
  }
}

// Shared memory of one factorisation CTA (doubles).
struct CholSmem {
  static constexpr int D = 0;                 // [2][32][T36] the factor CTA's L_KK^{-1}, by K % 2
  static constexpr int DL = D + 2 * 32 * T36; // [32][T36] a worker's copy of the step's L_KK^{-1}
  static constexpr int TQ = DL + 32 * T36;    // [32][T33] L_{K+1,K} (factor CTA)
  static constexpr int TP = TQ + 32 * T33;    // [32][T33] A_{K+1,K+1}, then its factor (factor CTA)
  static constexpr int COL = TP + 32 * T33;   // [2][32] pivot column
  static constexpr int TOTAL = COL + 64;
};

// Warp 0 factors the updated diagonal tile in Tp and inverts the factor into
// D; then the CTA stores both.
__device__ void factor_diag(double* sm, double* D, double* __restrict__ A, int n, int K,
                            double* __restrict__ dinv, int* info) {
  double* Tp = sm + CholSmem::TP;
  if ((threadIdx.x >> 5) == 0) potrf_inv_tile(Tp, sm + CholSmem::COL, D, K, n, info);
  __syncthreads();
  store_tile(A, n, K, K, Tp, true);
  double* out = dinv + (int64_t)K * 1024;
  for (int e = threadIdx.x; e < 1024; e += FT) out[e] = D[(e >> 5) * T36 + (e & 31)];
}

// One cluster of CL CTAs: CTA 0 makes every diagonal factor, CTAs 1..CL-1 are
// workers.  WB: tiles below the diagonal in the band.  Step K: CTA 0 divides
// tile row K+1 by L_KK^T with its own L_KK^{-1}, then forms and factors tile
// K+1 (its inverse into the other half of a double buffer, since the workers
// copy the current half during the same step); the workers divide tile rows
// K+2..K+WB (round robin) and then apply the rest of the trailing update, half
// a tile per warp.  Every CTA runs the same sequence of cluster barriers; the
// branches between them depend only on the step and the rank.
__global__ void __launch_bounds__(FT) band_chol_kernel(double* __restrict__ A, int n, int NB, int WB,
                                                       double* __restrict__ dinv, int* __restrict__ info) {
  extern __shared__ __align__(16) double sm[];
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  const int warp = threadIdx.x >> 5;
  constexpr int NW = CL - 1;  // workers
  double* Tq = sm + CholSmem::TQ;
  double* Tp = sm + CholSmem::TP;

  if (rank == 0) {
    load_tile(A, n, 0, 0, Tp);
    __syncthreads();
    factor_diag(sm, sm + CholSmem::D, A, n, 0, dinv, info);
  }
  cluster_arrive();
  cluster_wait();

  for (int K = 0; K < NB; ++K) {
    const int last = min(NB - 1, K + WB);
    double* Dk = sm + CholSmem::D + (K & 1) * 32 * T36;  // L_KK^{-1} in the factor CTA's layout
    if (rank == 0) {
      const bool next = K + 1 < NB;
      if (next) {
        load_tile(A, n, K + 1, K + 1, Tp);
        if (WB > 0) trsm_mma(A, n, K + 1, K, Dk, Tq);
      }
      __syncthreads();
      cluster_arrive();  // L_{K+1,K} is in L2
      if (next) {
        if (WB > 0) {
          syrk_smem(Tp, Tq);
          __syncthreads();
        }
        factor_diag(sm, sm + CholSmem::D + ((K + 1) & 1) * 32 * T36, A, n, K + 1, dinv, info);
      }
      cluster_wait();
    } else {
      const int I0 = K + 1 + rank;  // this worker's first tile row
      if (I0 <= last) {
        // L_KK^{-1} from the factor CTA's distributed shared memory, copied once
        // with all loads in flight: the step's divisions then read it locally
        const double* Dp = cluster.map_shared_rank(Dk, 0);
        double* Dl = sm + CholSmem::DL;
        constexpr int NV = (32 * T36 + FT - 1) / FT;
        double v[NV];
#pragma unroll
        for (int u = 0; u < NV; ++u) {
          const int e = threadIdx.x + FT * u;
          if (e < 32 * T36) v[u] = Dp[e];
        }
#pragma unroll
        for (int u = 0; u < NV; ++u) {
          const int e = threadIdx.x + FT * u;
          if (e < 32 * T36) Dl[e] = v[u];
        }
        __syncthreads();
        for (int I = I0; I <= last; I += NW) trsm_mma(A, n, I, K, Dl, nullptr);
      }
      __syncthreads();
      cluster_arrive();  // the step's L_IK are in L2
      cluster_wait();
      // the trailing update in half tiles: half tile u to warp (u / NW) % 8 of
      // worker 1 + u % NW
      int u = 0;
      for (int I = K + 1; I <= last; ++I)
        for (int J = K + 1; J <= I; ++J) {
          if (I == K + 1 && J == K + 1) continue;
          for (int h = 0; h < 2; ++h, ++u)
            if (1 + u % NW == rank && (u / NW) % 8 == warp) update_half_tile(A, n, I, J, K, h);
        }
    }
    cluster_arrive();  // updates and the next factor are in place
    cluster_wait();
  }
}

constexpr int CW = 16;     // columns of L^{-1} per column block
constexpr int SX = 20;     // row stride of a 32 x 16 block (doubles): B-fragment reads conflict-free
constexpr int NSLOT = 6;   // staged-tile ring

__device__ __forceinline__ void cp_async8z(double* dst, const double* src, bool ok) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(ok ? 8 : 0));
}
__device__ __forceinline__ void cp_async16(double* dst, const double* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_wait_ring() { asm volatile("cp.async.wait_group %0;\n" ::"n"(NSLOT - 2)); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::); }

// X tile (I, column block at c0) from X[32][SX] in shared memory to the
// requested outputs; a non-finite entry marks the factorisation failed (n + 1)
__device__ void write_block(const double* X, int I, int c0, int n, const BandInvOut& o, int* info) {
  const int t = threadIdx.x;
  bool bad = false;
  {
    const int r = t >> 3, c = 2 * (t & 7), gr = TS * I + r;
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const int gc = c0 + c + e;
      if (gr < n && gc < n) {
        const double v = X[r * SX + c + e];
        bad |= !isfinite(v);
        const int64_t at = (int64_t)gr * n + gc;
        if (o.L64) o.L64[at] = v;
        if (o.L32) o.L32[at] = (float)v;
      }
    }
  }
  if (o.LT64 || o.LT32) {
    const int c = t >> 4, r = 2 * (t & 15), gc = c0 + c;
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const int gr = TS * I + r + e;
      if (gr < n && gc < n) {
        const double v = X[(r + e) * SX + c];
        const int64_t at = (int64_t)gc * n + gr;
        if (o.LT64) o.LT64[at] = v;
        if (o.LT32) o.LT32[at] = (float)v;
      }
    }
  }
  if (bad) atomicCAS(info, 0, n + 1);
}

// Staged-tile stream of one column block (tile column J): for I = J+1 .. NB-1
// the tiles L_IK, K = max(J, I-WB) .. I-1, then L_II^{-1} (K == I).  The copy
// addresses of this thread are precomputed once; a tile costs one base
// address and a few adds.
struct TileStream {
  int I, K, J, WB;
  const double* A;
  const double* dinv;
  int n;
  int64_t n8;           // 8 rows of A
  int dst_l, dst_d;     // this thread's first shared-memory slot of an L tile / a L_II^{-1} tile
  int row_l, col_l;     // this thread's first row and column in an L tile
  int src_d;            // this thread's first element of a L_II^{-1} tile
  __device__ void start(int j, int wb, const double* a, const double* di, int nn) {
    J = j;
    WB = wb;
    I = j + 1;
    K = max(J, I - WB);
    A = a;
    dinv = di;
    n = nn;
    n8 = 8 * (int64_t)nn;
    const int t = threadIdx.x;
    row_l = t >> 5;
    col_l = t & 31;
    dst_l = row_l * T36 + col_l;
    dst_d = (t >> 4) * T36 + 2 * (t & 15);
    src_d = (t >> 4) * 32 + 2 * (t & 15);
  }
  __device__ void next() {
    if (K == I) {
      ++I;
      K = max(J, I - WB);
    } else {
      ++K;
    }
  }
  // L rows 8u + row_l (u = 0..3) / L_II^{-1} rows 16u + (t >> 4) (u = 0, 1)
  __device__ __forceinline__ void issue(double* st) const {
    if (K == I) {
      const double* src = dinv + (int64_t)I * 1024 + src_d;
      cp_async16(st + dst_d, src);
      cp_async16(st + dst_d + 16 * T36, src + 16 * 32);
    } else {
      const int r0 = TS * I + row_l;
      const double* src = A + (int64_t)r0 * n + TS * K + col_l;
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const bool ok = r0 + 8 * u < n;
        cp_async8z(st + dst_l + 8 * u * T36, ok ? src + u * n8 : A, ok);
      }
    }
  }
};

// Grid: one CTA per pair of column blocks (cb, NCB - 1 - cb).  Warp w owns the
// 8 x 8 output block (w / 2, w % 2) of the 32 x 16 block of every tile row.
// RM + 1: the ring's size, a power of two >= WB + 1.
__global__ void __launch_bounds__(FT) band_inverse_kernel(const double* __restrict__ A,
                                                          const double* __restrict__ dinv, int n, int NB, int WB,
                                                          int RM, BandInvOut out, int* __restrict__ info) {
  extern __shared__ __align__(16) double sm[];
  double* ring = sm;                             // [RM + 1][32][SX]: X_KJ of the recent tile rows
  double* stage = ring + (RM + 1) * 32 * SX;     // [NSLOT][32][T36]
  double* sacc = stage + NSLOT * 32 * T36;       // [32][SX]
  const int t = threadIdx.x, lane = t & 31, w = t >> 5, g = lane >> 2, q = lane & 3;
  const int ar = 8 * (w >> 1) + g, bcol = 8 * (w & 1);
  const int a_off = ar * T36 + q, b_off = q * SX + bcol + g, c_off = ar * SX + bcol + 2 * q;
  const int NCB = (n + CW - 1) / CW;
  for (int pass = 0; pass < 2; ++pass) {
    const int cb = pass == 0 ? (int)blockIdx.x : NCB - 1 - (int)blockIdx.x;
    if (pass == 1 && cb <= (int)blockIdx.x) break;
    const int c0 = CW * cb, J = c0 / TS, h = (c0 / CW) & 1;
    double* xj = ring + (J & RM) * 32 * SX;
    for (int e = t; e < 32 * CW; e += FT) {
      const int r = e >> 4, c = e & 15;
      xj[r * SX + c] = dinv[(int64_t)J * 1024 + r * 32 + CW * h + c];
    }
    __syncthreads();
    write_block(xj, J, c0, n, out, info);

    TileStream ps;
    ps.start(J, WB, A, dinv, n);
#pragma unroll 1
    for (int s = 0; s < NSLOT - 1; ++s) {
      if (ps.I < NB) {
        ps.issue(stage + s * 32 * T36);
        ps.next();
      }
      cp_commit();
    }
    int slot = 0;
#pragma unroll 1
    for (int I = J + 1; I < NB; ++I) {
      double acc[4][2] = {};  // four accumulator chains, summed at the tile row's end
      const int kb = max(J, I - WB);
#pragma unroll 1
      for (int K = kb; K <= I; ++K) {
        cp_wait_ring();
        __syncthreads();  // everyone's copies of this tile landed; the previous slot is consumed
        if (ps.I < NB) {
          ps.issue(stage + (slot == 0 ? NSLOT - 1 : slot - 1) * 32 * T36);
          ps.next();
        }
        cp_commit();
        const double* st = stage + slot * 32 * T36 + a_off;
        slot = slot + 1 == NSLOT ? 0 : slot + 1;
        if (K < I) {
          const double* xk = ring + (K & RM) * 32 * SX + b_off;
#pragma unroll
          for (int ks = 0; ks < 8; ++ks) dmma(acc[ks & 3][0], acc[ks & 3][1], st[4 * ks], xk[4 * ks * SX]);
        } else {
          // X_IJ = -L_II^{-1} (sum over K of L_IK X_KJ)
#pragma unroll
          for (int e = 0; e < 2; ++e) sacc[c_off + e] = (acc[0][e] + acc[1][e]) + (acc[2][e] + acc[3][e]);
          __syncthreads();
          double y[4][2] = {};
#pragma unroll
          for (int ks = 0; ks < 8; ++ks)
            dmma(y[ks & 3][0], y[ks & 3][1], -st[4 * ks], sacc[(4 * ks + q) * SX + bcol + g]);
          double* xi = ring + (I & RM) * 32 * SX;
#pragma unroll
          for (int e = 0; e < 2; ++e) xi[c_off + e] = (y[0][e] + y[1][e]) + (y[2][e] + y[3][e]);
          __syncthreads();
          write_block(xi, I, c0, n, out, info);
        }
      }
    }
    cp_wait_all();
    __syncthreads();
  }
}

int ring_mask(int WB) {
  int r = 1;
  while (r < WB + 1) r <<= 1;
  return r - 1;
}

size_t inverse_smem(int WB) {
  return sizeof(double) * ((size_t)(ring_mask(WB) + 1) * 32 * SX + NSLOT * 32 * T36 + 32 * SX);
}

}  // namespace

int band_tiles(int bw) { return (std::max(bw, 0) + TS - 1) / TS; }

// Whether the current device can run the factorisation cluster at all (it can on
// a whole B200; a partitioned or smaller device may not): asked once per device.
bool band_path_available() {
  static std::mutex mu;
  static std::map<int, bool> known;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return false;
  std::lock_guard<std::mutex> lk(mu);
  const auto it = known.find(dev);
  if (it != known.end()) return it->second;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(CL);
  cfg.blockDim = dim3(FT);
  cfg.dynamicSmemBytes = sizeof(double) * CholSmem::TOTAL;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = CL;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  int clusters = 0;
  const bool ok = cudaOccupancyMaxActiveClusters(&clusters, band_chol_kernel, &cfg) == cudaSuccess && clusters > 0;
  if (!ok) cudaGetLastError();
  known[dev] = ok;
  return ok;
}

size_t band_dinv_bytes(int n) { return sizeof(double) * 1024 * (size_t)std::max(1, (n + TS - 1) / TS); }

cudaError_t band_chol_inverse(double* A, int n, int bw, double* dinv, const BandInvOut& out, int* info,
                              cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const int NB = (n + TS - 1) / TS, WB = std::min(NB - 1, band_tiles(bw));
  if (WB > kBandMaxTiles) return cudaErrorInvalidValue;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(CL);
  cfg.blockDim = dim3(FT);
  cfg.dynamicSmemBytes = sizeof(double) * CholSmem::TOTAL;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = CL;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaError_t e = cudaLaunchKernelEx(&cfg, band_chol_kernel, A, n, NB, WB, dinv, info);
  if (e != cudaSuccess) return e;
  e = sf_launched(1);
  if (e != cudaSuccess) return e;
  static std::atomic<uint64_t> attr_done;
  e = once_per_device(attr_done, [] {
    return cudaFuncSetAttribute(band_inverse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)inverse_smem(kBandMaxTiles));
  });
  if (e != cudaSuccess) return e;
  const int ncb = (n + CW - 1) / CW;
  band_inverse_kernel<<<(ncb + 1) / 2, FT, inverse_smem(WB), s>>>(A, dinv, n, NB, WB, ring_mask(WB), out, info);
  return sf_launched(1);
}

}  // namespace simpfem
