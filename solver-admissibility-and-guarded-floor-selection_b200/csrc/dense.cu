// Dense FP64 factorisation of the coarsest-level matrix: the entry
// (chol_inverse), and the recursion that takes matrices whose band is too wide
// for the band path in bandchol.cu.
//
// The reference factors the assembled coarsest matrix with cp.linalg.cholesky,
// treats a failed factorisation (info != 0 or a non-finite factor) as the
// trigger for its eps*I regularisation (gpu_fem/multigrid_v4.py:1308-1337), and
// solves with two triangular solves per coarse correction
// (gpu_fem/multigrid_v4.py:1916-1917).  Here the setup produces L^{-1} directly
// so that each coarse solve is two bandwidth-bound triangular matrix-vector
// products instead of two latency-bound substitutions.
//
// Recursive algorithm on the row-major n x n arrays A (input, destroyed) and
// Li (output L^{-1}, lower, zero upper).  For a diagonal block of size m split
// at m1 (a multiple of 32):
//
//   chol_inv(11)                          -> Li11 = L11^{-1}
//   Li21 <- A21 * Li11^T                  (= L21, parked in Li21's storage)
//   A22  <- A22 - Li21 * Li21^T           (Schur complement, lower tiles)
//   chol_inv(22)                          -> Li22 = L22^{-1}
//   A21  <- Li21 * Li11                   (= L21 L11^{-1}, parked in A21)
//   Li21 <- -Li22 * A21                   (= -L22^{-1} L21 L11^{-1})
//
// Blocks of at most 32 rows are factored and inverted by one warp.  Every
// other flop is an FP64 GEMM whose K range is cut to the non-zero part of a
// triangular operand; the zero triangles are stored explicitly (Li starts
// zeroed), so the cut is exact.  For a dense matrix the work is n^3/3 for the
// factor plus n^3/3 for the inverse, as for potrf + trtri.  The coarsest
// matrix of the hierarchy is banded (a 27-point stencil in lexicographic node
// order: lower bandwidth ~3 (ny+1)(nz+1)); the band is measured from the data
// and the GEMMs are cut to it (chol_inv_rec), which leaves about 2 n^2 bw flops,
// nearly all of them in the fill-in of L^{-1}.
#include "common.cuh"

namespace simpfem {

namespace {

constexpr int GM = 64, GN = 64, GK = 16, GT = 128;

enum { TRI_NONE = 0, TRI_OPA_LOWER = 1, TRI_OPB_LOWER = 2, TRI_OPB_UPPER = 3 };

struct DGemm {
  int M, N, K;
  const double* A;
  int64_t lda;
  const double* B;
  int64_t ldb;
  double* C;
  int64_t ldc;
  double alpha, beta;
  int tri;        // which operand is triangular (restricts the K range per tile)
  int lower_out;  // skip output tiles entirely above the diagonal
  int tri_off = 0;  // TRI_OPB_LOWER: op(B)[k][j] is non-zero for k >= j + tri_off
};

// C = alpha * A op(B) + beta * C on the FP64 tensor cores (mma.sync m8n8k4):
// 64x64 CTA tiles, 4 warps each owning a 32x32 warp tile (4 x 4 MMA tiles),
// 16-deep K steps streamed through a 4-stage cp.async pipeline (8-byte copies,
// zero-filled outside the matrix, so any leading dimension works).  A is
// row-major (A[i*lda + p]) and kept [m][k] in shared memory;
//   TB = 0: op(B)[p][j] = B[p*ldb + j], kept [k][n];
//   TB = 1: op(B)[p][j] = B[j*ldb + p], kept [n][k].
// Row strides of 20 ([m][k], [n][k]) and 68 ([k][n]) doubles put the 32 values
// of one fragment read in 16 banks twice each, the minimum of two wavefronts.
constexpr int KST = 20, NST = 68, NSTAGE = 4;
constexpr int A_STAGE = GM * KST;                       // doubles per stage
constexpr int B_STAGE_T = GN * KST, B_STAGE_N = GK * NST;

__device__ __forceinline__ void dmma_m8n8k4(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

__device__ __forceinline__ void cp_async8(double* dst, const double* src, bool ok) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(ok ? 8 : 0));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

template <int TB>
__global__ void __launch_bounds__(GT) dgemm_kernel(DGemm g) {
  extern __shared__ __align__(16) double dsm[];
  double* As = dsm;                         // [NSTAGE][GM][KST]
  double* Bs = dsm + NSTAGE * A_STAGE;      // [NSTAGE][GN][KST] or [NSTAGE][GK][NST]
  constexpr int BSTG = TB ? B_STAGE_T : B_STAGE_N;
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  const int wm = w >> 1, wn = w & 1;
  const int i0 = blockIdx.y * GM, j0 = blockIdx.x * GN;
  if (g.lower_out && j0 > i0 + GM - 1) return;
  int kbeg = 0, kend = g.K;
  if (g.tri == TRI_OPA_LOWER) kend = min(kend, i0 + GM);
  if (g.tri == TRI_OPB_UPPER) kend = min(kend, j0 + GN);
  if (g.tri == TRI_OPB_LOWER) kbeg = max(0, j0 + g.tri_off);
  const int nk = kend > kbeg ? (kend - kbeg + GK - 1) / GK : 0;
  // copy mappings: "row-run" = one matrix row, 8 consecutive k; "k-run" = one
  // k row, 8 consecutive columns
  const int ar = t >> 1, ak = (t & 1) * 8;
  const int bkr = t >> 3, bj = (t & 7) * 8;

  auto issue = [&](int stage, int k0) {
    double* as = As + stage * A_STAGE;
    double* bs = Bs + stage * BSTG;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int i = i0 + ar, p = k0 + ak + q;
      const bool ok = i < g.M && p < g.K;
      cp_async8(as + ar * KST + ak + q, ok ? g.A + (int64_t)i * g.lda + p : g.A, ok);
    }
    if (TB == 1) {
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int j = j0 + ar, p = k0 + ak + q;
        const bool ok = j < g.N && p < g.K;
        cp_async8(bs + ar * KST + ak + q, ok ? g.B + (int64_t)j * g.ldb + p : g.B, ok);
      }
    } else {
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int j = j0 + bj + q, p = k0 + bkr;
        const bool ok = j < g.N && p < g.K;
        cp_async8(bs + bkr * NST + bj + q, ok ? g.B + (int64_t)p * g.ldb + j : g.B, ok);
      }
    }
  };

  double acc[4][4][2];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;

#pragma unroll
  for (int s = 0; s < NSTAGE - 1; ++s) {
    if (s < nk) issue(s, kbeg + s * GK);
    cp_async_commit();
  }
  for (int kt = 0; kt < nk; ++kt) {
    cp_async_wait<NSTAGE - 2>();  // this thread's copies of stage kt have landed
    __syncthreads();              // everyone's have, and stage kt - 1 is consumed
    if (kt + NSTAGE - 1 < nk) issue((kt + NSTAGE - 1) % NSTAGE, kbeg + (kt + NSTAGE - 1) * GK);
    cp_async_commit();
    const double* as = As + (kt % NSTAGE) * A_STAGE;
    const double* bs = Bs + (kt % NSTAGE) * BSTG;
#pragma unroll
    for (int kq = 0; kq < GK / 4; ++kq) {
      // fragments: A[row = lane/4][k = lane%4], B[k = lane%4][col = lane/4]
      const int kk = kq * 4 + (lane & 3);
      double af[4], bf[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) af[a] = as[(wm * 32 + a * 8 + (lane >> 2)) * KST + kk];
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const int nn = wn * 32 + b * 8 + (lane >> 2);
        bf[b] = TB ? bs[nn * KST + kk] : bs[kk * NST + nn];
      }
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) dmma_m8n8k4(acc[a][b][0], acc[a][b][1], af[a], bf[b]);
    }
  }
  cp_async_wait<0>();

  // accumulator fragment: row = lane/4, columns 2*(lane%4) + {0, 1}
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int i = i0 + wm * 32 + a * 8 + (lane >> 2);
    if (i >= g.M) continue;
    double* crow = g.C + (int64_t)i * g.ldc;
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int j = j0 + wn * 32 + b * 8 + (lane & 3) * 2 + e;
        if (j >= g.N) continue;
        const double v = g.alpha * acc[a][b][e];
        crow[j] = (g.beta == 0.0) ? v : v + g.beta * crow[j];
      }
  }
}

cudaError_t dgemm(const DGemm& g, int tb, cudaStream_t s) {
  if (g.M <= 0 || g.N <= 0) return cudaSuccess;
  const dim3 grid(div_up(g.N, GN), div_up(g.M, GM));
  const size_t smem = sizeof(double) * NSTAGE * (A_STAGE + (tb ? B_STAGE_T : B_STAGE_N));
  static std::atomic<uint64_t> attr_done[2];
  const cudaError_t ea = once_per_device(attr_done[tb], [&] {
    return tb == 0 ? cudaFuncSetAttribute(dgemm_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)
                   : cudaFuncSetAttribute(dgemm_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  });
  if (ea != cudaSuccess) return ea;
  if (tb == 0) dgemm_kernel<0><<<grid, GT, smem, s>>>(g);
  else dgemm_kernel<1><<<grid, GT, smem, s>>>(g);
  return sf_launched(1);
}

// One warp factors the m x m (m <= 32) diagonal block at offset o of A
// (right-looking, lane i holding row i in registers, the pivot column
// broadcast through shared memory and scaled by the reciprocal square root of
// the pivot) and writes its inverse into Li.  A non-positive or
// non-finite pivot records o + j + 1 in *info (first one wins) and continues
// with pivot 1 so the kernel stays finite.
__global__ void __launch_bounds__(32) chol_inv_leaf_kernel(const double* __restrict__ A, double* __restrict__ Li,
                                                           int64_t n, int o, int m, int* info) {
  __shared__ double S[32][33];
  __shared__ double col[32];
  __shared__ double dinv[32];
  const int lane = threadIdx.x;
  for (int r = 0; r < 32; ++r)
    S[r][lane] = (r < m && lane < m) ? A[(int64_t)(o + r) * n + o + lane] : (r == lane ? 1.0 : 0.0);
  __syncwarp();
  double row[32];
#pragma unroll
  for (int c = 0; c < 32; ++c) row[c] = S[lane][c];
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    double d = __shfl_sync(0xffffffffu, row[j], j);
    const bool bad = !(d > 0.0) || !isfinite(d);
    if (bad) {
      d = 1.0;
      if (lane == 0) atomicCAS(info, 0, o + j + 1);
    }
    const double rs = rsqrt(d);  // one long-latency op per pivot on the serial chain
    const double sd = d * rs;
    const double l = (lane > j) ? row[j] * rs : 0.0;
    if (lane == j) row[j] = sd;
    if (lane > j) row[j] = l;
    col[lane] = l;
    __syncwarp();
    // rows below the pivot: row[c] -= l_ij * l_cj for j < c (entries c > lane are
    // the unused upper triangle; l = 0 leaves rows <= j unchanged)
#pragma unroll
    for (int c = j + 1; c < 32; ++c) row[c] = fma(-l, col[c], row[c]);
    __syncwarp();
  }
#pragma unroll
  for (int c = 0; c < 32; ++c) S[lane][c] = (c <= lane) ? row[c] : 0.0;
  __syncwarp();
  dinv[lane] = 1.0 / S[lane][lane];
  __syncwarp();
  // lane c computes column c of L^{-1}: x[r] = (delta_rc - sum_{p<r} L[r][p] x[p]) / L[r][r],
  // the sum split over four independent partial sums to shorten the FMA chain
  double x[32];
#pragma unroll
  for (int r = 0; r < 32; ++r) {
    double acc[4] = {(r == lane) ? 1.0 : 0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int p = 0; p < r; ++p) acc[p & 3] = fma(-S[r][p], x[p], acc[p & 3]);
    x[r] = ((acc[0] + acc[1]) + (acc[2] + acc[3])) * dinv[r];
  }
  if (lane < m) {
#pragma unroll
    for (int r = 0; r < 32; ++r)
      if (r < m) Li[(int64_t)(o + r) * n + o + lane] = x[r];
  }
}

// bw: lower bandwidth of A (A[i][j] == 0 for i - j > bw).  Band Cholesky
// keeps L inside the band, so A21 and L21 are non-zero only in their top-right
// R x (m1 - C0) corner (R = min(m2, bw), C0 = max(0, m1 - bw)) and the Schur
// update touches only A22[0:R][0:R]; L^{-1} fills in, and its off-diagonal block
// is -Li22[:, 0:R] * X[0:R, :] with X = L21 Li11 (R x m1).  With bw >= m - 1 this
// is the dense algorithm; the skipped products are exact zeros.
cudaError_t chol_inv_rec(double* A, double* Li, int64_t n, int o, int m, int bw, int* info, cudaStream_t s) {
  if (m <= 32) {
    chol_inv_leaf_kernel<<<1, 32, 0, s>>>(A, Li, n, o, m, info);
    return sf_launched(1);
  }
  const int nb = (m + 31) / 32;
  const int m1 = 32 * ((nb + 1) / 2);
  const int m2 = m - m1;
  const int R = std::min(m2, bw), C0 = std::max(0, m1 - bw), W = m1 - C0;
  cudaError_t e = chol_inv_rec(A, Li, n, o, m1, bw, info, s);
  if (e != cudaSuccess) return e;
  double* A21 = A + (int64_t)(o + m1) * n + o;
  double* A22 = A + (int64_t)(o + m1) * n + o + m1;
  double* Li11 = Li + (int64_t)o * n + o;
  double* Li21 = Li + (int64_t)(o + m1) * n + o;
  double* Li22 = Li + (int64_t)(o + m1) * n + o + m1;
  if (R > 0) {
    // L21[0:R, C0:m1] <- A21[0:R, C0:m1] * Li11[C0:m1, C0:m1]^T  (op(B) upper triangular)
    e = dgemm(DGemm{R, W, W, A21 + C0, n, Li11 + (int64_t)C0 * n + C0, n, Li21 + C0, n, 1.0, 0.0, TRI_OPB_UPPER,
                    0},
              1, s);
    if (e != cudaSuccess) return e;
    // A22[0:R, 0:R] <- A22 - L21 L21^T  (lower tiles)
    e = dgemm(DGemm{R, R, W, Li21 + C0, n, Li21 + C0, n, A22, n, -1.0, 1.0, TRI_NONE, 1}, 1, s);
    if (e != cudaSuccess) return e;
  }
  e = chol_inv_rec(A, Li, n, o + m1, m2, bw, info, s);
  if (e != cudaSuccess) return e;
  if (R == 0) return cudaSuccess;  // L21 = 0: the off-diagonal block of L^{-1} stays zero
  // X = A21[0:R, 0:m1] <- L21[0:R, C0:m1] * Li11[C0:m1, 0:m1]  (Li11 lower: row C0 + k is non-zero for
  // columns j <= C0 + k)
  {
    DGemm g{R, m1, W, Li21 + C0, n, Li11 + (int64_t)C0 * n, n, A21, n, 1.0, 0.0, TRI_OPB_LOWER, 0};
    g.tri_off = -C0;
    e = dgemm(g, 0, s);
    if (e != cudaSuccess) return e;
  }
  // Li21 <- -Li22[:, 0:R] * X[0:R, :]  (Li22 lower triangular)
  return dgemm(DGemm{m2, m1, R, Li22, n, A21, n, Li21, n, -1.0, 0.0, TRI_OPA_LOWER, 0}, 0, s);
}

// lower bandwidth of a row-major n x n matrix: max over rows of i - (first
// column j <= i with A[i][j] != 0; NaN counts as non-zero); one warp per row
__global__ void lower_band_kernel(const double* __restrict__ A, int n, int* __restrict__ bw) {
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= n) return;
  const int i = (int)warp;
  const double* row = A + (int64_t)i * n;
  int first = i;
  for (int j0 = 0; j0 <= i; j0 += 32) {
    const int j = j0 + lane;
    const bool nz = j <= i && row[j] != 0.0;
    const unsigned b = __ballot_sync(0xffffffffu, nz);
    if (b) {
      first = j0 + __ffs((int)b) - 1;
      break;
    }
  }
  if (lane == 0 && i - first > 0) atomicMax(bw, i - first);
}

template <typename OT>
__global__ void transpose_kernel(const double* __restrict__ A, int n, OT* __restrict__ At) {
  __shared__ double T[32][33];
  const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int i = by + r, j = bx + threadIdx.x;
    T[r][threadIdx.x] = (i < n && j < n) ? A[(int64_t)i * n + j] : 0.0;
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int i = bx + r, j = by + threadIdx.x;
    if (i < n && j < n) At[(int64_t)i * n + j] = (OT)T[threadIdx.x][r];
  }
}

__global__ void nonfinite_flag_kernel(const double* __restrict__ A, int64_t n, int bad_code, int* info) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    if (!isfinite(A[i])) {
      atomicCAS(info, 0, bad_code);
      return;
    }
}

template <typename OT>
cudaError_t launch_transpose(const double* A, int n, OT* At, cudaStream_t s) {
  const int nb = div_up(n, 32);
  transpose_kernel<OT><<<dim3(nb, nb), dim3(32, 8), 0, s>>>(A, n, At);
  return sf_launched(1);
}

}  // namespace

cudaError_t chol_inverse(double* A, int n, double* work64, double* dinv, const BandInvOut& out, int* info_dev,
                         cudaStream_t s, int bw_known) {
  cudaError_t e = cudaMemsetAsync(info_dev, 0, 2 * sizeof(int), s);
  if (e != cudaSuccess) return e;
  if (n <= 0) return cudaSuccess;
  // the band (exact zeros below it) decides the path and the blocks multiplied
  int bw = std::min(bw_known, n - 1);
  if (bw_known < 0) {
    lower_band_kernel<<<div_up((int64_t)n * 32, 256), 256, 0, s>>>(A, n, info_dev + 1);
    e = sf_launched(1);
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(&bw, info_dev + 1, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return e;
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return e;
  }
  bw = std::max(bw, 0);
  if (band_tiles(bw) <= kBandMaxTiles && band_path_available())
    return band_chol_inverse(A, n, bw, dinv, out, info_dev, s);
  const int64_t nn = (int64_t)n * n;
  e = cudaMemsetAsync(work64, 0, sizeof(double) * (size_t)nn, s);
  if (e != cudaSuccess) return e;
  e = chol_inv_rec(A, work64, n, 0, n, bw, info_dev, s);
  if (e != cudaSuccess) return e;
  nonfinite_flag_kernel<<<(int)std::min<int64_t>(div_up(nn, 256), 148 * 16), 256, 0, s>>>(work64, nn, n + 1,
                                                                                          info_dev);
  e = sf_launched(1);
  if (e != cudaSuccess) return e;
  if (out.L64 && out.L64 != work64) {
    e = cudaMemcpyAsync(out.L64, work64, sizeof(double) * (size_t)nn, cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return e;
  }
  if (out.LT64 && (e = launch_transpose(work64, n, out.LT64, s)) != cudaSuccess) return e;
  if (out.L32 && (e = launch_convert(F64, F32, work64, out.L32, nn, nullptr, s)) != cudaSuccess) return e;
  if (out.LT32 && (e = launch_transpose(work64, n, out.LT32, s)) != cudaSuccess) return e;
  return cudaSuccess;
}

cudaError_t dense_chol_inverse(double* A, int n, double* Linv, double* dinv, int* info_dev, cudaStream_t s) {
  if (n > 0) {
    const cudaError_t e = cudaMemsetAsync(Linv, 0, sizeof(double) * (size_t)n * n, s);
    if (e != cudaSuccess) return e;
  }
  BandInvOut out;
  out.L64 = Linv;
  return chol_inverse(A, n, Linv, dinv, out, info_dev, s);
}

}  // namespace simpfem
