// Dense FP64 factorisation of the coarsest-level matrix.
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
// zeroed), so the cut is exact.  Total work n^3/3 for the factor plus n^3/3
// for the inverse, as for potrf + trtri.
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
};

// C = alpha * A op(B) + beta * C on the FP64 tensor cores (mma.sync m8n8k4):
// 64x64 CTA tiles, 4 warps each owning a 32x32 warp tile (4 x 4 MMA tiles),
// 16-deep K steps staged through padded shared memory with one
// register-staged prefetch of the next K step.  A is row-major (A[i*lda + p]);
//   TB = 0: op(B)[p][j] = B[p*ldb + j];  TB = 1: op(B)[p][j] = B[j*ldb + p].
// The shared-memory row stride of 68 doubles puts the 16 (k, m) pairs a half
// warp reads for one fragment in 16 distinct banks.
constexpr int SST = 68;

__device__ __forceinline__ void dmma_m8n8k4(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

template <int TB>
__global__ void __launch_bounds__(GT) dgemm_kernel(DGemm g) {
  __shared__ __align__(16) double As[2][GK][SST];
  __shared__ __align__(16) double Bs[2][GK][SST];
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  const int wm = w >> 1, wn = w & 1;
  const int i0 = blockIdx.y * GM, j0 = blockIdx.x * GN;
  if (g.lower_out && j0 > i0 + GM - 1) return;
  int kbeg = 0, kend = g.K;
  if (g.tri == TRI_OPA_LOWER) kend = min(kend, i0 + GM);
  if (g.tri == TRI_OPB_UPPER) kend = min(kend, j0 + GN);
  if (g.tri == TRI_OPB_LOWER) kbeg = j0;
  // loads: "row-run" = one matrix row, 8 consecutive k; "k-run" = one k row,
  // four pairs of consecutive columns 16 apart
  const int ar = t >> 1, ak = (t & 1) * 8;
  const int bkr = t >> 3, bj = (t & 7) * 2;
  double ra[8], rb[8];
  auto gload = [&](int k0) {
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int i = i0 + ar, p = k0 + ak + q;
      ra[q] = (i < g.M && p < g.K) ? g.A[(int64_t)i * g.lda + p] : 0.0;
    }
    if (TB == 1) {
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int j = j0 + ar, p = k0 + ak + q;
        rb[q] = (j < g.N && p < g.K) ? g.B[(int64_t)j * g.ldb + p] : 0.0;
      }
    } else {
#pragma unroll
      for (int h = 0; h < 4; ++h)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int j = j0 + bj + 16 * h + e, p = k0 + bkr;
          rb[2 * h + e] = (j < g.N && p < g.K) ? g.B[(int64_t)p * g.ldb + j] : 0.0;
        }
    }
  };
  auto sstore = [&](int buf) {
#pragma unroll
    for (int q = 0; q < 8; ++q) As[buf][ak + q][ar] = ra[q];
    if (TB == 1) {
#pragma unroll
      for (int q = 0; q < 8; ++q) Bs[buf][ak + q][ar] = rb[q];
    } else {
#pragma unroll
      for (int h = 0; h < 4; ++h)
        *reinterpret_cast<double2*>(&Bs[buf][bkr][bj + 16 * h]) = make_double2(rb[2 * h], rb[2 * h + 1]);
    }
  };

  double acc[4][4][2];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;

  int buf = 0;
  if (kbeg < kend) {
    gload(kbeg);
    sstore(0);
    __syncthreads();
  }
  for (int k0 = kbeg; k0 < kend; k0 += GK) {
    const bool more = k0 + GK < kend;
    if (more) gload(k0 + GK);
#pragma unroll
    for (int kq = 0; kq < GK / 4; ++kq) {
      // fragments: A[row = lane/4][k = lane%4], B[k = lane%4][col = lane/4]
      const int kk = kq * 4 + (lane & 3);
      double af[4], bf[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) af[a] = As[buf][kk][wm * 32 + a * 8 + (lane >> 2)];
#pragma unroll
      for (int b = 0; b < 4; ++b) bf[b] = Bs[buf][kk][wn * 32 + b * 8 + (lane >> 2)];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) dmma_m8n8k4(acc[a][b][0], acc[a][b][1], af[a], bf[b]);
    }
    if (more) sstore(buf ^ 1);
    __syncthreads();
    buf ^= 1;
  }

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
  if (tb == 0) dgemm_kernel<0><<<grid, GT, 0, s>>>(g);
  else dgemm_kernel<1><<<grid, GT, 0, s>>>(g);
  return sf_launched(1);
}

// One warp factors the m x m (m <= 32) diagonal block at offset o of A
// (right-looking, lane i holding row i in registers, the pivot column
// broadcast through shared memory, scaled by the pivot's reciprocal as
// LAPACK's potf2 does) and writes its inverse into Li.  A non-positive or
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
    const double sd = sqrt(d);
    const double rs = 1.0 / sd;
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
  // lane c computes column c of L^{-1}: x[r] = (delta_rc - sum_{p<r} L[r][p] x[p]) / L[r][r]
  double x[32];
#pragma unroll
  for (int r = 0; r < 32; ++r) {
    double acc = (r == lane) ? 1.0 : 0.0;
#pragma unroll
    for (int p = 0; p < r; ++p) acc = fma(-S[r][p], x[p], acc);
    x[r] = acc * dinv[r];
  }
  if (lane < m) {
#pragma unroll
    for (int r = 0; r < 32; ++r)
      if (r < m) Li[(int64_t)(o + r) * n + o + lane] = x[r];
  }
}

cudaError_t chol_inv_rec(double* A, double* Li, int64_t n, int o, int m, int* info, cudaStream_t s) {
  if (m <= 32) {
    chol_inv_leaf_kernel<<<1, 32, 0, s>>>(A, Li, n, o, m, info);
    return sf_launched(1);
  }
  const int nb = (m + 31) / 32;
  const int m1 = 32 * ((nb + 1) / 2);
  const int m2 = m - m1;
  cudaError_t e = chol_inv_rec(A, Li, n, o, m1, info, s);
  if (e != cudaSuccess) return e;
  double* A21 = A + (int64_t)(o + m1) * n + o;
  double* A22 = A + (int64_t)(o + m1) * n + o + m1;
  double* Li11 = Li + (int64_t)o * n + o;
  double* Li21 = Li + (int64_t)(o + m1) * n + o;
  double* Li22 = Li + (int64_t)(o + m1) * n + o + m1;
  // Li21 <- A21 * Li11^T  (op(B) = Li11^T is upper triangular)
  e = dgemm(DGemm{m2, m1, m1, A21, n, Li11, n, Li21, n, 1.0, 0.0, TRI_OPB_UPPER, 0}, 1, s);
  if (e != cudaSuccess) return e;
  // A22 <- A22 - Li21 * Li21^T  (lower tiles)
  e = dgemm(DGemm{m2, m2, m1, Li21, n, Li21, n, A22, n, -1.0, 1.0, TRI_NONE, 1}, 1, s);
  if (e != cudaSuccess) return e;
  e = chol_inv_rec(A, Li, n, o + m1, m2, info, s);
  if (e != cudaSuccess) return e;
  // A21 <- Li21 * Li11  (Li11 lower triangular)
  e = dgemm(DGemm{m2, m1, m1, Li21, n, Li11, n, A21, n, 1.0, 0.0, TRI_OPB_LOWER, 0}, 0, s);
  if (e != cudaSuccess) return e;
  // Li21 <- -Li22 * A21  (Li22 lower triangular)
  return dgemm(DGemm{m2, m1, m2, Li22, n, A21, n, Li21, n, -1.0, 0.0, TRI_OPA_LOWER, 0}, 0, s);
}

__global__ void transpose_kernel(const double* __restrict__ A, int n, double* __restrict__ At) {
  __shared__ double T[32][33];
  const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int i = by + r, j = bx + threadIdx.x;
    T[r][threadIdx.x] = (i < n && j < n) ? A[(int64_t)i * n + j] : 0.0;
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int i = bx + r, j = by + threadIdx.x;
    if (i < n && j < n) At[(int64_t)i * n + j] = T[threadIdx.x][r];
  }
}

__global__ void nonfinite_flag_kernel(const double* __restrict__ A, int64_t n, int bad_code, int* info) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    if (!isfinite(A[i])) {
      atomicCAS(info, 0, bad_code);
      return;
    }
}

}  // namespace

cudaError_t dense_chol_inverse(double* A, int n, double* Linv, int* info_dev, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(info_dev, 0, sizeof(int), s);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(Linv, 0, sizeof(double) * (size_t)n * n, s);
  if (e != cudaSuccess) return e;
  if (n <= 0) return cudaSuccess;
  e = chol_inv_rec(A, Linv, n, 0, n, info_dev, s);
  if (e != cudaSuccess) return e;
  const int64_t nn = (int64_t)n * n;
  nonfinite_flag_kernel<<<(int)std::min<int64_t>(div_up(nn, 256), 148 * 16), 256, 0, s>>>(Linv, nn, n + 1,
                                                                                          info_dev);
  return sf_launched(1);
}

cudaError_t launch_transpose(const double* A, int n, double* At, cudaStream_t s) {
  const int nb = div_up(n, 32);
  transpose_kernel<<<dim3(nb, nb), dim3(32, 8), 0, s>>>(A, n, At);
  return sf_launched(1);
}

}  // namespace simpfem
