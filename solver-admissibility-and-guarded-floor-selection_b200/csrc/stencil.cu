// Coarse-level operators of the Galerkin hierarchy as 27-point 3x3-block stencils.
//
// The reference assembles level 1 elementwise into CSR
// (gpu_fem/multigrid_v4.py:219-361, _build_level1_galerkin_struct +
// assemble_level1_galerkin) and forms level >= 2 with sparse triple products
// (gpu_fem/multigrid_v4.py:1275-1300); transfers are CSR SpMVs with
// kron(P_scalar, I3) restricted to free DOFs (gpu_fem/solver_v2.py:62-149,
// multigrid_v4.py:728-748).  On the structured grid every one of these is a
// stencil: the coarse operator of node n is 27 blocks of 3x3 coupling n to its
// neighbours n + o, and the trilinear transfers are separable products of 1-D
// weights.  Coefficients are stored structure-of-arrays,
// coef[(o * 9 + r * 3 + q) * nn + n], so a warp of consecutive nodes reads each
// coefficient with one coalesced access.
#include "common.cuh"

namespace simpfem {

__device__ __forceinline__ void node_ijk(const Grid& g, int64_t node, int& i, int& j, int& k) {
  const int NZ = g.nz + 1, NY = g.ny + 1;
  k = (int)(node % NZ);
  j = (int)((node / NZ) % NY);
  i = (int)(node / ((int64_t)NZ * NY));
}

__device__ __forceinline__ int64_t node_id(const Grid& g, int i, int j, int k) {
  return ((int64_t)i * (g.ny + 1) + j) * (g.nz + 1) + k;
}

template <typename VT, typename CT>
__device__ __forceinline__ VT coef_to(CT c) {
  return (VT)to_d(c);
}
template <>
__device__ __forceinline__ float coef_to<float, __nv_bfloat16>(__nv_bfloat16 c) {
  return __bfloat162float(c);
}

// One thread per (node, output component r): 81 coefficient loads (coalesced
// across the warp's consecutive nodes) and 81 gathered vector loads.  A
// neighbour outside the grid has zero coefficients (the assembly writes them),
// so its offset is clamped to 0 instead of branching and every load of the
// thread can be in flight at once.  32-bit node indices (levels >= 1 have at
// most 1/8 of the fine nodes; the launcher checks 3 * nn < 2^31).
template <typename VT, typename CT, int EPI>
__global__ void __launch_bounds__(256) stencil_kernel(Grid g, const CT* __restrict__ coef,
                                                      const uint8_t* __restrict__ mask, const VT* __restrict__ u,
                                                      EpiArgs ea) {
  if (guard_off(ea.guard)) return;
  const int nn = (int)g.nn;
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y;
  if (n >= nn) return;
  const int NZ1 = g.nz + 1, NY1 = g.ny + 1;
  const int k = n % NZ1, jq = n / NZ1;
  const int j = jq % NY1, i = jq / NY1;
  const int sx[3] = {i > 0 ? -NY1 * NZ1 : 0, 0, i < g.nx ? NY1 * NZ1 : 0};
  const int sy[3] = {j > 0 ? -NZ1 : 0, 0, j < g.ny ? NZ1 : 0};
  const int sz[3] = {k > 0 ? -1 : 0, 0, k < g.nz ? 1 : 0};
  const CT* cp = coef + (int64_t)(r * 3) * nn + n;
  VT acc = VT(0);
#pragma unroll
  for (int o = 0; o < 27; ++o) {
    const VT* um = u + 3 * (n + sx[o / 9] + sy[(o / 3) % 3] + sz[o % 3]);
#pragma unroll
    for (int q = 0; q < 3; ++q) acc += coef_to<VT, CT>(cp[(int64_t)(o * 9 + q) * nn]) * um[q];
  }
  const int dof = 3 * n + r;
  epilogue<VT, EPI>(ea, dof, mask[dof] != 0, acc, u[dof]);
}

template <typename VT, typename CT>
static cudaError_t stencil_dispatch(Epi epi, const Grid& g, const void* coef, const uint8_t* mask,
                                    const void* u, const EpiArgs& ea, cudaStream_t s) {
  if (3 * g.nn >= (int64_t(1) << 31)) return cudaErrorInvalidValue;
  const int bs = 256;
  const dim3 nb(div_up(g.nn, bs), 3);
  const CT* c = (const CT*)coef;
  const VT* uu = (const VT*)u;
  switch (epi) {
    case EPI_APPLY: stencil_kernel<VT, CT, EPI_APPLY><<<nb, bs, 0, s>>>(g, c, mask, uu, ea); break;
    case EPI_RESID: stencil_kernel<VT, CT, EPI_RESID><<<nb, bs, 0, s>>>(g, c, mask, uu, ea); break;
    case EPI_CHEB1: stencil_kernel<VT, CT, EPI_CHEB1><<<nb, bs, 0, s>>>(g, c, mask, uu, ea); break;
    case EPI_CHEB: stencil_kernel<VT, CT, EPI_CHEB><<<nb, bs, 0, s>>>(g, c, mask, uu, ea); break;
    case EPI_JAC: stencil_kernel<VT, CT, EPI_JAC><<<nb, bs, 0, s>>>(g, c, mask, uu, ea); break;
    default: return cudaErrorInvalidValue;
  }
  return sf_launched(1);
}

cudaError_t launch_stencil(DType vt, DType ct, Epi epi, const Grid& g, const void* coef,
                           const uint8_t* mask, const void* u, const EpiArgs& ea, cudaStream_t s) {
  if (vt == F64 && ct == F64) return stencil_dispatch<double, double>(epi, g, coef, mask, u, ea, s);
  if (vt == F32 && ct == F32) return stencil_dispatch<float, float>(epi, g, coef, mask, u, ea, s);
  if (vt == F32 && ct == BF16)
    return stencil_dispatch<float, __nv_bfloat16>(epi, g, coef, mask, u, ea, s);
  if (vt == F64 && ct == F32) return stencil_dispatch<double, float>(epi, g, coef, mask, u, ea, s);
  return cudaErrorInvalidValue;
}

// ----------------------------------------------------------------------------
// BF16 stencils of the mixed-precision cycle, node-major by neighbour column:
// coefC[n * 288 + col * 32 + oz * 9 + r * 3 + q] with col = ox * 3 + oy, i.e.
// the 27 coefficients coupling node n to its three z-neighbours in column
// (ox, oy) in one 64-byte slot (entries 27..31 zero).  Made from the FP64
// structure-of-arrays operator once per setup.
//
// Nine lanes per node, three nodes per warp: lane (t, col) loads its slot with
// four 16-byte loads and the 9 vector entries of its z-neighbours, forms its
// part of the node's three row sums, and the node's first lane adds the nine
// parts (in column order, through shared memory) and applies the epilogue with
// operands it read up front.  The row-per-thread kernel above chains 81 loads
// per thread (latency-bound on the small coarse levels) and a warp per node
// spends its issue slots on per-node index and reduction work; this split keeps
// both small.
constexpr int kColSlot = 32, kNodeStrideC = 9 * kColSlot;

// 32 nodes per block: coalesced reads along n of the FP64 operator, the tile
// transposed through shared memory, coalesced node-major BF16 writes
__global__ void __launch_bounds__(256) stencil_colmajor_bf16_kernel(int nn, const double* __restrict__ K64,
                                                                     __nv_bfloat16* __restrict__ out) {
  __shared__ __nv_bfloat16 tile[32 * kNodeStrideC];
  const int n0 = blockIdx.x * 32;
  const int nl = threadIdx.x & 31, c0 = threadIdx.x >> 5;
  const int cnt = min(32, nn - n0);
  for (int c = c0; c < kNodeStrideC; c += 8) {
    const int col = c / kColSlot, w = c % kColSlot;
    float v = 0.f;
    if (nl < cnt && w < 27) {
      const int o = col * 3 + w / 9;  // o = ox * 9 + oy * 3 + oz
      v = (float)K64[(int64_t)(o * 9 + w % 9) * nn + n0 + nl];
    }
    tile[nl * kNodeStrideC + c] = __float2bfloat16_rn(v);
  }
  __syncthreads();
  __nv_bfloat16* dst = out + (int64_t)n0 * kNodeStrideC;
  for (int e = threadIdx.x; e < cnt * kNodeStrideC; e += blockDim.x) dst[e] = tile[e];
}

cudaError_t launch_stencil_colmajor_bf16(int64_t nn, const double* K64, __nv_bfloat16* out, cudaStream_t s) {
  if (nn <= 0) return cudaSuccess;
  if (nn * kNodeStrideC >= (int64_t(1) << 31)) return cudaErrorInvalidValue;
  stencil_colmajor_bf16_kernel<<<div_up(nn, 32), 256, 0, s>>>((int)nn, K64, out);
  return sf_launched(1);
}

__device__ __forceinline__ float bf16_lo(unsigned w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf16_hi(unsigned w) { return __uint_as_float(w & 0xffff0000u); }

template <int EPI>
__global__ void __launch_bounds__(256) stencil_col_bf16_kernel(Grid g, const __nv_bfloat16* __restrict__ coefC,
                                                               const uint8_t* __restrict__ mask,
                                                               const float* __restrict__ u, EpiArgs ea) {
  __shared__ float part[8][27][3];
  if (guard_off(ea.guard)) return;
  const int nn = (int)g.nn;
  const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (warp * 3 >= nn) return;  // whole warps leave together
  const int t = lane / 9, col = lane - 9 * t;
  const int64_t n64 = warp * 3 + t;
  const bool act = lane < 27 && n64 < nn;
  const int n = act ? (int)n64 : 0;
  EpiOperands<float, EPI> eo;
  float xv[3];
  if (act && col == 0) {
    eo.load(ea, 3 * (int64_t)n, mask);
#pragma unroll
    for (int c = 0; c < 3; ++c) xv[c] = u[3 * n + c];
  }
  float p0 = 0.f, p1 = 0.f, p2 = 0.f;
  if (act) {
    const int NZ1 = g.nz + 1, NY1 = g.ny + 1;
    const int k = n % NZ1, jq = n / NZ1;
    const int j = jq % NY1, i = jq / NY1;
    const int ox = col / 3, oy = col % 3;
    // a neighbour outside the grid has zero coefficients: clamp it to the node itself
    const int dx = (ox == 0) ? (i > 0 ? -NY1 * NZ1 : 0) : (ox == 2 ? (i < g.nx ? NY1 * NZ1 : 0) : 0);
    const int dy = (oy == 0) ? (j > 0 ? -NZ1 : 0) : (oy == 2 ? (j < g.ny ? NZ1 : 0) : 0);
    const int base = n + dx + dy;
    const uint4* cp = reinterpret_cast<const uint4*>(coefC + (int64_t)n * kNodeStrideC + col * kColSlot);
    const uint4 q0 = cp[0], q1 = cp[1], q2 = cp[2], q3 = cp[3];
    const unsigned wv[16] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w,
                             q2.x, q2.y, q2.z, q2.w, q3.x, q3.y, q3.z, q3.w};
    float cf[28];
#pragma unroll
    for (int e = 0; e < 14; ++e) {
      cf[2 * e] = bf16_lo(wv[e]);
      cf[2 * e + 1] = bf16_hi(wv[e]);
    }
#pragma unroll
    for (int oz = 0; oz < 3; ++oz) {
      const int dz = (oz == 0) ? (k > 0 ? -1 : 0) : (oz == 2 ? (k < g.nz ? 1 : 0) : 0);
      const float* um = u + 3 * (base + dz);
      const float u0 = um[0], u1 = um[1], u2 = um[2];
      const float* c = cf + oz * 9;
      p0 = fmaf(c[0], u0, fmaf(c[1], u1, fmaf(c[2], u2, p0)));
      p1 = fmaf(c[3], u0, fmaf(c[4], u1, fmaf(c[5], u2, p1)));
      p2 = fmaf(c[6], u0, fmaf(c[7], u1, fmaf(c[8], u2, p2)));
    }
  }
  if (lane < 27) {
    part[wib][lane][0] = p0;
    part[wib][lane][1] = p1;
    part[wib][lane][2] = p2;
  }
  __syncwarp();
  if (act && col == 0) {
    float a0 = 0.f, a1 = 0.f, a2 = 0.f;
#pragma unroll
    for (int cc = 0; cc < 9; ++cc) {
      a0 += part[wib][lane + cc][0];
      a1 += part[wib][lane + cc][1];
      a2 += part[wib][lane + cc][2];
    }
    eo.apply(ea, 3 * (int64_t)n, 0, a0, xv[0]);
    eo.apply(ea, 3 * (int64_t)n + 1, 1, a1, xv[1]);
    eo.apply(ea, 3 * (int64_t)n + 2, 2, a2, xv[2]);
  }
}

cudaError_t launch_stencil_col_bf16(Epi epi, const Grid& g, const __nv_bfloat16* coefC, const uint8_t* mask,
                                    const float* u, const EpiArgs& ea, cudaStream_t s) {
  if (3 * g.nn >= (int64_t(1) << 31) || g.nn * kNodeStrideC >= (int64_t(1) << 31)) return cudaErrorInvalidValue;
  const int nb = div_up(div_up(g.nn, 3), 8);
  switch (epi) {
    case EPI_APPLY: stencil_col_bf16_kernel<EPI_APPLY><<<nb, 256, 0, s>>>(g, coefC, mask, u, ea); break;
    case EPI_RESID: stencil_col_bf16_kernel<EPI_RESID><<<nb, 256, 0, s>>>(g, coefC, mask, u, ea); break;
    case EPI_CHEB1: stencil_col_bf16_kernel<EPI_CHEB1><<<nb, 256, 0, s>>>(g, coefC, mask, u, ea); break;
    case EPI_CHEB: stencil_col_bf16_kernel<EPI_CHEB><<<nb, 256, 0, s>>>(g, coefC, mask, u, ea); break;
    case EPI_JAC: stencil_col_bf16_kernel<EPI_JAC><<<nb, 256, 0, s>>>(g, coefC, mask, u, ea); break;
    default: return cudaErrorInvalidValue;
  }
  return sf_launched(1);
}

// ----------------------------------------------------------------------------
// Level-1 Galerkin operator from the fine element moduli: for every coarse
// element C and sub-element stu, E_fine[child(C, stu)] * Q_stu with
// Q_stu = P24(stu)^T KE P24(stu), child clamped to the fine grid exactly as
// gpu_fem/multigrid_v4.py:285-289 does.  Q is given in corner-major order
// Q[stu][(a * 3 + r) * 24 + b * 3 + q] with a, b coarse-element corners.
__global__ void level1_assemble_kernel(Grid gc, Grid gf, const double* __restrict__ E,
                                       const double* __restrict__ Q, const uint8_t* __restrict__ mask,
                                       double* __restrict__ coef) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= 27 * gc.nn) return;
  const int o = (int)(idx / gc.nn);
  const int64_t n = idx - (int64_t)o * gc.nn;
  int i, j, k;
  node_ijk(gc, n, i, j, k);
  const int ox = o / 9 - 1, oy = (o / 3) % 3 - 1, oz = o % 3 - 1;
  const int mi = i + ox, mj = j + oy, mk = k + oz;
  double blk[9];
#pragma unroll
  for (int r = 0; r < 9; ++r) blk[r] = 0.0;
  const bool nb_ok = mi >= 0 && mj >= 0 && mk >= 0 && mi <= gc.nx && mj <= gc.ny && mk <= gc.nz;
  if (nb_ok) {
    for (int a = 0; a < 8; ++a) {
      const int ax = a >> 2, ay = (a >> 1) & 1, az = a & 1;
      const int bx = ax + ox, by = ay + oy, bz = az + oz;
      if (bx < 0 || bx > 1 || by < 0 || by > 1 || bz < 0 || bz > 1) continue;
      const int ci = i - ax, cj = j - ay, ck = k - az;
      if (ci < 0 || cj < 0 || ck < 0 || ci >= gc.nx || cj >= gc.ny || ck >= gc.nz) continue;
      const int b = bx * 4 + by * 2 + bz;
      double elem[9];
#pragma unroll
      for (int r = 0; r < 9; ++r) elem[r] = 0.0;
      for (int stu = 0; stu < 8; ++stu) {
        const int s_ = stu >> 2, t_ = (stu >> 1) & 1, u_ = stu & 1;
        const int fi = min(2 * ci + s_, gf.nx - 1);
        const int fj = min(2 * cj + t_, gf.ny - 1);
        const int fk = min(2 * ck + u_, gf.nz - 1);
        const double Ee = E[((int64_t)fi * gf.ny + fj) * gf.nz + fk];
        const double* q = Q + (int64_t)stu * 576;
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
          for (int c = 0; c < 3; ++c) elem[r * 3 + c] += Ee * q[(a * 3 + r) * 24 + b * 3 + c];
      }
#pragma unroll
      for (int r = 0; r < 9; ++r) blk[r] += elem[r];
    }
  }
  const int64_t m = nb_ok ? node_id(gc, mi, mj, mk) : 0;
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const bool keep = nb_ok && mask[3 * n + r] && mask[3 * m + c];
      coef[((int64_t)o * 9 + r * 3 + c) * gc.nn + n] = keep ? blk[r * 3 + c] : 0.0;
    }
}

cudaError_t launch_level1_assemble(const Grid& gc, const Grid& gf, const double* E_fine,
                                   const double* Q, const uint8_t* mask_c, double* coef,
                                   cudaStream_t s) {
  level1_assemble_kernel<<<div_up(27 * gc.nn, 128), 128, 0, s>>>(gc, gf, E_fine, Q, mask_c, coef);
  return sf_launched(1);
}

// ----------------------------------------------------------------------------
// 1-D trilinear weights, row-normalised as in gpu_fem/solver_v2.py:62-149:
// w[3 * f + (f - 2 * c + 1)] is the weight of coarse node c for fine node f.
__device__ __forceinline__ double w1(const double* w, int f, int c) {
  const int d = f - 2 * c;
  return (d < -1 || d > 1) ? 0.0 : w[3 * f + d + 1];
}

// K_c = R K_f P on stencils (Galerkin triple product of the reference's RAP loop).
// Coarse block (n, M = n + o) = sum over fine nodes f in the support of n and
// fine neighbours g = f + d of f in the support of M of
// P[f, n] K_f[f, g] P[g, M].  The trilinear weights factor per axis, so each
// axis contributes a list of at most 7 valid (f, d) pairs with weight
// w(f, I) w(g, I + m) (m the axis component of o), and the sum runs over the
// product of the three lists: only non-zero terms, no per-term bounds checks
// or weight lookups (the thread is otherwise bound by that scan of 27 x 27
// candidate pairs).
struct RapAxis {
  double w[7];
  int64_t off[7];  // fine-node offset (f - 2I) * node stride + d * stencil-block stride
  int cnt;
};

__device__ __forceinline__ void rap_axis(RapAxis& ax, const double* __restrict__ w, int I, int m, int nf,
                                         int64_t node_stride, int64_t blk_stride) {
  ax.cnt = 0;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int f = 2 * I + a - 1;
    if (f < 0 || f > nf) continue;
    const double wf = w1(w, f, I);
    if (wf == 0.0) continue;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const int gg = f + d - 1;
      if (gg < 0 || gg > nf) continue;
      const double wg = w1(w, gg, I + m);
      if (wg == 0.0) continue;
      ax.w[ax.cnt] = wf * wg;
      ax.off[ax.cnt] = (int64_t)(a - 1) * node_stride + (int64_t)d * blk_stride;
      ++ax.cnt;
    }
  }
}

__global__ void rap_kernel(Grid gf, Grid gc, const double* __restrict__ cf, const uint8_t* __restrict__ mask_c,
                           const double* __restrict__ wx, const double* __restrict__ wy,
                           const double* __restrict__ wz, double* __restrict__ cc) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= 27 * gc.nn) return;
  const int o = (int)(idx / gc.nn);
  const int64_t n = idx - (int64_t)o * gc.nn;
  int I, J, K;
  node_ijk(gc, n, I, J, K);
  const int mx = o / 9 - 1, my = (o / 3) % 3 - 1, mz = o % 3 - 1;
  const int MI = I + mx, MJ = J + my, MK = K + mz;
  double blk[9];
#pragma unroll
  for (int r = 0; r < 9; ++r) blk[r] = 0.0;
  const bool nb_ok = MI >= 0 && MJ >= 0 && MK >= 0 && MI <= gc.nx && MJ <= gc.ny && MK <= gc.nz;
  if (nb_ok) {
    const int64_t nn = gf.nn, NZ1 = gf.nz + 1, NY1 = gf.ny + 1;
    // stencil block of offset (dx, dy, dz) starts at ((dx * 9 + dy * 3 + dz) * 9) * nn
    RapAxis ax, ay, az;
    rap_axis(ax, wx, I, mx, gf.nx, NY1 * NZ1, 81 * nn);
    rap_axis(ay, wy, J, my, gf.ny, NZ1, 27 * nn);
    rap_axis(az, wz, K, mz, gf.nz, 1, 9 * nn);
    // index of the fine node (2I, 2J, 2K); every listed pair adds an offset that
    // lands on a fine node inside the grid
    const int64_t base = node_id(gf, 2 * I, 2 * J, 2 * K);
    for (int ex = 0; ex < ax.cnt; ++ex) {
      for (int ey = 0; ey < ay.cnt; ++ey) {
        const double wxy = ax.w[ex] * ay.w[ey];
        const int64_t bxy = base + ax.off[ex] + ay.off[ey];
#pragma unroll
        for (int ez = 0; ez < 7; ++ez) {
          if (ez >= az.cnt) break;
          const double pp = wxy * az.w[ez];
          const double* src = cf + (bxy + az.off[ez]);
#pragma unroll
          for (int r = 0; r < 9; ++r) blk[r] += pp * src[(int64_t)r * nn];
        }
      }
    }
  }
  const int64_t m = nb_ok ? node_id(gc, MI, MJ, MK) : 0;
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const bool keep = nb_ok && mask_c[3 * n + r] && mask_c[3 * m + c];
      cc[((int64_t)o * 9 + r * 3 + c) * gc.nn + n] = keep ? blk[r * 3 + c] : 0.0;
    }
}

cudaError_t launch_rap(const Grid& gf, const Grid& gc, const double* coef_f, const uint8_t* mask_c,
                       const double* wx, const double* wy, const double* wz, double* coef_c,
                       cudaStream_t s) {
  rap_kernel<<<div_up(27 * gc.nn, 128), 128, 0, s>>>(gf, gc, coef_f, mask_c, wx, wy, wz, coef_c);
  return sf_launched(1);
}

__global__ void stencil_diag_kernel(Grid g, const double* __restrict__ coef, const uint8_t* __restrict__ mask,
                                    double* __restrict__ dinv) {
  const int64_t dof = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (dof >= g.ndof) return;
  const int64_t n = dof / 3;
  const int r = (int)(dof - 3 * n);
  double d = coef[((int64_t)13 * 9 + r * 3 + r) * g.nn + n];
  d = fabs(d) > 1e-12 ? d : 1.0;
  dinv[dof] = mask[dof] ? 1.0 / d : 0.0;
}

cudaError_t launch_stencil_diag(const Grid& g, const double* coef, const uint8_t* mask,
                                double* dinv, cudaStream_t s) {
  stencil_diag_kernel<<<div_up(g.ndof, 256), 256, 0, s>>>(g, coef, mask, dinv);
  return sf_launched(1);
}

// ----------------------------------------------------------------------------
template <typename T>
__global__ void restrict_kernel(Grid gf, Grid gc, const double* __restrict__ wx, const double* __restrict__ wy,
                                const double* __restrict__ wz, const uint8_t* __restrict__ mask_c,
                                const T* __restrict__ fine, T* __restrict__ coarse, const int* guard) {
  if (guard_off(guard)) return;
  const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= gc.nn) return;
  int I, J, K;
  node_ijk(gc, n, I, J, K);
  // per-axis weights of the three fine nodes 2I - 1 .. 2I + 1 (0 outside the grid)
  double pw[3][3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int fi = 2 * I + a - 1, fj = 2 * J + a - 1, fk = 2 * K + a - 1;
    pw[0][a] = (fi < 0 || fi > gf.nx) ? 0.0 : w1(wx, fi, I);
    pw[1][a] = (fj < 0 || fj > gf.ny) ? 0.0 : w1(wy, fj, J);
    pw[2][a] = (fk < 0 || fk > gf.nz) ? 0.0 : w1(wz, fk, K);
  }
  T acc[3] = {T(0), T(0), T(0)};
#pragma unroll
  for (int d = 0; d < 27; ++d) {
    const int ax = d / 9, ay = (d / 3) % 3, az = d % 3;
    const T p = (T)(pw[0][ax] * pw[1][ay] * pw[2][az]);
    if (p == T(0)) continue;
    const int64_t f = node_id(gf, 2 * I + ax - 1, 2 * J + ay - 1, 2 * K + az - 1);
#pragma unroll
    for (int c = 0; c < 3; ++c) acc[c] += p * fine[3 * f + c];
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) coarse[3 * n + c] = mask_c[3 * n + c] ? acc[c] : T(0);
}

template <typename T>
__global__ void prolong_kernel(Grid gf, Grid gc, const double* __restrict__ wx, const double* __restrict__ wy,
                               const double* __restrict__ wz, const uint8_t* __restrict__ mask_f,
                               const T* __restrict__ coarse, T* __restrict__ fine, const int* guard) {
  if (guard_off(guard)) return;
  const int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= gf.nn) return;
  int i, j, k;
  node_ijk(gf, f, i, j, k);
  T acc[3] = {T(0), T(0), T(0)};
  // per-axis weights of the coarse parents floor(i/2) and floor(i/2) + 1 (0 outside)
  double qw[3][2];
#pragma unroll
  for (int b = 0; b < 2; ++b) {
    const int I = (i >> 1) + b, J = (j >> 1) + b, K = (k >> 1) + b;
    qw[0][b] = I > gc.nx ? 0.0 : w1(wx, i, I);
    qw[1][b] = J > gc.ny ? 0.0 : w1(wy, j, J);
    qw[2][b] = K > gc.nz ? 0.0 : w1(wz, k, K);
  }
  // coarse parents: floor(i/2) and floor(i/2)+1 (the latter only for odd i)
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const int I = (i >> 1) + (a >> 2), J = (j >> 1) + ((a >> 1) & 1), K = (k >> 1) + (a & 1);
    const T p = (T)(qw[0][a >> 2] * qw[1][(a >> 1) & 1] * qw[2][a & 1]);
    if (p == T(0)) continue;
    const int64_t n = node_id(gc, I, J, K);
#pragma unroll
    for (int c = 0; c < 3; ++c) acc[c] += p * coarse[3 * n + c];
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) fine[3 * f + c] = mask_f[3 * f + c] ? acc[c] : T(0);
}

cudaError_t launch_restrict(DType t, const Grid& gf, const Grid& gc, const double* wx,
                            const double* wy, const double* wz, const uint8_t* mask_c,
                            const void* fine, void* coarse, const int* guard, cudaStream_t s) {
  const int nb = div_up(gc.nn, 128);
  if (t == F64)
    restrict_kernel<double><<<nb, 128, 0, s>>>(gf, gc, wx, wy, wz, mask_c, (const double*)fine,
                                               (double*)coarse, guard);
  else
    restrict_kernel<float><<<nb, 128, 0, s>>>(gf, gc, wx, wy, wz, mask_c, (const float*)fine,
                                              (float*)coarse, guard);
  return sf_launched(1);
}

cudaError_t launch_prolong(DType t, const Grid& gf, const Grid& gc, const double* wx,
                           const double* wy, const double* wz, const uint8_t* mask_f,
                           const void* coarse, void* fine, const int* guard, cudaStream_t s) {
  const int nb = div_up(gf.nn, 128);
  if (t == F64)
    prolong_kernel<double><<<nb, 128, 0, s>>>(gf, gc, wx, wy, wz, mask_f, (const double*)coarse,
                                              (double*)fine, guard);
  else
    prolong_kernel<float><<<nb, 128, 0, s>>>(gf, gc, wx, wy, wz, mask_f, (const float*)coarse,
                                             (float*)fine, guard);
  return sf_launched(1);
}

// ----------------------------------------------------------------------------
// Dense free-DOF matrix of the coarsest stencil (row-major n x n; A zeroed first).
__global__ void stencil_to_dense_kernel(Grid g, const double* __restrict__ coef,
                                        const int32_t* __restrict__ didx, int64_t n,
                                        double* __restrict__ A) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= 27 * g.ndof) return;
  const int o = (int)(idx / g.ndof);
  const int64_t dof = idx - (int64_t)o * g.ndof;
  const int64_t p = didx[dof];
  if (p < 0) return;
  const int64_t node = dof / 3;
  const int r = (int)(dof - 3 * node);
  int i, j, k;
  node_ijk(g, node, i, j, k);
  const int mi = i + o / 9 - 1, mj = j + (o / 3) % 3 - 1, mk = k + o % 3 - 1;
  if (mi < 0 || mj < 0 || mk < 0 || mi > g.nx || mj > g.ny || mk > g.nz) return;
  const int64_t m = node_id(g, mi, mj, mk);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const int64_t q = didx[3 * m + c];
    if (q < 0) continue;
    A[p * n + q] = coef[((int64_t)o * 9 + r * 3 + c) * g.nn + node];
  }
}

cudaError_t launch_stencil_to_dense(const Grid& g, const double* coef, const int32_t* dense_idx,
                                    int64_t n, double* A, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(A, 0, sizeof(double) * n * n, s);
  if (e != cudaSuccess) return e;
  stencil_to_dense_kernel<<<div_up(27 * g.ndof, 256), 256, 0, s>>>(g, coef, dense_idx, n, A);
  return sf_launched(1);
}

// ----------------------------------------------------------------------------
template <typename A, typename B>
__global__ void convert_kernel(const A* __restrict__ src, B* __restrict__ dst, int64_t n, const int* guard) {
  if (guard_off(guard)) return;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = from_d<B>(to_d(src[i]));
}

template <>
__global__ void convert_kernel<double, float>(const double* __restrict__ src, float* __restrict__ dst,
                                              int64_t n, const int* guard) {
  if (guard_off(guard)) return;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = __double2float_rn(src[i]);
}

cudaError_t launch_convert(DType from, DType to, const void* src, void* dst, int64_t n,
                           const int* guard, cudaStream_t s) {
  const int nb = div_up(n, 256);
  if (from == F64 && to == F32)
    convert_kernel<double, float><<<nb, 256, 0, s>>>((const double*)src, (float*)dst, n, guard);
  else if (from == F32 && to == F64)
    convert_kernel<float, double><<<nb, 256, 0, s>>>((const float*)src, (double*)dst, n, guard);
  else if (from == F64 && to == BF16)
    convert_kernel<double, __nv_bfloat16><<<nb, 256, 0, s>>>((const double*)src,
                                                             (__nv_bfloat16*)dst, n, guard);
  else if (from == F64 && to == F64)
    convert_kernel<double, double><<<nb, 256, 0, s>>>((const double*)src, (double*)dst, n, guard);
  else if (from == F32 && to == F32)
    convert_kernel<float, float><<<nb, 256, 0, s>>>((const float*)src, (float*)dst, n, guard);
  else
    return cudaErrorInvalidValue;
  return sf_launched(1);
}

}  // namespace simpfem
