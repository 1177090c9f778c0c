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
__global__ void rap_kernel(Grid gf, Grid gc, const double* __restrict__ cf, const uint8_t* __restrict__ mask_c,
                           const double* __restrict__ wx, const double* __restrict__ wy,
                           const double* __restrict__ wz, double* __restrict__ cc) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= 27 * gc.nn) return;
  const int o = (int)(idx / gc.nn);
  const int64_t n = idx - (int64_t)o * gc.nn;
  int I, J, K;
  node_ijk(gc, n, I, J, K);
  const int MI = I + o / 9 - 1, MJ = J + (o / 3) % 3 - 1, MK = K + o % 3 - 1;
  double blk[9];
#pragma unroll
  for (int r = 0; r < 9; ++r) blk[r] = 0.0;
  const bool nb_ok = MI >= 0 && MJ >= 0 && MK >= 0 && MI <= gc.nx && MJ <= gc.ny && MK <= gc.nz;
  if (nb_ok) {
    for (int d1 = 0; d1 < 27; ++d1) {
      const int fi = 2 * I + d1 / 9 - 1, fj = 2 * J + (d1 / 3) % 3 - 1, fk = 2 * K + d1 % 3 - 1;
      if (fi < 0 || fj < 0 || fk < 0 || fi > gf.nx || fj > gf.ny || fk > gf.nz) continue;
      const double p1 = w1(wx, fi, I) * w1(wy, fj, J) * w1(wz, fk, K);
      if (p1 == 0.0) continue;
      const int64_t f1 = node_id(gf, fi, fj, fk);
      for (int of = 0; of < 27; ++of) {
        const int gi = fi + of / 9 - 1, gj = fj + (of / 3) % 3 - 1, gk = fk + of % 3 - 1;
        if (gi < 0 || gj < 0 || gk < 0 || gi > gf.nx || gj > gf.ny || gk > gf.nz) continue;
        const double p2 = w1(wx, gi, MI) * w1(wy, gj, MJ) * w1(wz, gk, MK);
        if (p2 == 0.0) continue;
        const double pp = p1 * p2;
        const double* src = cf + (int64_t)of * 9 * gf.nn + f1;
#pragma unroll
        for (int r = 0; r < 9; ++r) blk[r] += pp * src[(int64_t)r * gf.nn];
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
  T acc[3] = {T(0), T(0), T(0)};
  for (int d = 0; d < 27; ++d) {
    const int fi = 2 * I + d / 9 - 1, fj = 2 * J + (d / 3) % 3 - 1, fk = 2 * K + d % 3 - 1;
    if (fi < 0 || fj < 0 || fk < 0 || fi > gf.nx || fj > gf.ny || fk > gf.nz) continue;
    const T p = (T)(w1(wx, fi, I) * w1(wy, fj, J) * w1(wz, fk, K));
    if (p == T(0)) continue;
    const int64_t f = node_id(gf, fi, fj, fk);
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
  // coarse parents: floor(i/2) and floor(i/2)+1 (the latter only for odd i)
  for (int a = 0; a < 8; ++a) {
    const int I = (i >> 1) + (a >> 2), J = (j >> 1) + ((a >> 1) & 1), K = (k >> 1) + (a & 1);
    if (I > gc.nx || J > gc.ny || K > gc.nz) continue;
    const T p = (T)(w1(wx, i, I) * w1(wy, j, J) * w1(wz, k, K));
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
