// Fine-level hex8 operator for the structured SIMP mesh.
//
// Replaces the reference's MatrixFreeKff.matvec (gpu_fem/solver_v2.py:1182-1222:
// expand -> gather -> KE @ u_elem.T * E -> bincount -> restrict) and the fused
// FusedMatvec kernels (gpu_fem/cuda_fused_matvec.py:41-88, :112-246) with one
// deterministic sweep kernel:
//
//  * Node indices are computed from (i, j, k); there is no edof table.
//  * A block owns a (bj-1) x (bk-1) patch of node columns (one halo element
//    column on the low j and k sides) and sweeps cx node planes along x.  Each
//    thread computes one element per plane and carries the element's +x face
//    contribution in registers to the next plane, so every element is
//    evaluated once per sweep (plus the halo columns).
//  * The element product KE * u_e uses the reflection symmetry of the unit
//    cube: in the Walsh (+/-1) basis over the element's 2x2x2 nodes the 24x24
//    unit stiffness is block diagonal with eight 3x3 blocks, so
//    KE u = H (B (H u)) costs 72 add + 72 FMA + 72 add instead of 576 FMA.
//  * Per-node sums are reduced in shared memory in a fixed order (no atomics),
//    and the caller's epilogue (residual, Chebyshev or Jacobi update) is fused
//    into the store.
#include <stdio.h>

#include "common.cuh"

namespace simpfem {

__constant__ double c_wht64[8][9];
__constant__ float c_wht32[8][9];
__constant__ float c_keb16[576];   // KE rounded to bf16 (stored as float), corner-major order
__constant__ double c_kediag[24];  // KE diagonal, corner-major order
__constant__ double c_kenb[8][9];  // 3x3 node-diagonal blocks of KE per corner

// corner q = dx * 4 + dy * 2 + dz  <->  reference local node (gpu_fem/pub_simp_solver.py:196-207)
static const int kRefNodeOfCorner[8] = {0, 4, 3, 7, 1, 5, 2, 6};

void set_fine_constants(const double* ke576, const WhtBlocks& wb) {
  // KE in corner-major order: row (q * 3 + c) <- reference row (3 * a(q) + c)
  double kem[576];
  for (int q = 0; q < 8; ++q)
    for (int c = 0; c < 3; ++c)
      for (int q2 = 0; q2 < 8; ++q2)
        for (int c2 = 0; c2 < 3; ++c2)
          kem[(q * 3 + c) * 24 + q2 * 3 + c2] =
              ke576[(3 * kRefNodeOfCorner[q] + c) * 24 + 3 * kRefNodeOfCorner[q2] + c2];
  float keb[576];
  for (int i = 0; i < 576; ++i) keb[i] = __bfloat162float(__float2bfloat16_rn((float)kem[i]));
  double kd[24];
  for (int i = 0; i < 24; ++i) kd[i] = kem[i * 24 + i];
  double nb[8][9];
  for (int q = 0; q < 8; ++q)
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) nb[q][r * 3 + c] = kem[(q * 3 + r) * 24 + q * 3 + c];
  float w32[8][9];
  for (int b = 0; b < 8; ++b)
    for (int i = 0; i < 9; ++i) w32[b][i] = (float)wb.b[b][i];
  cudaMemcpyToSymbol(c_wht64, wb.b, sizeof(wb.b));
  cudaMemcpyToSymbol(c_wht32, w32, sizeof(w32));
  cudaMemcpyToSymbol(c_keb16, keb, sizeof(keb));
  cudaMemcpyToSymbol(c_kediag, kd, sizeof(kd));
  cudaMemcpyToSymbol(c_kenb, nb, sizeof(nb));
}

template <typename T>
__device__ __forceinline__ T wht_coef(int b, int i);
template <>
__device__ __forceinline__ double wht_coef<double>(int b, int i) { return c_wht64[b][i]; }
template <>
__device__ __forceinline__ float wht_coef<float>(int b, int i) { return c_wht32[b][i]; }

template <typename T>
__device__ __forceinline__ void wht8(T a[8]) {
#pragma unroll
  for (int m = 4; m >= 1; m >>= 1) {
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      if ((q & m) == 0) {
        T p = a[q], r = a[q | m];
        a[q] = p + r;
        a[q | m] = p - r;
      }
    }
  }
}

// f = E * KE * u for one element, u/f indexed [corner][component].
template <typename T>
__device__ __forceinline__ void elem_wht(const T (&u)[8][3], T E, T (&f)[8][3]) {
  T w[3][8];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
#pragma unroll
    for (int q = 0; q < 8; ++q) w[c][q] = u[q][c];
    wht8(w[c]);
  }
  T v[3][8];
#pragma unroll
  for (int b = 0; b < 8; ++b) {
    const T in0 = w[0][b ^ 4], in1 = w[1][b ^ 2], in2 = w[2][b ^ 1];
    v[0][b ^ 4] = E * (wht_coef<T>(b, 0) * in0 + wht_coef<T>(b, 1) * in1 + wht_coef<T>(b, 2) * in2);
    v[1][b ^ 2] = E * (wht_coef<T>(b, 3) * in0 + wht_coef<T>(b, 4) * in1 + wht_coef<T>(b, 5) * in2);
    v[2][b ^ 1] = E * (wht_coef<T>(b, 6) * in0 + wht_coef<T>(b, 7) * in1 + wht_coef<T>(b, 8) * in2);
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    wht8(v[c]);
#pragma unroll
    for (int q = 0; q < 8; ++q) f[q][c] = v[c][q];
  }
}

// f = E * (KE_bf16 @ bf16(u)) with FP32 accumulation (the reference's BF16 WMMA
// semantics, gpu_fem/cuda_fused_matvec.py:112-246).
__device__ __forceinline__ void elem_bf16(const float (&u)[8][3], float E, float (&f)[8][3]) {
  float ub[24];
#pragma unroll
  for (int q = 0; q < 8; ++q)
#pragma unroll
    for (int c = 0; c < 3; ++c) ub[q * 3 + c] = __bfloat162float(__float2bfloat16_rn(u[q][c]));
#pragma unroll
  for (int i = 0; i < 24; ++i) {
    float acc = 0.f;
#pragma unroll
    for (int j = 0; j < 24; ++j) acc = fmaf(c_keb16[j * 24 + i], ub[j], acc);
    f[i / 3][i % 3] = E * acc;
  }
}

template <typename T>
__device__ __forceinline__ void load_face(T (&uu)[4][3], const T* __restrict__ u, const Grid& g,
                                          int p, int je, int ke, bool colv) {
#pragma unroll
  for (int q2 = 0; q2 < 4; ++q2) {
    const int dj = q2 >> 1, dk = q2 & 1;
    const int j = je + dj, k = ke + dk;
    const bool ok = p >= 0 && p <= g.nx && j >= 0 && j <= g.ny && k >= 0 && k <= g.nz &&
                    (colv || q2 == 0);
    if (ok) {
      const int64_t node = ((int64_t)p * (g.ny + 1) + j) * (g.nz + 1) + k;
#pragma unroll
      for (int c = 0; c < 3; ++c) uu[q2][c] = u[3 * node + c];
    } else {
#pragma unroll
      for (int c = 0; c < 3; ++c) uu[q2][c] = T(0);
    }
  }
}

template <typename T, int EPI, int KMODE, int MAXT>
__global__ void __launch_bounds__(MAXT) fine_sweep_kernel(Grid g, SweepShape sh, const T* __restrict__ E,
                                                          const uint8_t* __restrict__ mask,
                                                          const T* __restrict__ u, EpiArgs ea) {
  if (guard_off(ea.guard)) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* S = reinterpret_cast<T*>(smem_raw);
  const int NT = sh.bj * sh.bk;
  const int t = threadIdx.x;
  const int tj = t / sh.bk, tk = t - tj * sh.bk;
  const int nbk = (g.nz + sh.bk - 1) / (sh.bk - 1);  // ceil((nz+1)/(bk-1))
  const int bjI = blockIdx.x / nbk, bkI = blockIdx.x - bjI * nbk;
  const int je = bjI * (sh.bj - 1) - 1 + tj;
  const int ke = bkI * (sh.bk - 1) - 1 + tk;
  const int i0 = blockIdx.y * sh.cx;
  const int i1 = min(i0 + sh.cx, g.nx + 1);
  const bool colv = je >= 0 && je < g.ny && ke >= 0 && ke < g.nz;
  const bool own = tj >= 1 && tk >= 1 && je <= g.ny && ke <= g.nz;

  T ulo[4][3], uhi[4][3], carry[4][3];
  load_face<T>(ulo, u, g, i0 - 1, je, ke, colv);
#pragma unroll
  for (int q2 = 0; q2 < 4; ++q2)
#pragma unroll
    for (int c = 0; c < 3; ++c) carry[q2][c] = T(0);

  for (int ie = i0 - 1; ie < i1; ++ie) {
    load_face<T>(uhi, u, g, ie + 1, je, ke, colv);
    const bool ev = colv && ie >= 0 && ie < g.nx;
    T f[8][3];
    if (ev) {
      T ue[8][3];
#pragma unroll
      for (int q2 = 0; q2 < 4; ++q2)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          ue[q2][c] = ulo[q2][c];
          ue[4 + q2][c] = uhi[q2][c];
        }
      const T Ee = E[((int64_t)ie * g.ny + je) * g.nz + ke];
      if (KMODE == 0) {
        elem_wht<T>(ue, Ee, f);
      } else {
        elem_bf16(reinterpret_cast<const float(&)[8][3]>(ue), (float)Ee,
                  reinterpret_cast<float(&)[8][3]>(f));
      }
    } else {
#pragma unroll
      for (int q = 0; q < 8; ++q)
#pragma unroll
        for (int c = 0; c < 3; ++c) f[q][c] = T(0);
    }
    if (ie >= i0) {
      T* buf = S + ((ie - i0) & 1) * 12 * NT;
#pragma unroll
      for (int q2 = 0; q2 < 4; ++q2)
#pragma unroll
        for (int c = 0; c < 3; ++c) buf[(q2 * 3 + c) * NT + t] = carry[q2][c] + f[q2][c];
      __syncthreads();
      if (own) {
        const int64_t node = ((int64_t)ie * (g.ny + 1) + je) * (g.nz + 1) + ke;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const T ku = ((buf[(0 * 3 + c) * NT + t] + buf[(2 * 3 + c) * NT + t - sh.bk]) +
                        buf[(1 * 3 + c) * NT + t - 1]) +
                       buf[(3 * 3 + c) * NT + t - sh.bk - 1];
          const int64_t dof = 3 * node + c;
          epilogue<T, EPI>(ea, dof, mask[dof] != 0, ku, ulo[0][c]);
        }
      }
    }
#pragma unroll
    for (int q2 = 0; q2 < 4; ++q2)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        carry[q2][c] = f[4 + q2][c];
        ulo[q2][c] = uhi[q2][c];
      }
  }
}

template <typename T, int EPI, int KMODE, int MAXT>
static cudaError_t launch_sweep(const Grid& g, const SweepShape& sh, const T* E, const uint8_t* mask,
                                const T* u, const EpiArgs& ea, cudaStream_t s) {
  const int NT = sh.bj * sh.bk;
  if (NT > MAXT || sh.bj < 2 || sh.bk < 2 || sh.cx < 1) return cudaErrorInvalidConfiguration;
  const size_t smem = (size_t)2 * 12 * NT * sizeof(T);
  static bool attr_done = false;
  if (!attr_done) {
    cudaFuncSetAttribute(fine_sweep_kernel<T, EPI, KMODE, MAXT>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr_done = true;
  }
  const int nbj = (g.ny + sh.bj - 1) / (sh.bj - 1);
  const int nbk = (g.nz + sh.bk - 1) / (sh.bk - 1);
  dim3 grid(nbj * nbk, div_up(g.nx + 1, sh.cx));
  fine_sweep_kernel<T, EPI, KMODE, MAXT><<<grid, NT, smem, s>>>(g, sh, E, mask, u, ea);
  return sf_launched(1);
}

constexpr int kMaxThreadsF64 = 256;
constexpr int kMaxThreadsF32 = 512;

cudaError_t launch_fine(DType t, Epi epi, const Grid& g, const SweepShape& sh, const void* E,
                        const uint8_t* mask, const void* u, const EpiArgs& ea, cudaStream_t s) {
#define SF_FINE_CASE(T, MAXT, E_)                                                              \
  case E_:                                                                                     \
    return launch_sweep<T, E_, 0, MAXT>(g, sh, (const T*)E, mask, (const T*)u, ea, s);
  if (t == F64) {
    switch (epi) {
      SF_FINE_CASE(double, kMaxThreadsF64, EPI_APPLY)
      SF_FINE_CASE(double, kMaxThreadsF64, EPI_RESID)
      SF_FINE_CASE(double, kMaxThreadsF64, EPI_CHEB1)
      SF_FINE_CASE(double, kMaxThreadsF64, EPI_CHEB)
      SF_FINE_CASE(double, kMaxThreadsF64, EPI_JAC)
    }
  } else if (t == F32) {
    switch (epi) {
      SF_FINE_CASE(float, kMaxThreadsF32, EPI_APPLY)
      SF_FINE_CASE(float, kMaxThreadsF32, EPI_RESID)
      SF_FINE_CASE(float, kMaxThreadsF32, EPI_CHEB1)
      SF_FINE_CASE(float, kMaxThreadsF32, EPI_CHEB)
      SF_FINE_CASE(float, kMaxThreadsF32, EPI_JAC)
    }
  } else if (t == BF16) {
    // BF16 operands (u and KE rounded to bf16), FP32 accumulation and FP32 vectors.
    switch (epi) {
      case EPI_APPLY:
        return launch_sweep<float, EPI_APPLY, 1, kMaxThreadsF32>(g, sh, (const float*)E, mask,
                                                                 (const float*)u, ea, s);
      case EPI_RESID:
        return launch_sweep<float, EPI_RESID, 1, kMaxThreadsF32>(g, sh, (const float*)E, mask,
                                                                 (const float*)u, ea, s);
      case EPI_CHEB1:
        return launch_sweep<float, EPI_CHEB1, 1, kMaxThreadsF32>(g, sh, (const float*)E, mask,
                                                                 (const float*)u, ea, s);
      case EPI_CHEB:
        return launch_sweep<float, EPI_CHEB, 1, kMaxThreadsF32>(g, sh, (const float*)E, mask,
                                                                (const float*)u, ea, s);
      case EPI_JAC:
        return launch_sweep<float, EPI_JAC, 1, kMaxThreadsF32>(g, sh, (const float*)E, mask,
                                                               (const float*)u, ea, s);
    }
  }
#undef SF_FINE_CASE
  return cudaErrorInvalidValue;
}

// ----------------------------------------------------------------------------
// diag(K_ff): per node, sum over the adjacent elements of E_e * KE_jj
// (MatrixFreeKff.extract_diagonal, gpu_fem/solver_v2.py:1228-1251).
__global__ void fine_diag_kernel(Grid g, const double* __restrict__ E, const uint8_t* __restrict__ mask,
                                 double* __restrict__ diag) {
  const int64_t node = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (node >= g.nn) return;
  const int NZ = g.nz + 1, NY = g.ny + 1;
  const int k = (int)(node % NZ);
  const int j = (int)((node / NZ) % NY);
  const int i = (int)(node / ((int64_t)NZ * NY));
  double acc[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    // element whose corner q sits on this node
    const int dx = q >> 2, dy = (q >> 1) & 1, dz = q & 1;
    const int ei = i - dx, ej = j - dy, ek = k - dz;
    if (ei < 0 || ej < 0 || ek < 0 || ei >= g.nx || ej >= g.ny || ek >= g.nz) continue;
    const double Ee = E[((int64_t)ei * g.ny + ej) * g.nz + ek];
#pragma unroll
    for (int c = 0; c < 3; ++c) acc[c] += Ee * c_kediag[q * 3 + c];
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) diag[3 * node + c] = mask[3 * node + c] ? acc[c] : 0.0;
}

cudaError_t launch_fine_diag(const Grid& g, const double* E, const uint8_t* mask, double /*kd*/,
                             double* diag, cudaStream_t s) {
  fine_diag_kernel<<<div_up(g.nn, 256), 256, 0, s>>>(g, E, mask, diag);
  return sf_launched(1);
}

// ----------------------------------------------------------------------------
// 3x3 node-block Jacobi (NodeBlockJacobiMF, gpu_fem/solver_v2.py:1268-1451):
// block(n) = sum_e E_e * KE[node block of n in e]; all-free nodes store the
// block inverse, partially constrained nodes store 1/diag for their free
// components (the reference's scalar fallback), constrained components 0.
__global__ void node_blocks_kernel(Grid g, const double* __restrict__ E, const uint8_t* __restrict__ mask,
                                   const double* __restrict__ diag_full, double* __restrict__ binv) {
  const int64_t node = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (node >= g.nn) return;
  const int NZ = g.nz + 1, NY = g.ny + 1;
  const int k = (int)(node % NZ);
  const int j = (int)((node / NZ) % NY);
  const int i = (int)(node / ((int64_t)NZ * NY));
  double B[9];
#pragma unroll
  for (int r = 0; r < 9; ++r) B[r] = 0.0;
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const int dx = q >> 2, dy = (q >> 1) & 1, dz = q & 1;
    const int ei = i - dx, ej = j - dy, ek = k - dz;
    if (ei < 0 || ej < 0 || ek < 0 || ei >= g.nx || ej >= g.ny || ek >= g.nz) continue;
    const double Ee = E[((int64_t)ei * g.ny + ej) * g.nz + ek];
#pragma unroll
    for (int r = 0; r < 9; ++r) B[r] += Ee * c_kenb[q][r];
  }
  const bool f0 = mask[3 * node], f1 = mask[3 * node + 1], f2 = mask[3 * node + 2];
  double out[9];
#pragma unroll
  for (int r = 0; r < 9; ++r) out[r] = 0.0;
  if (f0 && f1 && f2) {
    const double c00 = B[4] * B[8] - B[5] * B[7];
    const double c01 = B[5] * B[6] - B[3] * B[8];
    const double c02 = B[3] * B[7] - B[4] * B[6];
    const double det = B[0] * c00 + B[1] * c01 + B[2] * c02;
    const double id = 1.0 / det;
    out[0] = c00 * id;
    out[1] = (B[2] * B[7] - B[1] * B[8]) * id;
    out[2] = (B[1] * B[5] - B[2] * B[4]) * id;
    out[3] = c01 * id;
    out[4] = (B[0] * B[8] - B[2] * B[6]) * id;
    out[5] = (B[2] * B[3] - B[0] * B[5]) * id;
    out[6] = c02 * id;
    out[7] = (B[1] * B[6] - B[0] * B[7]) * id;
    out[8] = (B[0] * B[4] - B[1] * B[3]) * id;
  } else {
    const bool fr[3] = {f0, f1, f2};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      // without a scalar diagonal the reference leaves these components at 0
      if (fr[c] && diag_full != nullptr) {
        double d = diag_full[3 * node + c];
        d = fabs(d) > 1e-12 ? d : 1.0;
        out[c * 4] = 1.0 / d;
      }
    }
  }
#pragma unroll
  for (int r = 0; r < 9; ++r) binv[9 * node + r] = out[r];
}

cudaError_t launch_node_blocks(const Grid& g, const double* E, const uint8_t* mask,
                               const double* diag_full, double* binv, cudaStream_t s) {
  node_blocks_kernel<<<div_up(g.nn, 256), 256, 0, s>>>(g, E, mask, diag_full, binv);
  return sf_launched(1);
}

__global__ void node_block_apply_kernel(int64_t nn, const double* __restrict__ binv,
                                        const double* __restrict__ r, double* __restrict__ z,
                                        const int* guard) {
  if (guard_off(guard)) return;
  const int64_t node = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (node >= nn) return;
  const double r0 = r[3 * node], r1 = r[3 * node + 1], r2 = r[3 * node + 2];
  const double* B = binv + 9 * node;
#pragma unroll
  for (int c = 0; c < 3; ++c) z[3 * node + c] = B[3 * c] * r0 + B[3 * c + 1] * r1 + B[3 * c + 2] * r2;
}

cudaError_t launch_node_block_apply(const Grid& g, const double* binv, const double* r, double* z,
                                    const int* guard, cudaStream_t s) {
  node_block_apply_kernel<<<div_up(g.nn, 256), 256, 0, s>>>(g.nn, binv, r, z, guard);
  return sf_launched(1);
}

// ----------------------------------------------------------------------------
// Element strain energy u_e^T KE u_e (SolverV4 sensitivity, gpu_fem/solver_v4.py:257-264).
__global__ void element_energy_kernel(Grid g, const double* __restrict__ u, double* __restrict__ ce) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= g.ne()) return;
  const int ek = (int)(e % g.nz);
  const int ej = (int)((e / g.nz) % g.ny);
  const int ei = (int)(e / ((int64_t)g.nz * g.ny));
  double ue[8][3];
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const int dx = q >> 2, dy = (q >> 1) & 1, dz = q & 1;
    const int64_t node = ((int64_t)(ei + dx) * (g.ny + 1) + (ej + dy)) * (g.nz + 1) + (ek + dz);
#pragma unroll
    for (int c = 0; c < 3; ++c) ue[q][c] = u[3 * node + c];
  }
  double f[8][3];
  elem_wht<double>(ue, 1.0, f);
  double acc = 0.0;
#pragma unroll
  for (int q = 0; q < 8; ++q)
#pragma unroll
    for (int c = 0; c < 3; ++c) acc += f[q][c] * ue[q][c];
  ce[e] = acc;
}

cudaError_t launch_element_energy(const Grid& g, const double* u_full, double* ce, cudaStream_t s) {
  element_energy_kernel<<<div_up(g.ne(), 256), 256, 0, s>>>(g, u_full, ce);
  return sf_launched(1);
}

}  // namespace simpfem
