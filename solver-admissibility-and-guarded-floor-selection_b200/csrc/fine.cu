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
__constant__ float2 c_wht32x2[8][9];  // c_wht32 duplicated into both lanes of a pair
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
  SF_CUDA(cudaMemcpyToSymbol(c_wht64, wb.b, sizeof(wb.b)));
  SF_CUDA(cudaMemcpyToSymbol(c_wht32, w32, sizeof(w32)));
  float2 w32x2[8][9];
  for (int b = 0; b < 8; ++b)
    for (int i = 0; i < 9; ++i) w32x2[b][i] = make_float2(w32[b][i], w32[b][i]);
  SF_CUDA(cudaMemcpyToSymbol(c_wht32x2, w32x2, sizeof(w32x2)));
  SF_CUDA(cudaMemcpyToSymbol(c_keb16, keb, sizeof(keb)));
  SF_CUDA(cudaMemcpyToSymbol(c_kediag, kd, sizeof(kd)));
  SF_CUDA(cudaMemcpyToSymbol(c_kenb, nb, sizeof(nb)));
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

// Each block stages its (bj+1) x (bk+1) node tile of one x-plane in shared
// memory: a tile row is 3 (bk+1) consecutive values of u, so the block reads it
// with coalesced loads, one value per thread and row (no node is read four
// times).  Thread t loads the values t, t + NT, ... of the flattened tile; the
// offsets do not depend on the plane and are computed once.
constexpr int kTileLoads = 6;  // enough for every shape with bj >= 2, bk >= 3; launch checks
constexpr int kPlaneBufs = 4;  // node-plane tiles: two being read, two in flight

// One element copied global -> shared asynchronously (cp.async; zero-filled when
// ok is false, reading nothing from src, which is then any valid address).
template <typename T>
__device__ __forceinline__ void cp_async_elem(T* dst, const T* src, bool ok) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  if (sizeof(T) == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(ok ? 8 : 0));
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src), "r"(ok ? 4 : 0));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all_but_one() { asm volatile("cp.async.wait_group 1;\n" ::); }

template <typename T, int EPI, int KMODE, int MAXT>
__global__ void __launch_bounds__(MAXT) fine_sweep_kernel(Grid g, SweepShape sh, const T* __restrict__ E,
                                                          const uint8_t* __restrict__ mask,
                                                          const T* __restrict__ u, EpiArgs ea) {
  if (guard_off(ea.guard)) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int NT = sh.bj * sh.bk;
  const int W = 3 * (sh.bk + 1);   // values per tile row
  const int PV = (sh.bj + 1) * W;  // values per plane tile
  T* F = reinterpret_cast<T*>(smem_raw);  // face sums [2][12][NT]
  T* P = F + 24 * NT;                     // node-plane tiles [kPlaneBufs][PV]
  const int t = threadIdx.x;
  const int tj = t / sh.bk, tk = t - tj * sh.bk;
  const int nbk = (g.nz + sh.bk - 1) / (sh.bk - 1);  // ceil((nz+1)/(bk-1))
  const int bjI = blockIdx.x / nbk, bkI = blockIdx.x - bjI * nbk;
  const int jb = bjI * (sh.bj - 1) - 1;  // first tile node row = first element row (a halo)
  const int kb = bkI * (sh.bk - 1) - 1;
  const int je = jb + tj, ke = kb + tk;
  const int i0 = blockIdx.y * sh.cx;
  const int i1 = min(i0 + sh.cx, g.nx + 1);
  const bool colv = je >= 0 && je < g.ny && ke >= 0 && ke < g.nz;
  const bool own = tj >= 1 && tk >= 1 && je <= g.ny && ke <= g.nz;
  const int64_t NZ1 = g.nz + 1;
  const int64_t plane_vals = 3 * (int64_t)(g.ny + 1) * NZ1;

  int rel[kTileLoads];
  bool okq[kTileLoads];
#pragma unroll
  for (int q = 0; q < kTileLoads; ++q) {
    const int v = t + q * NT;
    const int row = v / W, col = v - row * W;
    const int j = jb + row, k = kb + col / 3;
    okq[q] = v < PV && j >= 0 && j <= g.ny && k >= 0 && k <= g.nz;
    rel[q] = okq[q] ? (int)(3 * ((int64_t)j * NZ1 + kb) + col) : 0;
  }
  // node plane p (zeros outside the mesh) into tile buffer p mod kPlaneBufs,
  // asynchronously; every call commits one copy group
  auto issue_plane = [&](int p) {
    const bool pv = p >= 0 && p <= g.nx;
    const int64_t base = pv ? (int64_t)p * plane_vals : 0;
    T* dst = P + (p & (kPlaneBufs - 1)) * PV;
#pragma unroll
    for (int q = 0; q < kTileLoads; ++q) {
      const int v = t + q * NT;
      if (q * NT < PV && v < PV) {
        const bool ok = pv && okq[q];
        cp_async_elem(dst + v, ok ? u + base + rel[q] : u, ok);
      }
    }
    cp_async_commit();
  };
  auto read_face = [&](int buf, T (&uu)[4][3]) {
    const T* src = P + buf * PV;
#pragma unroll
    for (int q2 = 0; q2 < 4; ++q2) {
      const int idx = (tj + (q2 >> 1)) * W + (tk + (q2 & 1)) * 3;
#pragma unroll
      for (int c = 0; c < 3; ++c) uu[q2][c] = src[idx + c];
    }
  };
  auto e_index = [&](int ie) { return ((int64_t)ie * g.ny + je) * g.nz + ke; };

  // prologue: planes i0-1 and i0 in the tile buffers, plane i0+1 in flight
  issue_plane(i0 - 1);
  issue_plane(i0);
  if (i0 + 1 <= i1) issue_plane(i0 + 1);
  else cp_async_commit();
  cp_async_wait_all_but_one();
  T Enext = (colv && i0 - 1 >= 0 && i0 - 1 < g.nx) ? E[e_index(i0 - 1)] : T(0);
  T carry[4][3];
#pragma unroll
  for (int q2 = 0; q2 < 4; ++q2)
#pragma unroll
    for (int c = 0; c < 3; ++c) carry[q2][c] = T(0);
  __syncthreads();

  // Element plane ie couples node planes ie and ie + 1, both read from the
  // rotating tile buffers (plane q in buffer q mod 4).  One barrier per plane:
  // the copy of plane ie + 3 is issued at the top (its buffer held plane ie - 1,
  // last read before the previous barrier), and before the barrier every thread
  // waits for its copies of plane ie + 2, so after it the next iteration's two
  // planes are complete and visible; the face sums alternate between two buffers.
  for (int ie = i0 - 1; ie < i1; ++ie) {
    if (ie + 3 <= i1) issue_plane(ie + 3);
    else cp_async_commit();
    const T Ee = Enext;
    Enext = (colv && ie + 1 < g.nx) ? E[e_index(ie + 1)] : T(0);
    const bool do_epi = own && ie >= i0;
    int64_t node = 0;
    if (do_epi) node = ((int64_t)ie * (g.ny + 1) + je) * NZ1 + ke;
    EpiOperands<T, EPI> eo;
    if (do_epi) eo.load(ea, 3 * node, mask);
    const int blo = ie & (kPlaneBufs - 1), bhi = (ie + 1) & (kPlaneBufs - 1);
    // the node's own value, read before the barrier: after it the next
    // iteration may overwrite this plane's buffer
    T xv[3];
    if (do_epi) {
      const T* xs = P + blo * PV + tj * W + tk * 3;
#pragma unroll
      for (int c = 0; c < 3; ++c) xv[c] = xs[c];
    }
    T f[8][3];
    if (colv && ie >= 0 && ie < g.nx) {
      T ue[8][3];
      read_face(blo, reinterpret_cast<T(&)[4][3]>(ue[0]));
      read_face(bhi, reinterpret_cast<T(&)[4][3]>(ue[4]));
      if (KMODE == 0) {
        elem_wht<T>(ue, Ee, f);
      } else {
        elem_bf16(reinterpret_cast<const float(&)[8][3]>(ue), (float)Ee, reinterpret_cast<float(&)[8][3]>(f));
      }
    } else {
#pragma unroll
      for (int q = 0; q < 8; ++q)
#pragma unroll
        for (int c = 0; c < 3; ++c) f[q][c] = T(0);
    }
    T* buf = F + (ie & 1) * 12 * NT;
    if (ie >= i0) {
#pragma unroll
      for (int q2 = 0; q2 < 4; ++q2)
#pragma unroll
        for (int c = 0; c < 3; ++c) buf[(q2 * 3 + c) * NT + t] = carry[q2][c] + f[q2][c];
    }
    cp_async_wait_all_but_one();
    __syncthreads();
    if (do_epi) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const T ku = ((buf[(0 * 3 + c) * NT + t] + buf[(2 * 3 + c) * NT + t - sh.bk]) +
                      buf[(1 * 3 + c) * NT + t - 1]) +
                     buf[(3 * 3 + c) * NT + t - sh.bk - 1];
        eo.apply(ea, 3 * node + c, c, ku, xv[c]);
      }
    }
#pragma unroll
    for (int q2 = 0; q2 < 4; ++q2)
#pragma unroll
      for (int c = 0; c < 3; ++c) carry[q2][c] = f[4 + q2][c];
  }
}

template <typename T>
static size_t sweep_smem(const SweepShape& sh) {
  const size_t NT = (size_t)sh.bj * sh.bk;
  const size_t PV = (size_t)(sh.bj + 1) * 3 * (sh.bk + 1);
  return (24 * NT + kPlaneBufs * PV) * sizeof(T);
}

template <typename T, int EPI, int KMODE, int MAXT>
static cudaError_t launch_sweep(const Grid& g, const SweepShape& sh, const T* E, const uint8_t* mask,
                                const T* u, const EpiArgs& ea, cudaStream_t s) {
  const int NT = sh.bj * sh.bk;
  if (NT > MAXT || sh.bj < 2 || sh.bk < 2 || sh.cx < 1) return cudaErrorInvalidConfiguration;
  if ((int64_t)(sh.bj + 1) * 3 * (sh.bk + 1) > (int64_t)kTileLoads * NT) return cudaErrorInvalidConfiguration;
  const size_t smem = sweep_smem<T>(sh);
  static std::atomic<uint64_t> attr_done;
  const cudaError_t ea0 = once_per_device(attr_done, [] {
    return cudaFuncSetAttribute(fine_sweep_kernel<T, EPI, KMODE, MAXT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                200 * 1024);
  });
  if (ea0 != cudaSuccess) return ea0;
  const int nbj = (g.ny + sh.bj - 1) / (sh.bj - 1);
  const int nbk = (g.nz + sh.bk - 1) / (sh.bk - 1);
  dim3 grid(nbj * nbk, div_up(g.nx + 1, sh.cx));
  fine_sweep_kernel<T, EPI, KMODE, MAXT><<<grid, NT, smem, s>>>(g, sh, E, mask, u, ea);
  return sf_launched(1);
}

// ----------------------------------------------------------------------------
// FP32 sweep with two elements per thread.  Thread (tj, tp) evaluates the
// k-adjacent element columns tk = 2tp and 2tp + 1 of the block's tile with the
// packed FP32 pair instructions of sm_100 (lane x: element 2tp, lane y: element
// 2tp + 1), which halves the arithmetic instruction count; it owns the nodes at
// those two positions.  The node tile is stored component-major in shared
// memory ([c][row][k], rows padded to an even length) so the dk = 0 corner pair
// of both elements is one aligned 64-bit load.  Elements outside the mesh get
// E = 0 (their corner values are zero-filled, so they contribute exactly 0)
// instead of a branch.  Same staging, barrier and summation order as
// fine_sweep_kernel; 32-bit indexing (the launcher checks ndof < 2^31).
__device__ __forceinline__ float2 f2sub(float2 a, float2 b) {
  return __ffma2_rn(b, make_float2(-1.f, -1.f), a);  // a - b, one rounding
}

__device__ __forceinline__ void wht8x2(float2 (&a)[8]) {
#pragma unroll
  for (int m = 4; m >= 1; m >>= 1) {
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      if ((q & m) == 0) {
        const float2 p = a[q], r = a[q | m];
        a[q] = __fadd2_rn(p, r);
        a[q | m] = f2sub(p, r);
      }
    }
  }
}

__device__ __forceinline__ void elem_wht_x2(const float2 (&u)[8][3], float2 E, float2 (&f)[8][3]) {
  float2 w[3][8];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
#pragma unroll
    for (int q = 0; q < 8; ++q) w[c][q] = u[q][c];
    wht8x2(w[c]);
  }
  float2 v[3][8];
#pragma unroll
  for (int b = 0; b < 8; ++b) {
    const float2 in0 = w[0][b ^ 4], in1 = w[1][b ^ 2], in2 = w[2][b ^ 1];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      float2 s = __fmul2_rn(c_wht32x2[b][3 * r], in0);
      s = __ffma2_rn(c_wht32x2[b][3 * r + 1], in1, s);
      s = __ffma2_rn(c_wht32x2[b][3 * r + 2], in2, s);
      v[r][b ^ (4 >> r)] = __fmul2_rn(E, s);
    }
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    wht8x2(v[c]);
#pragma unroll
    for (int q = 0; q < 8; ++q) f[q][c] = v[c][q];
  }
}

constexpr int kX2Threads = 256;
constexpr int kX2NodeLoads = 3;  // tile nodes per thread; launch checks

template <int EPI, int MINB>
__global__ void __launch_bounds__(kX2Threads, MINB) fine_sweep_x2_kernel(Grid g, SweepShape sh,
                                                                   const float* __restrict__ E,
                                                                   const uint8_t* __restrict__ mask,
                                                                   const float* __restrict__ u, EpiArgs ea) {
  if (guard_off(ea.guard)) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int HK = sh.bk >> 1, NT = sh.bj * HK, NE = sh.bj * sh.bk;
  const int NK1 = sh.bk + 1, NKP = sh.bk + 2;
  const int RP = (sh.bj + 1) * NKP;  // one component of one plane tile
  const int PV = 3 * RP;
  const int NN = (sh.bj + 1) * NK1;  // tile nodes
  float* F = reinterpret_cast<float*>(smem_raw);  // face sums [3][12][NE], plane q in q mod 3
  float* P = F + 36 * NE;                         // plane tiles [3][3][bj+1][NKP]
  const int t = threadIdx.x;
  const int tj = t / HK, tp = t - tj * HK, tk0 = 2 * tp;
  const int nbk = (g.nz + sh.bk - 1) / (sh.bk - 1);
  const int bjI = blockIdx.x / nbk, bkI = blockIdx.x - bjI * nbk;
  const int jb = bjI * (sh.bj - 1) - 1, kb = bkI * (sh.bk - 1) - 1;
  const int je = jb + tj, ke0 = kb + tk0, ke1 = ke0 + 1;
  const int i0 = blockIdx.y * sh.cx;
  const int i1 = min(i0 + sh.cx, g.nx + 1);
  const bool rowv = je >= 0 && je < g.ny;
  const bool colv0 = rowv && ke0 >= 0 && ke0 < g.nz, colv1 = rowv && ke1 >= 0 && ke1 < g.nz;
  const bool ownr = tj >= 1 && je <= g.ny;
  const bool own0 = ownr && tk0 >= 1 && ke0 <= g.nz, own1 = ownr && ke1 <= g.nz;
  const int NZ1 = g.nz + 1;
  const int64_t plane_vals = 3 * (int64_t)(g.ny + 1) * NZ1;

  int rel[kX2NodeLoads], sidx[kX2NodeLoads];
  bool okn[kX2NodeLoads];
#pragma unroll
  for (int s = 0; s < kX2NodeLoads; ++s) {
    const int n = t + s * NT;
    const int row = n / NK1, kk = n - row * NK1;
    const int j = jb + row, k = kb + kk;
    okn[s] = n < NN && j >= 0 && j <= g.ny && k >= 0 && k <= g.nz;
    rel[s] = okn[s] ? 3 * (j * NZ1 + k) : 0;
    sidx[s] = n < NN ? row * NKP + kk : -1;
  }
  // (the packed sweep stages its planes through registers: with cp.async it
  // needed 214 registers for the Jacobi epilogue and ran slower)
  auto load_plane = [&](int p, float (&r)[3 * kX2NodeLoads]) {
    const bool pv = p >= 0 && p <= g.nx;
    const float* base = u + (pv ? (int64_t)p * plane_vals : 0);
#pragma unroll
    for (int s = 0; s < kX2NodeLoads; ++s)
#pragma unroll
      for (int c = 0; c < 3; ++c) r[3 * s + c] = (pv && okn[s]) ? base[rel[s] + c] : 0.f;
  };
  auto store_plane = [&](int buf, const float (&r)[3 * kX2NodeLoads]) {
    float* dst = P + buf * PV;
#pragma unroll
    for (int s = 0; s < kX2NodeLoads; ++s)
      if (sidx[s] >= 0) {
#pragma unroll
        for (int c = 0; c < 3; ++c) dst[c * RP + sidx[s]] = r[3 * s + c];
      }
  };
  auto read_face2 = [&](int buf, float2 (&uu)[8][3], int q0) {
    const float* src = P + buf * PV;
#pragma unroll
    for (int q2 = 0; q2 < 4; ++q2) {
      const int base = (tj + (q2 >> 1)) * NKP + tk0 + (q2 & 1);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float* a = src + c * RP + base;
        uu[q0 + q2][c] = (q2 & 1) ? make_float2(a[0], a[1]) : *reinterpret_cast<const float2*>(a);
      }
    }
  };
  auto e_pair = [&](int ie) {
    const bool pv = ie >= 0 && ie < g.nx;
    const int idx = (ie * g.ny + je) * g.nz + ke0;
    return make_float2((pv && colv0) ? E[idx] : 0.f, (pv && colv1) ? E[idx + 1] : 0.f);
  };

  float pre[3 * kX2NodeLoads];
  load_plane(i0 - 1, pre);
  store_plane((i0 + 2) % 3, pre);
  load_plane(i0, pre);
  store_plane(i0 % 3, pre);
  if (i0 + 1 <= i1) load_plane(i0 + 1, pre);
  float2 En = e_pair(i0 - 1);
  __syncthreads();

  const int e0 = tj * sh.bk + tk0;
  const int em1 = tp == 0 ? e0 : e0 - 1;  // node 2tp is a halo when tp == 0
  for (int ie = i0 - 1; ie < i1; ++ie) {
    if (ie + 2 <= i1) store_plane((ie + 2) % 3, pre);
    if (ie + 3 <= i1) load_plane(ie + 3, pre);
    const float2 Ee = En;
    En = e_pair(ie + 1);
    const bool epi0 = own0 && ie >= i0, epi1 = own1 && ie >= i0;
    const int node0 = (ie * (g.ny + 1) + je) * NZ1 + ke0;
    const int blo = (ie + 3) % 3, bhi = (ie + 1) % 3;
    float2 f[8][3];
    {
      float2 ue[8][3];
      read_face2(blo, ue, 0);
      read_face2(bhi, ue, 4);
      elem_wht_x2(ue, Ee, f);
    }
    // epilogue operands after the element arithmetic (not live across its
    // register peak); the face-sum stores and the barrier cover their latency
    EpiOperands<float, EPI> eo0, eo1;
    if (epi0) eo0.load(ea, 3 * (int64_t)node0, mask);
    if (epi1) eo1.load(ea, 3 * (int64_t)node0 + 3, mask);
    float2 xv[3];
    if (epi0 || epi1) {
      const float* xs = P + blo * PV + tj * NKP + tk0;
#pragma unroll
      for (int c = 0; c < 3; ++c) xv[c] = *reinterpret_cast<const float2*>(xs + c * RP);
    }
    // face sums of node plane ie: this element plane's -x face added to the
    // +x face of element plane ie - 1, which this thread parked in the same
    // slots one iteration earlier; the +x face goes to plane ie + 1's buffer
    // (last read before the previous barrier)
    float* Fb = F + ((ie + 3) % 3) * 12 * NE;
    float* Fn = F + ((ie + 1) % 3) * 12 * NE;
#pragma unroll
    for (int q2 = 0; q2 < 4; ++q2)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        float2* slot = reinterpret_cast<float2*>(Fb + (q2 * 3 + c) * NE + e0);
        if (ie >= i0) *slot = __fadd2_rn(*slot, f[q2][c]);
        *reinterpret_cast<float2*>(Fn + (q2 * 3 + c) * NE + e0) = f[4 + q2][c];
      }
    __syncthreads();
    if (epi0 || epi1) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float2 a = *reinterpret_cast<const float2*>(Fb + (0 * 3 + c) * NE + e0);
        const float2 b = *reinterpret_cast<const float2*>(Fb + (2 * 3 + c) * NE + e0 - sh.bk);
        const float* p1 = Fb + (1 * 3 + c) * NE;
        const float* p3 = Fb + (3 * 3 + c) * NE - sh.bk;
        const float2 x1 = make_float2(p1[em1], p1[e0]);
        const float2 x3 = make_float2(p3[em1], p3[e0]);
        const float2 ku = __fadd2_rn(__fadd2_rn(__fadd2_rn(a, b), x1), x3);
        if (epi0) eo0.apply(ea, 3 * (int64_t)node0 + c, c, ku.x, xv[c].x);
        if (epi1) eo1.apply(ea, 3 * (int64_t)node0 + 3 + c, c, ku.y, xv[c].y);
      }
    }
  }
}

static bool x2_shape_ok(const Grid& g, const SweepShape& sh) {
  const int NT = sh.bj * sh.bk / 2;
  return sh.bk % 2 == 0 && sh.bk >= 4 && sh.bj >= 3 && sh.cx >= 1 && NT <= kX2Threads &&
         (sh.bj + 1) * (sh.bk + 1) <= kX2NodeLoads * NT && g.ndof < (int64_t(1) << 31);
}

template <int EPI>
static cudaError_t launch_sweep_f32(const Grid& g, const SweepShape& sh, const float* E, const uint8_t* mask,
                                    const float* u, const EpiArgs& ea, cudaStream_t s) {
  if (sh.variant == 1 || !x2_shape_ok(g, sh)) return launch_sweep<float, EPI, 0, 512>(g, sh, E, mask, u, ea, s);
  const int NT = sh.bj * sh.bk / 2, NE = sh.bj * sh.bk;
  const size_t smem = sizeof(float) * (36 * (size_t)NE + 9 * (size_t)(sh.bj + 1) * (sh.bk + 2));
  static std::atomic<uint64_t> attr_done[2];
  const int capped = sh.variant == 2 ? 1 : 0;
  const cudaError_t ea0 = once_per_device(attr_done[capped], [&] {
    return capped ? cudaFuncSetAttribute(fine_sweep_x2_kernel<EPI, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         200 * 1024)
                  : cudaFuncSetAttribute(fine_sweep_x2_kernel<EPI, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         200 * 1024);
  });
  if (ea0 != cudaSuccess) return ea0;
  const int nbj = (g.ny + sh.bj - 1) / (sh.bj - 1);
  const int nbk = (g.nz + sh.bk - 1) / (sh.bk - 1);
  dim3 grid(nbj * nbk, div_up(g.nx + 1, sh.cx));
  if (capped)
    fine_sweep_x2_kernel<EPI, 2><<<grid, NT, smem, s>>>(g, sh, E, mask, u, ea);
  else
    fine_sweep_x2_kernel<EPI, 1><<<grid, NT, smem, s>>>(g, sh, E, mask, u, ea);
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
      case EPI_APPLY:
        return launch_sweep_f32<EPI_APPLY>(g, sh, (const float*)E, mask, (const float*)u, ea, s);
      case EPI_RESID:
        return launch_sweep_f32<EPI_RESID>(g, sh, (const float*)E, mask, (const float*)u, ea, s);
      case EPI_CHEB1:
        return launch_sweep_f32<EPI_CHEB1>(g, sh, (const float*)E, mask, (const float*)u, ea, s);
      case EPI_CHEB:
        return launch_sweep_f32<EPI_CHEB>(g, sh, (const float*)E, mask, (const float*)u, ea, s);
      case EPI_JAC:
        return launch_sweep_f32<EPI_JAC>(g, sh, (const float*)E, mask, (const float*)u, ea, s);
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
