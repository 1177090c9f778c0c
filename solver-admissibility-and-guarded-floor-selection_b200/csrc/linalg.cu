// Vector, reduction, dense and Krylov kernels of the simpfem library.
//
// Reductions are deterministic: a fixed grid writes one partial per block and
// the last block to finish (ticket counter) sums the partials in block order,
// so every dot product is bitwise reproducible run to run.
#include <math.h>

#include "common.cuh"

namespace simpfem {

constexpr int kRedBlocks = 296;  // 2 x 148 SMs
constexpr int kRedThreads = 256;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum of up to 4 values (result valid in thread 0).
template <int ND>
__device__ __forceinline__ void block_sum(double (&v)[ND], double* sh /*32*ND*/) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < ND; ++k) {
    const double w = warp_sum(v[k]);
    if (lane == 0) sh[k * 32 + wid] = w;
  }
  __syncthreads();
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < ND; ++k) {
      double w = lane < nw ? sh[k * 32 + lane] : 0.0;
      v[k] = warp_sum(w);
    }
  }
}

// Finalisation by the last block to finish: out[k] = sum of the partials in
// block order (bitwise reproducible).  The block first stages every partial
// in shared memory with one parallel round of loads, so the ordered sum runs
// over shared memory instead of a serial chain of global loads.
template <int ND>
__device__ __forceinline__ bool last_block_finalize(const double (&v)[ND], RedWork w, double* out) {
  __shared__ bool is_last;
  __shared__ double stage[4 * kRedBlocks];
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < ND; ++k) w.partials[k * kRedBlocks + blockIdx.x] = v[k];
    __threadfence();
    const unsigned t = atomicAdd(w.ticket, 1u);
    is_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!is_last) return false;
  __threadfence();
  const int nb = (int)gridDim.x;
  for (int e = threadIdx.x; e < ND * nb; e += blockDim.x) {
    const int k = e / nb, b = e - k * nb;
    stage[k * kRedBlocks + b] = ((volatile double*)w.partials)[k * kRedBlocks + b];
  }
  __syncthreads();
  if (threadIdx.x < ND) {
    const int k = threadIdx.x;
    double s = 0.0;
    for (int b = 0; b < nb; ++b) s += stage[k * kRedBlocks + b];
    out[k] = s;
  }
  if (threadIdx.x == 0) *w.ticket = 0u;
  return true;
}

template <typename T>
__device__ __forceinline__ double dot_term(const DotSet& ds, int k, int64_t i) {
  const T a = ((const T*)ds.a[k])[i];
  const T b = ((const T*)ds.b[k])[i];
  if (ds.mode[k] == 0) return (double)a * (double)b;
  const T c = ((const T*)ds.c[k])[i];
  if (ds.mode[k] == 1) return (double)mul_rn(a, c) * (double)b;  // (a * c) * b
  if (ds.mode[k] == 3) return (double)mul_rn(a, c) * (double)mul_rn(b, c);  // (a * c) * (b * c)
  // mode 2: a * (b / c) on entries with c != 0
  return c != T(0) ? (double)a * (double)(b / c) : 0.0;
}

template <typename T, int ND>
__global__ void __launch_bounds__(kRedThreads) dots_kernel(int64_t n, DotSet ds, RedWork w, double* out,
                                                           const int* guard) {
  if (guard_off(guard)) return;
  __shared__ double sh[32 * 4];
  double v[ND];
#pragma unroll
  for (int k = 0; k < ND; ++k) v[k] = 0.0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  // four strided elements per pass: their loads are independent and in flight
  // together (one load per vector per thread left the kernel latency-bound)
  for (; i + 3 * stride < n; i += 4 * stride) {
#pragma unroll
    for (int k = 0; k < ND; ++k) {
      const double t0 = dot_term<T>(ds, k, i), t1 = dot_term<T>(ds, k, i + stride);
      const double t2 = dot_term<T>(ds, k, i + 2 * stride), t3 = dot_term<T>(ds, k, i + 3 * stride);
      v[k] += t0;
      v[k] += t1;
      v[k] += t2;
      v[k] += t3;
    }
  }
  for (; i < n; i += stride) {
#pragma unroll
    for (int k = 0; k < ND; ++k) v[k] += dot_term<T>(ds, k, i);
  }
  block_sum<ND>(v, sh);
  last_block_finalize<ND>(v, w, out);
}

static int red_blocks(int64_t n) {
  const int64_t b = (n + kRedThreads - 1) / kRedThreads;
  return (int)(b < kRedBlocks ? (b < 1 ? 1 : b) : kRedBlocks);
}

cudaError_t launch_dots(DType t, int64_t n, const DotSet& ds, RedWork w, double* out,
                        const int* guard, cudaStream_t s) {
  const int nb = red_blocks(n);
#define SF_DOTS(T)                                                                                 \
  switch (ds.nd) {                                                                                 \
    case 1: dots_kernel<T, 1><<<nb, kRedThreads, 0, s>>>(n, ds, w, out, guard); break;            \
    case 2: dots_kernel<T, 2><<<nb, kRedThreads, 0, s>>>(n, ds, w, out, guard); break;            \
    case 3: dots_kernel<T, 3><<<nb, kRedThreads, 0, s>>>(n, ds, w, out, guard); break;            \
    case 4: dots_kernel<T, 4><<<nb, kRedThreads, 0, s>>>(n, ds, w, out, guard); break;            \
    default: return cudaErrorInvalidValue;                                                         \
  }
  if (t == F64) {
    SF_DOTS(double)
  } else if (t == F32) {
    SF_DOTS(float)
  } else {
    return cudaErrorInvalidValue;
  }
#undef SF_DOTS
  return sf_launched(1);
}

// min, max and count(E > thr) of a double array (contrast classification,
// gpu_fem/multigrid_v4.py:1204-1239).
__global__ void __launch_bounds__(kRedThreads) minmax_kernel(int64_t n, const double* __restrict__ E,
                                                             double thr, RedWork w, double* out) {
  __shared__ double sh[32 * 3];
  double v[3] = {INFINITY, -INFINITY, 0.0};
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const double e = E[i];
    v[0] = fmin(v[0], e);
    v[1] = fmax(v[1], e);
    v[2] += (e > thr) ? 1.0 : 0.0;
  }
  // min/max reduce via shuffles
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v[0] = fmin(v[0], __shfl_down_sync(0xffffffffu, v[0], o));
    v[1] = fmax(v[1], __shfl_down_sync(0xffffffffu, v[1], o));
    v[2] += __shfl_down_sync(0xffffffffu, v[2], o);
  }
  if (lane == 0) {
    sh[wid] = v[0];
    sh[32 + wid] = v[1];
    sh[64 + wid] = v[2];
  }
  __syncthreads();
  __shared__ bool is_last;
  if (threadIdx.x == 0) {
    const int nw = blockDim.x >> 5;
    double a = INFINITY, b = -INFINITY, c = 0.0;
    for (int k = 0; k < nw; ++k) {
      a = fmin(a, sh[k]);
      b = fmax(b, sh[32 + k]);
      c += sh[64 + k];
    }
    w.partials[blockIdx.x] = a;
    w.partials[kRedBlocks + blockIdx.x] = b;
    w.partials[2 * kRedBlocks + blockIdx.x] = c;
    __threadfence();
    is_last = atomicAdd(w.ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (is_last && threadIdx.x == 0) {
    __threadfence();
    double a = INFINITY, b = -INFINITY, c = 0.0;
    volatile double* p = w.partials;
    for (int k = 0; k < (int)gridDim.x; ++k) {
      a = fmin(a, p[k]);
      b = fmax(b, p[kRedBlocks + k]);
      c += p[2 * kRedBlocks + k];
    }
    out[0] = a;
    out[1] = b;
    out[2] = c;
    *w.ticket = 0u;
  }
}

cudaError_t launch_minmax_count(int64_t n, const double* E, double thr, RedWork w, double* out3,
                                cudaStream_t s) {
  minmax_kernel<<<red_blocks(n), kRedThreads, 0, s>>>(n, E, thr, w, out3);
  return sf_launched(1);
}

// ----------------------------------------------------------------------------
// Elementwise kernels.
template <typename T>
__global__ void axpby_kernel(int64_t n, T alpha, const T* __restrict__ x, T beta, const T* __restrict__ y,
                             T* __restrict__ out, const int* guard) {
  if (guard_off(guard)) return;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  // out = alpha * x + beta * y, each product rounded (numpy semantics); a null
  // y means out = alpha * x, alpha == 1 skips the product.
  T a = alpha == T(1) ? x[i] : mul_rn(alpha, x[i]);
  if (y == nullptr) {
    out[i] = a;
    return;
  }
  T b = beta == T(1) ? y[i] : (beta == T(-1) ? -y[i] : mul_rn(beta, y[i]));
  out[i] = add_rn(a, b);
}

cudaError_t launch_axpby(DType t, int64_t n, double alpha, const void* x, double beta,
                         const void* y, void* out, const int* guard, cudaStream_t s) {
  const int nb = div_up(n, 256);
  if (t == F64)
    axpby_kernel<double><<<nb, 256, 0, s>>>(n, alpha, (const double*)x, beta, (const double*)y,
                                            (double*)out, guard);
  else
    axpby_kernel<float><<<nb, 256, 0, s>>>(n, (float)alpha, (const float*)x, (float)beta,
                                           (const float*)y, (float*)out, guard);
  return sf_launched(1);
}

template <typename T>
__global__ void fill_kernel(int64_t n, T v, T* __restrict__ out, const int* guard) {
  if (guard_off(guard)) return;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = v;
}

// out[i] = a pseudo-random value in [-0.5, 0.5) from a hash of (i, seed): test
// data for timing kernels on realistic (non-constant) vectors.
template <typename T>
__global__ void fill_hash_kernel(int64_t n, uint32_t seed, T* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t h = (uint32_t)i * 2654435761u ^ (uint32_t)(i >> 32) ^ seed;
  h ^= h >> 15;
  h *= 0x2c1b3c6du;
  h ^= h >> 12;
  out[i] = (T)((double)(h & 0xffffffu) * (1.0 / 16777216.0) - 0.5);
}

cudaError_t launch_fill_hash(DType t, int64_t n, uint32_t seed, void* out, cudaStream_t s) {
  const int nb = div_up(n, 256);
  if (t == F64)
    fill_hash_kernel<double><<<nb, 256, 0, s>>>(n, seed, (double*)out);
  else
    fill_hash_kernel<float><<<nb, 256, 0, s>>>(n, seed, (float*)out);
  return sf_launched(1);
}

cudaError_t launch_fill(DType t, int64_t n, double v, void* out, const int* guard, cudaStream_t s) {
  const int nb = div_up(n, 256);
  if (t == F64)
    fill_kernel<double><<<nb, 256, 0, s>>>(n, v, (double*)out, guard);
  else
    fill_kernel<float><<<nb, 256, 0, s>>>(n, (float)v, (float*)out, guard);
  return sf_launched(1);
}

cudaError_t launch_copy(DType t, int64_t n, const void* src, void* dst, const int* guard,
                        cudaStream_t s) {
  return launch_axpby(t, n, 1.0, src, 0.0, nullptr, dst, guard, s);
}

// First Chebyshev step from x0 = 0 (gpu_fem/multigrid_v4.py:1783-1812 with
// A(0) = 0): d = dinv * rhs; x = alpha * d.
template <typename T>
__global__ void cheb_zero_kernel(int64_t n, T alpha, const T* __restrict__ dinv, const T* __restrict__ rhs,
                                 T* __restrict__ d, T* __restrict__ x, const int* guard) {
  if (guard_off(guard)) return;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const T z = mul_rn(dinv[i], rhs[i]);
  d[i] = z;
  x[i] = mul_rn(alpha, z);
}

cudaError_t launch_cheb_zero(DType t, int64_t n, double alpha, const void* dinv, const void* rhs,
                             void* d, void* x, const int* guard, cudaStream_t s) {
  const int nb = div_up(n, 256);
  if (t == F64)
    cheb_zero_kernel<double><<<nb, 256, 0, s>>>(n, alpha, (const double*)dinv, (const double*)rhs,
                                                (double*)d, (double*)x, guard);
  else
    cheb_zero_kernel<float><<<nb, 256, 0, s>>>(n, (float)alpha, (const float*)dinv,
                                               (const float*)rhs, (float*)d, (float*)x, guard);
  return sf_launched(1);
}

// First damped-Jacobi step from x0 = 0: x = (omega * dinv) * rhs.
template <typename T>
__global__ void jac_zero_kernel(int64_t n, T omega, const T* __restrict__ dinv, const T* __restrict__ rhs,
                                T* __restrict__ x, const int* guard) {
  if (guard_off(guard)) return;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  x[i] = mul_rn(mul_rn(omega, dinv[i]), rhs[i]);
}

cudaError_t launch_jac_zero(DType t, int64_t n, double omega, const void* dinv, const void* rhs,
                            void* x, const int* guard, cudaStream_t s) {
  const int nb = div_up(n, 256);
  if (t == F64)
    jac_zero_kernel<double><<<nb, 256, 0, s>>>(n, omega, (const double*)dinv, (const double*)rhs,
                                               (double*)x, guard);
  else
    jac_zero_kernel<float><<<nb, 256, 0, s>>>(n, (float)omega, (const float*)dinv,
                                              (const float*)rhs, (float*)x, guard);
  return sf_launched(1);
}

template <typename T>
__global__ void expand_kernel(int64_t nf, const int32_t* __restrict__ idx, const T* __restrict__ src,
                              T* __restrict__ dst) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nf) dst[idx[i]] = src[i];
}
template <typename T>
__global__ void compress_kernel(int64_t nf, const int32_t* __restrict__ idx, const T* __restrict__ src,
                                T* __restrict__ dst) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nf) dst[i] = src[idx[i]];
}

cudaError_t launch_expand(DType t, int64_t n_free, const int32_t* free_idx, const void* src_free,
                          void* dst_full, cudaStream_t s) {
  const int nb = div_up(n_free, 256);
  if (t == F64)
    expand_kernel<double><<<nb, 256, 0, s>>>(n_free, free_idx, (const double*)src_free, (double*)dst_full);
  else
    expand_kernel<float><<<nb, 256, 0, s>>>(n_free, free_idx, (const float*)src_free, (float*)dst_full);
  return sf_launched(1);
}

cudaError_t launch_compress(DType t, int64_t n_free, const int32_t* free_idx,
                            const void* src_full, void* dst_free, cudaStream_t s) {
  const int nb = div_up(n_free, 256);
  if (t == F64)
    compress_kernel<double><<<nb, 256, 0, s>>>(n_free, free_idx, (const double*)src_full, (double*)dst_free);
  else
    compress_kernel<float><<<nb, 256, 0, s>>>(n_free, free_idx, (const float*)src_full, (float*)dst_free);
  return sf_launched(1);
}

__global__ void gather_idx_kernel(int64_t n, const int32_t* __restrict__ idx, const double* __restrict__ src,
                                  double* __restrict__ dst, const int* guard) {
  if (guard_off(guard)) return;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[idx[i]];
}
__global__ void scatter_idx_kernel(int64_t n, const int32_t* __restrict__ idx, const double* __restrict__ src,
                                   double* __restrict__ dst, const int* guard) {
  if (guard_off(guard)) return;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[idx[i]] = src[i];
}

cudaError_t launch_gather_idx(int64_t n, const int32_t* idx, const double* src, double* dst,
                              const int* guard, cudaStream_t s) {
  gather_idx_kernel<<<div_up(n, 256), 256, 0, s>>>(n, idx, src, dst, guard);
  return sf_launched(1);
}
cudaError_t launch_scatter_idx(int64_t n, const int32_t* idx, const double* src, double* dst,
                               const int* guard, cudaStream_t s) {
  scatter_idx_kernel<<<div_up(n, 256), 256, 0, s>>>(n, idx, src, dst, guard);
  return sf_launched(1);
}

// out = mask ? op(a) : 0 with
//   op 0: 1 / a          op 1: a * s          op 2: a / s (s_dev when given)
//   op 3: b * a          op 4: s (constant)   op 5: a
//   op 6: |a| > 1e-12 ? a : 1   (the reference's diagonal guard)
__global__ void vec_op_kernel(int64_t n, int op, const double* __restrict__ a, const double* __restrict__ b,
                              const uint8_t* __restrict__ mask, double s, const double* s_dev,
                              double* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const bool m = mask == nullptr || mask[i] != 0;
  double r = 0.0;
  if (m) {
    switch (op) {
      case 0: r = 1.0 / a[i]; break;
      case 1: r = a[i] * s; break;
      case 2: r = a[i] / (s_dev != nullptr ? *s_dev : s); break;
      case 3: r = b[i] * a[i]; break;
      case 4: r = s; break;
      case 5: r = a[i]; break;
      case 6: r = fabs(a[i]) > 1e-12 ? a[i] : 1.0; break;
      default: r = a[i];
    }
  }
  out[i] = r;
}

cudaError_t launch_vec_op(int64_t n, int op, const double* a, const double* b, const uint8_t* mask,
                          double s, const double* s_dev, double* out, cudaStream_t st) {
  vec_op_kernel<<<div_up(n, 256), 256, 0, st>>>(n, op, a, b, mask, s, s_dev, out);
  return sf_launched(1);
}

// Root-enrichment weights (gpu_fem/multigrid_v4.py:1150-1157):
// w = clip(|diag| / max|diag|, floor, 1) ** power on free DOFs.
__global__ void enrich_weight_kernel(int64_t n, const double* __restrict__ diag, const uint8_t* __restrict__ mask,
                                     const double* __restrict__ dmax, double wfloor, double wpow,
                                     double* __restrict__ w) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (!mask[i]) {
    w[i] = 0.0;
    return;
  }
  double v = fabs(diag[i]) / fmax(*dmax, 1e-300);
  v = fmin(fmax(v, wfloor), 1.0);
  if (fabs(wpow - 1.0) > 1e-12) v = pow(v, wpow);
  w[i] = v;
}

cudaError_t launch_enrich_weights(int64_t n, const double* diag, const uint8_t* mask,
                                  const double* dmax_dev, double wfloor, double wpow, double* w,
                                  cudaStream_t s) {
  enrich_weight_kernel<<<div_up(n, 256), 256, 0, s>>>(n, diag, mask, dmax_dev, wfloor, wpow, w);
  return sf_launched(1);
}

// out = mask ? (mode 0: w * r ; mode 1: clip(1 - w, floor, 1) * r ;
//               mode 2: w * (r - p) ; mode 3: clip(1 - w, floor, 1) * (r - p)) : 0
__global__ void enrich_rhs_kernel(int64_t n, int mode, const double* __restrict__ w, double wfloor,
                                  const double* __restrict__ r, const double* __restrict__ p,
                                  const uint8_t* __restrict__ mask, double* __restrict__ out,
                                  const int* guard) {
  if (guard_off(guard)) return;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (!mask[i]) {
    out[i] = 0.0;
    return;
  }
  double ww = w[i];
  if (mode == 1 || mode == 3) ww = fmin(fmax(1.0 - ww, wfloor), 1.0);
  const double rr = (mode >= 2) ? sub_rn(r[i], p[i]) : r[i];
  out[i] = mul_rn(ww, rr);
}

cudaError_t launch_enrich_rhs(int64_t n, int mode, const double* w, double wfloor, const double* r,
                              const double* p, const uint8_t* mask, double* out, const int* guard,
                              cudaStream_t s) {
  enrich_rhs_kernel<<<div_up(n, 256), 256, 0, s>>>(n, mode, w, wfloor, r, p, mask, out, guard);
  return sf_launched(1);
}

// y = M b over the triangle of a dense row-major M (lower: j <= i, upper: j >= i),
// one warp per row.
// y = L b (UPPER = 0: lower rows 0..row) or L^T b stored transposed (UPPER = 1),
// one warp per row, FP64 accumulation; the matrix may be stored in FP32 (the
// mixed cycle's copy).  Four strided loads per lane are in flight per pass.
template <int UPPER, typename MT>
__global__ void tri_matvec_kernel(const MT* __restrict__ M, int n, const double* __restrict__ b,
                                  double* __restrict__ y, const int* guard) {
  if (guard_off(guard)) return;
  const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= n) return;
  const MT* r = M + (int64_t)row * n;
  const int lo = UPPER ? row : 0, hi = UPPER ? n : row + 1;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
  int j = lo + lane;
  for (; j + 96 < hi; j += 128) {
    s0 += (double)r[j] * b[j];
    s1 += (double)r[j + 32] * b[j + 32];
    s2 += (double)r[j + 64] * b[j + 64];
    s3 += (double)r[j + 96] * b[j + 96];
  }
  for (; j < hi; j += 32) s0 += (double)r[j] * b[j];
  double s = (s0 + s1) + (s2 + s3);
  s = warp_sum(s);
  if (lane == 0) y[row] = s;
}

cudaError_t launch_coarsest_solve(const double* Linv, const double* LinvT, int n, const double* b, double* tmp,
                                  double* x, const int* guard, cudaStream_t s) {
  const int blocks = div_up((int64_t)n * 32, 256);
  tri_matvec_kernel<0, double><<<blocks, 256, 0, s>>>(Linv, n, b, tmp, guard);
  tri_matvec_kernel<1, double><<<blocks, 256, 0, s>>>(LinvT, n, tmp, x, guard);
  return sf_launched(2);
}

// The FP32 copy with 16-byte row starts (n % 4 == 0): one warp per row, the
// row read as float4 with eight of them per lane in flight, so the longest
// rows (n / 128 float4 per lane) take a few memory round trips instead of one
// per 128 entries.  The diagonal-aligned start of an upper row and the row's
// end are read as scalars.  FP64 accumulation in a fixed order per row.
__device__ __forceinline__ double dot4(float4 a, double2 b0, double2 b1) {
  return ((double)a.x * b0.x + (double)a.y * b0.y) + ((double)a.z * b1.x + (double)a.w * b1.y);
}

template <int UPPER>
__global__ void __launch_bounds__(256) tri_matvec_f32v_kernel(const float* __restrict__ M, int n,
                                                              const double* __restrict__ b,
                                                              double* __restrict__ y, const int* guard) {
  if (guard_off(guard)) return;
  const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= n) return;
  const float* r = M + (int64_t)row * n;
  const int lo = UPPER ? row : 0, hi = UPPER ? n : row + 1;
  const int lo4 = min(hi, (lo + 3) & ~3);  // first column of the float4 body
  const int nv = (hi - lo4) >> 2;          // float4 in the body
  const int t0 = lo4 + 4 * nv;             // first column of the scalar tail
  double acc[8];
#pragma unroll
  for (int u = 0; u < 8; ++u) acc[u] = 0.0;
  if (lane < lo4 - lo) acc[0] += (double)r[lo + lane] * b[lo + lane];
  if (lane < hi - t0) acc[1] += (double)r[t0 + lane] * b[t0 + lane];
  const float4* r4 = reinterpret_cast<const float4*>(r + lo4);
  const double2* b2 = reinterpret_cast<const double2*>(b + lo4);
  int v = lane;
  for (; v + 224 < nv; v += 256) {
    float4 a[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) a[u] = __ldg(r4 + v + 32 * u);
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int q = v + 32 * u;
      acc[u] += dot4(a[u], __ldg(b2 + 2 * q), __ldg(b2 + 2 * q + 1));
    }
  }
  for (; v < nv; v += 32) acc[2] += dot4(__ldg(r4 + v), __ldg(b2 + 2 * v), __ldg(b2 + 2 * v + 1));
  double s = ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
  s = warp_sum(s);
  if (lane == 0) y[row] = s;
}

cudaError_t launch_coarsest_solve_f32(const float* Linv, const float* LinvT, int n, const double* b, double* tmp,
                                      double* x, const int* guard, cudaStream_t s) {
  const int blocks = div_up((int64_t)n * 32, 256);
  const bool vec = n % 4 == 0 && ((uintptr_t)Linv & 15) == 0 && ((uintptr_t)LinvT & 15) == 0 &&
                   ((uintptr_t)b & 15) == 0 && ((uintptr_t)tmp & 15) == 0;
  if (vec) {
    tri_matvec_f32v_kernel<0><<<blocks, 256, 0, s>>>(Linv, n, b, tmp, guard);
    tri_matvec_f32v_kernel<1><<<blocks, 256, 0, s>>>(LinvT, n, tmp, x, guard);
  } else {
    tri_matvec_kernel<0, float><<<blocks, 256, 0, s>>>(Linv, n, b, tmp, guard);
    tri_matvec_kernel<1, float><<<blocks, 256, 0, s>>>(LinvT, n, tmp, x, guard);
  }
  return sf_launched(2);
}

__global__ void add_diag_kernel(double* A, int n, double eps) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) A[(int64_t)i * n + i] += eps;
}
cudaError_t launch_add_diag(double* A, int n, double eps, cudaStream_t s) {
  add_diag_kernel<<<div_up(n, 256), 256, 0, s>>>(A, n, eps);
  return sf_launched(1);
}

__global__ void diag_sum_kernel(const double* A, int n, double* out) {
  // single block
  __shared__ double sh[32];
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) v += A[(int64_t)i * n + i];
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += sh[k];
    *out = t;
  }
}
cudaError_t launch_diag_sum(const double* A, int n, double* out, cudaStream_t s) {
  diag_sum_kernel<<<1, 256, 0, s>>>(A, n, out);
  return sf_launched(1);
}

__global__ void all_finite_kernel(const double* A, int64_t n, int* flag) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && !isfinite(A[i])) *flag = 1;
}
cudaError_t launch_all_finite(const double* A, int64_t n, int* flag, cudaStream_t s) {
  all_finite_kernel<<<div_up(n, 256), 256, 0, s>>>(A, n, flag);
  return sf_launched(1);
}

// ----------------------------------------------------------------------------
// Krylov building blocks (_cupy_fgmres, gpu_fem/multigrid_v4.py:416-534), the
// Arnoldi state living on the device.

// h[0] = <v0, w>
cudaError_t launch_mgs_first(int64_t n, const double* v0, const double* w, RedWork rw, double* h0,
                             const int* guard, cudaStream_t s) {
  DotSet ds;
  ds.a[0] = v0;
  ds.b[0] = w;
  ds.nd = 1;
  return launch_dots(F64, n, ds, rw, h0, guard, s);
}

// w <- w - h_i * v_i ; out <- <v_next, w_new> (or <w_new, w_new> when v_next is null)
__global__ void __launch_bounds__(kRedThreads) mgs_step_kernel(int64_t n, const double* __restrict__ vi,
                                                               const double* __restrict__ vnext,
                                                               double* __restrict__ w,
                                                               const double* __restrict__ hi, RedWork rw,
                                                               double* out, const int* guard) {
  if (guard_off(guard)) return;
  __shared__ double sh[32];
  const double h = *hi;
  double v[1] = {0.0};
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  // four strided elements per pass (independent loads in flight together)
  for (; i + 3 * stride < n; i += 4 * stride) {
    double wv[4], vv[4], nv[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      wv[q] = w[i + q * stride];
      vv[q] = vi[i + q * stride];
      if (vnext != nullptr) nv[q] = vnext[i + q * stride];
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const double wn = sub_rn(wv[q], mul_rn(h, vv[q]));
      w[i + q * stride] = wn;
      v[0] += (vnext != nullptr ? nv[q] : wn) * wn;
    }
  }
  for (; i < n; i += stride) {
    const double wn = sub_rn(w[i], mul_rn(h, vi[i]));
    w[i] = wn;
    v[0] += (vnext != nullptr ? vnext[i] : wn) * wn;
  }
  block_sum<1>(v, sh);
  last_block_finalize<1>(v, rw, out);
}

cudaError_t launch_mgs_step(int64_t n, const double* vi, const double* vnext, double* w,
                            const double* hi, RedWork rw, double* out, const int* guard,
                            cudaStream_t s) {
  mgs_step_kernel<<<red_blocks(n), kRedThreads, 0, s>>>(n, vi, vnext, w, hi, rw, out, guard);
  return sf_launched(1);
}

// Krylov control (single thread).  Flags: see KrylovDev in internal.h.
__global__ void krylov_init_kernel(KrylovDev k, const int* parent) {
  int* f = k.flags;
  const bool pok = parent == nullptr || *parent != 0;
  const double bn = sqrt(k.sc[SC_BNORM2]);
  k.sc[SC_BNORM] = bn;
  for (int i = 0; i < NFLAGS; ++i) f[i] = 0;
  f[F_HISTN] = 0;
  if (!pok) {
    f[F_DONE] = 1;
  } else if (bn <= 1e-30) {
    f[F_DONE] = 1;
    f[F_CONV] = 1;
  }
  f[F_NOTDONE] = f[F_DONE] ? 0 : 1;
}

__global__ void krylov_restart_kernel(KrylovDev k, double tol, double* hist_host, int hist_cap) {
  int* f = k.flags;
  f[F_DID] = 0;
  f[F_CYC] = 0;
  if (f[F_DONE]) return;
  const double beta = sqrt(k.sc[SC_BETA2]);
  k.sc[SC_BETA] = beta;
  const double rel = beta / k.sc[SC_BNORM];
  if (hist_host != nullptr && f[F_HISTN] < hist_cap) hist_host[f[F_HISTN]] = rel;
  f[F_HISTN] += 1;
  if (rel <= tol) {
    f[F_DONE] = 1;
    f[F_CONV] = 1;
    f[F_NOTDONE] = 0;
    return;
  }
  f[F_CYC] = 1;
  f[F_DID] = 1;
  f[F_JF] = 0;
  k.g[0] = beta;
}

// Givens update of column j (the reference's host-side loop, done on the device).
__global__ void givens_kernel(KrylovDev k, int j, double tol, double* hist_host, int hist_cap) {
  int* f = k.flags;
  if (!f[F_CYC]) return;
  const int ld = k.restart + 1;
  double* H = k.H + (int64_t)j * ld;  // column j
  const double h_norm = sqrt(k.sc[SC_HSQ]);
  H[j + 1] = h_norm;
  k.sc[SC_HNORM] = h_norm;
  for (int i = 0; i < j; ++i) {
    const double a = H[i], b = H[i + 1];
    const double tmp = __dadd_rn(__dmul_rn(k.cs[i], a), __dmul_rn(k.sn[i], b));
    H[i + 1] = __dadd_rn(__dmul_rn(-k.sn[i], a), __dmul_rn(k.cs[i], b));
    H[i] = tmp;
  }
  const double hjj = H[j], hj1 = H[j + 1];
  const double denom = sqrt(__dadd_rn(__dmul_rn(hjj, hjj), __dmul_rn(hj1, hj1)));
  double c, sn;
  if (denom < 1e-300) {
    c = 1.0;
    sn = 0.0;
  } else {
    c = hjj / denom;
    sn = hj1 / denom;
  }
  k.cs[j] = c;
  k.sn[j] = sn;
  H[j] = __dadd_rn(__dmul_rn(c, hjj), __dmul_rn(sn, hj1));
  H[j + 1] = 0.0;
  const double gj = k.g[j];
  k.g[j + 1] = __dmul_rn(-sn, gj);
  k.g[j] = __dmul_rn(c, gj);
  f[F_TOTAL] += 1;
  f[F_JF] = j + 1;
  const double rel = fabs(k.g[j + 1]) / k.sc[SC_BNORM];
  if (hist_host != nullptr && f[F_HISTN] < hist_cap) hist_host[f[F_HISTN]] = rel;
  f[F_HISTN] += 1;
  if (rel <= tol) {
    f[F_CONV] = 1;
    f[F_DONE] = 1;
    f[F_NOTDONE] = 0;
    f[F_CYC] = 0;
  } else if (h_norm <= 1e-14) {
    // lucky breakdown: the reference reports convergence
    f[F_CONV] = 1;
    f[F_DONE] = 1;
    f[F_NOTDONE] = 0;
    f[F_BREAK] = 1;
    f[F_CYC] = 0;
  }
}

// dst = src / (*denom)   (V[j+1] = w / h_norm ; V[0] = r / beta)
__global__ void scale_vec_kernel(int64_t n, const double* __restrict__ src, const double* __restrict__ denom,
                                 double* __restrict__ dst, const int* guard) {
  if (guard_off(guard)) return;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[i] / *denom;
}

cudaError_t launch_scale_vec(int64_t n, const double* src, const double* denom_dev, double* dst,
                             const int* guard, cudaStream_t s) {
  scale_vec_kernel<<<div_up(n, 256), 256, 0, s>>>(n, src, denom_dev, dst, guard);
  return sf_launched(1);
}

// Back substitution R y = g[:jf] (column-oriented, R = triu(H[:jf, :jf])).
// A zero pivot (exactly singular R; the reference falls back to lstsq) sets y_j = 0.
__global__ void backsolve_kernel(KrylovDev k) {
  if (!k.flags[F_DID]) return;
  const int jf = k.flags[F_JF];
  const int ld = k.restart + 1;
  __shared__ double x[1024];
  for (int i = threadIdx.x; i < jf; i += blockDim.x) x[i] = k.g[i];
  __syncthreads();
  for (int j = jf - 1; j >= 0; --j) {
    if (threadIdx.x == 0) {
      const double r = k.H[(int64_t)j * ld + j];
      x[j] = (r != 0.0) ? x[j] / r : 0.0;
    }
    __syncthreads();
    const double xj = x[j];
    for (int i = threadIdx.x; i < j; i += blockDim.x) x[i] = __dsub_rn(x[i], __dmul_rn(xj, k.H[(int64_t)j * ld + i]));
    __syncthreads();
  }
  for (int i = threadIdx.x; i < jf; i += blockDim.x) k.y[i] = x[i];
}

cudaError_t launch_backsolve(KrylovDev k, cudaStream_t s) {
  backsolve_kernel<<<1, 256, 0, s>>>(k);
  return sf_launched(1);
}

// x <- x + y_0 Z_0 + y_1 Z_1 + ... (sequential per element, as the reference's loop)
__global__ void update_x_kernel(int64_t n, double* __restrict__ x, double* const* __restrict__ Z,
                                const double* __restrict__ y, const int* flags) {
  if (!flags[F_DID]) return;
  const int jf = flags[F_JF];
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double xi = x[i];
  for (int j = 0; j < jf; ++j) xi = __dadd_rn(xi, __dmul_rn(y[j], Z[j][i]));
  x[i] = xi;
}

cudaError_t launch_update_x(int64_t n, double* x, double* const* Z_dev, const double* y,
                            const int* flags, cudaStream_t s) {
  update_x_kernel<<<div_up(n, 256), 256, 0, s>>>(n, x, Z_dev, y, flags);
  return sf_launched(1);
}

// ----------------------------------------------------------------------------
// Scalar decisions of the safeguarded corrections (single thread).
//  OP_LS1: coarse-correction line search, first half
//          (gpu_fem/multigrid_v4.py:867-931): in  sc[0]=|c|^2 sc[1]=|r|^2
//          sc[2]=<Ac,Ac> sc[3]=<r,Ac> ; out sc[4]=applied scale, sc[7]=degenerate
//  OP_LS2: second half: in sc[5]=|trial|^2 ; p0 = acceptance ratio ; out sc[6]=accept
//  OP_RLF: root-local inner FGMRES acceptance (:964-1004): in sc[0]=|c|^2 sc[1]=|r|^2
//          sc[5]=|trial|^2 ; out sc[6]=accept (scale 1 in sc[4])
//  OP_RLL: root-local line search (:1006-1055): in sc[0..3] ; p1 = max scale ;
//          out sc[4]=scale, sc[6]=accept
__global__ void scalar_op_kernel(int op, double* sc, double p0, double p1, const int* guard) {
  if (guard_off(guard)) return;
  if (op == OP_LS1 || op == OP_RLL) {
    const double cn = sqrt(sc[0]), rn = sqrt(sc[1]);
    double deg = (cn <= 1e-300 || rn <= 1e-300) ? 1.0 : 0.0;
    const double denom = sc[2];
    if (denom <= 1e-300) deg = 1.0;
    const double raw = sc[3] / denom;
    const double applied = fmin(p1, fmax(0.0, raw));
    sc[4] = deg != 0.0 ? 0.0 : applied;
    sc[7] = deg;
    sc[8] = raw;
    if (op == OP_RLL) sc[6] = (deg == 0.0 && applied > 1e-12) ? 1.0 : 0.0;
  } else if (op == OP_LS2) {
    const double rn = sqrt(sc[1]);
    const double tn = sqrt(sc[5]);
    const bool reject = sc[7] != 0.0 || tn > p0 * rn;
    sc[6] = reject ? 0.0 : 1.0;
  } else if (op == OP_RLF) {
    const double cn = sqrt(sc[0]), rn = sqrt(sc[1]);
    const bool deg = cn <= 1e-300 || rn <= 1e-300;
    const double tn = sqrt(sc[5]);
    sc[4] = 1.0;
    sc[6] = (!deg && !(tn > rn)) ? 1.0 : 0.0;
  }
}

cudaError_t launch_scalar_op(int op, double* sc, double p0, double p1, const int* guard,
                             cudaStream_t s) {
  scalar_op_kernel<<<1, 1, 0, s>>>(op, sc, p0, p1, guard);
  return sf_launched(1);
}

// x <- accept ? x + s * c : x   (s = 1 uses x + c)
template <typename T>
__global__ void select_axpy_kernel(int64_t n, T* __restrict__ x, const T* __restrict__ c,
                                   const double* __restrict__ sc, int unit, const int* guard) {
  if (guard_off(guard)) return;
  if (sc[6] == 0.0) return;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const T s = (T)sc[4];
  x[i] = unit ? add_rn(x[i], c[i]) : add_rn(x[i], mul_rn(s, c[i]));
}

cudaError_t launch_select_axpy(DType t, int64_t n, void* x, const void* c, const double* sc,
                               int unit, const int* guard, cudaStream_t s) {
  if (t == F64)
    select_axpy_kernel<double><<<div_up(n, 256), 256, 0, s>>>(n, (double*)x, (const double*)c, sc,
                                                              unit, guard);
  else
    select_axpy_kernel<float><<<div_up(n, 256), 256, 0, s>>>(n, (float*)x, (const float*)c, sc,
                                                             unit, guard);
  return sf_launched(1);
}

// trial = r - s * Ac (s from sc[4], or 1 when unit) ; sc[5] = |trial|^2
template <typename T>
__global__ void __launch_bounds__(kRedThreads) trial_kernel(int64_t n, const T* __restrict__ r,
                                                            const T* __restrict__ Ac, double* sc,
                                                            int unit, T* __restrict__ trial,
                                                            RedWork rw, const int* guard) {
  if (guard_off(guard)) return;
  __shared__ double sh[32];
  const T s = (T)sc[4];
  double v[1] = {0.0};
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const T t = unit ? sub_rn(r[i], Ac[i]) : sub_rn(r[i], mul_rn(s, Ac[i]));
    if (trial != nullptr) trial[i] = t;
    v[0] += (double)t * (double)t;
  }
  block_sum<1>(v, sh);
  last_block_finalize<1>(v, rw, sc + 5);
}

cudaError_t launch_trial_residual(DType t, int64_t n, const void* r, const void* Ac, double* sc,
                                  int unit, void* trial, RedWork rw, const int* guard,
                                  cudaStream_t s) {
  if (t == F64)
    trial_kernel<double><<<red_blocks(n), kRedThreads, 0, s>>>(n, (const double*)r, (const double*)Ac,
                                                               sc, unit, (double*)trial, rw, guard);
  else
    trial_kernel<float><<<red_blocks(n), kRedThreads, 0, s>>>(n, (const float*)r, (const float*)Ac, sc,
                                                              unit, (float*)trial, rw, guard);
  return sf_launched(1);
}

// Select between the accepted trial residual and the old residual:
// out <- accept ? trial : r  (used when a corrected residual feeds a second correction)
template <typename T>
__global__ void select_vec_kernel(int64_t n, const T* trial, const T* r, const double* sc, T* out,
                                  const int* guard) {
  if (guard_off(guard)) return;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = sc[6] != 0.0 ? trial[i] : r[i];
}

cudaError_t launch_select_vec(DType t, int64_t n, const void* trial, const void* r,
                              const double* sc, void* out, const int* guard, cudaStream_t s) {
  if (t == F64)
    select_vec_kernel<double><<<div_up(n, 256), 256, 0, s>>>(n, (const double*)trial, (const double*)r,
                                                             sc, (double*)out, guard);
  else
    select_vec_kernel<float><<<div_up(n, 256), 256, 0, s>>>(n, (const float*)trial, (const float*)r,
                                                            sc, (float*)out, guard);
  return sf_launched(1);
}

cudaError_t launch_krylov_init(KrylovDev k, const int* parent, cudaStream_t s) {
  krylov_init_kernel<<<1, 1, 0, s>>>(k, parent);
  return sf_launched(1);
}
cudaError_t launch_krylov_restart(KrylovDev k, double tol, double* hist_host, int hist_cap,
                                  cudaStream_t s) {
  krylov_restart_kernel<<<1, 1, 0, s>>>(k, tol, hist_host, hist_cap);
  return sf_launched(1);
}
cudaError_t launch_givens(KrylovDev k, int j, double tol, double* hist_host, int hist_cap,
                          cudaStream_t s) {
  givens_kernel<<<1, 1, 0, s>>>(k, j, tol, hist_host, hist_cap);
  return sf_launched(1);
}

// ----------------------------------------------------------------------------
// Fixed-count Jacobi-PCG coarse solve (gpu_fem/solver_v2.py:781-810).
// sc: [0]=rz [1]=pAp [2]=rz_new [3]=alpha [4]=beta
__global__ void pcg_scalar_kernel(int which, double* sc, const int* guard) {
  if (guard_off(guard)) return;
  if (which == 0) {
    sc[3] = sc[0] / (sc[1] + 1e-300);
  } else {
    sc[4] = sc[2] / (sc[0] + 1e-300);
    sc[0] = sc[2];
  }
}

cudaError_t launch_pcg_scalar(int which, double* sc, const int* guard, cudaStream_t s) {
  pcg_scalar_kernel<<<1, 1, 0, s>>>(which, sc, guard);
  return sf_launched(1);
}

// x += alpha p ; r -= alpha Ap ; z = dinv r ; sc[2] = <r, z>
__global__ void __launch_bounds__(kRedThreads) pcg_xr_kernel(int64_t n, double* __restrict__ x,
                                                             double* __restrict__ r, double* __restrict__ z,
                                                             const double* __restrict__ p,
                                                             const double* __restrict__ Ap,
                                                             const double* __restrict__ dinv, double* sc,
                                                             RedWork rw, const int* guard) {
  if (guard_off(guard)) return;
  __shared__ double sh[32];
  const double alpha = sc[3];
  double v[1] = {0.0};
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    x[i] = __dadd_rn(x[i], __dmul_rn(alpha, p[i]));
    const double rn = __dsub_rn(r[i], __dmul_rn(alpha, Ap[i]));
    r[i] = rn;
    const double zn = __dmul_rn(dinv[i], rn);
    z[i] = zn;
    v[0] += rn * zn;
  }
  block_sum<1>(v, sh);
  last_block_finalize<1>(v, rw, sc + 2);
}

cudaError_t launch_pcg_xr(int64_t n, double* x, double* r, double* z, const double* p, const double* Ap,
                          const double* dinv, double* sc, RedWork rw, const int* guard, cudaStream_t s) {
  pcg_xr_kernel<<<red_blocks(n), kRedThreads, 0, s>>>(n, x, r, z, p, Ap, dinv, sc, rw, guard);
  return sf_launched(1);
}

// p = z + beta p
__global__ void pcg_p_kernel(int64_t n, const double* __restrict__ z, double* __restrict__ p,
                             const double* __restrict__ sc, const int* guard) {
  if (guard_off(guard)) return;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = __dadd_rn(z[i], __dmul_rn(sc[4], p[i]));
}

cudaError_t launch_pcg_p(int64_t n, const double* z, double* p, const double* sc, const int* guard,
                         cudaStream_t s) {
  pcg_p_kernel<<<div_up(n, 256), 256, 0, s>>>(n, z, p, sc, guard);
  return sf_launched(1);
}

// z = dinv * r (elementwise), guarded
__global__ void dmul_kernel(int64_t n, const double* __restrict__ dinv, const double* __restrict__ r,
                            double* __restrict__ z, const int* guard) {
  if (guard_off(guard)) return;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) z[i] = __dmul_rn(dinv[i], r[i]);
}

cudaError_t launch_dmul(int64_t n, const double* dinv, const double* r, double* z, const int* guard,
                        cudaStream_t s) {
  dmul_kernel<<<div_up(n, 256), 256, 0, s>>>(n, dinv, r, z, guard);
  return sf_launched(1);
}

}  // namespace simpfem
