// SIMP loop kernels around the guarded solve: the cone density filter, its
// transpose, and the optimality-criteria (OC) update.
//
// The reference filters with a row-normalised sparse matrix
// (gpu_fem/pub_simp_solver.py:90-117 _build_density_filter: weight
// rmin - dist for every element within distance < rmin, the element itself
// weight rmin, rows divided by their sums) and runs the OC bisection with one
// SpMV per step (gpu_fem/simp_gpu.py:212-294 _oc_step_cupy).  On the structured
// grid the filter is a stencil over the offsets within rmin, applied here
// directly (row sums from the in-grid offsets), and without a Heaviside
// projection the bisection's volume sum(H rn) equals sum_j (H^T 1)_j rn_j, so a
// bisection step is one fused pass over the design variables.
//
// Element index e = (i * ny + j) * nz + k.  Reductions are deterministic: every
// block writes a partial, one block sums them in block order.
#include <algorithm>
#include <mutex>

#include "common.cuh"
#include "gmg_impl.h"
#include "simpfem.h"

namespace simpfem {
namespace {

constexpr int kMaxOff = 343;  // offsets within radius <= 3.5 in a 7^3 box
constexpr int kSimpBlocks = 296, kSimpThreads = 256;

struct FilterOffsets {
  int n;
  int dx[kMaxOff], dy[kMaxOff], dz[kMaxOff];
  double w[kMaxOff];
};

__constant__ FilterOffsets c_off;

__device__ __forceinline__ double row_sum(int i, int j, int k, int nx, int ny, int nz) {
  double s = 0.0;
  for (int q = 0; q < c_off.n; ++q) {
    const int a = i + c_off.dx[q], b = j + c_off.dy[q], c = k + c_off.dz[q];
    if (a >= 0 && a < nx && b >= 0 && b < ny && c >= 0 && c < nz) s += c_off.w[q];
  }
  return s;
}

// y = H x (transpose = 0) or y = H^T x (transpose = 1); H symmetric in its
// weights, so (H^T x)_e = sum over neighbours f of w(e, f) x_f / rowsum_f
__global__ void cone_filter_kernel(int nx, int ny, int nz, int transpose, const double* __restrict__ x,
                                   double* __restrict__ y) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t ne = (int64_t)nx * ny * nz;
  if (e >= ne) return;
  const int k = (int)(e % nz), j = (int)((e / nz) % ny), i = (int)(e / ((int64_t)ny * nz));
  double acc = 0.0;
  for (int q = 0; q < c_off.n; ++q) {
    const int a = i + c_off.dx[q], b = j + c_off.dy[q], c = k + c_off.dz[q];
    if (a < 0 || a >= nx || b < 0 || b >= ny || c < 0 || c >= nz) continue;
    const int64_t f = ((int64_t)a * ny + b) * nz + c;
    const double wf = transpose ? c_off.w[q] / row_sum(a, b, c, nx, ny, nz) : c_off.w[q];
    acc += wf * x[f];
  }
  y[e] = transpose ? acc : acc / row_sum(i, j, k, nx, ny, nz);
}

__device__ __forceinline__ double block_reduce_sum(double v, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
  return t;
}

__device__ __forceinline__ double block_reduce_max(double v, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t = fmax(t, sh[w]);
  return t;
}

// the reference's OC candidate for multiplier lm (simp_gpu.py:271-276):
// rn = clip(clip(rho * sqrt(-dc_s / (lm * dv_s)), rho - move, rho + move), 1e-3, 1)
// with dc_s = min(dc, -1e-12), dv_s = max(dv, 1e-12)
__device__ __forceinline__ double oc_candidate(double rho, double dc, double dv, double lm, double move) {
  const double dcs = fmin(dc, -1e-12), dvs = fmax(dv, 1e-12);
  double r = rho * sqrt(-dcs / (lm * dvs));
  r = fmin(fmax(r, rho - move), rho + move);
  return fmin(fmax(r, 1e-3), 1.0);
}

// mode 0: partial sums of vw * rn(lm) (vw = H^T 1: the filtered volume sum(H rn));
// mode 1: write rn(lm) and partial maxima of |rn - rho|.  dv == nullptr: dv = 1.
__global__ void __launch_bounds__(kSimpThreads) oc_pass_kernel(int64_t n, const double* __restrict__ rho,
                                                               const double* __restrict__ dc,
                                                               const double* __restrict__ dv,
                                                               const double* __restrict__ vw, double lm,
                                                               double move, int mode, double* __restrict__ rn,
                                                               double* __restrict__ partials) {
  __shared__ double sh[32];
  double v = 0.0;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const double r = oc_candidate(rho[e], dc[e], dv ? dv[e] : 1.0, lm, move);
    if (mode == 0) {
      v += vw[e] * r;
    } else {
      rn[e] = r;
      v = fmax(v, fabs(r - rho[e]));
    }
  }
  const double t = mode == 0 ? block_reduce_sum(v, sh) : block_reduce_max(v, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = t;
}

// out = partials summed (mode 0) or maximised (mode 1) in block order
__global__ void oc_finish_kernel(int nb, int mode, const double* __restrict__ partials, double* __restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double s = 0.0;
  for (int b = 0; b < nb; ++b) s = mode == 0 ? s + partials[b] : fmax(s, partials[b]);
  *out = s;
}

// Heaviside projection of x and its derivative (pub_simp_solver.py:245-253):
// p = (tanh(b eta) + tanh(b (x - eta))) / den, dp = b (1 - tanh(b (x - eta))^2) / den,
// den = tanh(b eta) + tanh(b (1 - eta)); dc (optional) is multiplied by dp into dcdp.
__global__ void heaviside_kernel(int64_t n, const double* __restrict__ x, double beta, double eta, double tbe,
                                 double den, double* __restrict__ p, double* __restrict__ dp,
                                 const double* __restrict__ dc, double* __restrict__ dcdp) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const double t = tanh(beta * (x[e] - eta));
  if (p) p[e] = (tbe + t) / den;
  const double d = beta * (1.0 - t * t) / den;
  if (dp) dp[e] = d;
  if (dcdp) dcdp[e] = dc[e] * d;
}

// partial sums of tanh(b eta) + tanh(b (x - eta)) (the projected volume times den)
__global__ void __launch_bounds__(kSimpThreads) projected_sum_kernel(int64_t n, const double* __restrict__ x,
                                                                     double beta, double eta, double tbe,
                                                                     double* __restrict__ partials) {
  __shared__ double sh[32];
  double v = 0.0;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
    v += tbe + tanh(beta * (x[e] - eta));
  const double t = block_reduce_sum(v, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = t;
}

FilterOffsets make_offsets(double rmin) {
  FilterOffsets o{};
  const int r = (int)floor(rmin);
  o.n = 0;
  // the element itself first, weight rmin, then the other offsets in
  // lexicographic order, weight rmin - dist (kept when dist <= rmin - 1e-10)
  o.dx[0] = o.dy[0] = o.dz[0] = 0;
  o.w[0] = rmin;
  o.n = 1;
  for (int a = -r; a <= r; ++a)
    for (int b = -r; b <= r; ++b)
      for (int c = -r; c <= r; ++c) {
        if (a == 0 && b == 0 && c == 0) continue;
        const double d = sqrt((double)(a * a + b * b + c * c));
        if (d > rmin - 1e-10) continue;
        o.dx[o.n] = a;
        o.dy[o.n] = b;
        o.dz[o.n] = c;
        o.w[o.n] = rmin - d;
        ++o.n;
      }
  return o;
}

}  // namespace
}  // namespace simpfem

using namespace simpfem;

#define SIMP_API_BEGIN try {
#define SIMP_API_END                        \
  }                                         \
  catch (const CudaFailure&) {              \
    return SIMPFEM_ECUDA;                   \
  }                                         \
  catch (const InvalidArg& e) {             \
    set_error(e.msg);                       \
    return SIMPFEM_EINVAL;                  \
  }                                         \
  catch (const std::exception& e) {         \
    set_error(e.what());                    \
    return SIMPFEM_EINTERNAL;               \
  }                                         \
  return SIMPFEM_OK;

namespace {
// the offsets live in constant memory, loaded when the radius or device changes
// (one radius at a time: a call with a new radius must not overlap filter
// launches of another radius on other streams)
std::mutex g_filter_mutex;
void set_filter(double rmin, cudaStream_t s) {
  std::lock_guard<std::mutex> lk(g_filter_mutex);
  static double cur = -1.0;
  static int dev_set = -1;
  int dev = 0;
  SF_CUDA(cudaGetDevice(&dev));
  if (cur == rmin && dev_set == dev) return;
  const FilterOffsets o = make_offsets(rmin);
  SF_CUDA(cudaMemcpyToSymbolAsync(c_off, &o, sizeof(o), 0, cudaMemcpyHostToDevice, s));
  SF_CUDA(cudaStreamSynchronize(s));
  cur = rmin;
  dev_set = dev;
}
}  // namespace

extern "C" {

int simpfem_cone_filter(int nx, int ny, int nz, double rmin, int transpose, const double* x, double* y,
                        void* stream) {
  SIMP_API_BEGIN
  if (nx < 1 || ny < 1 || nz < 1 || !x || !y || x == y) throw InvalidArg{"simpfem_cone_filter: bad argument"};
  if (!(rmin >= 1.0 && rmin <= 3.5)) throw InvalidArg{"simpfem_cone_filter: rmin must be in [1, 3.5]"};
  cudaStream_t s = (cudaStream_t)stream;
  set_filter(rmin, s);
  const int64_t ne = (int64_t)nx * ny * nz;
  cone_filter_kernel<<<div_up(ne, 256), 256, 0, s>>>(nx, ny, nz, transpose ? 1 : 0, x, y);
  SF_CUDA(sf_launched(1));
  SIMP_API_END
}

size_t simpfem_oc_work_bytes(void) { return sizeof(double) * (kSimpBlocks + 2); }

int simpfem_oc_update(int64_t n, const double* rho, const double* dc, const double* dv, const double* vol_w,
                      double volfrac, double move, double* rho_new, double* work, size_t work_bytes,
                      double* change_host, double* lambda_host, int* steps_host, void* stream) {
  SIMP_API_BEGIN
  if (n < 1 || !rho || !dc || !vol_w || !rho_new || !work) throw InvalidArg{"simpfem_oc_update: null argument"};
  if (work_bytes < simpfem_oc_work_bytes()) throw InvalidArg{"simpfem_oc_update: workspace too small"};
  cudaStream_t s = (cudaStream_t)stream;
  double* partials = work;
  double* out = work + kSimpBlocks;
  const int nb = (int)std::min<int64_t>(kSimpBlocks, div_up(n, kSimpThreads));
  const double target = volfrac * (double)n;
  double l1 = 0.0, l2 = 1e9, lm = 0.5 * (l1 + l2);
  int steps = 0;
  // the reference's bisection (simp_gpu.py:268-290): at most 100 steps, stop
  // when l2 - l1 < 1e-9; the candidate of the last midpoint is the update
  for (int it = 0; it < 100; ++it) {
    lm = 0.5 * (l1 + l2);
    oc_pass_kernel<<<nb, kSimpThreads, 0, s>>>(n, rho, dc, dv, vol_w, lm, move, 0, nullptr, partials);
    oc_finish_kernel<<<1, 32, 0, s>>>(nb, 0, partials, out);
    SF_CUDA(sf_launched(2));
    double vol = 0.0;
    SF_CUDA(cudaMemcpyAsync(&vol, out, sizeof(double), cudaMemcpyDeviceToHost, s));
    SF_CUDA(cudaStreamSynchronize(s));
    ++steps;
    if (vol > target) l1 = lm;
    else l2 = lm;
    if (l2 - l1 < 1e-9) break;
  }
  oc_pass_kernel<<<nb, kSimpThreads, 0, s>>>(n, rho, dc, dv, vol_w, lm, move, 1, rho_new, partials);
  oc_finish_kernel<<<1, 32, 0, s>>>(nb, 1, partials, out);
  SF_CUDA(sf_launched(2));
  double ch = 0.0;
  SF_CUDA(cudaMemcpyAsync(&ch, out, sizeof(double), cudaMemcpyDeviceToHost, s));
  SF_CUDA(cudaStreamSynchronize(s));
  if (change_host) *change_host = ch;
  if (lambda_host) *lambda_host = lm;
  if (steps_host) *steps_host = steps;
  SIMP_API_END
}

int simpfem_heaviside(int64_t n, const double* x, double beta, double eta, double* proj, double* dproj,
                      void* stream) {
  SIMP_API_BEGIN
  if (n < 1 || !x || (!proj && !dproj)) throw InvalidArg{"simpfem_heaviside: bad argument"};
  if (!(beta > 0.0)) throw InvalidArg{"simpfem_heaviside: beta must be positive"};
  const double tbe = tanh(beta * eta), den = tbe + tanh(beta * (1.0 - eta));
  cudaStream_t s = (cudaStream_t)stream;
  heaviside_kernel<<<div_up(n, 256), 256, 0, s>>>(n, x, beta, eta, tbe, den, proj, dproj, nullptr, nullptr);
  SF_CUDA(sf_launched(1));
  SIMP_API_END
}

size_t simpfem_oc_projected_work_bytes(int64_t n) {
  return sizeof(double) * (5 * (size_t)std::max<int64_t>(n, 1) + kSimpBlocks + 2);
}

int simpfem_oc_update_projected(int nx, int ny, int nz, double rmin, const double* rho, const double* rho_f,
                                const double* dc_phys, double beta, double eta, double volfrac, double move,
                                double* rho_new, double* work, size_t work_bytes, double* change_host,
                                double* lambda_host, int* steps_host, void* stream) {
  SIMP_API_BEGIN
  const int64_t n = (int64_t)nx * ny * nz;
  if (nx < 1 || ny < 1 || nz < 1 || !rho || !rho_f || !dc_phys || !rho_new || !work)
    throw InvalidArg{"simpfem_oc_update_projected: null argument"};
  if (work_bytes < simpfem_oc_projected_work_bytes(n))
    throw InvalidArg{"simpfem_oc_update_projected: workspace too small"};
  if (!(beta > 1e-6)) throw InvalidArg{"simpfem_oc_update_projected: beta must exceed 1e-6 (else simpfem_oc_update)"};
  if (!(rmin >= 1.0 && rmin <= 3.5)) throw InvalidArg{"simpfem_oc_update_projected: rmin must be in [1, 3.5]"};
  cudaStream_t s = (cudaStream_t)stream;
  set_filter(rmin, s);
  double* dh = work;
  double* dcdh = dh + n;  // dc * dh, then reused for the filtered candidate
  double* dcd = dcdh + n;
  double* dvd = dcd + n;
  double* rn = dvd + n;
  double* partials = rn + n;
  double* out = partials + kSimpBlocks;
  const double tbe = tanh(beta * eta), den = tbe + tanh(beta * (1.0 - eta));
  const int eb = div_up(n, 256);
  // sensitivities in the design space (simp_gpu.py:245-258): H^T (dc dh), H^T dh
  heaviside_kernel<<<eb, 256, 0, s>>>(n, rho_f, beta, eta, tbe, den, nullptr, dh, dc_phys, dcdh);
  cone_filter_kernel<<<eb, 256, 0, s>>>(nx, ny, nz, 1, dcdh, dcd);
  cone_filter_kernel<<<eb, 256, 0, s>>>(nx, ny, nz, 1, dh, dvd);
  SF_CUDA(sf_launched(3));
  double* rnf = dcdh;
  const int nb = (int)std::min<int64_t>(kSimpBlocks, div_up(n, kSimpThreads));
  const double target = volfrac * (double)n;
  double l1 = 0.0, l2 = 1e9, lm = 0.5 * (l1 + l2);
  int steps = 0;
  // the bisection of simp_gpu.py:268-290 with the projected volume of each candidate:
  // sum(tanh(b eta) + tanh(b (H rn - eta))) / den against volfrac n
  for (int it = 0; it < 100; ++it) {
    lm = 0.5 * (l1 + l2);
    oc_pass_kernel<<<nb, kSimpThreads, 0, s>>>(n, rho, dcd, dvd, nullptr, lm, move, 1, rn, partials);
    cone_filter_kernel<<<eb, 256, 0, s>>>(nx, ny, nz, 0, rn, rnf);
    projected_sum_kernel<<<nb, kSimpThreads, 0, s>>>(n, rnf, beta, eta, tbe, partials);
    oc_finish_kernel<<<1, 32, 0, s>>>(nb, 0, partials, out);
    SF_CUDA(sf_launched(4));
    double vol = 0.0;
    SF_CUDA(cudaMemcpyAsync(&vol, out, sizeof(double), cudaMemcpyDeviceToHost, s));
    SF_CUDA(cudaStreamSynchronize(s));
    ++steps;
    if (vol / den > target) l1 = lm;
    else l2 = lm;
    if (l2 - l1 < 1e-9) break;
  }
  oc_pass_kernel<<<nb, kSimpThreads, 0, s>>>(n, rho, dcd, dvd, nullptr, lm, move, 1, rho_new, partials);
  oc_finish_kernel<<<1, 32, 0, s>>>(nb, 1, partials, out);
  SF_CUDA(sf_launched(2));
  double ch = 0.0;
  SF_CUDA(cudaMemcpyAsync(&ch, out, sizeof(double), cudaMemcpyDeviceToHost, s));
  SF_CUDA(cudaStreamSynchronize(s));
  if (change_host) *change_host = ch;
  if (lambda_host) *lambda_host = lm;
  if (steps_host) *steps_host = steps;
  SIMP_API_END
}

}  // extern "C"
