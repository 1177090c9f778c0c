// Learned floor proposer: a small 3D CNN, forward, backward and Adam on the GPU.
// No counterpart in the reference.
//
//   x (N, 1, 16^3) -- the density average-pooled to 16^3 (pool16_kernel)
//   conv 1->16  s1 -> 16^3, conv 16->16 s2 -> 8^3, conv 16->32 s2 -> 4^3,
//   conv 32->32 s2 -> 2^3   (3x3x3, pad 1, ReLU after each)
//   mean over 8 positions (32) ++ 2 probe features -> dense 34 -> 3 -> softmax
//
// Weights are stored and read as bfloat16, biases and every activation and
// accumulation in float32; the float32 master copy is what Adam updates (the
// gradient is taken with respect to the bfloat16 weights).  Parameter layout:
// W1 b1 W2 b2 W3 b3 W4 b4 Wfc bfc, weights [cout][cin][kz][ky][kx].
// Every reduction (weight and bias gradients, the loss) runs in a fixed order,
// so a training run is bitwise reproducible.
//
// The network is tiny (49,017 parameters, at most ~70 MFLOP per sample): one
// thread per output value for the convolutions and one block per parameter for
// the weight gradients keep every launch short and deterministic; none of it is
// on the solver's hot path (one forward per guarded solve).
#include <math.h>

#include <cstring>

#include "common.cuh"
#include "gmg_impl.h"
#include "simpfem.h"

namespace simpfem {
namespace {

constexpr int kS0 = 16, kVox = kS0 * kS0 * kS0, kFeat = 2, kClass = 3;
constexpr int kCin[4] = {1, 16, 16, 32}, kCout[4] = {16, 16, 32, 32}, kStride[4] = {1, 2, 2, 2};
constexpr int kSin[4] = {16, 16, 8, 4}, kSout[4] = {16, 8, 4, 2};
constexpr int kHidden = 32, kZ = kHidden + kFeat;

struct Layout {
  int w[5], b[5], n;
};
constexpr Layout layout() {
  Layout L{};
  int o = 0;
  for (int l = 0; l < 4; ++l) {
    L.w[l] = o;
    o += kCout[l] * kCin[l] * 27;
    L.b[l] = o;
    o += kCout[l];
  }
  L.w[4] = o;
  o += kClass * kZ;
  L.b[4] = o;
  o += kClass;
  L.n = o;
  return L;
}
constexpr Layout kL = layout();
static_assert(kL.n == 49017, "parameter count");

__global__ void to_bf16_kernel(int n, const float* __restrict__ src, __nv_bfloat16* __restrict__ dst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = __float2bfloat16_rn(src[i]);
}

// y = relu(conv(x) + b); one thread per output value
__global__ void conv_fwd_kernel(int N, int cin, int cout, int sin, int sout, int stride,
                                const float* __restrict__ x, const __nv_bfloat16* __restrict__ W,
                                const float* __restrict__ b, float* __restrict__ y) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t total = (int64_t)N * cout * sout * sout * sout;
  if (idx >= total) return;
  const int t = (int)(idx % (sout * sout * sout));
  const int ox = t % sout, oy = (t / sout) % sout, oz = t / (sout * sout);
  const int64_t nc = idx / (sout * sout * sout);
  const int co = (int)(nc % cout), n = (int)(nc / cout);
  float acc = b[co];
  for (int ci = 0; ci < cin; ++ci) {
    const float* xin = x + ((int64_t)n * cin + ci) * sin * sin * sin;
    const __nv_bfloat16* w = W + ((int64_t)co * cin + ci) * 27;
#pragma unroll
    for (int kz = 0; kz < 3; ++kz) {
      const int iz = oz * stride + kz - 1;
      if (iz < 0 || iz >= sin) continue;
#pragma unroll
      for (int ky = 0; ky < 3; ++ky) {
        const int iy = oy * stride + ky - 1;
        if (iy < 0 || iy >= sin) continue;
#pragma unroll
        for (int kx = 0; kx < 3; ++kx) {
          const int ix = ox * stride + kx - 1;
          if (ix < 0 || ix >= sin) continue;
          acc = fmaf(__bfloat162float(w[(kz * 3 + ky) * 3 + kx]), xin[(iz * sin + iy) * sin + ix], acc);
        }
      }
    }
  }
  y[idx] = fmaxf(acc, 0.f);
}

// head: g = mean of the last activation, z = [g, feats], logits, softmax,
// per-sample cross-entropy (labels may be null), one thread per sample
__global__ void head_fwd_kernel(int N, const float* __restrict__ a4, const float* __restrict__ feats,
                                const __nv_bfloat16* __restrict__ Wfc, const float* __restrict__ bfc,
                                const int32_t* __restrict__ labels, float* __restrict__ z, float* __restrict__ prob,
                                float* __restrict__ loss_n) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  float zz[kZ];
  for (int c = 0; c < kHidden; ++c) {
    float s = 0.f;
    for (int p = 0; p < 8; ++p) s += a4[((int64_t)n * kHidden + c) * 8 + p];
    zz[c] = s * 0.125f;
  }
  zz[kHidden] = feats[2 * n];
  zz[kHidden + 1] = feats[2 * n + 1];
  float lg[kClass], mx = -INFINITY;
  for (int k = 0; k < kClass; ++k) {
    float s = bfc[k];
    for (int j = 0; j < kZ; ++j) s = fmaf(__bfloat162float(Wfc[k * kZ + j]), zz[j], s);
    lg[k] = s;
    mx = fmaxf(mx, s);
  }
  float den = 0.f;
  for (int k = 0; k < kClass; ++k) den += expf(lg[k] - mx);
  for (int k = 0; k < kClass; ++k) prob[n * kClass + k] = expf(lg[k] - mx) / den;
  for (int j = 0; j < kZ; ++j) z[n * kZ + j] = zz[j];
  if (labels) {
    // a label outside the rungs gives a NaN loss (and no one-hot term in the gradient)
    const int lab = labels[n];
    float l = NAN;
    for (int k = 0; k < kClass; ++k)
      if (k == lab) l = -(lg[k] - mx - logf(den));
    loss_n[n] = l;
  }
}

// dlogits = (p - onehot) / N; dWfc, dbfc (one thread per parameter, samples in order)
__global__ void head_bwd_params_kernel(int N, const float* __restrict__ prob, const int32_t* __restrict__ labels,
                                       const float* __restrict__ z, float* __restrict__ gWfc,
                                       float* __restrict__ gbfc) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kClass * kZ + kClass) return;
  const float invN = 1.f / (float)N;
  if (p < kClass * kZ) {
    const int k = p / kZ, j = p % kZ;
    float s = 0.f;
    for (int n = 0; n < N; ++n) s += ((prob[n * kClass + k] - (labels[n] == k ? 1.f : 0.f)) * invN) * z[n * kZ + j];
    gWfc[p] = s;
  } else {
    const int k = p - kClass * kZ;
    float s = 0.f;
    for (int n = 0; n < N; ++n) s += (prob[n * kClass + k] - (labels[n] == k ? 1.f : 0.f)) * invN;
    gbfc[k] = s;
  }
}

// d4 = (dz / 8) broadcast over the 8 positions of the last activation
__global__ void head_bwd_data_kernel(int N, const float* __restrict__ prob, const int32_t* __restrict__ labels,
                                     const __nv_bfloat16* __restrict__ Wfc, float* __restrict__ d4) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= N * kHidden * 8) return;
  const int n = idx / (kHidden * 8), c = (idx / 8) % kHidden;
  const float invN = 1.f / (float)N;
  float s = 0.f;
  for (int k = 0; k < kClass; ++k)
    s = fmaf((prob[n * kClass + k] - (labels[n] == k ? 1.f : 0.f)) * invN, __bfloat162float(Wfc[k * kZ + c]), s);
  d4[idx] = s * 0.125f;
}

// dx = conv^T(dy * relu'(y)); one thread per input value
__global__ void conv_bwd_data_kernel(int N, int cin, int cout, int sin, int sout, int stride,
                                     const float* __restrict__ dy, const float* __restrict__ y,
                                     const __nv_bfloat16* __restrict__ W, float* __restrict__ dx) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t total = (int64_t)N * cin * sin * sin * sin;
  if (idx >= total) return;
  const int t = (int)(idx % (sin * sin * sin));
  const int ix = t % sin, iy = (t / sin) % sin, iz = t / (sin * sin);
  const int64_t nc = idx / (sin * sin * sin);
  const int ci = (int)(nc % cin), n = (int)(nc / cin);
  float acc = 0.f;
  for (int co = 0; co < cout; ++co) {
    const int64_t ybase = ((int64_t)n * cout + co) * sout * sout * sout;
    const __nv_bfloat16* w = W + ((int64_t)co * cin + ci) * 27;
#pragma unroll
    for (int kz = 0; kz < 3; ++kz) {
      const int tz = iz + 1 - kz;
      if (tz < 0 || tz % stride) continue;
      const int oz = tz / stride;
      if (oz >= sout) continue;
#pragma unroll
      for (int ky = 0; ky < 3; ++ky) {
        const int ty = iy + 1 - ky;
        if (ty < 0 || ty % stride) continue;
        const int oy = ty / stride;
        if (oy >= sout) continue;
#pragma unroll
        for (int kx = 0; kx < 3; ++kx) {
          const int tx = ix + 1 - kx;
          if (tx < 0 || tx % stride) continue;
          const int ox = tx / stride;
          if (ox >= sout) continue;
          const int64_t o = ybase + (oz * sout + oy) * sout + ox;
          if (y[o] > 0.f) acc = fmaf(__bfloat162float(w[(kz * 3 + ky) * 3 + kx]), dy[o], acc);
        }
      }
    }
  }
  dx[idx] = acc;
}

// weight and bias gradients: one block per weight (co, ci, k) and one block per
// bias co (the last cout blocks); 256 threads reduce over (n, output position)
// in a fixed order
__global__ void __launch_bounds__(256) conv_bwd_param_kernel(int N, int cin, int cout, int sin, int sout, int stride,
                                                             const float* __restrict__ dy, const float* __restrict__ y,
                                                             const float* __restrict__ x, float* __restrict__ gW,
                                                             float* __restrict__ gb) {
  __shared__ float red[256];
  const int nw = cout * cin * 27;
  const int p = blockIdx.x;
  const int so3 = sout * sout * sout;
  const int64_t m = (int64_t)N * so3;
  float s = 0.f;
  if (p < nw) {
    const int k = p % 27, ci = (p / 27) % cin, co = p / (27 * cin);
    const int kz = k / 9, ky = (k / 3) % 3, kx = k % 3;
    for (int64_t q = threadIdx.x; q < m; q += blockDim.x) {
      const int o = (int)(q % so3);
      const int n = (int)(q / so3);
      const int ox = o % sout, oy = (o / sout) % sout, oz = o / (sout * sout);
      const int iz = oz * stride + kz - 1, iy = oy * stride + ky - 1, ix = ox * stride + kx - 1;
      if (iz < 0 || iz >= sin || iy < 0 || iy >= sin || ix < 0 || ix >= sin) continue;
      const int64_t yo = ((int64_t)n * cout + co) * so3 + o;
      if (y[yo] > 0.f) s = fmaf(dy[yo], x[((int64_t)n * cin + ci) * sin * sin * sin + (iz * sin + iy) * sin + ix], s);
    }
  } else {
    const int co = p - nw;
    for (int64_t q = threadIdx.x; q < m; q += blockDim.x) {
      const int o = (int)(q % so3);
      const int n = (int)(q / so3);
      const int64_t yo = ((int64_t)n * cout + co) * so3 + o;
      if (y[yo] > 0.f) s += dy[yo];
    }
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    if (p < nw) gW[p] = red[0];
    else gb[p - nw] = red[0];
  }
}

__global__ void loss_sum_kernel(int N, const float* __restrict__ loss_n, float* __restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  float s = 0.f;
  for (int n = 0; n < N; ++n) s += loss_n[n];
  *out = s / (float)N;
}

__global__ void adam_kernel(int n, float* __restrict__ theta, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  theta[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// adaptive average pooling of one density field (element order (i*ny + j)*nz + k)
// to 16^3: window i covers [floor(i*n/16), ceil((i+1)*n/16)) along each axis
__global__ void pool16_kernel(int nx, int ny, int nz, const double* __restrict__ d, float* __restrict__ out) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= kVox) return;
  const int c = idx % kS0, b = (idx / kS0) % kS0, a = idx / (kS0 * kS0);
  const int x0 = a * nx / kS0, x1 = ((a + 1) * nx + kS0 - 1) / kS0;
  const int y0 = b * ny / kS0, y1 = ((b + 1) * ny + kS0 - 1) / kS0;
  const int z0 = c * nz / kS0, z1 = ((c + 1) * nz + kS0 - 1) / kS0;
  double s = 0.0;
  for (int i = x0; i < x1; ++i)
    for (int j = y0; j < y1; ++j)
      for (int k = z0; k < z1; ++k) s += d[((int64_t)i * ny + j) * nz + k];
  out[idx] = (float)(s / ((double)(x1 - x0) * (y1 - y0) * (z1 - z0)));
}

}  // namespace
}  // namespace simpfem

using namespace simpfem;

struct simpfem_cnn {
  int max_batch = 0;
  int64_t step = 0;
  DevBuf theta, wbf, grad, m, v;
  DevBuf act[5];   // act[0] unused (the input is the caller's), act[1..4] layer outputs
  DevBuf dact[5];  // gradients of the layer outputs act[1..4] (dact[0] unused)
  DevBuf z, prob, loss_n, loss;
};

namespace {

void forward(simpfem_cnn* h, const float* x, const float* feats, const int32_t* labels, int N, cudaStream_t s) {
  to_bf16_kernel<<<div_up(kL.n, 256), 256, 0, s>>>(kL.n, h->theta.as<float>(), h->wbf.as<__nv_bfloat16>());
  SF_CUDA(sf_launched(1));
  const float* in = x;
  for (int l = 0; l < 4; ++l) {
    const int64_t total = (int64_t)N * kCout[l] * kSout[l] * kSout[l] * kSout[l];
    conv_fwd_kernel<<<div_up(total, 256), 256, 0, s>>>(
        N, kCin[l], kCout[l], kSin[l], kSout[l], kStride[l], in, h->wbf.as<__nv_bfloat16>() + kL.w[l],
        h->theta.as<float>() + kL.b[l], h->act[l + 1].as<float>());
    SF_CUDA(sf_launched(1));
    in = h->act[l + 1].as<float>();
  }
  head_fwd_kernel<<<div_up(N, 128), 128, 0, s>>>(N, h->act[4].as<float>(), feats,
                                                 h->wbf.as<__nv_bfloat16>() + kL.w[4], h->theta.as<float>() + kL.b[4],
                                                 labels, h->z.as<float>(), h->prob.as<float>(), h->loss_n.as<float>());
  SF_CUDA(sf_launched(1));
}

void backward(simpfem_cnn* h, const float* x, const int32_t* labels, int N, cudaStream_t s) {
  float* g = h->grad.as<float>();
  head_bwd_params_kernel<<<1, 128, 0, s>>>(N, h->prob.as<float>(), labels, h->z.as<float>(), g + kL.w[4],
                                          g + kL.b[4]);
  head_bwd_data_kernel<<<div_up(N * kHidden * 8, 256), 256, 0, s>>>(
      N, h->prob.as<float>(), labels, h->wbf.as<__nv_bfloat16>() + kL.w[4], h->dact[4].as<float>());
  SF_CUDA(sf_launched(2));
  for (int l = 3; l >= 0; --l) {
    const float* xin = l == 0 ? x : h->act[l].as<float>();
    const int nblk = kCout[l] * kCin[l] * 27 + kCout[l];
    conv_bwd_param_kernel<<<nblk, 256, 0, s>>>(N, kCin[l], kCout[l], kSin[l], kSout[l], kStride[l],
                                               h->dact[l + 1].as<float>(), h->act[l + 1].as<float>(), xin,
                                               g + kL.w[l], g + kL.b[l]);
    SF_CUDA(sf_launched(1));
    if (l > 0) {
      const int64_t total = (int64_t)N * kCin[l] * kSin[l] * kSin[l] * kSin[l];
      conv_bwd_data_kernel<<<div_up(total, 256), 256, 0, s>>>(
          N, kCin[l], kCout[l], kSin[l], kSout[l], kStride[l], h->dact[l + 1].as<float>(), h->act[l + 1].as<float>(),
          h->wbf.as<__nv_bfloat16>() + kL.w[l], h->dact[l].as<float>());
      SF_CUDA(sf_launched(1));
    }
  }
}

void check_batch(simpfem_cnn* h, int N) {
  if (N < 1 || N > h->max_batch) throw InvalidArg{"simpfem_cnn: batch size outside [1, max_batch]"};
}

}  // namespace

#define CNN_API_BEGIN try {
#define CNN_API_END                         \
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

extern "C" {

int simpfem_cnn_n_params(void) { return kL.n; }

int simpfem_cnn_create(int max_batch, simpfem_cnn** out) {
  CNN_API_BEGIN
  if (!out || max_batch < 1 || max_batch > 65536) throw InvalidArg{"simpfem_cnn_create: bad argument"};
  auto* h = new simpfem_cnn();
  try {
    h->max_batch = max_batch;
    h->theta.alloc(4 * kL.n);
    h->wbf.alloc(2 * kL.n);
    h->grad.alloc(4 * kL.n);
    h->m.alloc(4 * kL.n);
    h->v.alloc(4 * kL.n);
    SF_CUDA(cudaMemset(h->theta.p, 0, 4 * kL.n));
    SF_CUDA(cudaMemset(h->grad.p, 0, 4 * kL.n));
    SF_CUDA(cudaMemset(h->m.p, 0, 4 * kL.n));
    SF_CUDA(cudaMemset(h->v.p, 0, 4 * kL.n));
    for (int l = 0; l < 4; ++l) {
      const size_t sz = 4 * (size_t)max_batch * kCout[l] * kSout[l] * kSout[l] * kSout[l];
      h->act[l + 1].alloc(sz);
      h->dact[l + 1].alloc(sz);
    }
    h->z.alloc(4 * (size_t)max_batch * kZ);
    h->prob.alloc(4 * (size_t)max_batch * kClass);
    h->loss_n.alloc(4 * (size_t)max_batch);
    h->loss.alloc(4);
  } catch (...) {
    delete h;
    throw;
  }
  *out = h;
  CNN_API_END
}

int simpfem_cnn_destroy(simpfem_cnn* h) {
  delete h;
  return SIMPFEM_OK;
}

int simpfem_cnn_set_params(simpfem_cnn* h, const float* host, int n) {
  CNN_API_BEGIN
  if (!h || !host || n != kL.n) throw InvalidArg{"simpfem_cnn_set_params: bad argument"};
  SF_CUDA(cudaMemcpy(h->theta.p, host, 4 * (size_t)n, cudaMemcpyHostToDevice));
  SF_CUDA(cudaMemset(h->m.p, 0, 4 * kL.n));
  SF_CUDA(cudaMemset(h->v.p, 0, 4 * kL.n));
  h->step = 0;
  CNN_API_END
}

int simpfem_cnn_get_params(simpfem_cnn* h, float* host, int n) {
  CNN_API_BEGIN
  if (!h || !host || n != kL.n) throw InvalidArg{"simpfem_cnn_get_params: bad argument"};
  SF_CUDA(cudaMemcpy(host, h->theta.p, 4 * (size_t)n, cudaMemcpyDeviceToHost));
  CNN_API_END
}

int simpfem_cnn_pool16(int nx, int ny, int nz, const double* density, float* out, void* stream) {
  CNN_API_BEGIN
  if (nx < 1 || ny < 1 || nz < 1 || !density || !out) throw InvalidArg{"simpfem_cnn_pool16: bad argument"};
  if ((int64_t)nx * ny * nz > (int64_t)1 << 31 || (int64_t)(nx + 1) * kS0 > INT32_MAX)
    throw InvalidArg{"simpfem_cnn_pool16: grid too large"};
  pool16_kernel<<<div_up(kVox, 256), 256, 0, (cudaStream_t)stream>>>(nx, ny, nz, density, out);
  SF_CUDA(sf_launched(1));
  CNN_API_END
}

int simpfem_cnn_forward(simpfem_cnn* h, const float* x, const float* feats, int N, float* prob, void* stream) {
  CNN_API_BEGIN
  if (!h || !x || !feats || !prob) throw InvalidArg{"simpfem_cnn_forward: null argument"};
  check_batch(h, N);
  cudaStream_t s = (cudaStream_t)stream;
  forward(h, x, feats, nullptr, N, s);
  SF_CUDA(cudaMemcpyAsync(prob, h->prob.p, 4 * (size_t)N * kClass, cudaMemcpyDeviceToDevice, s));
  CNN_API_END
}

int simpfem_cnn_loss_grad(simpfem_cnn* h, const float* x, const float* feats, const int32_t* labels, int N,
                          float* grad_host, float* loss_host, void* stream) {
  CNN_API_BEGIN
  if (!h || !x || !feats || !labels) throw InvalidArg{"simpfem_cnn_loss_grad: null argument"};
  check_batch(h, N);
  cudaStream_t s = (cudaStream_t)stream;
  forward(h, x, feats, labels, N, s);
  backward(h, x, labels, N, s);
  loss_sum_kernel<<<1, 32, 0, s>>>(N, h->loss_n.as<float>(), h->loss.as<float>());
  SF_CUDA(sf_launched(1));
  if (loss_host) SF_CUDA(cudaMemcpyAsync(loss_host, h->loss.p, 4, cudaMemcpyDeviceToHost, s));
  if (grad_host) SF_CUDA(cudaMemcpyAsync(grad_host, h->grad.p, 4 * (size_t)kL.n, cudaMemcpyDeviceToHost, s));
  if (loss_host || grad_host) SF_CUDA(cudaStreamSynchronize(s));
  CNN_API_END
}

int simpfem_cnn_adam_step(simpfem_cnn* h, float lr, float beta1, float beta2, float eps, void* stream) {
  CNN_API_BEGIN
  if (!h) throw InvalidArg{"simpfem_cnn_adam_step: null handle"};
  h->step += 1;
  const float c1 = 1.f - powf(beta1, (float)h->step), c2 = 1.f - powf(beta2, (float)h->step);
  adam_kernel<<<div_up(kL.n, 256), 256, 0, (cudaStream_t)stream>>>(
      kL.n, h->theta.as<float>(), h->grad.as<float>(), h->m.as<float>(), h->v.as<float>(), lr, beta1, beta2, eps, c1,
      c2);
  SF_CUDA(sf_launched(1));
  CNN_API_END
}

}  // extern "C"
