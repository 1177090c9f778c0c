// simpfem_true_residual_noalloc: the recomputed true-residual guard for callers
// that may not allocate device memory.
//
// Who needs it: a host framework that owns every byte of device memory through
// its own pool (an optimisation loop or a plugin host) may forbid raw
// cudaMalloc/cudaFree from the libraries it calls, because an allocation
// outside the pool bypasses its accounting and a cudaFree synchronises the whole
// device.  simpfem_true_residual keeps work buffers in the mesh handle and sizes
// them on first use; this variant takes full-layout vectors and a residual
// output from the caller and keeps its only scratch -- the per-block partial
// sums and the completion ticket of the deterministic reduction -- in a
// fixed-size array compiled into the library.
//
// Limits and sharing:
//  * at most kMaxDofs = 8,388,608 DOFs (4096 blocks x 2048 entries), i.e. about
//    2.7 million elements; larger meshes are rejected with SIMPFEM_EINVAL;
//  * the array (about 64 KB) is resident on every GPU that loads the library
//    until the process exits;
//  * every call on a device shares the one array: two calls whose kernels
//    overlap on that GPU (different streams, or threads racing) corrupt each
//    other's sums.  Serialise the calls per device.  The ticket is cleared at
//    the start of each call; the partials are fully rewritten by each call.
//  * the first call on a device looks up the array's device address with that
//    device current (cudaGetSymbolAddress) and caches it; make that first call
//    before any stream capture.
#include <math.h>

#include <cstring>
#include <mutex>

#include "gmg_impl.h"
#include "simpfem.h"

namespace {

constexpr int kNaThreads = 256;
constexpr int kNaPerThread = 8;
constexpr int kNaPerBlock = kNaThreads * kNaPerThread;  // 2048 entries per block
constexpr int kNaMaxBlocks = 4096;
constexpr int64_t kMaxDofs = (int64_t)kNaMaxBlocks * kNaPerBlock;
// layout: partials of |r|^2 [kNaMaxBlocks] | partials of |b|^2 [kNaMaxBlocks] | result[2] | ticket
constexpr size_t kScratchBytes = sizeof(double) * (2 * kNaMaxBlocks + 2) + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_na_mutex;
void* g_na_ptr[kMaxDevices] = {};

__device__ __forceinline__ double na_warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// |r|^2 and |b|^2 over the free DOFs (mask[i] != 0), with one partial per block
// and the last block summing the partials in block order (bitwise
// reproducible).  The residual is already zero at constrained DOFs; b is
// masked here so loads a caller leaves at constrained DOFs do not count, as in
// simpfem_true_residual, which compresses b to its free entries.
__global__ void __launch_bounds__(kNaThreads) na_norms_kernel(int64_t n, const double* __restrict__ r,
                                                              const double* __restrict__ b,
                                                              const uint8_t* __restrict__ mask,
                                                              unsigned char* scratch) {
  double* pr = reinterpret_cast<double*>(scratch);
  double* pb = pr + kNaMaxBlocks;
  double* res = pb + kNaMaxBlocks;
  unsigned* ticket = reinterpret_cast<unsigned*>(res + 2);
  __shared__ double sh[2][kNaThreads / 32];
  __shared__ bool last;
  const int64_t base = (int64_t)blockIdx.x * kNaPerBlock;
  double a = 0.0, c = 0.0;
#pragma unroll
  for (int k = 0; k < kNaPerThread; ++k) {
    const int64_t i = base + (int64_t)k * kNaThreads + threadIdx.x;
    if (i < n) {
      a += r[i] * r[i];
      if (mask[i]) c += b[i] * b[i];
    }
  }
  a = na_warp_sum(a);
  c = na_warp_sum(c);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
    sh[0][wid] = a;
    sh[1][wid] = c;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double sa = 0.0, sc = 0.0;
    for (int w = 0; w < kNaThreads / 32; ++w) {
      sa += sh[0][w];
      sc += sh[1][w];
    }
    pr[blockIdx.x] = sa;
    pb[blockIdx.x] = sc;
    __threadfence();
    last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    const volatile double* vr = pr;
    const volatile double* vb = pb;
    double sa = 0.0, sc = 0.0;
    for (int k = 0; k < (int)gridDim.x; ++k) {
      sa += vr[k];
      sc += vb[k];
    }
    res[0] = sa;
    res[1] = sc;
  }
}

// Device address of the scratch array for the current device (looked up once).
unsigned char* scratch_for_current_device() {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    simpfem::set_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    throw simpfem::CudaFailure(e);
  }
  if (dev < 0 || dev >= kMaxDevices) throw simpfem::InvalidArg{"simpfem_true_residual_noalloc: device index too large"};
  std::lock_guard<std::mutex> lk(g_na_mutex);
  if (g_na_ptr[dev] == nullptr) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      simpfem::set_error(std::string("cudaGetSymbolAddress(no-alloc scratch): ") + cudaGetErrorString(e));
      throw simpfem::CudaFailure(e != cudaSuccess ? e : cudaErrorInvalidSymbol);
    }
    g_na_ptr[dev] = p;
  }
  return static_cast<unsigned char*>(g_na_ptr[dev]);
}

}  // namespace

using namespace simpfem;

extern "C" int simpfem_true_residual_noalloc(simpfem_mesh* mh, const double* E, const double* b_full,
                                             const double* x_full, double* r_full, double* out_host,
                                             void* stream) {
  try {
    if (!mh || !E || !b_full || !x_full || !r_full || !out_host)
      throw InvalidArg{"simpfem_true_residual_noalloc: null argument"};
    Mesh& m = mh->impl;
    const int64_t n = m.g.ndof;
    if (n > kMaxDofs)
      throw InvalidArg{"simpfem_true_residual_noalloc: mesh has " + std::to_string(n) +
                       " DOFs, above the no-alloc maximum of " + std::to_string(kMaxDofs)};
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned char* scratch = scratch_for_current_device();
    double* res = reinterpret_cast<double*>(scratch) + 2 * kNaMaxBlocks;
    SF_CUDA(cudaMemsetAsync(res + 2, 0, sizeof(unsigned), s));
    EpiArgs ea;
    ea.y = r_full;
    ea.b = b_full;
    fine_apply(m, F64, EPI_RESID, E, x_full, ea, s);
    const int blocks = (int)((n + kNaPerBlock - 1) / kNaPerBlock);
    na_norms_kernel<<<blocks, kNaThreads, 0, s>>>(n, r_full, b_full, m.mask.as<uint8_t>(), scratch);
    SF_CUDA(sf_launched(1));
    double h[2];
    SF_CUDA(cudaMemcpyAsync(h, res, sizeof(h), cudaMemcpyDeviceToHost, s));
    SF_CUDA(cudaStreamSynchronize(s));
    *out_host = sqrt(h[0]) / sqrt(h[1]);
  } catch (const CudaFailure&) {
    return SIMPFEM_ECUDA;
  } catch (const InvalidArg& e) {
    set_error(e.msg);
    return SIMPFEM_EINVAL;
  } catch (const std::exception& e) {
    set_error(e.what());
    return SIMPFEM_EINTERNAL;
  }
  return SIMPFEM_OK;
}
