// Device helpers shared by the simpfem kernels.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "internal.h"

namespace simpfem {

// Explicitly rounded arithmetic: the vector updates mirror the reference's
// numpy/CuPy expressions operation by operation (one rounding per operator),
// so contraction into FMA is suppressed where the reference rounds twice.
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }

template <typename T>
__device__ __forceinline__ float to_f(T v) { return (float)v; }
template <>
__device__ __forceinline__ float to_f<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }

template <typename T>
__device__ __forceinline__ double to_d(T v) { return (double)v; }
template <>
__device__ __forceinline__ double to_d<__nv_bfloat16>(__nv_bfloat16 v) {
  return (double)__bfloat162float(v);
}

template <typename T>
__device__ __forceinline__ T from_d(double v) { return (T)v; }
template <>
__device__ __forceinline__ __nv_bfloat16 from_d<__nv_bfloat16>(double v) {
  return __float2bfloat16_rn((float)v);
}

__device__ __forceinline__ bool guard_off(const int* g) { return g != nullptr && *g == 0; }

// Per-DOF epilogue shared by the fine and coarse operators.
template <typename T, int EPI>
__device__ __forceinline__ void epilogue(const EpiArgs& ea, int64_t dof, bool free_dof, T ku, T x) {
  if (EPI == EPI_APPLY) {
    ((T*)ea.y)[dof] = free_dof ? ku : T(0);
  } else if (EPI == EPI_RESID) {
    ((T*)ea.y)[dof] = free_dof ? sub_rn(((const T*)ea.b)[dof], ku) : T(0);
  } else if (EPI == EPI_CHEB1) {
    if (free_dof) {
      T r = sub_rn(((const T*)ea.b)[dof], ku);
      T z = mul_rn(((const T*)ea.dinv)[dof], r);
      ((T*)ea.d)[dof] = z;
      ((T*)ea.xo)[dof] = add_rn(x, mul_rn((T)ea.s1, z));
    } else {
      ((T*)ea.d)[dof] = T(0);
      ((T*)ea.xo)[dof] = T(0);
    }
  } else if (EPI == EPI_CHEB) {
    if (free_dof) {
      T r = sub_rn(((const T*)ea.b)[dof], ku);
      T z = mul_rn(((const T*)ea.dinv)[dof], r);
      T dn = mul_rn((T)ea.s1, add_rn(z, mul_rn((T)ea.s2, ((T*)ea.d)[dof])));
      ((T*)ea.d)[dof] = dn;
      ((T*)ea.xo)[dof] = add_rn(x, dn);
    } else {
      ((T*)ea.d)[dof] = T(0);
      ((T*)ea.xo)[dof] = T(0);
    }
  } else if (EPI == EPI_JAC) {
    if (free_dof) {
      T r = sub_rn(((const T*)ea.b)[dof], ku);
      T w = mul_rn((T)ea.s1, ((const T*)ea.dinv)[dof]);
      ((T*)ea.xo)[dof] = add_rn(x, mul_rn(w, r));
    } else {
      ((T*)ea.xo)[dof] = T(0);
    }
  }
}

// The same per-DOF epilogues for the three DOFs of one node, with the operands
// read into registers by load() ahead of the element arithmetic so their
// latency overlaps it; apply() then evaluates exactly epilogue()'s expressions.
template <typename T, int EPI>
struct EpiOperands {
  bool fr[3];
  T b[3], di[3], dd[3];
  __device__ __forceinline__ void load(const EpiArgs& ea, int64_t dof0, const uint8_t* __restrict__ mask) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      fr[c] = mask[dof0 + c] != 0;
      if (EPI != EPI_APPLY) b[c] = ((const T*)ea.b)[dof0 + c];
      if (EPI == EPI_CHEB1 || EPI == EPI_CHEB || EPI == EPI_JAC) di[c] = ((const T*)ea.dinv)[dof0 + c];
      if (EPI == EPI_CHEB) dd[c] = ((const T*)ea.d)[dof0 + c];
    }
  }
  __device__ __forceinline__ void apply(const EpiArgs& ea, int64_t dof, int c, T ku, T x) const {
    if (EPI == EPI_APPLY) {
      ((T*)ea.y)[dof] = fr[c] ? ku : T(0);
    } else if (EPI == EPI_RESID) {
      ((T*)ea.y)[dof] = fr[c] ? sub_rn(b[c], ku) : T(0);
    } else if (EPI == EPI_CHEB1) {
      if (fr[c]) {
        const T z = mul_rn(di[c], sub_rn(b[c], ku));
        ((T*)ea.d)[dof] = z;
        ((T*)ea.xo)[dof] = add_rn(x, mul_rn((T)ea.s1, z));
      } else {
        ((T*)ea.d)[dof] = T(0);
        ((T*)ea.xo)[dof] = T(0);
      }
    } else if (EPI == EPI_CHEB) {
      if (fr[c]) {
        const T z = mul_rn(di[c], sub_rn(b[c], ku));
        const T dn = mul_rn((T)ea.s1, add_rn(z, mul_rn((T)ea.s2, dd[c])));
        ((T*)ea.d)[dof] = dn;
        ((T*)ea.xo)[dof] = add_rn(x, dn);
      } else {
        ((T*)ea.d)[dof] = T(0);
        ((T*)ea.xo)[dof] = T(0);
      }
    } else if (EPI == EPI_JAC) {
      if (fr[c]) {
        const T w = mul_rn((T)ea.s1, di[c]);
        ((T*)ea.xo)[dof] = add_rn(x, mul_rn(w, sub_rn(b[c], ku)));
      } else {
        ((T*)ea.xo)[dof] = T(0);
      }
    }
  }
};

inline int div_up(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

}  // namespace simpfem
