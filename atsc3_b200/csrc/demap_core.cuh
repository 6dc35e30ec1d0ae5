// demap_core.cuh -- the per-cell max-log arithmetic shared by the demapper
// kernels (demap.cu, timeint.cu): the point metric in the operation order of
// lab/m44_ldm.py:2447-2450 and the per-bit minima of :2483-2486.  Float32
// for the decode path; float64 for the drop-in of the reference's default
// float64 demap_llr_fast (lab/m16_demap_fast.py:80-119).
#pragma once

#include <cuda_runtime.h>

namespace atsc3 {

// Rounded-to-nearest arithmetic of one value type (no contraction).
template <typename T> struct DemapArith;
template <> struct DemapArith<float> {
  static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
  static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
  static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
  static __device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
  static __device__ __forceinline__ float min(float a, float b) { return fminf(a, b); }
  static __device__ __forceinline__ float inf() { return __int_as_float(0x7f800000); }
};
template <> struct DemapArith<double> {
  static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
  static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
  static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
  static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
  static __device__ __forceinline__ double min(double a, double b) { return fmin(a, b); }
  static __device__ __forceinline__ double inf() { return __longlong_as_double(0x7ff0000000000000ll); }
};

template <typename T>
__device__ __forceinline__ T point_metric(T zr, T zi, T pr, T pi, T p2) {
  using A = DemapArith<T>;
  T q = A::mul(zr, pr);
  q = A::add(q, A::mul(zi, pi));
  q = A::mul(q, (T)-2);
  return A::add(q, p2);
}

template <typename T> struct NoDeduce { using type = T; };

// min over the labels of one cell, split by each label bit.
// mn[i][b]: minimum of q over labels whose bit i (0 = MSB) equals b;
// *qmin (nullable) the minimum over all labels.
template <int NB, typename T = float>
__device__ __forceinline__ void cell_minima(T zr, T zi, const T *spr,
                                            const T *spi, const T *sp2,
                                            T (&mn)[NB][2],
                                            typename NoDeduce<T>::type *qmin) {
  using A = DemapArith<T>;
  constexpr int M = 1 << NB;
  constexpr int LB = NB < 4 ? NB : 4;   // label bits inside a block
  constexpr int BLK = 1 << LB;
  const T inf = A::inf();
#pragma unroll
  for (int i = 0; i < NB; ++i) mn[i][0] = mn[i][1] = inf;
  T all = inf;
  for (int k0 = 0; k0 < M; k0 += BLK) {
    T bmin = inf;
#pragma unroll
    for (int u = 0; u < BLK; ++u) {
      const int k = k0 + u;
      const T q = point_metric<T>(zr, zi, spr[k], spi[k], sp2[k]);
#pragma unroll
      for (int p = 0; p < LB; ++p) {       // label bit p <-> y index NB-1-p
        const int i = NB - 1 - p;
        if ((u >> p) & 1) mn[i][1] = A::min(mn[i][1], q);
        else mn[i][0] = A::min(mn[i][0], q);
      }
      bmin = A::min(bmin, q);
    }
#pragma unroll
    for (int p = LB; p < NB; ++p) {
      const int i = NB - 1 - p;
      if ((k0 >> p) & 1) mn[i][1] = A::min(mn[i][1], bmin);
      else mn[i][0] = A::min(mn[i][0], bmin);
    }
    all = A::min(all, bmin);
  }
  if (qmin) *qmin = all;
}

}  // namespace atsc3
