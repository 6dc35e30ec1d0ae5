// demap_core.cuh -- the per-cell max-log arithmetic shared by the demapper
// kernels (demap.cu, timeint.cu): the point metric in the operation order of
// lab/m44_ldm.py:2447-2450 and the per-bit minima of :2483-2486.
#pragma once

#include <cuda_runtime.h>

namespace atsc3 {

__device__ __forceinline__ float point_metric(float zr, float zi, float pr,
                                              float pi, float p2) {
  float q = __fmul_rn(zr, pr);
  q = __fadd_rn(q, __fmul_rn(zi, pi));
  q = __fmul_rn(q, -2.0f);
  return __fadd_rn(q, p2);
}

// min over the labels of one cell, split by each label bit.
// mn[i][b]: minimum of q over labels whose bit i (0 = MSB) equals b.
template <int NB>
__device__ __forceinline__ void cell_minima(float zr, float zi,
                                            const float *spr, const float *spi,
                                            const float *sp2, float (&mn)[NB][2],
                                            float *qmin) {
  constexpr int M = 1 << NB;
  constexpr int LB = NB < 4 ? NB : 4;   // label bits inside a block
  constexpr int BLK = 1 << LB;
  const float inf = __int_as_float(0x7f800000);
#pragma unroll
  for (int i = 0; i < NB; ++i) mn[i][0] = mn[i][1] = inf;
  float all = inf;
  for (int k0 = 0; k0 < M; k0 += BLK) {
    float bmin = inf;
#pragma unroll
    for (int u = 0; u < BLK; ++u) {
      const int k = k0 + u;
      const float q = point_metric(zr, zi, spr[k], spi[k], sp2[k]);
#pragma unroll
      for (int p = 0; p < LB; ++p) {       // label bit p <-> y index NB-1-p
        const int i = NB - 1 - p;
        if ((u >> p) & 1) mn[i][1] = fminf(mn[i][1], q);
        else mn[i][0] = fminf(mn[i][0], q);
      }
      bmin = fminf(bmin, q);
    }
#pragma unroll
    for (int p = LB; p < NB; ++p) {
      const int i = NB - 1 - p;
      if ((k0 >> p) & 1) mn[i][1] = fminf(mn[i][1], bmin);
      else mn[i][0] = fminf(mn[i][0], bmin);
    }
    all = fminf(all, bmin);
  }
  if (qmin) *qmin = all;
}

}  // namespace atsc3
