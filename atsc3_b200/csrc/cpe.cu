// cpe.cu -- common phase error correction of an OFDM cell pool (sm_100a):
// the decision-directed per-symbol complex gain of lab/m6_cells.py:176-209
// (cpe_correct; the same algorithm as lab/m9_gpu.py:283-299 and
// lab/m9_fast.py:619-753), the stage before the demapper.
//
//   z = pool / sqrt(mean |pool|^2)
//   per OFDM symbol, `iters` times:
//     hard = nearest point of the cell's region alphabet (argmin |z - p|,
//            first minimum wins), or the known dummy value (region 2);
//     c = sum conj(hard)*z / max(sum |hard|^2, 1e-12);  z /= c;  gain *= c
//
// Float64 throughout.  One CTA per symbol (symbols are contiguous ranges of
// the pool); the alphabets sit in shared memory; the per-symbol sums are a
// fixed-order tree reduction, so results are deterministic.  Agreement with
// the numpy reference is to float64 rounding (its sums are BLAS dot products
// and numpy pairwise means, summed in other orders); hard decisions agree.

#include <cuda_runtime.h>

#include <algorithm>

#include "../../include/atsc3_fec.h"
#include "common.cuh"

namespace atsc3 {

constexpr int CPE_T = 256;

struct CpeArgs {
  const double2 *pool;
  int64_t n;
  const int32_t *sym_ptr;
  int nsym;
  const uint8_t *region;
  const double2 *alph0;
  int m0;
  const double2 *alph1;
  int m1;
  const double2 *dummy;
  int iters;
  double *work;          // [0]: sqrt(mean power); [1 ..]: power partials
  double2 *out;
  double2 *gains;
};

// Smith's algorithm for a / b (Smith, CACM 5(8), 1962), the form numpy's
// complex128 division uses
__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
  if (fabs(b.x) >= fabs(b.y)) {
    const double rat = b.y / b.x;
    const double scl = 1.0 / (b.x + b.y * rat);
    return make_double2((a.x + a.y * rat) * scl, (a.y - a.x * rat) * scl);
  }
  const double rat = b.x / b.y;
  const double scl = 1.0 / (b.y + b.x * rat);
  return make_double2((a.x * rat + a.y) * scl, (a.y * rat - a.x) * scl);
}

// per-block partial sums of |pool|^2 (hypot squared, as numpy's abs**2)
__global__ void __launch_bounds__(CPE_T) cpe_power_kernel(const CpeArgs a) {
  __shared__ double red[CPE_T];
  const int64_t per = (a.n + gridDim.x - 1) / gridDim.x;
  const int64_t lo = per * blockIdx.x;
  const int64_t hi = min(a.n, lo + per);
  double s = 0.0;
  for (int64_t i = lo + threadIdx.x; i < hi; i += CPE_T) {
    const double h = hypot(a.pool[i].x, a.pool[i].y);
    s += h * h;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = CPE_T / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) a.work[1 + blockIdx.x] = red[0];
}

__global__ void cpe_scale_kernel(const CpeArgs a, int nparts) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0.0;
    for (int b = 0; b < nparts; ++b) s += a.work[1 + b];
    a.work[0] = sqrt(s / (double)a.n);
  }
}

__global__ void __launch_bounds__(CPE_T) cpe_symbol_kernel(const CpeArgs a) {
  extern __shared__ double2 sp[];
  double2 *p0 = sp, *p1 = sp + a.m0;
  __shared__ double rnr[CPE_T], rni[CPE_T], rd[CPE_T];
  __shared__ double2 cshared;
  for (int k = threadIdx.x; k < a.m0; k += CPE_T) p0[k] = a.alph0[k];
  for (int k = threadIdx.x; k < a.m1; k += CPE_T) p1[k] = a.alph1[k];
  const int s = blockIdx.x;
  const int64_t lo = a.sym_ptr[s], hi = a.sym_ptr[s + 1];
  const double rt = a.work[0];
  // unit mean power over the whole pool
  for (int64_t i = lo + threadIdx.x; i < hi; i += CPE_T) {
    const double2 q = a.pool[i];
    a.out[i] = make_double2(q.x / rt, q.y / rt);
  }
  __syncthreads();
  double2 ctot = make_double2(1.0, 0.0);
  for (int it = 0; it < a.iters; ++it) {
    double nr = 0.0, ni = 0.0, dd = 0.0;
    for (int64_t i = lo + threadIdx.x; i < hi; i += CPE_T) {
      const double2 z = a.out[i];
      const int r = a.region[i];
      // region 0 / 1: nearest point of that alphabet; 2: the known dummy
      // value; anything else (or a missing table) contributes nothing
      double2 h = make_double2(0.0, 0.0);
      if (r == 2) {
        if (a.dummy) h = a.dummy[i];
      } else if (r < 2) {
        const double2 *p = r == 0 ? p0 : p1;
        const int m = r == 0 ? a.m0 : a.m1;
        if (m > 0) {
          double best = hypot(z.x - p[0].x, z.y - p[0].y);
          int bi = 0;
          for (int k = 1; k < m; ++k) {
            const double d = hypot(z.x - p[k].x, z.y - p[k].y);
            if (d < best) { best = d; bi = k; }
          }
          h = p[bi];
        }
      }
      nr += h.x * z.x + h.y * z.y;      // conj(h) * z
      ni += h.x * z.y - h.y * z.x;
      dd += h.x * h.x + h.y * h.y;
    }
    rnr[threadIdx.x] = nr;
    rni[threadIdx.x] = ni;
    rd[threadIdx.x] = dd;
    __syncthreads();
    for (int w = CPE_T / 2; w > 0; w >>= 1) {
      if ((int)threadIdx.x < w) {
        rnr[threadIdx.x] += rnr[threadIdx.x + w];
        rni[threadIdx.x] += rni[threadIdx.x + w];
        rd[threadIdx.x] += rd[threadIdx.x + w];
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      const double den = fmax(rd[0], 1e-12);
      cshared = make_double2(rnr[0] / den, rni[0] / den);
    }
    __syncthreads();
    const double2 c = cshared;
    for (int64_t i = lo + threadIdx.x; i < hi; i += CPE_T) a.out[i] = cdiv(a.out[i], c);
    ctot = make_double2(ctot.x * c.x - ctot.y * c.y, ctot.x * c.y + ctot.y * c.x);
    __syncthreads();
  }
  if (threadIdx.x == 0) a.gains[s] = ctot;
}

}  // namespace atsc3

extern "C" {

int32_t atsc3_cpe_workspace(int64_t *work_bytes) {
  ATSC3_ARG(work_bytes != nullptr, "null output");
  *work_bytes = (1 + 1024) * 8;
  return 0;
}

int32_t atsc3_cpe_correct(const double *pool, int64_t ncells,
                          const int32_t *sym_ptr, int32_t nsym,
                          const uint8_t *region, const double *alphabet0,
                          int32_t m0, const double *alphabet1, int32_t m1,
                          const double *dummy, int32_t iters, double *out,
                          double *gains, void *work, void *stream) {
  using namespace atsc3;
  ATSC3_ARG(ncells >= 0 && nsym >= 0 && iters >= 0, "negative size");
  ATSC3_ARG(m0 >= 1 && m1 >= 0 && m0 <= 4096 && m1 <= 4096,
            "alphabets of 1..4096 (and 0..4096) points");
  if (ncells == 0 || nsym == 0) return 0;
  ATSC3_ARG(pool && sym_ptr && region && alphabet0 && out && gains && work,
            "null pointer");
  ATSC3_ARG(m1 == 0 || alphabet1 != nullptr, "alphabet1 required");
  CpeArgs a;
  a.pool = (const double2 *)pool;
  a.n = ncells;
  a.sym_ptr = sym_ptr;
  a.nsym = nsym;
  a.region = region;
  a.alph0 = (const double2 *)alphabet0;
  a.m0 = m0;
  a.alph1 = (const double2 *)(alphabet1 ? alphabet1 : alphabet0);
  a.m1 = m1;
  a.dummy = (const double2 *)dummy;
  a.iters = iters;
  a.work = (double *)work;
  a.out = (double2 *)out;
  a.gains = (double2 *)gains;
  cudaStream_t st = (cudaStream_t)stream;
  const int nparts = (int)std::min<int64_t>(1024, (ncells + CPE_T - 1) / CPE_T);
  cpe_power_kernel<<<nparts, CPE_T, 0, st>>>(a);
  cpe_scale_kernel<<<1, 32, 0, st>>>(a, nparts);
  const int smem = (m0 + m1) * 16;
  if (smem > 48 * 1024)
    ATSC3_CUDA(cudaFuncSetAttribute((const void *)cpe_symbol_kernel,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    smem));
  cpe_symbol_kernel<<<nsym, CPE_T, smem, st>>>(a);
  ATSC3_CUDA(cudaGetLastError());
  return 0;
}

}  // extern "C"
