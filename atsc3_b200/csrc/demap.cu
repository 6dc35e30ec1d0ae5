// demap.cu -- NUC max-log soft demapper with the BICM bit de-interleaver
// fused into its epilogue (sm_100a).
//
// Reference semantics: lab/m44_ldm.py:2431-2494 (`_point_metric`,
// `demap_batch_qam`), the float32 form of lab/m6_bicm.py:213-225
// (`demap_llr`) and lab/m16_demap_fast.py:80-119 (`demap_llr_fast`):
//
//   q_k   = ((zr*pr_k + zi*pi_k) * -2) + |p_k|^2      every op rounded to f32
//   a_i   = min over labels with bit i = 1 of q_k       (y0 = MSB)
//   b_i   = min over labels with bit i = 0 of q_k
//   llr_i = (a_i - b_i) / sigma2                        IEEE f32 division
//   lam[lam_of_q[MOD*s + i]] = llr_i                    (lab/m9_fast.py:1120)
//
// The |z|^2 term common to every point cancels in a_i - b_i
// (lab/m16_demap_fast.py:27-58), so it is only used by the sigma2 estimator.
//
// Work split: one thread per cell; the alphabet (Re, Im, |p|^2, 3*M floats)
// is staged in shared memory; cells (float2) and per-cell sigma2 are read
// coalesced.  Per-bit minima: labels are walked in blocks of 16; the four
// low label bits are compile-time constants inside a block, the high bits
// are constant across it and take the block minimum once.  This is the
// point-distance work of K=2 -- no tensor-core shape.

#include <cuda_runtime.h>

#include "../../include/atsc3_fec.h"
#include "common.cuh"
#include "demap_core.cuh"

namespace atsc3 {

template <int NB>
__global__ void __launch_bounds__(256) demap_kernel(
    const float2 *__restrict__ cells, int64_t ld_cells, int nblk, int ncell,
    const float *__restrict__ pts, int sigma_mode,
    const float *__restrict__ sigma2, int64_t ld_sigma, float s2scalar,
    const int32_t *__restrict__ lam_of_q, float *__restrict__ out,
    int64_t ld_out) {
  constexpr int M = 1 << NB;
  extern __shared__ float sp[];
  float *spr = sp, *spi = sp + M, *sp2 = sp + 2 * M;
  for (int k = threadIdx.x; k < 3 * M; k += blockDim.x) sp[k] = pts[k];
  __syncthreads();
  const int64_t total = (int64_t)nblk * ncell;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int b = (int)(g / ncell);
    const int s = (int)(g - (int64_t)b * ncell);
    const float2 z = cells[(size_t)b * ld_cells + s];
    float mn[NB][2];
    cell_minima<NB>(z.x, z.y, spr, spi, sp2, mn, nullptr);
    float s2 = s2scalar;
    if (sigma_mode == 1) s2 = sigma2[(size_t)b * ld_sigma + s];
    else if (sigma_mode == 2) s2 = sigma2[b];
    float *o = out + (size_t)b * ld_out;
#pragma unroll
    for (int i = 0; i < NB; ++i) {
      float d = __fsub_rn(mn[i][1], mn[i][0]);
      if (sigma_mode != 3) d = __fdiv_rn(d, s2);
      const int q = s * NB + i;
      o[lam_of_q ? __ldg(lam_of_q + q) : q] = d;
    }
  }
}

// sigma2[b] = max(mean_s(|z|^2 + min_k q_k), 1e-9); float64 accumulation.
template <int NB>
__global__ void __launch_bounds__(256) row_sigma_kernel(
    const float2 *__restrict__ cells, int64_t ld_cells, int ncell,
    const float *__restrict__ pts, float *__restrict__ sigma2) {
  constexpr int M = 1 << NB;
  extern __shared__ float sp[];
  __shared__ double red[32];
  float *spr = sp, *spi = sp + M, *sp2 = sp + 2 * M;
  for (int k = threadIdx.x; k < 3 * M; k += blockDim.x) sp[k] = pts[k];
  __syncthreads();
  const int b = blockIdx.x;
  double acc = 0.0;
  for (int s = threadIdx.x; s < ncell; s += blockDim.x) {
    const float2 z = cells[(size_t)b * ld_cells + s];
    float mn[NB][2], qmin;
    cell_minima<NB>(z.x, z.y, spr, spi, sp2, mn, &qmin);
    const float z2 = __fadd_rn(__fmul_rn(z.x, z.x), __fmul_rn(z.y, z.y));
    acc += (double)__fadd_rn(z2, qmin);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    const float m = (float)(t / (double)ncell);
    sigma2[b] = fmaxf(m, 1e-9f);
  }
}

// ---- float64: the drop-in for the reference's default float64
// demap_llr_fast (lab/m16_demap_fast.py:80-119; m = |p|^2 - 2 Re(y p*), the
// per-bit minima, / sigma2).  Same work split, double arithmetic, cells as
// double2 (complex128), output in q order or through lam_of_q.
template <int NB>
__global__ void __launch_bounds__(256) demap_f64_kernel(
    const double2 *__restrict__ cells, int64_t ld_cells, int nblk, int ncell,
    const double *__restrict__ pts, int sigma_mode,
    const double *__restrict__ sigma2, int64_t ld_sigma, double s2scalar,
    const int32_t *__restrict__ lam_of_q, double *__restrict__ out,
    int64_t ld_out) {
  using A = DemapArith<double>;
  constexpr int M = 1 << NB;
  extern __shared__ double spd[];
  double *spr = spd, *spi = spd + M, *sp2 = spd + 2 * M;
  for (int k = threadIdx.x; k < 3 * M; k += blockDim.x) spd[k] = pts[k];
  __syncthreads();
  const int64_t total = (int64_t)nblk * ncell;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int b = (int)(g / ncell);
    const int s = (int)(g - (int64_t)b * ncell);
    const double2 z = cells[(size_t)b * ld_cells + s];
    double mn[NB][2];
    cell_minima<NB, double>(z.x, z.y, spr, spi, sp2, mn, nullptr);
    double s2 = s2scalar;
    if (sigma_mode == 1) s2 = sigma2[(size_t)b * ld_sigma + s];
    else if (sigma_mode == 2) s2 = sigma2[b];
    double *o = out + (size_t)b * ld_out;
#pragma unroll
    for (int i = 0; i < NB; ++i) {
      const double d = A::div(A::sub(mn[i][1], mn[i][0]), s2);
      const int q = s * NB + i;
      o[lam_of_q ? __ldg(lam_of_q + q) : q] = d;
    }
  }
}

// sigma2[b] = max(mean_s(|z|^2 + min_k q_k), 1e-9) in float64 (the estimate
// of lab/m16_demap_fast.py:104-106).
template <int NB>
__global__ void __launch_bounds__(256) row_sigma_f64_kernel(
    const double2 *__restrict__ cells, int64_t ld_cells, int ncell,
    const double *__restrict__ pts, double *__restrict__ sigma2) {
  using A = DemapArith<double>;
  constexpr int M = 1 << NB;
  extern __shared__ double spd[];
  __shared__ double red[32];
  double *spr = spd, *spi = spd + M, *sp2 = spd + 2 * M;
  for (int k = threadIdx.x; k < 3 * M; k += blockDim.x) spd[k] = pts[k];
  __syncthreads();
  const int b = blockIdx.x;
  double acc = 0.0;
  for (int s = threadIdx.x; s < ncell; s += blockDim.x) {
    const double2 z = cells[(size_t)b * ld_cells + s];
    double mn[NB][2], qmin;
    cell_minima<NB, double>(z.x, z.y, spr, spi, sp2, mn, &qmin);
    const double z2 = A::add(A::mul(z.x, z.x), A::mul(z.y, z.y));
    acc += A::add(z2, qmin);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    sigma2[b] = fmax(t / (double)ncell, 1e-9);
  }
}

typedef void (*DemapF64Fn)(const double2 *, int64_t, int, int, const double *,
                           int, const double *, int64_t, double,
                           const int32_t *, double *, int64_t);
typedef void (*SigmaF64Fn)(const double2 *, int64_t, int, const double *,
                           double *);

static DemapF64Fn demap_f64_fn(int nb) {
  switch (nb) {
    case 2: return demap_f64_kernel<2>;
    case 4: return demap_f64_kernel<4>;
    case 6: return demap_f64_kernel<6>;
    case 8: return demap_f64_kernel<8>;
    case 10: return demap_f64_kernel<10>;
    case 12: return demap_f64_kernel<12>;
  }
  return nullptr;
}

static SigmaF64Fn sigma_f64_fn(int nb) {
  switch (nb) {
    case 2: return row_sigma_f64_kernel<2>;
    case 4: return row_sigma_f64_kernel<4>;
    case 6: return row_sigma_f64_kernel<6>;
    case 8: return row_sigma_f64_kernel<8>;
    case 10: return row_sigma_f64_kernel<10>;
    case 12: return row_sigma_f64_kernel<12>;
  }
  return nullptr;
}

typedef void (*DemapFn)(const float2 *, int64_t, int, int, const float *, int,
                        const float *, int64_t, float, const int32_t *,
                        float *, int64_t);
typedef void (*SigmaFn)(const float2 *, int64_t, int, const float *, float *);

static DemapFn demap_fn(int nb) {
  switch (nb) {
    case 2: return demap_kernel<2>;
    case 4: return demap_kernel<4>;
    case 6: return demap_kernel<6>;
    case 8: return demap_kernel<8>;
    case 10: return demap_kernel<10>;
    case 12: return demap_kernel<12>;
  }
  return nullptr;
}

static SigmaFn sigma_fn(int nb) {
  switch (nb) {
    case 2: return row_sigma_kernel<2>;
    case 4: return row_sigma_kernel<4>;
    case 6: return row_sigma_kernel<6>;
    case 8: return row_sigma_kernel<8>;
    case 10: return row_sigma_kernel<10>;
    case 12: return row_sigma_kernel<12>;
  }
  return nullptr;
}

static int num_sms() {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
  }
  return sms;
}

int32_t demap_launch(const float *cells, int64_t ld_cells, int nblk, int ncell,
                     const float *pts, int nbits, int sigma_mode,
                     const float *sigma2, int64_t ld_sigma, float s2scalar,
                     const int32_t *lam_of_q, float *out, int64_t ld_out,
                     cudaStream_t st) {
  ATSC3_ARG(nblk >= 0 && ncell >= 0, "negative size");
  ATSC3_ARG(sigma_mode >= 0 && sigma_mode <= 3, "sigma_mode must be 0..3");
  DemapFn fn = demap_fn(nbits);
  ATSC3_ARG(fn != nullptr, "nbits must be 2, 4, 6, 8, 10 or 12");
  if (nblk == 0 || ncell == 0) return 0;
  ATSC3_ARG(cells && pts && out, "null pointer");
  ATSC3_ARG(ld_cells >= ncell, "ld_cells < ncell");
  ATSC3_ARG(ld_out >= (int64_t)ncell * nbits, "ld_out < ncell*nbits");
  ATSC3_ARG(((uintptr_t)cells & 7) == 0, "cells must be 8-byte aligned");
  ATSC3_ARG(!(sigma_mode == 1 || sigma_mode == 2) || sigma2 != nullptr,
            "sigma2 array required");
  ATSC3_ARG(sigma_mode != 1 || ld_sigma >= ncell, "ld_sigma < ncell");
  const int smem = 3 * (1 << nbits) * 4;
  if (smem > 48 * 1024)
    ATSC3_CUDA(cudaFuncSetAttribute((const void *)fn,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    smem));
  const int64_t total = (int64_t)nblk * ncell;
  int64_t grid = (total + 255) / 256;
  const int64_t cap = (int64_t)num_sms() * 8;
  if (grid > cap) grid = cap;
  fn<<<(unsigned)grid, 256, smem, st>>>((const float2 *)cells, ld_cells, nblk,
                                        ncell, pts, sigma_mode, sigma2,
                                        ld_sigma, s2scalar, lam_of_q, out,
                                        ld_out);
  ATSC3_CUDA(cudaGetLastError());
  return 0;
}

int32_t demap_f64_launch(const double *cells, int64_t ld_cells, int nblk,
                         int ncell, const double *pts, int nbits,
                         int sigma_mode, const double *sigma2,
                         int64_t ld_sigma, double s2scalar,
                         const int32_t *lam_of_q, double *out, int64_t ld_out,
                         cudaStream_t st) {
  ATSC3_ARG(nblk >= 0 && ncell >= 0, "negative size");
  ATSC3_ARG(sigma_mode >= 0 && sigma_mode <= 2, "sigma_mode must be 0..2");
  DemapF64Fn fn = demap_f64_fn(nbits);
  ATSC3_ARG(fn != nullptr, "nbits must be 2, 4, 6, 8, 10 or 12");
  if (nblk == 0 || ncell == 0) return 0;
  ATSC3_ARG(cells && pts && out, "null pointer");
  ATSC3_ARG(ld_cells >= ncell, "ld_cells < ncell");
  ATSC3_ARG(ld_out >= (int64_t)ncell * nbits, "ld_out < ncell*nbits");
  ATSC3_ARG(((uintptr_t)cells & 15) == 0, "cells must be 16-byte aligned");
  ATSC3_ARG(sigma_mode == 0 || sigma2 != nullptr, "sigma2 array required");
  ATSC3_ARG(sigma_mode != 1 || ld_sigma >= ncell, "ld_sigma < ncell");
  const int smem = 3 * (1 << nbits) * 8;
  if (smem > 48 * 1024)
    ATSC3_CUDA(cudaFuncSetAttribute((const void *)fn,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    smem));
  const int64_t total = (int64_t)nblk * ncell;
  int64_t grid = (total + 255) / 256;
  const int64_t cap = (int64_t)num_sms() * 8;
  if (grid > cap) grid = cap;
  fn<<<(unsigned)grid, 256, smem, st>>>((const double2 *)cells, ld_cells, nblk,
                                        ncell, pts, sigma_mode, sigma2,
                                        ld_sigma, s2scalar, lam_of_q, out,
                                        ld_out);
  ATSC3_CUDA(cudaGetLastError());
  return 0;
}

int32_t row_sigma_f64_launch(const double *cells, int64_t ld_cells, int nblk,
                             int ncell, const double *pts, int nbits,
                             double *sigma2, cudaStream_t st) {
  SigmaF64Fn fn = sigma_f64_fn(nbits);
  ATSC3_ARG(fn != nullptr, "nbits must be 2, 4, 6, 8, 10 or 12");
  ATSC3_ARG(nblk >= 0 && ncell > 0, "bad size");
  if (nblk == 0) return 0;
  ATSC3_ARG(cells && pts && sigma2, "null pointer");
  ATSC3_ARG(ld_cells >= ncell, "ld_cells < ncell");
  ATSC3_ARG(((uintptr_t)cells & 15) == 0, "cells must be 16-byte aligned");
  const int smem = 3 * (1 << nbits) * 8;
  if (smem > 48 * 1024)
    ATSC3_CUDA(cudaFuncSetAttribute((const void *)fn,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    smem));
  fn<<<nblk, 256, smem, st>>>((const double2 *)cells, ld_cells, ncell, pts,
                              sigma2);
  ATSC3_CUDA(cudaGetLastError());
  return 0;
}

int32_t row_sigma_launch(const float *cells, int64_t ld_cells, int nblk,
                         int ncell, const float *pts, int nbits, float *sigma2,
                         cudaStream_t st) {
  SigmaFn fn = sigma_fn(nbits);
  ATSC3_ARG(fn != nullptr, "nbits must be 2, 4, 6, 8, 10 or 12");
  ATSC3_ARG(nblk >= 0 && ncell > 0, "bad size");
  if (nblk == 0) return 0;
  ATSC3_ARG(cells && pts && sigma2, "null pointer");
  ATSC3_ARG(((uintptr_t)cells & 7) == 0, "cells must be 8-byte aligned");
  const int smem = 3 * (1 << nbits) * 4;
  if (smem > 48 * 1024)
    ATSC3_CUDA(cudaFuncSetAttribute((const void *)fn,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    smem));
  fn<<<nblk, 256, smem, st>>>((const float2 *)cells, ld_cells, ncell, pts,
                              sigma2);
  ATSC3_CUDA(cudaGetLastError());
  return 0;
}

// ---- uneven batches: every block its own constellation ---------------------
// One CTA per chunk of up to 256 cells of one block (chunk_blk / chunk_start
// built on the host); the CTA stages its block's alphabet (up to 4096
// points) and dispatches on the block's bits per symbol.
struct DemapBatchArgs {
  const float2 *cells;
  const int64_t *cell_off;
  const int32_t *ncell;
  const int32_t *nbits;
  const float *pts;
  const int64_t *pts_off;     // floats, 3*M per alphabet
  const float *sigma2;        // one per block
  const int32_t *lq;
  const int64_t *lq_off;
  float *llr;
  const int64_t *llr_off;
  const int32_t *chunk_blk;
  const int32_t *chunk_start;
};

template <int NB>
__device__ __forceinline__ void demap_cell_batch(const DemapBatchArgs &a, int b,
                                                 int s, const float *sp) {
  constexpr int M = 1 << NB;
  const float2 z = a.cells[a.cell_off[b] + s];
  float mn[NB][2];
  cell_minima<NB>(z.x, z.y, sp, sp + M, sp + 2 * M, mn, nullptr);
  const float s2 = a.sigma2[b];
  const int32_t *lq = a.lq + a.lq_off[b];
  float *o = a.llr + a.llr_off[b];
#pragma unroll
  for (int i = 0; i < NB; ++i)
    o[__ldg(lq + s * NB + i)] = __fdiv_rn(__fsub_rn(mn[i][1], mn[i][0]), s2);
}

__global__ void __launch_bounds__(256) demap_batch_kernel(const DemapBatchArgs a) {
  extern __shared__ float sp[];
  const int b = a.chunk_blk[blockIdx.x];
  const int s = a.chunk_start[blockIdx.x] + threadIdx.x;
  const int nb = a.nbits[b];
  const int M3 = 3 << nb;
  const float *src = a.pts + a.pts_off[b];
  for (int k = threadIdx.x; k < M3; k += blockDim.x) sp[k] = src[k];
  __syncthreads();
  if (s >= a.ncell[b]) return;
  switch (nb) {
    case 2: demap_cell_batch<2>(a, b, s, sp); break;
    case 4: demap_cell_batch<4>(a, b, s, sp); break;
    case 6: demap_cell_batch<6>(a, b, s, sp); break;
    case 8: demap_cell_batch<8>(a, b, s, sp); break;
    case 10: demap_cell_batch<10>(a, b, s, sp); break;
    case 12: demap_cell_batch<12>(a, b, s, sp); break;
  }
}

}  // namespace atsc3

extern "C" {

int32_t atsc3_demap_batch(const float *cells, const int64_t *cell_off,
                          const int32_t *ncell, const int32_t *nbits,
                          const float *pts, const int64_t *pts_off,
                          const float *sigma2, const int32_t *lq,
                          const int64_t *lq_off, float *llr,
                          const int64_t *llr_off, const int32_t *chunk_blk,
                          const int32_t *chunk_start, int32_t nchunks,
                          int32_t max_nbits, void *stream) {
  using namespace atsc3;
  ATSC3_ARG(nchunks >= 0, "negative size");
  if (nchunks == 0) return 0;
  ATSC3_ARG(cells && cell_off && ncell && nbits && pts && pts_off && sigma2 &&
                lq && lq_off && llr && llr_off && chunk_blk && chunk_start,
            "null pointer");
  ATSC3_ARG(max_nbits >= 2 && max_nbits <= 12, "max_nbits must be 2..12");
  const int smem = 3 * (1 << max_nbits) * 4;
  if (smem > 48 * 1024)
    ATSC3_CUDA(cudaFuncSetAttribute((const void *)demap_batch_kernel,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  DemapBatchArgs a{(const float2 *)cells, cell_off, ncell, nbits, pts, pts_off,
                   sigma2, lq, lq_off, llr, llr_off, chunk_blk, chunk_start};
  demap_batch_kernel<<<nchunks, 256, smem, (cudaStream_t)stream>>>(a);
  ATSC3_CUDA(cudaGetLastError());
  return 0;
}


int32_t atsc3_demap(const float *cells, int64_t ld_cells, int32_t nblk,
                    int32_t ncell, const float *pts, int32_t nbits,
                    int32_t sigma_mode, const float *sigma2, int64_t ld_sigma,
                    float sigma2_scalar, const int32_t *lam_of_q, float *out,
                    int64_t ld_out, void *stream) {
  return atsc3::demap_launch(cells, ld_cells, nblk, ncell, pts, nbits,
                             sigma_mode, sigma2, ld_sigma, sigma2_scalar,
                             lam_of_q, out, ld_out, (cudaStream_t)stream);
}

int32_t atsc3_demap_f64(const double *cells, int64_t ld_cells, int32_t nblk,
                        int32_t ncell, const double *pts, int32_t nbits,
                        int32_t sigma_mode, const double *sigma2,
                        int64_t ld_sigma, double sigma2_scalar,
                        const int32_t *lam_of_q, double *out, int64_t ld_out,
                        void *stream) {
  return atsc3::demap_f64_launch(cells, ld_cells, nblk, ncell, pts, nbits,
                                 sigma_mode, sigma2, ld_sigma, sigma2_scalar,
                                 lam_of_q, out, ld_out, (cudaStream_t)stream);
}

int32_t atsc3_demap_row_sigma2_f64(const double *cells, int64_t ld_cells,
                                   int32_t nblk, int32_t ncell,
                                   const double *pts, int32_t nbits,
                                   double *sigma2, void *stream) {
  return atsc3::row_sigma_f64_launch(cells, ld_cells, nblk, ncell, pts, nbits,
                                     sigma2, (cudaStream_t)stream);
}

int32_t atsc3_demap_row_sigma2(const float *cells, int64_t ld_cells,
                               int32_t nblk, int32_t ncell, const float *pts,
                               int32_t nbits, float *sigma2, void *stream) {
  return atsc3::row_sigma_launch(cells, ld_cells, nblk, ncell, pts, nbits,
                                 sigma2, (cudaStream_t)stream);
}

}  // extern "C"
