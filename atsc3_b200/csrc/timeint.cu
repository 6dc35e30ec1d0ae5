// timeint.cu -- the time de-interleavers of A/322 7.1.4 / 7.1.5 fused into
// the demapper's cell load (sm_100a): each thread computes where its FEC
// Block cell sits in the received PLP cell stream, reads it (and its sigma2)
// from there, and demaps it exactly as demap.cu does (same float32 operation
// order, bit de-interleaver in the epilogue).  The de-interleaved cell array
// is never written.
//
// Index maps (restated from the reference receiver):
//  * Hybrid TI, twisted block de-interleaver (A/322 7.1.5.4;
//    lab/m6_tbi.py:75-88 fec_block, cached as one gather in
//    lab/m9_fast.py:1087-1093): in a TI block of Nr rows (cells per FEC
//    Block) and Nc columns (FEC Blocks), cell r of FEC Block j was sent at
//    position Nr * ((j - (r mod Nc)) mod Nc) + r; TI block t starts at
//    t * per_ti in the PLP stream.  Closed form for TI blocks without
//    virtual FEC Blocks; with virtual Blocks (and any other map) the caller
//    passes the index table.
//  * Convolutional TI (A/322 7.1.4; lab/m10_cti.py:97-100, 126-141): the
//    pre-CTI cell i leaves the interleaver at q = i + Nrows * ((start_row +
//    i) mod Nrows); FEC Block b's cell s is pre-CTI cell C + b*ncell + s.
// A cell whose source position lies outside the received stream (the
// convolutional interleaver's fill, an index -1 in a table) is an erasure:
// its LLRs are 0.

#include <cuda_runtime.h>

#include "../../include/atsc3_fec.h"
#include "common.cuh"
#include "demap_core.cuh"

namespace atsc3 {

struct GatherArgs {
  const float2 *cells;     // received PLP cell stream
  int64_t ncells;          // its length
  int nblk, ncell;
  const float *pts;
  int gmode;               // 0 table, 1 hybrid TI (twisted block), 2 CTI
  const int32_t *src;      // mode 0: (nblk, ncell) source positions, -1 = none
  int64_t p0, p1, p2;      // mode 1: stream offset, Nc, per_ti
                           // mode 2: C, Nrows, start_row
  int sigma_mode;          // 0 scalar, 1 per received cell, 2 per FEC Block
  const float *sigma2;
  float s2scalar;
  const int32_t *lam_of_q;
  float *out;
  int64_t ld_out;
};

__device__ __forceinline__ int64_t gather_source(const GatherArgs &a, int b,
                                                 int s) {
  if (a.gmode == 0) return (int64_t)__ldg(a.src + (size_t)b * a.ncell + s);
  if (a.gmode == 1) {
    const int nc = (int)a.p1;
    const int t = b / nc;
    const int j = b - t * nc;
    int k = j - s % nc;
    k += k < 0 ? nc : 0;
    return a.p0 + (int64_t)t * a.p2 + (int64_t)a.ncell * k + s;
  }
  const int64_t i = a.p0 + (int64_t)b * a.ncell + s;
  const int64_t r = (a.p2 + i) % a.p1;
  return i + a.p1 * r;
}

template <int NB>
__global__ void __launch_bounds__(256) demap_gather_kernel(const GatherArgs a) {
  constexpr int M = 1 << NB;
  extern __shared__ float sp[];
  float *spr = sp, *spi = sp + M, *sp2 = sp + 2 * M;
  for (int k = threadIdx.x; k < 3 * M; k += blockDim.x) sp[k] = a.pts[k];
  __syncthreads();
  const int64_t total = (int64_t)a.nblk * a.ncell;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int b = (int)(g / a.ncell);
    const int s = (int)(g - (int64_t)b * a.ncell);
    const int64_t src = gather_source(a, b, s);
    float *o = a.out + (size_t)b * a.ld_out;
    if (src < 0 || src >= a.ncells) {
#pragma unroll
      for (int i = 0; i < NB; ++i) {
        const int q = s * NB + i;
        o[a.lam_of_q ? __ldg(a.lam_of_q + q) : q] = 0.f;
      }
      continue;
    }
    const float2 z = a.cells[src];
    float mn[NB][2];
    cell_minima<NB>(z.x, z.y, spr, spi, sp2, mn, nullptr);
    float s2 = a.s2scalar;
    if (a.sigma_mode == 1) s2 = a.sigma2[src];
    else if (a.sigma_mode == 2) s2 = a.sigma2[b];
#pragma unroll
    for (int i = 0; i < NB; ++i) {
      const float d = __fdiv_rn(__fsub_rn(mn[i][1], mn[i][0]), s2);
      const int q = s * NB + i;
      o[a.lam_of_q ? __ldg(a.lam_of_q + q) : q] = d;
    }
  }
}

typedef void (*GatherFn)(const GatherArgs);

static GatherFn gather_fn(int nb) {
  switch (nb) {
    case 2: return demap_gather_kernel<2>;
    case 4: return demap_gather_kernel<4>;
    case 6: return demap_gather_kernel<6>;
    case 8: return demap_gather_kernel<8>;
    case 10: return demap_gather_kernel<10>;
    case 12: return demap_gather_kernel<12>;
  }
  return nullptr;
}

}  // namespace atsc3

extern "C" {

int32_t atsc3_demap_gather(const float *cells, int64_t ncells, int32_t nblk,
                           int32_t ncell, const float *pts, int32_t nbits,
                           int32_t gather_mode, const int32_t *src_index,
                           int64_t p0, int64_t p1, int64_t p2,
                           int32_t sigma_mode, const float *sigma2,
                           float sigma2_scalar, const int32_t *lam_of_q,
                           float *out, int64_t ld_out, void *stream) {
  using namespace atsc3;
  ATSC3_ARG(nblk >= 0 && ncell >= 0 && ncells >= 0, "negative size");
  ATSC3_ARG(gather_mode >= 0 && gather_mode <= 2, "gather_mode must be 0..2");
  ATSC3_ARG(sigma_mode >= 0 && sigma_mode <= 2, "sigma_mode must be 0..2");
  GatherFn fn = gather_fn(nbits);
  ATSC3_ARG(fn != nullptr, "nbits must be 2, 4, 6, 8, 10 or 12");
  if (nblk == 0 || ncell == 0) return 0;
  ATSC3_ARG(cells && pts && out, "null pointer");
  ATSC3_ARG(((uintptr_t)cells & 7) == 0, "cells must be 8-byte aligned");
  ATSC3_ARG(ld_out >= (int64_t)ncell * nbits, "ld_out < ncell*nbits");
  ATSC3_ARG(sigma_mode == 0 || sigma2 != nullptr, "sigma2 array required");
  if (gather_mode == 0) ATSC3_ARG(src_index != nullptr, "src_index required");
  if (gather_mode == 1) {
    ATSC3_ARG(p1 >= 1 && p0 >= 0, "hybrid TI needs Nc >= 1 and offset >= 0");
    ATSC3_ARG(p2 >= (int64_t)ncell * p1, "per_ti < Nr * Nc");
  }
  if (gather_mode == 2)
    ATSC3_ARG(p1 >= 1 && p0 >= 0 && p2 >= 0, "CTI needs Nrows >= 1, C >= 0, start_row >= 0");
  GatherArgs a;
  a.cells = (const float2 *)cells;
  a.ncells = ncells;
  a.nblk = nblk;
  a.ncell = ncell;
  a.pts = pts;
  a.gmode = gather_mode;
  a.src = src_index;
  a.p0 = p0;
  a.p1 = p1;
  a.p2 = p2;
  a.sigma_mode = sigma_mode;
  a.sigma2 = sigma2;
  a.s2scalar = sigma2_scalar;
  a.lam_of_q = lam_of_q;
  a.out = out;
  a.ld_out = ld_out;
  const int smem = 3 * (1 << nbits) * 4;
  if (smem > 48 * 1024)
    ATSC3_CUDA(cudaFuncSetAttribute((const void *)fn,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    smem));
  int dev = 0, sms = 148;
  ATSC3_CUDA(cudaGetDevice(&dev));
  ATSC3_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int64_t total = (int64_t)nblk * ncell;
  int64_t grid = (total + 255) / 256;
  if (grid > (int64_t)sms * 8) grid = (int64_t)sms * 8;
  fn<<<(unsigned)grid, 256, smem, (cudaStream_t)stream>>>(a);
  ATSC3_CUDA(cudaGetLastError());
  return 0;
}

}  // extern "C"
