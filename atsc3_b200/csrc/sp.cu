// sp.cu -- exact (log-tanh) sum-product decoding in float64 for the blocks
// min-sum could not close (sm_100a): the near-miss rescue of the reference
// receiver, lab/m16_margin.py:325-390 (sum_product_decode_batch), called from
// lab/m44_ldm.py:2527-2554 on rows whose unsatisfied-check count is small.
//
// Per iteration (it = 0 .. iters), for every block still decoding:
//   syndrome of tot (hard decision tot < 0); zero -> converged at `it`;
//   it == iters -> stop with the current decisions;
//   else per check, per edge e:  v = tot[var(e)] - m[e],
//        t = tanh(clip(v, -38, 38) / 2), parity of (t < 0),
//        lt = log(clip(|t|, 1e-300, 1)), lsum = sum of lt over the check,
//        m[e] = +-2 atanh(clip(exp(clip(lsum - lt, -700, -1e-16)), 0,
//               1 - 1e-16)), negative when parity ^ (t < 0);
//   per variable: tot = llr + sum of its messages in ascending check order.
// tanh, log, exp and atanh are CUDA's float64 functions (not restated); the
// messages agree with the numpy float64 reference to rounding, the decisions
// (bits, convergence, iteration) are what the tests compare.
//
// Launch shape: one thread per (block, check) and per (block, bit); four
// launches per iteration on the caller's stream; a block that has finished
// is skipped by every kernel.  This path runs on a handful of blocks per
// frame, so it is not on the throughput-critical path.

#include <cuda_runtime.h>

#include "../../include/atsc3_fec.h"
#include "common.cuh"

namespace atsc3 {

struct SpArgs {
  const int32_t *cptr, *cidx, *vptr, *vedge;
  int n, nc, nedges, nblk, iters;
  const double *llr;
  int64_t ld_llr;
  double *tot;       // (nblk, n)
  double *msg;       // (nblk, nedges)
  int32_t *st;       // [0, nblk): active (1) / done (0); [nblk, 2nblk): bad
                     // accumulator; [2nblk, 3nblk): iteration a block ended
  uint8_t *bits;
  int64_t ld_bits;
  uint8_t *conv;
  int32_t *its;
  int32_t *bad;
};

__global__ void __launch_bounds__(256) sp_init_kernel(const SpArgs a) {
  const int64_t total = (int64_t)a.nblk * a.n;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int b = (int)(g / a.n);
    const int v = (int)(g - (int64_t)b * a.n);
    a.tot[g] = a.llr[(size_t)b * a.ld_llr + v];
  }
  const int64_t te = (int64_t)a.nblk * a.nedges;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < te;
       g += (int64_t)gridDim.x * blockDim.x)
    a.msg[g] = 0.0;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < a.nblk;
       g += (int64_t)gridDim.x * blockDim.x) {
    a.st[g] = 1;
    a.st[a.nblk + g] = 0;
    a.st[2 * a.nblk + g] = -1;
  }
}

__device__ __forceinline__ double sp_t(double v) {
  const double x = fmin(fmax(v, -38.0), 38.0) * 0.5;
  return tanh(x);
}

__device__ __forceinline__ double sp_lt(double t) {
  return log(fmin(fmax(fabs(t), 1e-300), 1.0));
}

// syndrome of tot and (upd) the check update, one thread per (block, check)
__global__ void __launch_bounds__(256) sp_check_kernel(const SpArgs a, int upd) {
  const int64_t total = (int64_t)a.nblk * a.nc;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int b = (int)(g / a.nc);
    if (!a.st[b]) continue;
    const int c = (int)(g - (int64_t)b * a.nc);
    const int e0 = __ldg(a.cptr + c), e1 = __ldg(a.cptr + c + 1);
    const double *tot = a.tot + (size_t)b * a.n;
    double *m = a.msg + (size_t)b * a.nedges;
    int syn = 0, par = 0;
    double lsum = 0.0;
    for (int e = e0; e < e1; ++e) {
      const double tv = tot[__ldg(a.cidx + e)];
      syn ^= tv < 0.0 ? 1 : 0;
      if (upd) {
        const double t = sp_t(tv - m[e]);
        par ^= t < 0.0 ? 1 : 0;
        lsum += sp_lt(t);
      }
    }
    if (syn) atomicAdd(a.st + a.nblk + b, 1);
    if (!upd) continue;
    for (int e = e0; e < e1; ++e) {
      const double tv = tot[__ldg(a.cidx + e)];
      const double t = sp_t(tv - m[e]);
      const double le = fmin(fmax(lsum - sp_lt(t), -700.0), -1e-16);
      const double mag = fmin(fmax(exp(le), 0.0), 1.0 - 1e-16);
      const double mn = 2.0 * atanh(mag);
      m[e] = (par ^ (t < 0.0 ? 1 : 0)) ? -mn : mn;
    }
  }
}

// per block: converged (zero syndrome) or out of iterations.  counts
// (nullable, one CTA launch): [0] blocks still decoding after this
// iteration, [1] blocks stopped unconverged at this iteration.
__global__ void sp_status_kernel(const SpArgs a, int it, int32_t *counts) {
  __shared__ int s_act, s_stop;
  if (threadIdx.x == 0) {
    s_act = 0;
    s_stop = 0;
  }
  __syncthreads();
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < a.nblk;
       b += gridDim.x * blockDim.x) {
    if (!a.st[b]) continue;
    const int badct = a.st[a.nblk + b];
    a.st[a.nblk + b] = 0;
    if (badct == 0 || it >= a.iters) {
      a.st[b] = 0;
      a.st[2 * a.nblk + b] = it;
      a.conv[b] = badct == 0 ? 1 : 0;
      a.its[b] = it;
      a.bad[b] = badct;
      if (badct) atomicAdd(&s_stop, 1);
    } else {
      atomicAdd(&s_act, 1);
    }
  }
  __syncthreads();
  if (counts && threadIdx.x == 0 && blockIdx.x == 0) {
    counts[0] = s_act;
    counts[1] = s_stop;
  }
}

// hard decisions of the blocks that ended at this iteration
__global__ void __launch_bounds__(256) sp_bits_kernel(const SpArgs a, int it) {
  const int64_t total = (int64_t)a.nblk * a.n;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int b = (int)(g / a.n);
    if (a.st[2 * a.nblk + b] != it) continue;
    const int v = (int)(g - (int64_t)b * a.n);
    a.bits[(size_t)b * a.ld_bits + v] = a.tot[g] < 0.0 ? 1 : 0;
  }
}

// tot = llr + messages in ascending check order (vedge), still-active blocks
__global__ void __launch_bounds__(256) sp_var_kernel(const SpArgs a) {
  const int64_t total = (int64_t)a.nblk * a.n;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int b = (int)(g / a.n);
    if (!a.st[b]) continue;
    const int v = (int)(g - (int64_t)b * a.n);
    const double *m = a.msg + (size_t)b * a.nedges;
    double s = a.llr[(size_t)b * a.ld_llr + v];
    const int k1 = __ldg(a.vptr + v + 1);
    for (int k = __ldg(a.vptr + v); k < k1; ++k) s += m[__ldg(a.vedge + k)];
    a.tot[g] = s;
  }
}

}  // namespace atsc3

extern "C" {

int32_t atsc3_ldpc_sp_workspace(int32_t n, int32_t nedges, int32_t nblk,
                                int64_t *work_bytes) {
  ATSC3_ARG(work_bytes != nullptr, "null output");
  ATSC3_ARG(n > 0 && nedges > 0 && nblk >= 0, "bad size");
  *work_bytes = (int64_t)nblk * ((int64_t)n + nedges) * 8 + (int64_t)nblk * 12;
  return 0;
}

int32_t atsc3_ldpc_sp_decode(const int32_t *cptr, const int32_t *cidx,
                             const int32_t *vptr, const int32_t *vedge,
                             int32_t n, int32_t nc, int32_t nedges,
                             const double *llr, int64_t ld_llr, int32_t nblk,
                             int32_t iters, uint8_t *bits, int64_t ld_bits,
                             uint8_t *conv, int32_t *its, int32_t *bad,
                             void *work, void *stream) {
  using namespace atsc3;
  ATSC3_ARG(n > 0 && nc > 0 && nedges > 0 && nblk >= 0 && iters >= 0, "bad size");
  if (nblk == 0) return 0;
  ATSC3_ARG(cptr && cidx && vptr && vedge && llr && bits && conv && its && bad && work,
            "null pointer");
  ATSC3_ARG(ld_llr >= n && ld_bits >= n, "leading dimension below n");
  ATSC3_ARG(((uintptr_t)work & 7) == 0 && ((uintptr_t)llr & 7) == 0,
            "llr and work must be 8-byte aligned");
  SpArgs a;
  a.cptr = cptr;
  a.cidx = cidx;
  a.vptr = vptr;
  a.vedge = vedge;
  a.n = n;
  a.nc = nc;
  a.nedges = nedges;
  a.nblk = nblk;
  a.iters = iters;
  a.llr = llr;
  a.ld_llr = ld_llr;
  a.tot = (double *)work;
  a.msg = a.tot + (size_t)nblk * n;
  a.st = (int32_t *)(a.msg + (size_t)nblk * nedges);
  a.bits = bits;
  a.ld_bits = ld_bits;
  a.conv = conv;
  a.its = its;
  a.bad = bad;
  cudaStream_t st = (cudaStream_t)stream;
  int dev = 0, sms = 148;
  ATSC3_CUDA(cudaGetDevice(&dev));
  ATSC3_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  auto grid = [&](int64_t work_items) {
    int64_t g = (work_items + 255) / 256;
    const int64_t cap = (int64_t)sms * 16;
    return (unsigned)(g < 1 ? 1 : (g > cap ? cap : g));
  };
  sp_init_kernel<<<grid((int64_t)nblk * (n > nedges ? n : nedges)), 256, 0, st>>>(a);
  for (int it = 0; it <= iters; ++it) {
    const int upd = it < iters ? 1 : 0;
    sp_check_kernel<<<grid((int64_t)nblk * nc), 256, 0, st>>>(a, upd);
    sp_status_kernel<<<1, 256, 0, st>>>(a, it, nullptr);
    sp_bits_kernel<<<grid((int64_t)nblk * n), 256, 0, st>>>(a, it);
    if (upd) sp_var_kernel<<<grid((int64_t)nblk * n), 256, 0, st>>>(a);
  }
  ATSC3_CUDA(cudaGetLastError());
  return 0;
}

int32_t atsc3_ldpc_sp_step(const int32_t *cptr, const int32_t *cidx,
                           const int32_t *vptr, const int32_t *vedge,
                           int32_t n, int32_t nc, int32_t nedges,
                           const double *llr, int64_t ld_llr, int32_t nblk,
                           int32_t it, int32_t last, uint8_t *bits,
                           int64_t ld_bits, uint8_t *conv, int32_t *its,
                           int32_t *bad, void *work, int32_t *counts,
                           void *stream) {
  using namespace atsc3;
  ATSC3_ARG(n > 0 && nc > 0 && nedges > 0 && nblk >= 0 && it >= 0, "bad size");
  if (nblk == 0) return 0;
  ATSC3_ARG(cptr && cidx && vptr && vedge && llr && bits && conv && its && bad &&
                work && counts, "null pointer");
  ATSC3_ARG(ld_llr >= n && ld_bits >= n, "leading dimension below n");
  ATSC3_ARG(((uintptr_t)work & 7) == 0 && ((uintptr_t)llr & 7) == 0,
            "llr and work must be 8-byte aligned");
  SpArgs a;
  a.cptr = cptr;
  a.cidx = cidx;
  a.vptr = vptr;
  a.vedge = vedge;
  a.n = n;
  a.nc = nc;
  a.nedges = nedges;
  a.nblk = nblk;
  // the last step retires every block still decoding (as iteration `iters`
  // of a full decode does); any other step retires only converged blocks
  a.iters = last ? it : it + 1;
  a.llr = llr;
  a.ld_llr = ld_llr;
  a.tot = (double *)work;
  a.msg = a.tot + (size_t)nblk * n;
  a.st = (int32_t *)(a.msg + (size_t)nblk * nedges);
  a.bits = bits;
  a.ld_bits = ld_bits;
  a.conv = conv;
  a.its = its;
  a.bad = bad;
  cudaStream_t st = (cudaStream_t)stream;
  int dev = 0, sms = 148;
  ATSC3_CUDA(cudaGetDevice(&dev));
  ATSC3_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  auto grid = [&](int64_t work_items) {
    int64_t g = (work_items + 255) / 256;
    const int64_t cap = (int64_t)sms * 16;
    return (unsigned)(g < 1 ? 1 : (g > cap ? cap : g));
  };
  if (it == 0)
    sp_init_kernel<<<grid((int64_t)nblk * (n > nedges ? n : nedges)), 256, 0, st>>>(a);
  const int upd = last ? 0 : 1;
  sp_check_kernel<<<grid((int64_t)nblk * nc), 256, 0, st>>>(a, upd);
  sp_status_kernel<<<1, 256, 0, st>>>(a, it, counts);
  sp_bits_kernel<<<grid((int64_t)nblk * n), 256, 0, st>>>(a, it);
  if (upd) sp_var_kernel<<<grid((int64_t)nblk * n), 256, 0, st>>>(a);
  ATSC3_CUDA(cudaGetLastError());
  return 0;
}

}  // extern "C"
