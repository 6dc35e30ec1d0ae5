// wms.cu -- unrolled weighted min-sum with a hand-written backward (sm_100a).
//
// Forward, flooding schedule, iterations t = 1..T (messages m^(0) = 0,
// posterior tot^(0) = llr):
//   x_e   = tot^(t-1)[v(e)] - m^(t-1)_e                       (bit -> check)
//   mu_e  = min over the other edges of |x|  (min1, or min2 at the first
//           minimum; first-minimum rule with strict <)
//   m_e^(t) = sgn_e * relu(alpha[t][d] * mu_e - beta[t][d]),
//           sgn_e = (product of signs of the check's x) * sign(x_e),
//           sign(x) = -1 iff x < 0, d = degree bucket of the check
//   tot^(t)[v] = llr[v] + sum_e m^(t)_e    (ascending edge order)
// Output: tot^(T).  With alpha = a, beta = 0 this is the normalised min-sum
// of lab/ldpc_kernel.c for T fixed iterations (no early stop).
//
// Memory: per iteration one 16-byte record per check {min1, min2, first,
// second, sign bits of x} (checkpoint), never the per-edge messages: every
// m^(t)_e is recomputed from the record.  The backward walks t = T..1,
// recomputing tot^(t-1) from the records of iteration t-1, then
//   G_e   = gtot^(t)[v(e)] - gx^(t+1)_e                       (dL/dm^(t)_e)
//   a_e = alpha*mu_e - beta > 0:  galpha += G sgn mu, gbeta -= G sgn,
//                                 gmu_e = G sgn alpha
//   gx^(t)_first  += sign(x_first)  * sum_{e != first} gmu_e
//   gx^(t)_second += sign(x_second) * gmu_first
//   gtot^(t-1)[v] = sum_e gx^(t)_e
// (signs and the arg-min choice are piecewise constant).  REC selects the
// stored record precision: float (FP32 messages) or bfloat16 minima (BF16
// messages, the low-precision variant).
//
// Tables are CSR (cptr/cidx check-major; vptr/vedge variable-major edge ids,
// vchk/vpos the check and position of each variable-major edge).  Parameter
// gradients are reduced per CTA in shared memory, one atomicAdd per CTA and
// parameter.

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "../../include/atsc3_fec.h"
#include "common.cuh"

namespace atsc3 {

struct WmsTables {
  const int32_t *cptr, *cidx, *vptr, *vedge, *vchk, *vpos;
  const int8_t *cbucket;     // degree bucket per check
  int n, nc, ne, nbucket;
};

struct WmsRec {              // 16 bytes
  float min1, min2;
  uint16_t first, second;
  uint32_t sx;               // bit j: x_j < 0
};

template <bool BF16>
__device__ __forceinline__ float rq(float v) {
  if constexpr (BF16) return __bfloat162float(__float2bfloat16_rn(v));
  return v;
}

// m for position j from a record (alpha/beta of that iteration and bucket)
__device__ __forceinline__ float wms_msg(const WmsRec &r, int j, int deg,
                                         float al, float be) {
  const float mu = (j == r.first) ? r.min2 : r.min1;
  const float a = __fsub_rn(__fmul_rn(al, mu), be);
  if (!(a > 0.f)) return 0.f;
  const uint32_t par = __popc(r.sx & ((deg >= 32) ? 0xFFFFFFFFu : ((1u << deg) - 1u))) & 1u;
  const uint32_t neg = par ^ ((r.sx >> j) & 1u);
  return neg ? -a : a;
}

// ---- forward: check update of iteration t (1-based) ------------------------
template <bool BF16>
__global__ void wms_check_fwd(WmsTables T, int nblk, const float *tot,
                              const WmsRec *rprev, WmsRec *rnew,
                              const float *alpha, const float *beta, int tprev) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= (int64_t)nblk * T.nc) return;
  const int b = (int)(g / T.nc), c = (int)(g - (int64_t)b * T.nc);
  const int e0 = T.cptr[c], deg = T.cptr[c + 1] - e0;
  const float *tb = tot + (size_t)b * T.n;
  WmsRec ro;
  float al = 0.f, be = 0.f;
  if (tprev > 0) {
    ro = rprev[(size_t)b * T.nc + c];
    const int d = T.cbucket[c];
    al = alpha[(tprev - 1) * T.nbucket + d];
    be = beta[(tprev - 1) * T.nbucket + d];
  }
  float min1 = __int_as_float(0x7f800000), min2 = min1;
  int first = 0, second = 0;
  uint32_t sx = 0;
  for (int j = 0; j < deg; ++j) {
    const float mo = tprev > 0 ? wms_msg(ro, j, deg, al, be) : 0.f;
    const float x = __fsub_rn(tb[T.cidx[e0 + j]], mo);
    if (x < 0.f) sx |= 1u << j;
    const float mag = fabsf(x);
    if (mag < min1) { min2 = min1; second = first; min1 = mag; first = j; }
    else if (mag < min2) { min2 = mag; second = j; }
  }
  WmsRec r;
  r.min1 = rq<BF16>(min1);
  r.min2 = rq<BF16>(min2);
  r.first = (uint16_t)first;
  r.second = (uint16_t)second;
  r.sx = sx;
  rnew[(size_t)b * T.nc + c] = r;
}

// ---- forward: variable update (tot^(t) from the records of iteration t) ----
__global__ void wms_var_fwd(WmsTables T, int nblk, const float *llr,
                            const WmsRec *rec, const float *alpha,
                            const float *beta, int t, float *tot) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= (int64_t)nblk * T.n) return;
  const int b = (int)(g / T.n), v = (int)(g - (int64_t)b * T.n);
  float s = llr[(size_t)b * T.n + v];
  if (t > 0) {
    const WmsRec *rb = rec + (size_t)b * T.nc;
    for (int k = T.vptr[v]; k < T.vptr[v + 1]; ++k) {
      const int c = T.vchk[k];
      const int d = T.cbucket[c];
      const WmsRec r = rb[c];
      s = __fadd_rn(s, wms_msg(r, T.vpos[k], T.cptr[c + 1] - T.cptr[c],
                               alpha[(t - 1) * T.nbucket + d],
                               beta[(t - 1) * T.nbucket + d]));
    }
  }
  tot[(size_t)b * T.n + v] = s;
}

// ---- backward: check step of iteration t ------------------------------------
// tot: tot^(t-1) (recomputed); rprev: records of t-1 (null for t = 1);
// rcur: records of t; gtot: dL/dtot^(t); gx_next: dL/dx^(t+1) (null at T);
// writes gx (dL/dx^(t)) and accumulates galpha/gbeta[t-1][bucket].
template <int MAXB>
__global__ void wms_check_bwd(WmsTables T, int nblk, const float *tot,
                              const WmsRec *rprev, const WmsRec *rcur,
                              const float *alpha, const float *beta, int t,
                              const float *gtot, const float *gx_next,
                              float *gx, float *galpha, float *gbeta) {
  __shared__ float sa[MAXB], sb[MAXB];
  for (int i = threadIdx.x; i < MAXB; i += blockDim.x) sa[i] = sb[i] = 0.f;
  __syncthreads();
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g < (int64_t)nblk * T.nc) {
    const int b = (int)(g / T.nc), c = (int)(g - (int64_t)b * T.nc);
    const int e0 = T.cptr[c], deg = T.cptr[c + 1] - e0;
    const int d = T.cbucket[c];
    const float al = alpha[(t - 1) * T.nbucket + d];
    const float be = beta[(t - 1) * T.nbucket + d];
    const WmsRec r = rcur[(size_t)b * T.nc + c];
    WmsRec rp;
    float alp = 0.f, bep = 0.f;
    if (t > 1) {
      rp = rprev[(size_t)b * T.nc + c];
      alp = alpha[(t - 2) * T.nbucket + d];
      bep = beta[(t - 2) * T.nbucket + d];
    }
    const float *tb = tot + (size_t)b * T.n;
    const float *gt = gtot + (size_t)b * T.n;
    const size_t eb = (size_t)b * T.ne;
    const uint32_t par = __popc(r.sx & ((deg >= 32) ? 0xFFFFFFFFu : ((1u << deg) - 1u))) & 1u;
    float ga = 0.f, gb = 0.f, gmu_rest = 0.f, gmu_first = 0.f;
    for (int j = 0; j < deg; ++j) {
      const float G = gt[T.cidx[e0 + j]] - (gx_next ? gx_next[eb + e0 + j] : 0.f);
      const float mu = (j == r.first) ? r.min2 : r.min1;
      const float a = al * mu - be;
      if (a > 0.f) {
        const float sg = (par ^ ((r.sx >> j) & 1u)) ? -1.f : 1.f;
        const float gaj = G * sg;
        ga += gaj * mu;
        gb -= gaj;
        const float gmu = gaj * al;
        if (j == r.first) gmu_first += gmu; else gmu_rest += gmu;
      }
    }
    // x^(t)_first and x^(t)_second: recompute their signs from tot^(t-1)
    for (int j = 0; j < deg; ++j) {
      float gxv = 0.f;
      if (j == r.first || j == r.second) {
        const float mo = t > 1 ? wms_msg(rp, j, deg, alp, bep) : 0.f;
        const float x = __fsub_rn(tb[T.cidx[e0 + j]], mo);
        const float sx = x < 0.f ? -1.f : 1.f;
        if (j == r.first) gxv += sx * gmu_rest;
        if (j == r.second && deg > 1) gxv += sx * gmu_first;
      }
      gx[eb + e0 + j] = gxv;
    }
    atomicAdd(&sa[d], ga);
    atomicAdd(&sb[d], gb);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < T.nbucket; i += blockDim.x) {
    if (sa[i] != 0.f) atomicAdd(&galpha[(t - 1) * T.nbucket + i], sa[i]);
    if (sb[i] != 0.f) atomicAdd(&gbeta[(t - 1) * T.nbucket + i], sb[i]);
  }
}

// ---- backward: gtot^(t-1)[v] = sum of gx^(t) over v's edges --------------------
__global__ void wms_var_bwd(WmsTables T, int nblk, const float *gx,
                            float *gtot_prev) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= (int64_t)nblk * T.n) return;
  const int b = (int)(g / T.n), v = (int)(g - (int64_t)b * T.n);
  const float *gb = gx + (size_t)b * T.ne;
  float s = 0.f;
  for (int k = T.vptr[v]; k < T.vptr[v + 1]; ++k) s += gb[T.vedge[k]];
  gtot_prev[(size_t)b * T.n + v] = s;
}

static inline unsigned nblocks(int64_t work, int th) {
  return (unsigned)((work + th - 1) / th);
}

}  // namespace atsc3

extern "C" {

// tables: int32 pointers (device) cptr, cidx, vptr, vedge, vchk, vpos; int8 cbucket.
int32_t atsc3_wms_forward(const int32_t *cptr, const int32_t *cidx,
                          const int32_t *vptr, const int32_t *vedge,
                          const int32_t *vchk, const int32_t *vpos,
                          const int8_t *cbucket, int32_t n, int32_t nc,
                          int32_t ne, int32_t nbucket, int32_t nblk,
                          int32_t iters, const float *llr, const float *alpha,
                          const float *beta, int32_t bf16, void *records,
                          float *tot_out, void *stream) {
  using namespace atsc3;
  ATSC3_ARG(n > 0 && nc > 0 && ne > 0 && nbucket > 0 && nbucket <= 127, "bad sizes");
  ATSC3_ARG(iters >= 1 && nblk >= 0, "bad sizes");
  if (nblk == 0) return 0;
  ATSC3_ARG(cptr && cidx && vptr && vedge && vchk && vpos && cbucket && llr &&
                alpha && beta && records && tot_out,
            "null pointer");
  WmsTables T{cptr, cidx, vptr, vedge, vchk, vpos, cbucket, n, nc, ne, nbucket};
  cudaStream_t st = (cudaStream_t)stream;
  WmsRec *rec = reinterpret_cast<WmsRec *>(records);
  const size_t per = (size_t)nblk * nc;
  // tot^(0) = llr
  wms_var_fwd<<<nblocks((int64_t)nblk * n, 256), 256, 0, st>>>(T, nblk, llr, rec, alpha, beta, 0, tot_out);
  for (int t = 1; t <= iters; ++t) {
    WmsRec *rn = rec + (size_t)(t - 1) * per;
    const WmsRec *rp = t > 1 ? rec + (size_t)(t - 2) * per : nullptr;
    if (bf16)
      wms_check_fwd<true><<<nblocks((int64_t)nblk * nc, 256), 256, 0, st>>>(T, nblk, tot_out, rp, rn, alpha, beta, t - 1);
    else
      wms_check_fwd<false><<<nblocks((int64_t)nblk * nc, 256), 256, 0, st>>>(T, nblk, tot_out, rp, rn, alpha, beta, t - 1);
    wms_var_fwd<<<nblocks((int64_t)nblk * n, 256), 256, 0, st>>>(T, nblk, llr, rn, alpha, beta, t, tot_out);
  }
  ATSC3_CUDA(cudaGetLastError());
  return 0;
}

// gtot: (nblk, n) dL/dtot^(T) on input, overwritten with dL/dllr on output.
// work: tot buffer (nblk*n floats) + two edge buffers (2*nblk*ne floats).
int32_t atsc3_wms_backward(const int32_t *cptr, const int32_t *cidx,
                           const int32_t *vptr, const int32_t *vedge,
                           const int32_t *vchk, const int32_t *vpos,
                           const int8_t *cbucket, int32_t n, int32_t nc,
                           int32_t ne, int32_t nbucket, int32_t nblk,
                           int32_t iters, const float *llr, const float *alpha,
                           const float *beta, const void *records, float *gtot,
                           float *galpha, float *gbeta, float *work,
                           void *stream) {
  using namespace atsc3;
  ATSC3_ARG(n > 0 && nc > 0 && ne > 0 && nbucket > 0 && nbucket <= 127, "bad sizes");
  ATSC3_ARG(iters >= 1 && nblk >= 0, "bad sizes");
  if (nblk == 0) return 0;
  ATSC3_ARG(gtot && galpha && gbeta && work && records, "null pointer");
  WmsTables T{cptr, cidx, vptr, vedge, vchk, vpos, cbucket, n, nc, ne, nbucket};
  cudaStream_t st = (cudaStream_t)stream;
  const WmsRec *rec = reinterpret_cast<const WmsRec *>(records);
  const size_t per = (size_t)nblk * nc;
  float *tot = work;
  float *gxa = work + (size_t)nblk * n;
  float *gxb = gxa + (size_t)nblk * ne;
  float *gx_next = nullptr;
  for (int t = iters; t >= 1; --t) {
    // recompute tot^(t-1) from the records of iteration t-1
    const WmsRec *rp = t > 1 ? rec + (size_t)(t - 2) * per : nullptr;
    wms_var_fwd<<<nblocks((int64_t)nblk * n, 256), 256, 0, st>>>(T, nblk, llr, rp, alpha, beta, t - 1, tot);
    float *gx = (gx_next == gxa) ? gxb : gxa;
    // per-CTA gradient partials in shared memory, one entry per bucket
    // (check degrees: a handful; block rows: up to 127)
    if (nbucket <= 64)
      wms_check_bwd<64><<<nblocks((int64_t)nblk * nc, 256), 256, 0, st>>>(
          T, nblk, tot, rp, rec + (size_t)(t - 1) * per, alpha, beta, t, gtot,
          gx_next, gx, galpha, gbeta);
    else
      wms_check_bwd<128><<<nblocks((int64_t)nblk * nc, 256), 256, 0, st>>>(
          T, nblk, tot, rp, rec + (size_t)(t - 1) * per, alpha, beta, t, gtot,
          gx_next, gx, galpha, gbeta);
    // gtot^(t-1): the edges of tot^(t-1) through x^(t)
    wms_var_bwd<<<nblocks((int64_t)nblk * n, 256), 256, 0, st>>>(T, nblk, gx, gtot);
    gx_next = gx;
  }
  ATSC3_CUDA(cudaGetLastError());
  return 0;
}

}  // extern "C"
