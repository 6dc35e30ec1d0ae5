// ldpc_flood.cu -- flooding normalised min-sum LDPC decoder for sm_100a.
//
// Algorithm (bit-exact restatement of lab/ldpc_kernel.c:65-146, the
// Felbs/atsc3 compiled kernel, and -- with `TORCH` -- of the float64 numpy /
// torch decoders lab/m3_ldpc.py:560-630 and lab/m9_gpu.py:168-211):
//
//   for it = 0 .. iters:
//     syndrome of sign(tot) over every check            (ldpc_kernel.c:96-101)
//     zero -> retire (its = it, conv = 1, bad = 0)      (:102-108)
//     it == iters -> retire (conv = 0, bad = #unsat)    (:109-113)
//     check update: v_e = tot[var_e] - m_e; first-minimum tie rule, strict <;
//       m_e = +-(e == first ? min2 : min1) * alpha, sign = parity ^ (v_e < 0)
//                                                       (:116-134)
//     variable update: s = +0; s += m_e in vedge order; tot = llr + s
//                                                       (:137-142)
//
// Layout: one thread-block CLUSTER owns one codeword at a time and keeps its
// whole decoder state in the cluster's distributed shared memory:
//   * tot[] (the posterior LLRs), partitioned by variable: CTA r holds
//     variables [r*2^nvlog2, (r+1)*2^nvlog2), so a variable index is its own
//     DSMEM address (rank = i >> nvlog2, offset = i & mask);
//   * one record per check instead of one message per edge (compressed
//     min-sum state): min1*alpha, min2*alpha, the first-minimum position and
//     one sign bit per edge.  Every edge message is recomputed exactly from
//     it, so nothing is rounded differently from the per-edge reference.
// Checks are partitioned over the cluster in runs of ncp.  Check phase: each
// thread owns one check, gathers tot of its variables through DSMEM,
// computes the syndrome bit and the new record in one pass.  Variable
// phase: each thread owns one variable and gathers its checks' records in
// the reference's summation order.  Two cluster barriers per iteration.
// The channel LLRs stay in global memory (read once per iteration,
// coalesced).  Clusters are persistent and stride over codewords.
//
// Tables (built on the host, see build_tables): sliced-ELL lists of 32
// checks / 32 variables per warp, padded with sentinels.

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "../../include/atsc3_fec.h"
#include "common.cuh"
#include "ldpc_plan.h"

namespace atsc3 {

// ---------------------------------------------------------------------------
// host: tables
// ---------------------------------------------------------------------------

int record_bytes(int dtype, int dmax_c) {
  if (dtype == 0) {
    if (dmax_c <= 56) return 16;
    if (dmax_c <= 128) return 32;
    return 0;
  }
  if (dmax_c <= 96) return 32;
  return 0;
}

int plan_smem_bytes(int dtype, int rec_bytes, int ncp, int nvlog2) {
  const int tsz = dtype ? 8 : 4;
  return (1 << nvlog2) * tsz + ncp * rec_bytes + 256;
}

int build_tables(const int32_t *cptr, const int32_t *cidx,
                 const int32_t *vptr, const int32_t *vedge, int n, int nc,
                 int nedges, int cluster, int *ncp_out, int *nvlog2_out,
                 std::vector<uint16_t> &cent, std::vector<int32_t> &cslice,
                 std::vector<uint32_t> &vent, std::vector<int32_t> &vslice,
                 int *dmax_c_out, int *dmax_v_out) {
  if (n <= 0 || nc <= 0 || nedges < 0) {
    set_error("invalid argument: empty code");
    return -3;
  }
  if (n > 65535) {
    set_error("unsupported: codeword length above 65535");
    return -4;
  }
  if (cluster < 1 || cluster > 16 || (cluster & (cluster - 1))) {
    set_error("invalid argument: cluster must be 1, 2, 4, 8 or 16");
    return -3;
  }
  if (cptr[0] != 0 || cptr[nc] != nedges || vptr[0] != 0 ||
      vptr[n] != nedges) {
    set_error("invalid argument: CSR pointers do not span the edges");
    return -3;
  }
  int dmax_c = 0;
  for (int c = 0; c < nc; ++c) {
    int d = cptr[c + 1] - cptr[c];
    if (d < 0) {
      set_error("invalid argument: cptr not monotone");
      return -3;
    }
    dmax_c = std::max(dmax_c, d);
  }
  if (dmax_c > ATSC3_MAX_ROW_DEG) {
    set_error("check degree above 128");
    return -1;
  }
  std::vector<int32_t> chk_of_edge(nedges);
  for (int c = 0; c < nc; ++c)
    for (int e = cptr[c]; e < cptr[c + 1]; ++e) {
      if (cidx[e] < 0 || cidx[e] >= n) {
        set_error("invalid argument: cidx out of range");
        return -3;
      }
      chk_of_edge[e] = c;
    }
  int dmax_v = 0;
  std::vector<uint8_t> seen(nedges, 0);
  for (int i = 0; i < n; ++i) {
    int d = vptr[i + 1] - vptr[i];
    if (d < 0) {
      set_error("invalid argument: vptr not monotone");
      return -3;
    }
    dmax_v = std::max(dmax_v, d);
    for (int k = vptr[i]; k < vptr[i + 1]; ++k) {
      int e = vedge[k];
      if (e < 0 || e >= nedges || seen[e] || cidx[e] != i) {
        set_error("invalid argument: vedge is not the variable-major "
                  "permutation of cidx");
        return -3;
      }
      seen[e] = 1;
    }
  }
  // partition
  int per = (nc + cluster - 1) / cluster;
  int ncp = (per + 31) / 32 * 32;
  if (ncp > 65536) {
    set_error("unsupported: more than 65536 checks per CTA");
    return -4;
  }
  int nvper = (n + cluster - 1) / cluster;
  int nvlog2 = 5;
  while ((1 << nvlog2) < nvper) ++nvlog2;
  // check-phase sliced ELL
  int nslc = (nc + 31) / 32;
  cslice.assign(nslc + 1, 0);
  for (int s = 0; s < nslc; ++s) {
    int dm = 0;
    for (int l = 0; l < 32; ++l) {
      int c = 32 * s + l;
      if (c < nc) dm = std::max(dm, cptr[c + 1] - cptr[c]);
    }
    cslice[s + 1] = cslice[s] + dm;
  }
  cent.assign((size_t)cslice[nslc] * 32, 0xFFFFu);
  for (int s = 0; s < nslc; ++s)
    for (int l = 0; l < 32; ++l) {
      int c = 32 * s + l;
      if (c >= nc) continue;
      for (int k = 0; k < cptr[c + 1] - cptr[c]; ++k)
        cent[((size_t)cslice[s] + k) * 32 + l] = (uint16_t)cidx[cptr[c] + k];
    }
  // variable-phase sliced ELL: (check offset in its CTA, CTA rank, position)
  int nslv = (n + 31) / 32;
  vslice.assign(nslv + 1, 0);
  for (int s = 0; s < nslv; ++s) {
    int dm = 0;
    for (int l = 0; l < 32; ++l) {
      int i = 32 * s + l;
      if (i < n) dm = std::max(dm, vptr[i + 1] - vptr[i]);
    }
    vslice[s + 1] = vslice[s] + dm;
  }
  vent.assign((size_t)vslice[nslv] * 32, 0xFFFFFFFFu);
  for (int s = 0; s < nslv; ++s)
    for (int l = 0; l < 32; ++l) {
      int i = 32 * s + l;
      if (i >= n) continue;
      for (int k = 0; k < vptr[i + 1] - vptr[i]; ++k) {
        int e = vedge[vptr[i] + k];
        int c = chk_of_edge[e];
        uint32_t pos = (uint32_t)(e - cptr[c]);
        uint32_t rank = (uint32_t)(c / ncp), off = (uint32_t)(c % ncp);
        vent[((size_t)vslice[s] + k) * 32 + l] = off | (rank << 16) |
                                                  (pos << 20);
      }
    }
  *ncp_out = ncp;
  *nvlog2_out = nvlog2;
  *dmax_c_out = dmax_c;
  *dmax_v_out = dmax_v;
  return 0;
}

// ---------------------------------------------------------------------------
// device: per-check records
// ---------------------------------------------------------------------------
//
// float, 16 B : {A, B, S0, F | S1<<8}       positions 0..55
// float, 32 B : {A, B, S0, F}{S1, S2, S3, 0} positions 0..127
// double, 32 B: {A.lo, A.hi, B.lo, B.hi}{S0, F, S1, S2} positions 0..95
// A = min1*alpha, B = min2*alpha, F = position of the first minimum,
// S = sign bit of each edge's message (1 = negative).

template <typename T, int RB> struct Rec;

template <> struct Rec<float, 16> {
  static constexpr int NV = 1;
  __device__ static float A(const uint4 *r) { return __uint_as_float(r[0].x); }
  __device__ static float B(const uint4 *r) { return __uint_as_float(r[0].y); }
  __device__ static int F(const uint4 *r) { return (int)(r[0].w & 0xFFu); }
  __device__ static uint32_t sign(const uint4 *r, int j) {
    return j < 32 ? (r[0].z >> j) & 1u : (r[0].w >> (j - 24)) & 1u;
  }
  __device__ static bool need_hi(int) { return false; }
  __device__ static void pack(uint4 *r, float A, float B, int F,
                              uint64_t lo, uint64_t) {
    r[0] = make_uint4(__float_as_uint(A), __float_as_uint(B), (uint32_t)lo,
                      (uint32_t)F | ((uint32_t)(lo >> 32) << 8));
  }
};

template <> struct Rec<float, 32> {
  static constexpr int NV = 2;
  __device__ static float A(const uint4 *r) { return __uint_as_float(r[0].x); }
  __device__ static float B(const uint4 *r) { return __uint_as_float(r[0].y); }
  __device__ static int F(const uint4 *r) { return (int)r[0].w; }
  __device__ static uint32_t sign(const uint4 *r, int j) {
    uint32_t w = j < 32 ? r[0].z : (j < 64 ? r[1].x : (j < 96 ? r[1].y : r[1].z));
    return (w >> (j & 31)) & 1u;
  }
  __device__ static bool need_hi(int j) { return j >= 32; }
  __device__ static void pack(uint4 *r, float A, float B, int F, uint64_t lo,
                              uint64_t hi) {
    r[0] = make_uint4(__float_as_uint(A), __float_as_uint(B), (uint32_t)lo,
                      (uint32_t)F);
    r[1] = make_uint4((uint32_t)(lo >> 32), (uint32_t)hi,
                      (uint32_t)(hi >> 32), 0u);
  }
};

template <> struct Rec<double, 32> {
  static constexpr int NV = 2;
  __device__ static double A(const uint4 *r) {
    return __hiloint2double((int)r[0].y, (int)r[0].x);
  }
  __device__ static double B(const uint4 *r) {
    return __hiloint2double((int)r[0].w, (int)r[0].z);
  }
  __device__ static int F(const uint4 *r) { return (int)r[1].y; }
  __device__ static uint32_t sign(const uint4 *r, int j) {
    uint32_t w = j < 32 ? r[1].x : (j < 64 ? r[1].z : r[1].w);
    return (w >> (j & 31)) & 1u;
  }
  __device__ static bool need_hi(int) { return true; }
  __device__ static void pack(uint4 *r, double A, double B, int F, uint64_t lo,
                              uint64_t hi) {
    r[0] = make_uint4((uint32_t)__double2loint(A), (uint32_t)__double2hiint(A),
                      (uint32_t)__double2loint(B), (uint32_t)__double2hiint(B));
    r[1] = make_uint4((uint32_t)lo, (uint32_t)F, (uint32_t)(lo >> 32),
                      (uint32_t)hi);
  }
};

struct FloodArgs {
  const void *llr;
  int64_t ld_llr;
  int nblk, n, nc, iters;
  double alpha;
  const uint16_t *cent;
  const int32_t *cslice;
  int nslc;
  const uint32_t *vent;
  const int32_t *vslice;
  int nslv;
  int ncp, nvlog2;
  uint8_t *bits;
  int64_t ld_bits;
  uint8_t *hard;
  int64_t ld_hard;
  uint8_t *conv;
  int32_t *its;
  int32_t *bad;
};

template <typename T> __device__ __forceinline__ T pos_inf();
template <> __device__ __forceinline__ float pos_inf<float>() {
  return __int_as_float(0x7f800000);
}
template <> __device__ __forceinline__ double pos_inf<double>() {
  return __longlong_as_double(0x7ff0000000000000LL);
}

__device__ __forceinline__ uint64_t low_mask64(int d) {
  return d >= 64 ? ~0ull : ((1ull << d) - 1ull);
}

// Semantics of the per-codeword decoder: SEM_KERNEL = lab/ldpc_kernel.c;
// SEM_TORCH = lab/m9_gpu.py in float32/float64; SEM_TORCH_BF16 / _F16 =
// lab/m9_gpu.py with dtype bfloat16 / float16, whose torch operations each
// compute in float32 and round the result to the narrow type: the decoder
// keeps float32 values that are all exact in the narrow type and rounds every
// subtraction, scaled minimum and partial sum the same way.
constexpr int SEM_KERNEL = 0, SEM_TORCH = 1, SEM_TORCH_BF16 = 2, SEM_TORCH_F16 = 3;

template <int SEM> __device__ __forceinline__ float narrow(float x) {
  if constexpr (SEM == SEM_TORCH_BF16) return __bfloat162float(__float2bfloat16_rn(x));
  else if constexpr (SEM == SEM_TORCH_F16) return __half2float(__float2half_rn(x));
  else return x;
}
template <int SEM> __device__ __forceinline__ double narrow(double x) { return x; }

// Geometry and tables of one code, as the per-codeword decoder sees them.
struct CwView {
  int n, nc, ncp, nvlog2, nslc, nslv;
  const uint16_t *cent;
  const int32_t *cslice;
  const uint32_t *vent;
  const int32_t *vslice;
};

// Decode ONE codeword with the whole cluster (every CTA of the cluster calls
// this with the same arguments).  sm: this CTA's shared memory for the
// codeword (posteriors, records, partial counts).  Writes bits_row /
// hard_row (nullable) and *conv, *its, *bad (rank 0).  Ends after a
// __syncthreads, with no distributed-shared-memory access in flight.
template <typename T, int RB, int SEM>
__device__ __forceinline__ void flood_codeword(
    const CwView &g, const T *lam, int iters, T alpha, unsigned char *sm,
    int rank, int CL, uint8_t *bits_row, uint8_t *hard_row, uint8_t *conv,
    int32_t *its, int32_t *bad) {
  using R = Rec<T, RB>;
  constexpr int NV = R::NV;
  constexpr bool TORCH = SEM != SEM_KERNEL;
  // the narrow types scale by alpha rounded to them (torch: alpha * sign
  // computed in float32, then rounded)
  alpha = narrow<SEM>(alpha);
  const int nvp = 1 << g.nvlog2;
  const uint32_t vmask = (uint32_t)nvp - 1u;
  T *tot = reinterpret_cast<T *>(sm);
  uint4 *rec = reinterpret_cast<uint4 *>(sm + (size_t)nvp * sizeof(T));
  int *part = reinterpret_cast<int *>(sm + (size_t)nvp * sizeof(T) +
                                      (size_t)g.ncp * RB);
  int *sbad = part + 32;
  const uint32_t tot_sa = smem_u32(tot);
  const uint32_t rec_sa = smem_u32(rec);
  const uint32_t part_sa = smem_u32(part);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nwarps = blockDim.x >> 5;
  const int cs0 = rank * (g.ncp >> 5);
  const int cs1 = min(g.nslc, cs0 + (g.ncp >> 5));
  const int vs0 = rank * (nvp >> 5);
  const int vs1 = min(g.nslv, vs0 + (nvp >> 5));
  const int cbase = rank * g.ncp;
  const int vbase = rank * nvp;
  const int vend = min(g.n, vbase + nvp);

  for (int i = vbase + tid; i < vend; i += blockDim.x) tot[i - vbase] = lam[i];
  for (int q = tid; q < g.ncp * NV; q += blockDim.x)
    rec[q] = make_uint4(0u, 0u, 0u, 0u);
  if (tid == 0) *sbad = 0;
  __syncthreads();
  cluster_sync_all();

  for (int it = 0;; ++it) {
    // ---------------- check phase (syndrome + new records) ----------------
    int mybad = 0;
    for (int s = cs0 + warp; s < cs1; s += nwarps) {
      const int c = (s << 5) + lane;
      const int e0 = __ldg(g.cslice + s);
      const int dm = __ldg(g.cslice + s + 1) - e0;
      if (c < g.nc) {
        const uint16_t *ent = g.cent + ((size_t)e0 << 5) + lane;
        uint4 ro[NV];
#pragma unroll
        for (int q = 0; q < NV; ++q) ro[q] = rec[(c - cbase) * NV + q];
        const T Ao = R::A(ro), Bo = R::B(ro);
        const int Fo = R::F(ro);
        T min1 = pos_inf<T>(), min2 = pos_inf<T>();
        int first = 0, deg = 0;
        uint32_t syn = 0;
        uint64_t slo = 0, shi = 0;
        for (int k0 = 0; k0 < dm; k0 += 8) {
          uint32_t vi[8];
          T t[8];
#pragma unroll
          for (int u = 0; u < 8; ++u)
            vi[u] = (k0 + u < dm) ? (uint32_t)__ldg(ent + ((k0 + u) << 5))
                                  : 0xFFFFu;
#pragma unroll
          for (int u = 0; u < 8; ++u)
            t[u] = vi[u] != 0xFFFFu
                       ? dsmem_ld<T>(dsmem_map(
                             tot_sa + (vi[u] & vmask) * (uint32_t)sizeof(T),
                             vi[u] >> g.nvlog2))
                       : T(0);
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            if (vi[u] == 0xFFFFu) continue;
            const int j = k0 + u;
            syn ^= (t[u] < T(0)) ? 1u : 0u;
            T mo = (j == Fo) ? Bo : Ao;
            if (R::sign(ro, j)) mo = -mo;
            const T v = narrow<SEM>(sub_rn(t[u], mo));
            const uint64_t sg = (v < T(0)) ? 1ull : 0ull;
            if (j < 64) slo |= sg << j; else shi |= sg << (j - 64);
            const T mag = fabs(v);
            if (mag < min1) { min2 = min1; min1 = mag; first = j; }
            else if (mag < min2) { min2 = mag; }
            deg = j + 1;
          }
        }
        const int par = (__popcll(slo) + __popcll(shi)) & 1;
        if (par) {
          slo ^= low_mask64(deg);
          shi ^= deg > 64 ? low_mask64(deg - 64) : 0ull;
        }
        uint4 rn[NV];
        R::pack(rn, narrow<SEM>(mul_rn(min1, alpha)), narrow<SEM>(mul_rn(min2, alpha)),
                first, slo, shi);
#pragma unroll
        for (int q = 0; q < NV; ++q) rec[(c - cbase) * NV + q] = rn[q];
        mybad += (int)syn;
      }
    }
    mybad = __reduce_add_sync(0xffffffffu, mybad);
    if (lane == 0 && mybad) atomicAdd(sbad, mybad);
    __syncthreads();
    if (tid < CL)
      dsmem_st_u32(dsmem_map(part_sa + (uint32_t)(((it & 1) * 16 + rank) * 4),
                             (uint32_t)tid),
                   (uint32_t)*sbad);
    cluster_sync_all();
    int badct = 0;
    for (int r = 0; r < CL; ++r) badct += part[(it & 1) * 16 + r];
    if (tid == 0) *sbad = 0;
    const bool done = (badct == 0) && (!TORCH || it > 0);
    if (done || it >= iters) {
      // ---------------- retire: hard decisions and status ------------------
      if (bits_row)
        for (int i = vbase + tid; i < vend; i += blockDim.x)
          bits_row[i] = tot[i - vbase] < T(0) ? 1 : 0;
      if (hard_row) {
        for (int w0 = vbase; w0 < vend; w0 += 32 * nwarps) {
          const int i = w0 + (warp << 5) + lane;
          const bool ng = i < vend && tot[i - vbase] < T(0);
          const uint32_t m = __ballot_sync(0xffffffffu, ng);
          const int base = w0 + (warp << 5);
          if (lane == 0 && base < vend) {
            const uint32_t word = __byte_perm(__brev(m), 0u, 0x0123u);
            if (base + 32 <= vend) {
              *reinterpret_cast<uint32_t *>(hard_row + (base >> 3)) = word;
            } else {
              const int nbyte = (vend - base + 7) >> 3;
              for (int q = 0; q < nbyte; ++q)
                hard_row[(base >> 3) + q] = (uint8_t)(word >> (8 * q));
            }
          }
        }
      }
      if (rank == 0 && tid == 0) {
        *conv = done ? 1 : 0;
        *its = it;
        *bad = done ? 0 : badct;
      }
      // outputs read posteriors the next codeword's prologue overwrites
      __syncthreads();
      return;
    }
    // ---------------- variable phase --------------------------------------
    for (int s = vs0 + warp; s < vs1; s += nwarps) {
      const int i = (s << 5) + lane;
      const int e0 = __ldg(g.vslice + s);
      const int dm = __ldg(g.vslice + s + 1) - e0;
      if (i < g.n) {
        const uint32_t *ent = g.vent + ((size_t)e0 << 5) + lane;
        const T li = lam[i];
        T acc = TORCH ? li : T(0);
        for (int k0 = 0; k0 < dm; k0 += 4) {
          uint32_t en[4];
          uint4 rr[4][NV];
#pragma unroll
          for (int u = 0; u < 4; ++u)
            en[u] = (k0 + u < dm) ? __ldg(ent + ((k0 + u) << 5)) : 0xFFFFFFFFu;
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            if (en[u] == 0xFFFFFFFFu) continue;
            const uint32_t ra = dsmem_map(
                rec_sa + (en[u] & 0xFFFFu) * (uint32_t)RB, (en[u] >> 16) & 15u);
            rr[u][0] = dsmem_ld_v4(ra);
            if (NV > 1 && R::need_hi((int)(en[u] >> 20)))
              rr[u][NV - 1] = dsmem_ld_v4(ra + 16u);
          }
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            if (en[u] == 0xFFFFFFFFu) continue;
            const int j = (int)(en[u] >> 20);
            T m = (j == R::F(rr[u])) ? R::B(rr[u]) : R::A(rr[u]);
            if (R::sign(rr[u], j)) m = -m;
            acc = narrow<SEM>(add_rn(acc, m));
          }
        }
        tot[i - vbase] = TORCH ? acc : add_rn(li, acc);
      }
    }
    __syncthreads();
    cluster_sync_all();
  }
}

template <typename T, int RB, int SEM>
__global__ void __launch_bounds__(1024, 1) ldpc_flood_kernel(const FloodArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int rank = (int)cluster_ctarank();
  const int CL = (int)cluster_nctarank();
  const CwView g{a.n, a.nc, a.ncp, a.nvlog2, a.nslc, a.nslv,
                 a.cent, a.cslice, a.vent, a.vslice};
  for (int b = (int)cluster_id_x(); b < a.nblk; b += (int)ncluster_x()) {
    const T *lam = reinterpret_cast<const T *>(a.llr) + (size_t)b * a.ld_llr;
    flood_codeword<T, RB, SEM>(
        g, lam, a.iters, (T)a.alpha, smem, rank, CL,
        a.bits ? a.bits + (size_t)b * a.ld_bits : nullptr,
        a.hard ? a.hard + (size_t)b * a.ld_hard : nullptr, a.conv + b,
        a.its + b, a.bad + b);
  }
  // no CTA may leave while a peer can still read its shared memory
  __syncthreads();
  cluster_sync_all();
}

// ---------------------------------------------------------------------------
// host: plans and launch
// ---------------------------------------------------------------------------

typedef void (*FloodFn)(const FloodArgs);

static FloodFn flood_fn(int dtype, int rb, int semantics) {
  if (dtype == 0 && rb == 16) {
    switch (semantics) {
      case SEM_KERNEL: return ldpc_flood_kernel<float, 16, SEM_KERNEL>;
      case SEM_TORCH: return ldpc_flood_kernel<float, 16, SEM_TORCH>;
      case SEM_TORCH_BF16: return ldpc_flood_kernel<float, 16, SEM_TORCH_BF16>;
      case SEM_TORCH_F16: return ldpc_flood_kernel<float, 16, SEM_TORCH_F16>;
    }
  }
  if (dtype == 0 && rb == 32) {
    switch (semantics) {
      case SEM_KERNEL: return ldpc_flood_kernel<float, 32, SEM_KERNEL>;
      case SEM_TORCH: return ldpc_flood_kernel<float, 32, SEM_TORCH>;
      case SEM_TORCH_BF16: return ldpc_flood_kernel<float, 32, SEM_TORCH_BF16>;
      case SEM_TORCH_F16: return ldpc_flood_kernel<float, 32, SEM_TORCH_F16>;
    }
  }
  if (dtype == 1 && rb == 32)
    return semantics == SEM_TORCH ? ldpc_flood_kernel<double, 32, SEM_TORCH> : nullptr;
  return nullptr;
}

static int max_dyn_smem(int dev) {
  int v = 0;
  cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  return v;
}

struct OccKey {
  FloodFn fn;
  int cl, smem, threads, dev;
  bool operator==(const OccKey &o) const {
    return fn == o.fn && cl == o.cl && smem == o.smem && threads == o.threads &&
           dev == o.dev;
  }
};
struct OccHash {
  size_t operator()(const OccKey &k) const {
    return std::hash<void *>()((void *)k.fn) ^ ((size_t)k.cl << 3) ^
           ((size_t)k.smem << 9) ^ ((size_t)k.threads << 27) ^
           ((size_t)k.dev << 40);
  }
};
static std::mutex g_occ_mu;
static std::unordered_map<OccKey, int, OccHash> g_occ;

// The kernel attributes are set once per (function, device) to the device
// limits, so plans of different shared-memory sizes can share a function.
static std::mutex g_attr_mu;
static std::unordered_map<uint64_t, int> g_attr_done;

static int32_t prepare_fn(FloodFn fn, int dev) {
  const uint64_t key = (uint64_t)(uintptr_t)fn ^ ((uint64_t)dev << 56);
  {
    std::lock_guard<std::mutex> g(g_attr_mu);
    if (g_attr_done.count(key)) return 0;
  }
  ATSC3_CUDA(cudaFuncSetAttribute((const void *)fn,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  max_dyn_smem(dev)));
  ATSC3_CUDA(cudaFuncSetAttribute(
      (const void *)fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  std::lock_guard<std::mutex> g(g_attr_mu);
  g_attr_done[key] = 1;
  return 0;
}

static int32_t max_clusters(FloodFn fn, int cl, int smem, int threads, int dev,
                            int *out) {
  OccKey key{fn, cl, smem, threads, dev};
  {
    std::lock_guard<std::mutex> g(g_occ_mu);
    auto it = g_occ.find(key);
    if (it != g_occ.end()) {
      *out = it->second;
      return 0;
    }
  }
  int32_t rc = prepare_fn(fn, dev);
  if (rc) return rc;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(cl, 1, 1);
  cfg.blockDim = dim3(threads, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cl;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int n = 0;
  ATSC3_CUDA(cudaOccupancyMaxActiveClusters(&n, (const void *)fn, &cfg));
  {
    std::lock_guard<std::mutex> g(g_occ_mu);
    g_occ[key] = n;
  }
  *out = n;
  return 0;
}

int32_t flood_launch(const atsc3_ldpc_plan *p, const void *llr, int64_t ld_llr,
                     int nblk, int iters, double alpha, int semantics,
                     uint8_t *bits, int64_t ld_bits, uint8_t *hard,
                     int64_t ld_hard, uint8_t *conv, int32_t *its,
                     int32_t *bad, int threads, cudaStream_t stream,
                     int max_clusters_cap) {
  ATSC3_ARG(p != nullptr, "null plan");
  ATSC3_ARG(nblk >= 0, "nblk < 0");
  ATSC3_ARG(iters >= 0, "iters < 0");
  ATSC3_ARG(semantics >= SEM_KERNEL && semantics <= SEM_TORCH_F16,
            "semantics must be 0, 1, 2 or 3");
  ATSC3_ARG(!(semantics != SEM_KERNEL && iters == 0), "semantics 1-3 need iters >= 1");
  ATSC3_ARG(!(p->dtype == 1 && semantics != SEM_TORCH),
            "float64 messages are only offered with semantics 1");
  ATSC3_ARG(ld_llr >= p->n, "ld_llr < n");
  ATSC3_ARG(bits == nullptr || ld_bits >= p->n, "ld_bits < n");
  ATSC3_ARG(hard == nullptr || (ld_hard >= (p->n + 7) / 8 && ld_hard % 4 == 0 &&
                                ((uintptr_t)hard & 3) == 0),
            "hard needs ld_hard >= ceil(n/8), a multiple of 4, 4-byte aligned");
  if (nblk == 0) return 0;
  ATSC3_ARG(conv && its && bad, "null status output");
  ATSC3_ARG(llr != nullptr, "null llr");
  if (threads <= 0) threads = 1024;
  ATSC3_ARG(threads % 32 == 0 && threads >= 64 && threads <= 1024,
            "threads must be a multiple of 32 in [64, 1024]");
  FloodFn fn = flood_fn(p->dtype, p->rec_bytes, semantics);
  if (!fn) {
    set_error("unsupported: no kernel for this dtype/record/semantics");
    return -4;
  }
  int ncl = 0;
  int32_t rc = max_clusters(fn, p->cluster, p->smem_bytes, threads, p->device,
                            &ncl);
  if (rc) return rc;
  if (ncl <= 0) {
    set_error("unsupported: cluster configuration cannot be resident");
    return -4;
  }
  rc = prepare_fn(fn, p->device);
  if (rc) return rc;
  if (max_clusters_cap > 0) ncl = std::min(ncl, max_clusters_cap);
  ncl = std::min(ncl, nblk);
  FloodArgs a;
  a.llr = llr;
  a.ld_llr = ld_llr;
  a.nblk = nblk;
  a.n = p->n;
  a.nc = p->nc;
  a.iters = iters;
  a.alpha = alpha;
  a.cent = p->d_cent;
  a.cslice = p->d_cslice;
  a.nslc = p->nslc;
  a.vent = p->d_vent;
  a.vslice = p->d_vslice;
  a.nslv = p->nslv;
  a.ncp = p->ncp;
  a.nvlog2 = p->nvlog2;
  a.bits = bits;
  a.ld_bits = ld_bits;
  a.hard = hard;
  a.ld_hard = ld_hard;
  a.conv = conv;
  a.its = its;
  a.bad = bad;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(ncl * p->cluster, 1, 1);
  cfg.blockDim = dim3(threads, 1, 1);
  cfg.dynamicSmemBytes = p->smem_bytes;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = p->cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  ATSC3_CUDA(cudaLaunchKernelEx(&cfg, fn, a));
  return 0;
}

int32_t plan_create(const int32_t *cptr, const int32_t *cidx,
                    const int32_t *vptr, const int32_t *vedge, int n, int nc,
                    int nedges, int dtype, int cluster, atsc3_ldpc_plan **out) {
  ATSC3_ARG(out != nullptr, "null output");
  ATSC3_ARG(cptr && cidx && vptr && vedge, "null CSR table");
  ATSC3_ARG(dtype == 0 || dtype == 1, "dtype must be 0 or 1");
  *out = nullptr;
  int dev = 0;
  ATSC3_CUDA(cudaGetDevice(&dev));
  const int smax = max_dyn_smem(dev);
  // degree check first, so -1 wins over every other complaint
  int dmax_c = 0;
  for (int c = 0; c < nc; ++c) dmax_c = std::max(dmax_c, cptr[c + 1] - cptr[c]);
  if (dmax_c > ATSC3_MAX_ROW_DEG) {
    set_error("check degree above 128");
    return -1;
  }
  const int rb = record_bytes(dtype, dmax_c);
  if (!rb) {
    set_error("unsupported: check degree too high for float64 records");
    return -4;
  }
  int cl = cluster;
  if (cl == 0) {
    for (cl = 1; cl <= 16; cl <<= 1) {
      int per = (nc + cl - 1) / cl;
      int ncp = (per + 31) / 32 * 32;
      int nvl = 5;
      while ((1 << nvl) < (n + cl - 1) / cl) ++nvl;
      if (plan_smem_bytes(dtype, rb, ncp, nvl) <= smax) break;
    }
    if (cl > 16) {
      set_error("unsupported: code state does not fit 16 CTAs of shared memory");
      return -4;
    }
  }
  auto *p = new atsc3_ldpc_plan();
  std::vector<uint16_t> cent;
  std::vector<int32_t> cslice, vslice;
  std::vector<uint32_t> vent;
  int rc = build_tables(cptr, cidx, vptr, vedge, n, nc, nedges, cl, &p->ncp,
                        &p->nvlog2, cent, cslice, vent, vslice, &p->dmax_c,
                        &p->dmax_v);
  if (rc) {
    delete p;
    return rc;
  }
  p->n = n;
  p->nc = nc;
  p->nedges = nedges;
  p->cluster = cl;
  p->dtype = dtype;
  p->rec_bytes = rb;
  p->nslc = (nc + 31) / 32;
  p->nslv = (n + 31) / 32;
  p->device = dev;
  p->smem_bytes = plan_smem_bytes(dtype, rb, p->ncp, p->nvlog2);
  if (p->smem_bytes > smax) {
    delete p;
    set_error("unsupported: per-CTA shared memory above the device limit; "
              "use a larger cluster");
    return -4;
  }
  auto up = [&](void **dst, const void *src, size_t bytes) -> cudaError_t {
    cudaError_t e = cudaMalloc(dst, bytes ? bytes : 4);
    if (e != cudaSuccess) return e;
    p->table_bytes += (int64_t)bytes;
    return bytes ? cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice)
                 : cudaSuccess;
  };
  cudaError_t e = up((void **)&p->d_cent, cent.data(), cent.size() * 2);
  if (e == cudaSuccess) e = up((void **)&p->d_cslice, cslice.data(), cslice.size() * 4);
  if (e == cudaSuccess) e = up((void **)&p->d_vent, vent.data(), vent.size() * 4);
  if (e == cudaSuccess) e = up((void **)&p->d_vslice, vslice.data(), vslice.size() * 4);
  if (e != cudaSuccess) {
    atsc3_ldpc_plan_destroy(p);
    return cuda_fail(e, "plan table upload");
  }
  *out = p;
  return 0;
}

// ---------------------------------------------------------------------------
// the reference ABI: host pointers in, host pointers out
// ---------------------------------------------------------------------------

static uint64_t fnv1a(uint64_t h, const void *p, size_t bytes) {
  const unsigned char *c = (const unsigned char *)p;
  for (size_t i = 0; i < bytes; ++i) {
    h ^= c[i];
    h *= 1099511628211ull;
  }
  return h;
}

// A code's plan for the host-pointer entry point: the edge-buffer
// quasi-cyclic plan when the tables are an A/322 code (Type A or B) that
// decoder takes (atsc3_ldpc_qc_detect2), else the CSR plan.  Both are bit-exact with
// lab/ldpc_kernel.c.
struct HostPlanEntry {
  atsc3_ldpc_plan *plan;
  atsc3_ldpc_qce_plan *qce;
  uint64_t hash;
};
static std::mutex g_hp_mu;
static std::unordered_map<uint64_t, HostPlanEntry> g_hp;   // by content hash

static uint64_t content_hash(const int32_t *cptr, const int32_t *cidx,
                             const int32_t *vptr, const int32_t *vedge, int n,
                             int nc, int ne, int dev) {
  uint64_t h = 1469598103934665603ull;
  int hdr[4] = {n, nc, ne, dev};
  h = fnv1a(h, hdr, sizeof(hdr));
  h = fnv1a(h, cptr, (size_t)(nc + 1) * 4);
  h = fnv1a(h, cidx, (size_t)ne * 4);
  h = fnv1a(h, vptr, (size_t)(n + 1) * 4);
  h = fnv1a(h, vedge, (size_t)ne * 4);
  return h;
}

static thread_local cudaStream_t t_stream = nullptr;

int32_t minsum_f32_host(const float *llr, int32_t nblk, int32_t n, int32_t nc,
                        int32_t nedges, const int32_t *cptr,
                        const int32_t *cidx, const int32_t *vptr,
                        const int32_t *vedge, int32_t iters, float alpha,
                        uint8_t *bits, uint8_t *conv, int32_t *its,
                        int32_t *bad) {
  ATSC3_ARG(cptr && cidx && vptr && vedge, "null CSR table");
  ATSC3_ARG(n > 0 && nc > 0 && nedges >= 0 && nblk >= 0 && iters >= 0,
            "negative size");
  for (int c = 0; c < nc; ++c)
    if (cptr[c + 1] - cptr[c] > ATSC3_MAX_ROW_DEG) {
      set_error("check degree above 128");
      return -1;
    }
  if (nblk == 0) return 0;
  ATSC3_ARG(llr && bits && conv && its && bad, "null buffer");
  int dev = 0;
  ATSC3_CUDA(cudaGetDevice(&dev));
  const uint64_t h = content_hash(cptr, cidx, vptr, vedge, n, nc, nedges, dev);
  atsc3_ldpc_plan *plan = nullptr;
  atsc3_ldpc_qce_plan *qce = nullptr;
  {
    std::lock_guard<std::mutex> g(g_hp_mu);
    auto it = g_hp.find(h);
    if (it != g_hp.end()) {
      plan = it->second.plan;
      qce = it->second.qce;
    }
  }
  if (!plan && !qce) {
    std::vector<int32_t> rowptr((size_t)n / 360 + 1), addr((size_t)nedges + 1);
    int32_t kq[3] = {0, 0, 0};
    if (atsc3_ldpc_qc_detect2(cptr, cidx, vptr, vedge, n, nc, nedges, kq,
                              rowptr.data(), addr.data()) == 0) {
      const int32_t rc = atsc3_ldpc_qce_plan_create2(n, kq[0], kq[1], kq[2], rowptr.data(),
                                                     addr.data(), 0, &qce);
      if (rc != 0 && rc != -4) return rc;   // -4: a structure it does not take
      if (rc) qce = nullptr;
    }
    if (!qce) {
      int32_t rc = plan_create(cptr, cidx, vptr, vedge, n, nc, nedges, 0, 0, &plan);
      if (rc) return rc;
    }
    std::lock_guard<std::mutex> g(g_hp_mu);
    auto it = g_hp.find(h);
    if (it != g_hp.end()) {
      if (plan) atsc3_ldpc_plan_destroy(plan);
      if (qce) atsc3_ldpc_qce_plan_destroy(qce);
      plan = it->second.plan;
      qce = it->second.qce;
    } else {
      g_hp[h] = HostPlanEntry{plan, qce, h};
    }
  }
  if (!t_stream) ATSC3_CUDA(cudaStreamCreateWithFlags(&t_stream, cudaStreamNonBlocking));
  cudaStream_t st = t_stream;
  const size_t nl = (size_t)nblk * n;
  char *buf = nullptr;
  const size_t o_llr = 0, o_bits = nl * 4, o_conv = o_bits + ((nl + 15) & ~15ull);
  const size_t o_its = o_conv + (((size_t)nblk + 15) & ~15ull);
  const size_t o_bad = o_its + (size_t)nblk * 4;
  const size_t total = o_bad + (size_t)nblk * 4;
  ATSC3_CUDA(cudaMallocAsync((void **)&buf, total, st));
  int32_t rc = 0;
  cudaError_t e = cudaMemcpyAsync(buf + o_llr, llr, nl * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) {
    if (qce)
      rc = atsc3_ldpc_qce_decode(qce, (const float *)(buf + o_llr), n, nblk, iters,
                                 alpha, 0, (uint8_t *)(buf + o_bits), n, nullptr, 0,
                                 (uint8_t *)(buf + o_conv), (int32_t *)(buf + o_its),
                                 (int32_t *)(buf + o_bad), 0, st);
    else
      rc = flood_launch(plan, buf + o_llr, n, nblk, iters, (double)alpha, 0,
                        (uint8_t *)(buf + o_bits), n, nullptr, 0,
                        (uint8_t *)(buf + o_conv), (int32_t *)(buf + o_its),
                        (int32_t *)(buf + o_bad), 0, st, 0);
    if (rc == 0) {
      e = cudaMemcpyAsync(bits, buf + o_bits, nl, cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = cudaMemcpyAsync(conv, buf + o_conv, nblk, cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = cudaMemcpyAsync(its, buf + o_its, (size_t)nblk * 4, cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = cudaMemcpyAsync(bad, buf + o_bad, (size_t)nblk * 4, cudaMemcpyDeviceToHost, st);
    }
  }
  cudaError_t e2 = cudaFreeAsync(buf, st);
  cudaError_t e3 = cudaStreamSynchronize(st);
  if (rc) return rc;
  if (e != cudaSuccess) return cuda_fail(e, "ldpc_minsum_f32 copy");
  if (e2 != cudaSuccess) return cuda_fail(e2, "ldpc_minsum_f32 free");
  if (e3 != cudaSuccess) return cuda_fail(e3, "ldpc_minsum_f32 sync");
  return 0;
}

}  // namespace atsc3

// ---------------------------------------------------------------------------
// exported C ABI
// ---------------------------------------------------------------------------

extern "C" {

int32_t ldpc_kernel_abi(void) { return 1; }

int32_t ldpc_minsum_f32(const float *llr, int32_t nblk, int32_t n, int32_t nc,
                        int32_t nedges, const int32_t *cptr,
                        const int32_t *cidx, const int32_t *vptr,
                        const int32_t *vedge, int32_t iters, float alpha,
                        uint8_t *bits, uint8_t *conv, int32_t *its,
                        int32_t *bad, float *work) {
  (void)work;
  return atsc3::minsum_f32_host(llr, nblk, n, nc, nedges, cptr, cidx, vptr,
                                vedge, iters, alpha, bits, conv, its, bad);
}

int32_t atsc3_ldpc_plan_create(const int32_t *cptr, const int32_t *cidx,
                               const int32_t *vptr, const int32_t *vedge,
                               int32_t n, int32_t nc, int32_t nedges,
                               int32_t dtype, int32_t cluster,
                               atsc3_ldpc_plan **out) {
  return atsc3::plan_create(cptr, cidx, vptr, vedge, n, nc, nedges, dtype,
                            cluster, out);
}

void atsc3_ldpc_plan_destroy(atsc3_ldpc_plan *p) {
  if (!p) return;
  cudaFree(p->d_cent);
  cudaFree(p->d_cslice);
  cudaFree(p->d_vent);
  cudaFree(p->d_vslice);
  delete p;
}

int32_t atsc3_ldpc_plan_info(const atsc3_ldpc_plan *p, int64_t *info) {
  ATSC3_ARG(p && info, "null argument");
  info[0] = p->n;
  info[1] = p->nc;
  info[2] = p->nedges;
  info[3] = p->cluster;
  info[4] = p->smem_bytes;
  info[5] = p->rec_bytes;
  info[6] = p->dmax_c;
  info[7] = p->dmax_v;
  info[8] = p->table_bytes;
  info[9] = p->dtype;
  return 0;
}

int32_t atsc3_ldpc_flood_config(const atsc3_ldpc_plan *plan, int32_t threads,
                                int32_t semantics, int32_t *out) {
  ATSC3_ARG(plan && out, "null argument");
  if (threads <= 0) threads = 1024;
  atsc3::FloodFn fn = atsc3::flood_fn(plan->dtype, plan->rec_bytes, semantics);
  ATSC3_ARG(fn != nullptr, "no kernel for this dtype/semantics");
  int ncl = 0;
  int32_t rc = atsc3::max_clusters(fn, plan->cluster, plan->smem_bytes, threads,
                                   plan->device, &ncl);
  if (rc) return rc;
  out[0] = ncl;
  out[1] = plan->cluster;
  out[2] = plan->smem_bytes;
  out[3] = threads;
  return 0;
}

int32_t atsc3_ldpc_decode_flood(const atsc3_ldpc_plan *plan, const void *llr,
                                int64_t ld_llr, int32_t nblk, int32_t iters,
                                double alpha, int32_t semantics, uint8_t *bits,
                                int64_t ld_bits, uint8_t *hard, int64_t ld_hard,
                                uint8_t *conv, int32_t *its, int32_t *bad,
                                int32_t threads, void *stream) {
  return atsc3::flood_launch(plan, llr, ld_llr, nblk, iters, alpha, semantics,
                             bits, ld_bits, hard, ld_hard, conv, its, bad,
                             threads, (cudaStream_t)stream, 0);
}

int32_t atsc3_ldpc_tables_host(const int32_t *cptr, const int32_t *cidx,
                               const int32_t *vptr, const int32_t *vedge,
                               int32_t n, int32_t nc, int32_t nedges,
                               int32_t cluster, int64_t *sizes, uint16_t *cent,
                               int32_t *cslice, uint32_t *vent,
                               int32_t *vslice) {
  ATSC3_ARG(cptr && cidx && vptr && vedge && sizes, "null argument");
  std::vector<uint16_t> c;
  std::vector<int32_t> cs, vs;
  std::vector<uint32_t> v;
  int ncp = 0, nvl = 0, dmc = 0, dmv = 0;
  int rc = atsc3::build_tables(cptr, cidx, vptr, vedge, n, nc, nedges, cluster,
                               &ncp, &nvl, c, cs, v, vs, &dmc, &dmv);
  if (rc) return rc;
  sizes[0] = (int64_t)c.size();
  sizes[1] = (int64_t)cs.size();
  sizes[2] = (int64_t)v.size();
  sizes[3] = (int64_t)vs.size();
  sizes[4] = ncp;
  sizes[5] = nvl;
  if (cent) std::memcpy(cent, c.data(), c.size() * 2);
  if (cslice) std::memcpy(cslice, cs.data(), cs.size() * 4);
  if (vent) std::memcpy(vent, v.data(), v.size() * 4);
  if (vslice) std::memcpy(vslice, vs.data(), vs.size() * 4);
  return 0;
}

}  // extern "C"

// ===========================================================================
// uneven batches: one persistent launch over codewords of different codes
// ===========================================================================

namespace atsc3 {

struct BatchPlanDev {
  CwView g;
  int rb;
  int pad[3];
};

struct BatchArgs {
  const BatchPlanDev *plans;
  const int32_t *bplan;      // plan index of each block
  const int32_t *order;      // queue position -> block (most work first)
  const float *llr;
  const int64_t *llr_off;    // floats
  uint8_t *hard;
  const int64_t *hard_off;   // bytes, 4-byte aligned
  uint8_t *conv;
  int32_t *its;
  int32_t *bad;
  int32_t *counter;          // zeroed before the launch
  int nblk, iters;
  float alpha;
};

// Clusters pull blocks from a device queue: rank 0 takes the next position
// and writes the block index into every CTA's slot (shared word 0); the
// codeword's state starts at shared byte 16.
__global__ void __launch_bounds__(1024, 1) ldpc_batch_kernel(const BatchArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  int *slot = reinterpret_cast<int *>(smem);
  const uint32_t slot_sa = smem_u32(slot);
  const int rank = (int)cluster_ctarank();
  const int CL = (int)cluster_nctarank();
  for (;;) {
    if (rank == 0 && threadIdx.x == 0) {
      const int q = atomicAdd(a.counter, 1);
      const int b = q < a.nblk ? __ldg(a.order + q) : -1;
      for (int r = 0; r < CL; ++r) dsmem_st_u32(dsmem_map(slot_sa, (uint32_t)r), (uint32_t)b);
    }
    cluster_sync_all();
    const int b = *slot;
    cluster_sync_all();            // everyone has read the slot
    if (b < 0) break;
    const BatchPlanDev P = a.plans[__ldg(a.bplan + b)];
    const float *lam = a.llr + __ldg(a.llr_off + b);
    uint8_t *hr = a.hard ? a.hard + __ldg(a.hard_off + b) : nullptr;
    if (P.rb == 16)
      flood_codeword<float, 16, SEM_KERNEL>(P.g, lam, a.iters, a.alpha, smem + 16,
                                       rank, CL, nullptr, hr, a.conv + b,
                                       a.its + b, a.bad + b);
    else
      flood_codeword<float, 32, SEM_KERNEL>(P.g, lam, a.iters, a.alpha, smem + 16,
                                       rank, CL, nullptr, hr, a.conv + b,
                                       a.its + b, a.bad + b);
  }
  __syncthreads();
  cluster_sync_all();
}

}  // namespace atsc3

extern "C" {

int32_t atsc3_ldpc_batch_prepare(const atsc3_ldpc_plan *const *plans,
                                 int32_t nplans, void *desc,
                                 int32_t *cluster_out, int32_t *smem_out) {
  using namespace atsc3;
  ATSC3_ARG(plans && nplans > 0 && desc && cluster_out && smem_out, "bad argument");
  std::vector<BatchPlanDev> h(nplans);
  int cl = plans[0]->cluster, smem = 0;
  for (int i = 0; i < nplans; ++i) {
    const atsc3_ldpc_plan *p = plans[i];
    ATSC3_ARG(p && p->dtype == 0, "batch plans must be float32 CSR plans");
    ATSC3_ARG(p->cluster == cl, "batch plans must share one cluster size");
    ATSC3_ARG(p->rec_bytes == 16 || p->rec_bytes == 32, "record size");
    h[i].g = CwView{p->n, p->nc, p->ncp, p->nvlog2, p->nslc, p->nslv,
                    p->d_cent, p->d_cslice, p->d_vent, p->d_vslice};
    h[i].rb = p->rec_bytes;
    smem = std::max(smem, p->smem_bytes);
  }
  ATSC3_CUDA(cudaMemcpy(desc, h.data(), h.size() * sizeof(BatchPlanDev),
                        cudaMemcpyHostToDevice));
  *cluster_out = cl;
  *smem_out = smem + 16;
  return 0;
}

int32_t atsc3_ldpc_batch_desc_bytes(int32_t nplans, int64_t *bytes) {
  ATSC3_ARG(nplans > 0 && bytes, "bad argument");
  *bytes = (int64_t)nplans * (int64_t)sizeof(atsc3::BatchPlanDev);
  return 0;
}

int32_t atsc3_ldpc_batch_decode(const void *desc, int32_t cluster, int32_t smem,
                                const int32_t *bplan, const int32_t *order,
                                int32_t nblk, const float *llr,
                                const int64_t *llr_off, uint8_t *hard,
                                const int64_t *hard_off, uint8_t *conv,
                                int32_t *its, int32_t *bad, int32_t iters,
                                float alpha, int32_t *counter, int32_t threads,
                                int32_t cap_clusters, void *stream) {
  using namespace atsc3;
  ATSC3_ARG(desc && bplan && order && llr && llr_off && conv && its && bad &&
                counter,
            "null pointer");
  ATSC3_ARG(cluster >= 1 && cluster <= 16, "cluster");
  ATSC3_ARG(iters >= 0 && nblk >= 0, "negative size");
  if (nblk == 0) return 0;
  if (threads <= 0) threads = 1024;
  ATSC3_ARG(threads % 32 == 0 && threads >= 64 && threads <= 1024, "threads");
  int dev = 0;
  ATSC3_CUDA(cudaGetDevice(&dev));
  FloodFn fn = reinterpret_cast<FloodFn>(ldpc_batch_kernel);
  int32_t rc = prepare_fn(fn, dev);
  if (rc) return rc;
  int ncl = 0;
  rc = max_clusters(fn, cluster, smem, threads, dev, &ncl);
  if (rc) return rc;
  if (ncl <= 0) {
    set_error("unsupported: batch cluster configuration cannot be resident");
    return -4;
  }
  if (cap_clusters > 0) ncl = std::min(ncl, cap_clusters);
  ncl = std::min(ncl, nblk);
  BatchArgs a;
  a.plans = reinterpret_cast<const BatchPlanDev *>(desc);
  a.bplan = bplan;
  a.order = order;
  a.llr = llr;
  a.llr_off = llr_off;
  a.hard = hard;
  a.hard_off = hard_off;
  a.conv = conv;
  a.its = its;
  a.bad = bad;
  a.counter = counter;
  a.nblk = nblk;
  a.iters = iters;
  a.alpha = alpha;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(ncl * cluster, 1, 1);
  cfg.blockDim = dim3(threads, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = (cudaStream_t)stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  ATSC3_CUDA(cudaLaunchKernelEx(&cfg, ldpc_batch_kernel, a));
  return 0;
}

}  // extern "C"

