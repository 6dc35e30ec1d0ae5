// ldpc_qc.cu -- flooding normalised min-sum for the quasi-cyclic A/322 Type B
// codes (sm_100a), bit-exact with lab/ldpc_kernel.c.
//
// Structure used (A/322 6.1.3.2, the construction of lab/m3_ldpc.py:166-212
// for Type B): with Z = 360, Q = (N-K)/360 and table entry x of information
// group g written x = Q*u + r, information bit m = 360*g + mm sits in check
// a = Q*((u + mm) mod 360) + r.  So check a = Q*k + r is row k of BLOCK ROW
// r, every (r, g) pair holds at most one circulant (verified on the host),
// and the parity bits form the dual diagonal: check (r, k) also holds parity
// bits K + 360*(r-1) + k and K + 360*r + k (r >= 1), or K + k and
// K + 360*(Q-1) + k-1 (r = 0, the latter only for k >= 1).
//
// Consequences exploited here:
//  * a check's columns, sorted ascending, are its information circulants in
//    block-column order followed by its two parity bits, so each edge's
//    position inside its check is a per-circulant constant;
//  * a variable's edges in ascending check order (the reference's summation
//    order, vedge = stable argsort of cidx) are its column's circulants sorted
//    by (u, r) and rotated: the ones with u + mm >= 360 wrap to small k and
//    come first.  s0[g*360 + mm] (precomputed, one byte) is where the
//    rotation starts;
//  * a warp of 32 consecutive checks (or bits) reads 32 consecutive
//    posteriors (or records) per circulant: coalesced DSMEM traffic, and the
//    only tables are a few KB of circulant descriptors.
//
// State per codeword lives in the distributed shared memory of one cluster,
// as in ldpc_flood.cu: posteriors partitioned by bit index (power of two per
// CTA), check records (min1*alpha, min2*alpha, signs, first position)
// partitioned by block row.  Work is split per CTA by block rows (check
// phase) and by edge-balanced runs of 32-bit chunks (variable phase).

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "../../include/atsc3_fec.h"
#include "common.cuh"

namespace atsc3 {

constexpr int QZ = 360;
constexpr int QCHUNK = 12;                 // ceil(360 / 32) warps per row/column
constexpr int QMAXCL = 16;

struct QcPlan {
  int n = 0, K = 0, Q = 0, nbi = 0;
  int cluster = 1, nvlog2 = 0, rows_per_cta = 0, ncp = 0, smem = 0;
  int di_max = 0, dc_max = 0, device = 0;
  int64_t table_bytes = 0;
  int rb[QMAXCL + 1] = {0};     // block rows of CTA c: [rb[c], rb[c+1])
  int wb[QMAXCL + 1] = {0};     // variable-phase work items of CTA c
  int2 *d_rdesc = nullptr;      // per row circulant: {360*g - u, u}
  int32_t *d_rptr = nullptr;    // (Q+1)
  int4 *d_cdesc = nullptr;      // per column circulant: {rank | pos<<8, rowoff, u, 0}
  int32_t *d_cptr = nullptr;    // (nbi+1)
  uint8_t *d_s0 = nullptr;      // (nbi*360) rotation start
  int32_t *d_rowinfo = nullptr; // per row: rank | (d_r << 8), rowoff  (2*Q)
};

struct QcTables {
  std::vector<int2> rdesc;
  std::vector<int32_t> rptr;
  std::vector<int4> cdesc;
  std::vector<int32_t> cptr;
  std::vector<uint8_t> s0;
  std::vector<int32_t> rowinfo;
};

// Host: derive the block-row / block-column descriptors from the Annex A
// address rows.  Returns 0, -3 or -4 (not a dup-free Type B code).
int qc_build(int n, int K, int Q, const int32_t *rowptr, const int32_t *addr,
             int cluster, QcPlan *p, QcTables *t) {
  if (n % QZ || K % QZ || Q <= 0 || (n - K) != Q * QZ) {
    set_error("invalid argument: not a 360-circulant Type B code");
    return -3;
  }
  if (cluster < 1 || cluster > QMAXCL || (cluster & (cluster - 1))) {
    set_error("invalid argument: cluster must be 1, 2, 4, 8 or 16");
    return -3;
  }
  if (n > 65535) {
    set_error("unsupported: codeword length above 65535");
    return -4;
  }
  const int nbi = K / QZ;
  struct Circ { int g, r, u; };
  std::vector<std::vector<Circ>> rows(Q), cols(nbi);
  for (int g = 0; g < nbi; ++g) {
    for (int e = rowptr[g]; e < rowptr[g + 1]; ++e) {
      int x = addr[e];
      if (x < 0 || x >= n - K) {
        set_error("invalid argument: address outside the parity range");
        return -3;
      }
      Circ c{g, x % Q, x / Q};
      rows[c.r].push_back(c);
      cols[g].push_back(c);
    }
  }
  int di = 0;
  for (int r = 0; r < Q; ++r) {
    auto &R = rows[r];
    std::sort(R.begin(), R.end(), [](const Circ &a, const Circ &b) {
      return a.g < b.g;
    });
    for (size_t i = 1; i < R.size(); ++i)
      if (R[i].g == R[i - 1].g) {
        set_error("unsupported: two circulants share a block (use the CSR "
                  "decoder)");
        return -4;
      }
    di = std::max(di, (int)R.size());
  }
  if (di + 2 > 64) {
    set_error("unsupported: block-row degree above 62");
    return -4;
  }
  // partition block rows over the cluster (contiguous, balanced by count)
  p->n = n; p->K = K; p->Q = Q; p->nbi = nbi; p->cluster = cluster;
  p->di_max = di;
  p->dc_max = 0;
  int per = (Q + cluster - 1) / cluster;
  for (int c = 0; c <= cluster; ++c) p->rb[c] = std::min(Q, c * per);
  p->rows_per_cta = per;
  p->ncp = per * QZ;
  std::vector<int> rrank(Q), rowoff(Q);
  for (int r = 0; r < Q; ++r) {
    rrank[r] = r / per;
    rowoff[r] = (r - p->rb[rrank[r]]) * QZ;
  }
  int nvper = (n + cluster - 1) / cluster, nvl = 5;
  while ((1 << nvl) < nvper) ++nvl;
  p->nvlog2 = nvl;
  // row descriptors
  t->rptr.assign(Q + 1, 0);
  t->rdesc.clear();
  for (int r = 0; r < Q; ++r) {
    for (auto &c : rows[r]) t->rdesc.push_back(make_int2(QZ * c.g - c.u, c.u));
    t->rptr[r + 1] = (int)t->rdesc.size();
  }
  t->rowinfo.assign(2 * Q, 0);
  for (int r = 0; r < Q; ++r) {
    t->rowinfo[2 * r] = rrank[r] | ((int)rows[r].size() << 8);
    t->rowinfo[2 * r + 1] = rowoff[r];
  }
  // column descriptors, sorted by (u, r): the summation order before rotation
  t->cptr.assign(nbi + 1, 0);
  t->cdesc.clear();
  t->s0.assign((size_t)nbi * QZ, 0);
  for (int g = 0; g < nbi; ++g) {
    auto &Cc = cols[g];
    std::sort(Cc.begin(), Cc.end(), [](const Circ &a, const Circ &b) {
      return a.u != b.u ? a.u < b.u : a.r < b.r;
    });
    p->dc_max = std::max(p->dc_max, (int)Cc.size());
    for (auto &c : Cc) {
      int pos = 0;
      for (auto &o : rows[c.r]) {
        if (o.g == g) break;
        ++pos;
      }
      t->cdesc.push_back(make_int4(rrank[c.r] | (pos << 8), rowoff[c.r], c.u, 0));
    }
    t->cptr[g + 1] = (int)t->cdesc.size();
    for (int mm = 0; mm < QZ; ++mm) {
      int s = 0;
      for (auto &c : Cc) s += (c.u + mm < QZ) ? 1 : 0;
      t->s0[(size_t)g * QZ + mm] = (uint8_t)s;
    }
  }
  // variable-phase work items: (block column b, chunk q), w = b*12 + q,
  // split into CL runs of equal edge count
  const int ncols = nbi + Q;
  std::vector<int64_t> wcost((size_t)ncols * QCHUNK);
  int64_t total = 0;
  for (int b = 0; b < ncols; ++b) {
    int deg = b < nbi ? (int)cols[b].size() : 2;
    for (int q = 0; q < QCHUNK; ++q) {
      int lanes = std::min(32, QZ - 32 * q);
      wcost[(size_t)b * QCHUNK + q] = (int64_t)lanes * deg + 8;
      total += wcost[(size_t)b * QCHUNK + q];
    }
  }
  int64_t acc = 0;
  int c = 1;
  p->wb[0] = 0;
  for (int w = 0; w < (int)wcost.size() && c < cluster; ++w) {
    acc += wcost[w];
    while (c < cluster && acc * cluster >= total * c) p->wb[c++] = w + 1;
  }
  while (c <= cluster) p->wb[c++] = (int)wcost.size();
  p->smem = (1 << nvl) * 4 + p->ncp * 16 + 256;
  return 0;
}

struct QcArgs {
  const float *llr;
  int64_t ld_llr;
  int nblk, n, K, Q, iters;
  float alpha;
  int nvlog2, ncp;
  int rb[QMAXCL + 1];
  int wb[QMAXCL + 1];
  const int2 *rdesc;
  const int32_t *rptr;
  const int4 *cdesc;
  const int32_t *cptr;
  const uint8_t *s0;
  const int32_t *rowinfo;
  int nbi;
  uint8_t *bits;
  int64_t ld_bits;
  uint8_t *hard;
  int64_t ld_hard;
  uint8_t *conv;
  int32_t *its;
  int32_t *bad;
};

__device__ __forceinline__ float qc_msg(uint4 r, int pos) {
  const float A = __uint_as_float(r.x), B = __uint_as_float(r.y);
  float m = (pos == (int)(r.w & 0xFFu)) ? B : A;
  const uint32_t s = pos < 32 ? (r.z >> pos) : (r.w >> (pos - 24));
  return (s & 1u) ? -m : m;
}

// DI: unroll bound of information circulants per block row (>= di_max).
template <bool TORCH, int DI>
__global__ void __launch_bounds__(1024, 1) ldpc_qc_kernel(const QcArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int rank = (int)cluster_ctarank();
  const int CL = (int)cluster_nctarank();
  const int nvp = 1 << a.nvlog2;
  const uint32_t vmask = (uint32_t)nvp - 1u;
  float *tot = reinterpret_cast<float *>(smem);
  uint4 *rec = reinterpret_cast<uint4 *>(smem + (size_t)nvp * 4);
  int *part = reinterpret_cast<int *>(smem + (size_t)nvp * 4 + (size_t)a.ncp * 16);
  int *sbad = part + 32;
  const uint32_t tot_sa = smem_u32(tot);
  const uint32_t rec_sa = smem_u32(rec);
  const uint32_t part_sa = smem_u32(part);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nwarps = blockDim.x >> 5;
  const int r0 = a.rb[rank], r1 = a.rb[rank + 1];
  const int ncitems = (r1 - r0) * QCHUNK;
  const int w0 = a.wb[rank], w1 = a.wb[rank + 1];
  const int vbase = rank * nvp;
  const int vend = min(a.n, vbase + nvp);
  const int K = a.K, Q = a.Q;

  if (tid == 0) *sbad = 0;

  for (int b = (int)cluster_id_x(); b < a.nblk; b += (int)ncluster_x()) {
    const float *lam = a.llr + (size_t)b * a.ld_llr;
    for (int i = vbase + tid; i < vend; i += blockDim.x) tot[i - vbase] = lam[i];
    for (int q = tid; q < a.ncp; q += blockDim.x) rec[q] = make_uint4(0u, 0u, 0u, 0u);
    __syncthreads();
    cluster_sync_all();

    for (int it = 0;; ++it) {
      // ---------------- check phase ----------------------------------------
      int mybad = 0;
      for (int w = warp; w < ncitems; w += nwarps) {
        const int r = r0 + w / QCHUNK;
        const int k = (w % QCHUNK) * 32 + lane;
        if (k < QZ) {
          const int rp = __ldg(a.rptr + r);
          const int d = __ldg(a.rptr + r + 1) - rp;
          const int li = (r - r0) * QZ + k;
          const uint4 ro = rec[li];
          const float Ao = __uint_as_float(ro.x), Bo = __uint_as_float(ro.y);
          const int Fo = (int)(ro.w & 0xFFu);
          float t[DI + 2];
#pragma unroll
          for (int i = 0; i < DI; ++i) {
            if (i < d) {
              const int2 ds = __ldg(a.rdesc + rp + i);
              const uint32_t v = (uint32_t)(ds.x + k + (k < ds.y ? QZ : 0));
              t[i] = dsmem_ld_f32(dsmem_map(tot_sa + (v & vmask) * 4u, v >> a.nvlog2));
            }
          }
          const uint32_t pa = (uint32_t)(r >= 1 ? K + QZ * (r - 1) + k : K + k);
          const bool hasb = r >= 1 || k >= 1;
          const uint32_t pb = (uint32_t)(r >= 1 ? K + QZ * r + k : K + QZ * (Q - 1) + k - 1);
          const float ta = dsmem_ld_f32(dsmem_map(tot_sa + (pa & vmask) * 4u, pa >> a.nvlog2));
          float tb = 0.f;
          if (hasb) tb = dsmem_ld_f32(dsmem_map(tot_sa + (pb & vmask) * 4u, pb >> a.nvlog2));
          float min1 = __int_as_float(0x7f800000), min2 = min1;
          int first = 0;
          uint32_t syn = 0;
          uint64_t sg = 0;
          auto edge = [&](float tv, int j) {
            syn ^= tv < 0.f ? 1u : 0u;
            float mo = (j == Fo) ? Bo : Ao;
            const uint32_t so = j < 32 ? (ro.z >> j) : (ro.w >> (j - 24));
            if (so & 1u) mo = -mo;
            const float v = __fsub_rn(tv, mo);
            if (v < 0.f) sg |= 1ull << j;
            const float mag = fabsf(v);
            if (mag < min1) { min2 = min1; min1 = mag; first = j; }
            else if (mag < min2) { min2 = mag; }
          };
#pragma unroll
          for (int i = 0; i < DI; ++i)
            if (i < d) edge(t[i], i);
          edge(ta, d);
          if (hasb) edge(tb, d + 1);
          const int deg = d + (hasb ? 2 : 1);
          if (__popcll(sg) & 1) sg ^= (deg >= 64 ? ~0ull : ((1ull << deg) - 1ull));
          rec[li] = make_uint4(__float_as_uint(__fmul_rn(min1, a.alpha)),
                               __float_as_uint(__fmul_rn(min2, a.alpha)),
                               (uint32_t)sg,
                               (uint32_t)first | ((uint32_t)(sg >> 32) << 8));
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
      for (int q = 0; q < CL; ++q) badct += part[(it & 1) * 16 + q];
      if (tid == 0) *sbad = 0;
      const bool done = (badct == 0) && (!TORCH || it > 0);
      if (done || it >= a.iters) {
        if (a.bits) {
          uint8_t *bo = a.bits + (size_t)b * a.ld_bits;
          for (int i = vbase + tid; i < vend; i += blockDim.x)
            bo[i] = tot[i - vbase] < 0.f ? 1 : 0;
        }
        if (a.hard) {
          uint8_t *ho = a.hard + (size_t)b * a.ld_hard;
          for (int wq = vbase; wq < vend; wq += 32 * nwarps) {
            const int i = wq + (warp << 5) + lane;
            const bool ng = i < vend && tot[i - vbase] < 0.f;
            const uint32_t m = __ballot_sync(0xffffffffu, ng);
            const int base = wq + (warp << 5);
            if (lane == 0 && base < vend) {
              const uint32_t word = __byte_perm(__brev(m), 0u, 0x0123u);
              if (base + 32 <= vend) {
                *reinterpret_cast<uint32_t *>(ho + (base >> 3)) = word;
              } else {
                const int nbyte = (vend - base + 7) >> 3;
                for (int q = 0; q < nbyte; ++q)
                  ho[(base >> 3) + q] = (uint8_t)(word >> (8 * q));
              }
            }
          }
        }
        if (rank == 0 && tid == 0) {
          a.conv[b] = done ? 1 : 0;
          a.its[b] = it;
          a.bad[b] = done ? 0 : badct;
        }
        break;
      }
      // ---------------- variable phase -------------------------------------
      for (int w = w0 + warp; w < w1; w += nwarps) {
        const int bc = w / QCHUNK;
        const int mm = (w % QCHUNK) * 32 + lane;
        if (mm < QZ) {
          const int lamidx = bc * QZ + mm;
          const float li = lam[lamidx];
          float acc = TORCH ? li : 0.f;
          if (bc < a.nbi) {
            const int cs = __ldg(a.cptr + bc);
            const int d = __ldg(a.cptr + bc + 1) - cs;
            const int s0 = __ldg(a.s0 + (size_t)bc * QZ + mm);
            for (int t0 = 0; t0 < d; t0 += 4) {
              uint4 rr[4];
              int pos[4];
#pragma unroll
              for (int u = 0; u < 4; ++u) {
                pos[u] = -1;
                if (t0 + u < d) {
                  int i = s0 + t0 + u;
                  if (i >= d) i -= d;
                  const int4 ds = __ldg(a.cdesc + cs + i);
                  int kk = ds.z + mm;
                  if (kk >= QZ) kk -= QZ;
                  pos[u] = ds.x >> 8;
                  rr[u] = dsmem_ld_v4(dsmem_map(
                      rec_sa + (uint32_t)(ds.y + kk) * 16u, (uint32_t)(ds.x & 0xFF)));
                }
              }
#pragma unroll
              for (int u = 0; u < 4; ++u)
                if (pos[u] >= 0) acc = __fadd_rn(acc, qc_msg(rr[u], pos[u]));
            }
          } else {
            const int tt = bc - a.nbi;           // parity block column
            const int2 ri = __ldg(reinterpret_cast<const int2 *>(a.rowinfo) + tt);
            const int dt = ri.x >> 8;
            const int p1 = tt >= 1 ? dt + 1 : dt;
            const uint4 m1 = dsmem_ld_v4(dsmem_map(
                rec_sa + (uint32_t)(ri.y + mm) * 16u, (uint32_t)(ri.x & 0xFF)));
            int rank2 = -1, off2 = 0, p2 = 0;
            if (tt + 1 < Q) {
              const int2 r2 = __ldg(reinterpret_cast<const int2 *>(a.rowinfo) + tt + 1);
              rank2 = r2.x & 0xFF;
              off2 = r2.y + mm;
              p2 = r2.x >> 8;
            } else if (mm + 1 < QZ) {
              const int2 r2 = __ldg(reinterpret_cast<const int2 *>(a.rowinfo));
              rank2 = r2.x & 0xFF;
              off2 = r2.y + mm + 1;
              p2 = (r2.x >> 8) + 1;
            }
            uint4 m2 = make_uint4(0u, 0u, 0u, 0u);
            if (rank2 >= 0)
              m2 = dsmem_ld_v4(dsmem_map(rec_sa + (uint32_t)off2 * 16u, (uint32_t)rank2));
            acc = __fadd_rn(acc, qc_msg(m1, p1));
            if (rank2 >= 0) acc = __fadd_rn(acc, qc_msg(m2, p2));
          }
          const float nv = TORCH ? acc : __fadd_rn(li, acc);
          const uint32_t owner = (uint32_t)lamidx >> a.nvlog2;
          if ((int)owner == rank) {
            tot[lamidx - vbase] = nv;
          } else {
            dsmem_st_u32(dsmem_map(tot_sa + ((uint32_t)lamidx & vmask) * 4u, owner),
                         __float_as_uint(nv));
          }
        }
      }
      __syncthreads();
      cluster_sync_all();
    }
  }
  __syncthreads();
  cluster_sync_all();
}

typedef void (*QcFn)(const QcArgs);

static QcFn qc_fn(int semantics, int di) {
  if (di <= 8) return semantics ? ldpc_qc_kernel<true, 8> : ldpc_qc_kernel<false, 8>;
  if (di <= 16) return semantics ? ldpc_qc_kernel<true, 16> : ldpc_qc_kernel<false, 16>;
  if (di <= 32) return semantics ? ldpc_qc_kernel<true, 32> : ldpc_qc_kernel<false, 32>;
  return nullptr;
}

static std::mutex g_qc_mu;
static std::unordered_map<uint64_t, int> g_qc_occ;
static std::unordered_map<uint64_t, int> g_qc_attr;

static int32_t qc_prepare(QcFn fn, int dev) {
  const uint64_t key = (uint64_t)(uintptr_t)fn ^ ((uint64_t)dev << 56);
  {
    std::lock_guard<std::mutex> g(g_qc_mu);
    if (g_qc_attr.count(key)) return 0;
  }
  int smax = 0;
  cudaDeviceGetAttribute(&smax, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  ATSC3_CUDA(cudaFuncSetAttribute((const void *)fn,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  ATSC3_CUDA(cudaFuncSetAttribute(
      (const void *)fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  std::lock_guard<std::mutex> g(g_qc_mu);
  g_qc_attr[key] = 1;
  return 0;
}

static int32_t qc_max_clusters(QcFn fn, int cl, int smem, int threads, int dev,
                               int *out) {
  const uint64_t key = ((uint64_t)(uintptr_t)fn * 1315423911ull) ^
                       ((uint64_t)cl << 1) ^ ((uint64_t)smem << 8) ^
                       ((uint64_t)threads << 30) ^ ((uint64_t)dev << 44);
  {
    std::lock_guard<std::mutex> g(g_qc_mu);
    auto it = g_qc_occ.find(key);
    if (it != g_qc_occ.end()) {
      *out = it->second;
      return 0;
    }
  }
  int32_t rc = qc_prepare(fn, dev);
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
  std::lock_guard<std::mutex> g(g_qc_mu);
  g_qc_occ[key] = n;
  *out = n;
  return 0;
}

}  // namespace atsc3

struct atsc3_ldpc_qc_plan {
  atsc3::QcPlan p;
};

extern "C" {

int32_t atsc3_ldpc_qc_plan_create(int32_t n, int32_t kldpc, int32_t qldpc,
                                  const int32_t *rowptr, const int32_t *addr,
                                  int32_t cluster, atsc3_ldpc_qc_plan **out) {
  using namespace atsc3;
  ATSC3_ARG(out && rowptr && addr, "null argument");
  *out = nullptr;
  int dev = 0;
  ATSC3_CUDA(cudaGetDevice(&dev));
  int smax = 0;
  ATSC3_CUDA(cudaDeviceGetAttribute(&smax, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  auto *h = new atsc3_ldpc_qc_plan();
  QcTables t;
  int rc = -4;
  if (cluster == 0) {
    for (int cl = 1; cl <= QMAXCL; cl <<= 1) {
      rc = qc_build(n, kldpc, qldpc, rowptr, addr, cl, &h->p, &t);
      if (rc == -3) break;
      if (rc == 0 && h->p.smem <= smax) break;
      rc = -4;
    }
  } else {
    rc = qc_build(n, kldpc, qldpc, rowptr, addr, cluster, &h->p, &t);
    if (rc == 0 && h->p.smem > smax) {
      set_error("unsupported: per-CTA shared memory above the device limit");
      rc = -4;
    }
  }
  if (rc) {
    if (rc == -4 && cluster == 0) set_error("unsupported: no cluster size fits");
    delete h;
    return rc;
  }
  h->p.device = dev;
  auto up = [&](void **dst, const void *src, size_t bytes) -> cudaError_t {
    cudaError_t e = cudaMalloc(dst, bytes ? bytes : 16);
    if (e != cudaSuccess) return e;
    h->p.table_bytes += (int64_t)bytes;
    return bytes ? cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice) : cudaSuccess;
  };
  cudaError_t e = up((void **)&h->p.d_rdesc, t.rdesc.data(), t.rdesc.size() * 8);
  if (e == cudaSuccess) e = up((void **)&h->p.d_rptr, t.rptr.data(), t.rptr.size() * 4);
  if (e == cudaSuccess) e = up((void **)&h->p.d_cdesc, t.cdesc.data(), t.cdesc.size() * 16);
  if (e == cudaSuccess) e = up((void **)&h->p.d_cptr, t.cptr.data(), t.cptr.size() * 4);
  if (e == cudaSuccess) e = up((void **)&h->p.d_s0, t.s0.data(), t.s0.size());
  if (e == cudaSuccess) e = up((void **)&h->p.d_rowinfo, t.rowinfo.data(), t.rowinfo.size() * 4);
  if (e != cudaSuccess) {
    atsc3_ldpc_qc_plan_destroy(h);
    return cuda_fail(e, "qc plan upload");
  }
  *out = h;
  return 0;
}

void atsc3_ldpc_qc_plan_destroy(atsc3_ldpc_qc_plan *h) {
  if (!h) return;
  cudaFree(h->p.d_rdesc);
  cudaFree(h->p.d_rptr);
  cudaFree(h->p.d_cdesc);
  cudaFree(h->p.d_cptr);
  cudaFree(h->p.d_s0);
  cudaFree(h->p.d_rowinfo);
  delete h;
}

int32_t atsc3_ldpc_qc_plan_info(const atsc3_ldpc_qc_plan *h, int64_t *info) {
  ATSC3_ARG(h && info, "null argument");
  info[0] = h->p.n;
  info[1] = h->p.K;
  info[2] = h->p.Q;
  info[3] = h->p.cluster;
  info[4] = h->p.smem;
  info[5] = h->p.di_max;
  info[6] = h->p.dc_max;
  info[7] = h->p.table_bytes;
  info[8] = h->p.rows_per_cta;
  info[9] = h->p.nvlog2;
  return 0;
}

int32_t atsc3_ldpc_qc_tables_host(int32_t n, int32_t kldpc, int32_t qldpc,
                                  const int32_t *rowptr, const int32_t *addr,
                                  int32_t cluster, int32_t *meta,
                                  int32_t *rdesc, int32_t *rptr,
                                  int32_t *cdesc, int32_t *cptr, uint8_t *s0,
                                  int32_t *rowinfo) {
  using namespace atsc3;
  ATSC3_ARG(meta && rowptr && addr, "null argument");
  QcPlan p;
  QcTables t;
  int rc = qc_build(n, kldpc, qldpc, rowptr, addr, cluster, &p, &t);
  if (rc) return rc;
  // meta: [0] rdesc entries [1] cdesc entries [2] nvlog2 [3] ncp
  //       [4] rows/CTA [5] di_max [6] dc_max [7] smem [8..8+CL] rb [25..] wb
  meta[0] = (int32_t)t.rdesc.size();
  meta[1] = (int32_t)t.cdesc.size();
  meta[2] = p.nvlog2;
  meta[3] = p.ncp;
  meta[4] = p.rows_per_cta;
  meta[5] = p.di_max;
  meta[6] = p.dc_max;
  meta[7] = p.smem;
  for (int c = 0; c <= QMAXCL; ++c) {
    meta[8 + c] = p.rb[c];
    meta[25 + c] = p.wb[c];
  }
  if (rdesc) std::memcpy(rdesc, t.rdesc.data(), t.rdesc.size() * 8);
  if (rptr) std::memcpy(rptr, t.rptr.data(), t.rptr.size() * 4);
  if (cdesc) std::memcpy(cdesc, t.cdesc.data(), t.cdesc.size() * 16);
  if (cptr) std::memcpy(cptr, t.cptr.data(), t.cptr.size() * 4);
  if (s0) std::memcpy(s0, t.s0.data(), t.s0.size());
  if (rowinfo) std::memcpy(rowinfo, t.rowinfo.data(), t.rowinfo.size() * 4);
  return 0;
}

int32_t atsc3_ldpc_qc_config(const atsc3_ldpc_qc_plan *h, int32_t threads,
                             int32_t semantics, int32_t *out) {
  using namespace atsc3;
  ATSC3_ARG(h && out, "null argument");
  if (threads <= 0) threads = 1024;
  QcFn fn = qc_fn(semantics, h->p.di_max);
  ATSC3_ARG(fn != nullptr, "no kernel for this degree");
  int ncl = 0;
  int32_t rc = qc_max_clusters(fn, h->p.cluster, h->p.smem, threads, h->p.device, &ncl);
  if (rc) return rc;
  out[0] = ncl;
  out[1] = h->p.cluster;
  out[2] = h->p.smem;
  out[3] = threads;
  return 0;
}

int32_t atsc3_ldpc_qc_decode(const atsc3_ldpc_qc_plan *h, const float *llr,
                             int64_t ld_llr, int32_t nblk, int32_t iters,
                             float alpha, int32_t semantics, uint8_t *bits,
                             int64_t ld_bits, uint8_t *hard, int64_t ld_hard,
                             uint8_t *conv, int32_t *its, int32_t *bad,
                             int32_t threads, void *stream) {
  using namespace atsc3;
  ATSC3_ARG(h != nullptr, "null plan");
  const QcPlan &p = h->p;
  ATSC3_ARG(nblk >= 0 && iters >= 0, "negative size");
  ATSC3_ARG(semantics == 0 || semantics == 1, "semantics must be 0 or 1");
  ATSC3_ARG(!(semantics == 1 && iters == 0), "semantics 1 needs iters >= 1");
  ATSC3_ARG(ld_llr >= p.n, "ld_llr < n");
  ATSC3_ARG(bits == nullptr || ld_bits >= p.n, "ld_bits < n");
  ATSC3_ARG(hard == nullptr || (ld_hard >= (p.n + 7) / 8 && ld_hard % 4 == 0 &&
                                ((uintptr_t)hard & 3) == 0),
            "hard needs ld_hard >= ceil(n/8), a multiple of 4, 4-byte aligned");
  if (nblk == 0) return 0;
  ATSC3_ARG(conv && its && bad, "null status output");
  ATSC3_ARG(llr != nullptr, "null llr");
  if (threads <= 0) threads = 1024;
  ATSC3_ARG(threads % 32 == 0 && threads >= 64 && threads <= 1024,
            "threads must be a multiple of 32 in [64, 1024]");
  QcFn fn = qc_fn(semantics, p.di_max);
  if (!fn) {
    set_error("unsupported: block-row degree too high");
    return -4;
  }
  int ncl = 0;
  int32_t rc = qc_max_clusters(fn, p.cluster, p.smem, threads, p.device, &ncl);
  if (rc) return rc;
  rc = qc_prepare(fn, p.device);
  if (rc) return rc;
  if (ncl <= 0) {
    set_error("unsupported: cluster configuration cannot be resident");
    return -4;
  }
  ncl = std::min(ncl, nblk);
  QcArgs a;
  std::memset(&a, 0, sizeof(a));
  a.llr = llr;
  a.ld_llr = ld_llr;
  a.nblk = nblk;
  a.n = p.n;
  a.K = p.K;
  a.Q = p.Q;
  a.iters = iters;
  a.alpha = alpha;
  a.nvlog2 = p.nvlog2;
  a.ncp = p.ncp;
  for (int c = 0; c <= QMAXCL; ++c) {
    a.rb[c] = p.rb[c];
    a.wb[c] = p.wb[c];
  }
  a.rdesc = p.d_rdesc;
  a.rptr = p.d_rptr;
  a.cdesc = p.d_cdesc;
  a.cptr = p.d_cptr;
  a.s0 = p.d_s0;
  a.rowinfo = p.d_rowinfo;
  a.nbi = p.nbi;
  a.bits = bits;
  a.ld_bits = ld_bits;
  a.hard = hard;
  a.ld_hard = ld_hard;
  a.conv = conv;
  a.its = its;
  a.bad = bad;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(ncl * p.cluster, 1, 1);
  cfg.blockDim = dim3(threads, 1, 1);
  cfg.dynamicSmemBytes = p.smem;
  cfg.stream = (cudaStream_t)stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = p.cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  ATSC3_CUDA(cudaLaunchKernelEx(&cfg, fn, a));
  return 0;
}

}  // extern "C"
