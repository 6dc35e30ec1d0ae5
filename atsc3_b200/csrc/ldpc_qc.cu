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
  int n = 0, K = 0, Q = 0, nbi = 0, nb = 0;
  int cluster = 1, cpc = 0, rows_per_cta = 0, ncp = 0, smem = 0;
  int dr_max = 0, dc_max = 0, device = 0;
  int64_t table_bytes = 0;
  int rb[QMAXCL + 1] = {0};     // block rows of CTA c: [rb[c], rb[c+1])
  int wb[QMAXCL + 1] = {0};     // variable-phase work items of CTA c
  int4 *d_rdesc = nullptr;      // per row edge slot
  int32_t *d_rptr = nullptr;    // (Q+1)
  int4 *d_cdesc = nullptr;      // per column edge slot
  int32_t *d_cptr = nullptr;    // (nb+1)
  uint8_t *d_s0 = nullptr;      // (nb*360) rotation start
};

// One edge slot of a block row or block column, shared by its 360 checks
// (bits):  x = owner CTA rank | WRAP flag << 8 | position << 16,
//          y = byte offset of the 360-entry block in the owner's shared
//              memory (posterior column for a row slot, record row for a
//              column slot), z = circulant shift u, w = unused.
// Row slot, check (r, k): target posterior index (k - u) mod 360.
// Column slot, bit mm:    target record index (u + mm) mod 360.
// WRAP marks the dual-diagonal wrap edge, absent for check (0, 0) and for
// the last codeword bit.
constexpr int QWRAP = 1 << 8;

struct QcTables {
  std::vector<int4> rdesc;
  std::vector<int32_t> rptr;
  std::vector<int4> cdesc;
  std::vector<int32_t> cptr;
  std::vector<uint8_t> s0;
};

// Host: derive the descriptors from the Annex A address rows.  Returns 0,
// -3 or -4 (not a dup-free Type B code).
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
  const int nbi = K / QZ, nb = n / QZ;
  struct Slot { int col, row, u, pos, wrap; };
  std::vector<std::vector<Slot>> rows(Q), cols(nb);
  for (int g = 0; g < nbi; ++g)
    for (int e = rowptr[g]; e < rowptr[g + 1]; ++e) {
      int x = addr[e];
      if (x < 0 || x >= n - K) {
        set_error("invalid argument: address outside the parity range");
        return -3;
      }
      rows[x % Q].push_back(Slot{g, x % Q, x / Q, 0, 0});
    }
  int drm = 0;
  for (int r = 0; r < Q; ++r) {
    auto &R = rows[r];
    std::sort(R.begin(), R.end(), [](const Slot &a, const Slot &b) {
      return a.col < b.col;
    });
    for (size_t i = 1; i < R.size(); ++i)
      if (R[i].col == R[i - 1].col) {
        set_error("unsupported: two circulants share a block (use the CSR "
                  "decoder)");
        return -4;
      }
    // dual diagonal: bits K+360(r-1)+k and K+360r+k (r >= 1); K+k and
    // K+360(Q-1)+k-1 (r = 0, absent for k = 0)
    if (r >= 1) {
      R.push_back(Slot{nbi + r - 1, r, 0, 0, 0});
      R.push_back(Slot{nbi + r, r, 0, 0, 0});
    } else {
      R.push_back(Slot{nbi, 0, 0, 0, 0});
      R.push_back(Slot{nbi + Q - 1, 0, 1, 0, QWRAP});
    }
    for (int i = 0; i < (int)R.size(); ++i) {
      R[i].pos = i;
      cols[R[i].col].push_back(R[i]);
    }
    drm = std::max(drm, (int)R.size());
  }
  if (drm > 64) {
    set_error("unsupported: block-row degree above 64");
    return -4;
  }
  p->n = n; p->K = K; p->Q = Q; p->nbi = nbi; p->nb = nb;
  p->cluster = cluster;
  p->dr_max = drm;
  // record rows and posterior columns, both split evenly over the cluster
  const int per = (Q + cluster - 1) / cluster;
  const int cpc = (nb + cluster - 1) / cluster;
  for (int c = 0; c <= cluster; ++c) p->rb[c] = std::min(Q, c * per);
  p->rows_per_cta = per;
  p->ncp = per * QZ;
  p->cpc = cpc;
  const int tot_bytes = cpc * QZ * 4;
  auto col_rank = [&](int b) { return b / cpc; };
  auto col_base = [&](int b) { return (b % cpc) * QZ * 4; };
  auto row_rank = [&](int r) { return r / per; };
  auto row_base = [&](int r) { return tot_bytes + (r % per) * QZ * 16; };
  t->rptr.assign(Q + 1, 0);
  t->rdesc.clear();
  for (int r = 0; r < Q; ++r) {
    for (auto &sl : rows[r])
      t->rdesc.push_back(make_int4(col_rank(sl.col) | sl.wrap | (sl.pos << 16),
                                   col_base(sl.col), sl.u, 0));
    t->rptr[r + 1] = (int)t->rdesc.size();
  }
  // column slots sorted by (u, row): ascending check order before rotation
  t->cptr.assign(nb + 1, 0);
  t->cdesc.clear();
  t->s0.assign((size_t)nb * QZ, 0);
  int dcm = 0;
  for (int b = 0; b < nb; ++b) {
    auto &Cc = cols[b];
    std::sort(Cc.begin(), Cc.end(), [](const Slot &a, const Slot &c) {
      return a.u != c.u ? a.u < c.u : a.row < c.row;
    });
    dcm = std::max(dcm, (int)Cc.size());
    for (auto &sl : Cc)
      t->cdesc.push_back(make_int4(row_rank(sl.row) | sl.wrap | (sl.pos << 16),
                                   row_base(sl.row), sl.u, 0));
    t->cptr[b + 1] = (int)t->cdesc.size();
    for (int mm = 0; mm < QZ; ++mm) {
      int s = 0;
      for (auto &sl : Cc) s += (sl.u + mm < QZ) ? 1 : 0;
      t->s0[(size_t)b * QZ + mm] = (uint8_t)s;
    }
  }
  p->dc_max = dcm;
  // variable-phase work items (column b, chunk q), w = b*12 + q, split into
  // CL runs of equal edge count
  std::vector<int64_t> wcost((size_t)nb * QCHUNK);
  int64_t total = 0;
  for (int b = 0; b < nb; ++b)
    for (int q = 0; q < QCHUNK; ++q) {
      int lanes = std::min(32, QZ - 32 * q);
      wcost[(size_t)b * QCHUNK + q] = (int64_t)lanes * (int64_t)cols[b].size() + 16;
      total += wcost[(size_t)b * QCHUNK + q];
    }
  int64_t acc = 0;
  int c = 1;
  p->wb[0] = 0;
  for (int w = 0; w < (int)wcost.size() && c < cluster; ++w) {
    acc += wcost[w];
    while (c < cluster && acc * cluster >= total * c) p->wb[c++] = w + 1;
  }
  while (c <= cluster) p->wb[c++] = (int)wcost.size();
  p->smem = tot_bytes + p->ncp * 16 + 256;
  return 0;
}

struct QcArgs {
  const float *llr;
  int64_t ld_llr;
  int nblk, n, iters;
  float alpha;
  int cpc, ncp;
  uint32_t cpc_inv;              // ceil(2^32 / cpc): bc / cpc for bc < 2^16
  int rb[QMAXCL + 1];
  int wb[QMAXCL + 1];
  const int4 *rdesc;
  const int32_t *rptr;
  const int4 *cdesc;
  const int32_t *cptr;
  const uint8_t *s0;
  // optional learned weights: record minima become relu(min*w_a - w_b) with
  // (w_a, w_b) = (walpha, wbeta)[min(it, wT-1)][dbucket[check degree]];
  // null -> (alpha, 0), which is bit-identical to min*alpha
  const float *walpha;
  const float *wbeta;
  const int8_t *dbucket;
  int wT, wnb;
  uint8_t *bits;
  int64_t ld_bits;
  uint8_t *hard;
  int64_t ld_hard;
  uint8_t *conv;
  int32_t *its;
  int32_t *bad;
};

// edge message from a record {A, B, S, F | S1 << 8} for edge position pos
__device__ __forceinline__ float qc_msg(uint4 r, uint32_t pos) {
  const float m = (pos == (r.w & 0xFFu)) ? __uint_as_float(r.y)
                                         : __uint_as_float(r.x);
  const uint32_t s = pos < 32u ? (r.z >> pos) : (r.w >> (pos - 24u));
  return __uint_as_float(__float_as_uint(m) ^ (s << 31));
}

// NCH: chunks of 8 edge slots per block row (compile-time, so every edge
// position is a constant); MASK: sign-mask type.  DSMEM loads are issued
// unconditionally -- an absent slot reads a harmless local address and is
// masked out arithmetically -- so the loads of a chunk are straight-line
// code the hardware can overlap.
template <bool TORCH, int NCH, typename MASK, int NT>
__global__ void __launch_bounds__(NT, 1) ldpc_qc_kernel(const QcArgs a) {
  // variable-phase record loads in flight per thread (register budget)
  constexpr int VB = NT >= 1024 ? 4 : (NT >= 768 ? 6 : 8);
  extern __shared__ __align__(16) unsigned char smem[];
  const int rank = (int)cluster_ctarank();
  const int CL = (int)cluster_nctarank();
  const int tot_bytes = a.cpc * QZ * 4;
  float *tot = reinterpret_cast<float *>(smem);
  uint4 *rec = reinterpret_cast<uint4 *>(smem + tot_bytes);
  int *part = reinterpret_cast<int *>(smem + tot_bytes + (size_t)a.ncp * 16);
  int *sbad = part + 32;
  const uint32_t sm_sa = smem_u32(smem);
  const uint32_t part_sa = smem_u32(part);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nwarps = blockDim.x >> 5;
  const int r0 = a.rb[rank], r1 = a.rb[rank + 1];
  const int ncitems = (r1 - r0) * QCHUNK;
  const int w0 = a.wb[rank], w1 = a.wb[rank + 1];
  const int vbase = rank * a.cpc * QZ;
  const int vend = min(a.n, vbase + a.cpc * QZ);
  constexpr int MB = (int)sizeof(MASK) * 8;
  const uint32_t dummy = sm_sa;                      // own, always mapped

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
        const int rl = w / QCHUNK;
        const int r = r0 + rl;
        const int k0 = (w - rl * QCHUNK) * 32 + lane;
        const bool kv = k0 < QZ;
        const int k = kv ? k0 : QZ - 1;
        const int rp = __ldg(a.rptr + r);
        const int deg = __ldg(a.rptr + r + 1) - rp;
        const int4 *ds = a.rdesc + rp;
        const int li = rl * QZ + k;
        const uint4 ro = rec[li];
        const float Ao = __uint_as_float(ro.x), Bo = __uint_as_float(ro.y);
        const uint32_t Fo = ro.w & 0xFFu;
        MASK So = (MASK)ro.z;
        if constexpr (MB > 32) So |= (MASK)(ro.w >> 8) << 32;
        float min1 = __int_as_float(0x7f800000), min2 = min1;
        uint32_t first = 0;
        MASK sv = 0, st = 0, live = 0;
#pragma unroll
        for (int c = 0; c < NCH; ++c) {
          float t[8];
          uint32_t ad[8];
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            const int j = c * 8 + u;
            const int4 d = __ldg(ds + min(j, deg - 1));
            const bool on = j < deg && !((d.x & QWRAP) && k == 0);
            int o = k - d.z;
            o += o < 0 ? QZ : 0;
            ad[u] = on ? dsmem_map(sm_sa + (uint32_t)(d.y + 4 * o), (uint32_t)(d.x & 0xFF))
                       : dummy;
            if (on) live |= (MASK)1 << j;
          }
#pragma unroll
          for (int u = 0; u < 8; ++u) t[u] = dsmem_ld_f32(ad[u]);
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            const int j = c * 8 + u;
            const MASK bit = (MASK)1 << j;
            if (live & bit) {
              if (t[u] < 0.f) st |= bit;
              float mo = ((uint32_t)j == Fo) ? Bo : Ao;
              if (So & bit) mo = -mo;
              const float v = __fsub_rn(t[u], mo);
              if (v < 0.f) sv |= bit;
              const float mag = fabsf(v);
              if (mag < min1) { min2 = min1; min1 = mag; first = (uint32_t)j; }
              else if (mag < min2) { min2 = mag; }
            }
          }
        }
        int par, syn;
        if constexpr (MB > 32) {
          par = __popcll((unsigned long long)sv) & 1;
          syn = __popcll((unsigned long long)st) & 1;
        } else {
          par = __popc((uint32_t)sv) & 1;
          syn = __popc((uint32_t)st) & 1;
        }
        if (par) sv ^= live;
        if (kv) {
          uint32_t hi = 0;
          if constexpr (MB > 32) hi = (uint32_t)((unsigned long long)sv >> 32) << 8;
          float wa = a.alpha, wb = 0.f;
          if (a.walpha) {
            int nl;
            if constexpr (MB > 32) nl = __popcll((unsigned long long)live);
            else nl = __popc((uint32_t)live);
            const int wi = min(it, a.wT - 1) * a.wnb + __ldg(a.dbucket + nl);
            wa = __ldg(a.walpha + wi);
            wb = __ldg(a.wbeta + wi);
          }
          float A = __fsub_rn(__fmul_rn(min1, wa), wb);
          float B = __fsub_rn(__fmul_rn(min2, wa), wb);
          A = A > 0.f ? A : 0.f;
          B = B > 0.f ? B : 0.f;
          rec[li] = make_uint4(__float_as_uint(A), __float_as_uint(B),
                               (uint32_t)sv, first | hi);
          mybad += syn;
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
          // whole bytes: 360-bit columns are 45-byte aligned
          uint8_t *ho = a.hard + (size_t)b * a.ld_hard;
          for (int by = (vbase >> 3) + tid; by < (vend >> 3); by += blockDim.x) {
            uint32_t v = 0;
            const float *tp = tot + (by * 8 - vbase);
#pragma unroll
            for (int q = 0; q < 8; ++q) v |= (tp[q] < 0.f ? 1u : 0u) << (7 - q);
            ho[by] = (uint8_t)v;
          }
        }
        if (rank == 0 && tid == 0) {
          a.conv[b] = done ? 1 : 0;
          a.its[b] = it;
          a.bad[b] = done ? 0 : badct;
        }
        // the packing above reads posteriors other threads overwrite in the
        // next codeword's prologue
        __syncthreads();
        break;
      }
      // ---------------- variable phase -------------------------------------
      for (int w = w0 + warp; w < w1; w += nwarps) {
        const int bc = w / QCHUNK;
        const int mm0 = (w - bc * QCHUNK) * 32 + lane;
        const bool mv = mm0 < QZ;
        const int mm = mv ? mm0 : QZ - 1;
        const int lamidx = bc * QZ + mm;
        const float li = lam[lamidx];
        float acc = TORCH ? li : 0.f;
        const int cs = __ldg(a.cptr + bc);
        const int d = __ldg(a.cptr + bc + 1) - cs;
        const int s0 = __ldg(a.s0 + lamidx);
        const int4 *ds = a.cdesc + cs;
        if (d == 2) {
          // dual-diagonal parity column (warp-uniform): two slots, no padding
          uint32_t ad[2], pos[2];
          bool on[2];
#pragma unroll
          for (int u = 0; u < 2; ++u) {
            int i = s0 + u;
            i -= i >= 2 ? 2 : 0;
            const int4 e = __ldg(ds + i);
            on[u] = !((e.x & QWRAP) && mm == QZ - 1);
            int o = e.z + mm;
            o -= o >= QZ ? QZ : 0;
            pos[u] = (uint32_t)e.x >> 16;
            ad[u] = on[u] ? dsmem_map(sm_sa + (uint32_t)(e.y + 16 * o),
                                      (uint32_t)(e.x & 0xFF))
                          : dummy;
          }
          const uint4 q0 = dsmem_ld_v4(ad[0]);
          const uint4 q1 = dsmem_ld_v4(ad[1]);
          if (on[0]) acc = __fadd_rn(acc, qc_msg(q0, pos[0]));
          if (on[1]) acc = __fadd_rn(acc, qc_msg(q1, pos[1]));
        } else
        for (int t0 = 0; t0 < d; t0 += VB) {
          uint32_t ad[VB], pos[VB];
          bool on[VB];
#pragma unroll
          for (int u = 0; u < VB; ++u) {
            int i = s0 + t0 + u;
            i -= i >= d ? d : 0;
            i = min(i, d - 1);
            const int4 e = __ldg(ds + i);
            on[u] = t0 + u < d && !((e.x & QWRAP) && mm == QZ - 1);
            int o = e.z + mm;
            o -= o >= QZ ? QZ : 0;
            pos[u] = (uint32_t)e.x >> 16;
            ad[u] = on[u] ? dsmem_map(sm_sa + (uint32_t)(e.y + 16 * o),
                                      (uint32_t)(e.x & 0xFF))
                          : dummy;
          }
          uint4 rr[VB];
#pragma unroll
          for (int u = 0; u < VB; ++u) rr[u] = dsmem_ld_v4(ad[u]);
#pragma unroll
          for (int u = 0; u < VB; ++u)
            if (on[u]) acc = __fadd_rn(acc, qc_msg(rr[u], pos[u]));
        }
        if (mv) {
          const float nv = TORCH ? acc : __fadd_rn(li, acc);
          const int owner = (int)__umulhi((uint32_t)bc, a.cpc_inv);   // bc / cpc
          const uint32_t off = (uint32_t)((bc - owner * a.cpc) * QZ + mm) * 4u;
          if (owner == rank) tot[off >> 2] = nv;
          else dsmem_st_u32(dsmem_map(sm_sa + off, (uint32_t)owner), __float_as_uint(nv));
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

#define ATSC3_QC_FN(NCH, MASK)                                              \
  (nt == 1024 ? (semantics ? ldpc_qc_kernel<true, NCH, MASK, 1024>           \
                           : ldpc_qc_kernel<false, NCH, MASK, 1024>)         \
   : nt == 768 ? (semantics ? ldpc_qc_kernel<true, NCH, MASK, 768>           \
                            : ldpc_qc_kernel<false, NCH, MASK, 768>)         \
               : (semantics ? ldpc_qc_kernel<true, NCH, MASK, 512>           \
                            : ldpc_qc_kernel<false, NCH, MASK, 512>))

// The CTA size picks the build: > 768 threads -> 1024-thread build (64
// registers, 4 record loads in flight per thread), > 512 -> 768 (85, 6),
// else 512 (128, 8).
static QcFn qc_fn(int semantics, int dr, int threads) {
  const int nt = threads > 768 ? 1024 : (threads > 512 ? 768 : 512);
  if (dr <= 8) return ATSC3_QC_FN(1, uint32_t);
  if (dr <= 16) return ATSC3_QC_FN(2, uint32_t);
  if (dr <= 24) return ATSC3_QC_FN(3, uint32_t);
  if (dr <= 32) return ATSC3_QC_FN(4, uint32_t);
  if (dr <= 40) return ATSC3_QC_FN(5, unsigned long long);
  if (dr <= 56) return ATSC3_QC_FN(7, unsigned long long);
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
  cudaError_t e = up((void **)&h->p.d_rdesc, t.rdesc.data(), t.rdesc.size() * 16);
  if (e == cudaSuccess) e = up((void **)&h->p.d_rptr, t.rptr.data(), t.rptr.size() * 4);
  if (e == cudaSuccess) e = up((void **)&h->p.d_cdesc, t.cdesc.data(), t.cdesc.size() * 16);
  if (e == cudaSuccess) e = up((void **)&h->p.d_cptr, t.cptr.data(), t.cptr.size() * 4);
  if (e == cudaSuccess) e = up((void **)&h->p.d_s0, t.s0.data(), t.s0.size());
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
  delete h;
}

int32_t atsc3_ldpc_qc_plan_info(const atsc3_ldpc_qc_plan *h, int64_t *info) {
  ATSC3_ARG(h && info, "null argument");
  info[0] = h->p.n;
  info[1] = h->p.K;
  info[2] = h->p.Q;
  info[3] = h->p.cluster;
  info[4] = h->p.smem;
  info[5] = h->p.dr_max;
  info[6] = h->p.dc_max;
  info[7] = h->p.table_bytes;
  info[8] = h->p.rows_per_cta;
  info[9] = h->p.cpc;
  return 0;
}

int32_t atsc3_ldpc_qc_tables_host(int32_t n, int32_t kldpc, int32_t qldpc,
                                  const int32_t *rowptr, const int32_t *addr,
                                  int32_t cluster, int32_t *meta,
                                  int32_t *rdesc, int32_t *rptr,
                                  int32_t *cdesc, int32_t *cptr, uint8_t *s0) {
  using namespace atsc3;
  ATSC3_ARG(meta && rowptr && addr, "null argument");
  QcPlan p;
  QcTables t;
  int rc = qc_build(n, kldpc, qldpc, rowptr, addr, cluster, &p, &t);
  if (rc) return rc;
  meta[0] = (int32_t)t.rdesc.size();
  meta[1] = (int32_t)t.cdesc.size();
  meta[2] = p.cpc;
  meta[3] = p.ncp;
  meta[4] = p.rows_per_cta;
  meta[5] = p.dr_max;
  meta[6] = p.dc_max;
  meta[7] = p.smem;
  for (int c = 0; c <= QMAXCL; ++c) {
    meta[8 + c] = p.rb[c];
    meta[25 + c] = p.wb[c];
  }
  if (rdesc) std::memcpy(rdesc, t.rdesc.data(), t.rdesc.size() * 16);
  if (rptr) std::memcpy(rptr, t.rptr.data(), t.rptr.size() * 4);
  if (cdesc) std::memcpy(cdesc, t.cdesc.data(), t.cdesc.size() * 16);
  if (cptr) std::memcpy(cptr, t.cptr.data(), t.cptr.size() * 4);
  if (s0) std::memcpy(s0, t.s0.data(), t.s0.size());
  return 0;
}

int32_t atsc3_ldpc_qc_config(const atsc3_ldpc_qc_plan *h, int32_t threads,
                             int32_t semantics, int32_t *out) {
  using namespace atsc3;
  ATSC3_ARG(h && out, "null argument");
  if (threads <= 0) threads = 1024;
  QcFn fn = qc_fn(semantics, h->p.dr_max, threads);
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

int32_t atsc3_ldpc_qc_decode_weighted(
    const atsc3_ldpc_qc_plan *h, const float *llr, int64_t ld_llr,
    int32_t nblk, int32_t iters, float alpha, int32_t semantics,
    const float *walpha, const float *wbeta, int32_t wT, int32_t wnb,
    const int8_t *dbucket, uint8_t *bits, int64_t ld_bits, uint8_t *hard,
    int64_t ld_hard, uint8_t *conv, int32_t *its, int32_t *bad,
    int32_t threads, void *stream);

int32_t atsc3_ldpc_qc_decode(const atsc3_ldpc_qc_plan *h, const float *llr,
                             int64_t ld_llr, int32_t nblk, int32_t iters,
                             float alpha, int32_t semantics, uint8_t *bits,
                             int64_t ld_bits, uint8_t *hard, int64_t ld_hard,
                             uint8_t *conv, int32_t *its, int32_t *bad,
                             int32_t threads, void *stream) {
  return atsc3_ldpc_qc_decode_weighted(h, llr, ld_llr, nblk, iters, alpha,
                                       semantics, nullptr, nullptr, 0, 0,
                                       nullptr, bits, ld_bits, hard, ld_hard,
                                       conv, its, bad, threads, stream);
}

int32_t atsc3_ldpc_qc_decode_weighted(
    const atsc3_ldpc_qc_plan *h, const float *llr, int64_t ld_llr,
    int32_t nblk, int32_t iters, float alpha, int32_t semantics,
    const float *walpha, const float *wbeta, int32_t wT, int32_t wnb,
    const int8_t *dbucket, uint8_t *bits, int64_t ld_bits, uint8_t *hard,
    int64_t ld_hard, uint8_t *conv, int32_t *its, int32_t *bad,
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
  QcFn fn = qc_fn(semantics, p.dr_max, threads);
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
  a.iters = iters;
  a.alpha = alpha;
  a.cpc = p.cpc;
  a.cpc_inv = (uint32_t)((0x100000000ull + (uint64_t)p.cpc - 1) / (uint64_t)p.cpc);
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
  if (walpha) {
    ATSC3_ARG(wbeta && dbucket && wT > 0 && wnb > 0,
              "weights need wbeta, dbucket, wT > 0, wnb > 0");
    a.walpha = walpha;
    a.wbeta = wbeta;
    a.dbucket = dbucket;
    a.wT = wT;
    a.wnb = wnb;
  }
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

namespace atsc3 {
// Device the plan's tables were built on (internal; used by the
// allocation-free entry point to refuse a plan from another GPU).
int qc_plan_device(const atsc3_ldpc_qc_plan *h) { return h->p.device; }
}  // namespace atsc3
