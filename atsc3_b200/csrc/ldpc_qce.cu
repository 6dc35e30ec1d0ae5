// ldpc_qce.cu -- flooding normalised min-sum for every quasi-cyclic A/322
// code (Type B, and Type A with its identity rows) with an EDGE-BUFFER layout
// (sm_100a), bit-exact with lab/ldpc_kernel.c (kernel semantics) and
// lab/m9_gpu.py:168-211 (torch semantics), float32; the same source, templated on
// the value type, also builds a float64 decoder (8-byte slots, no learned
// weights).
//
// The code structure used is the one of ldpc_qc.cu (360x360 circulants,
// dual-diagonal parity part, edge order inside a check = block-column order,
// a bit's summation order = its column's circulant list sorted by (shift,
// row) and rotated at s0[col*360 + mm]), except that a block may hold more
// than one circulant here, and a Type A code adds identity block rows: a
// bit's checks there come after its accumulator checks, so its sum is two
// rotated segments (s0, then s0b), and its few accumulator rows of high
// degree take a loop path ("heavy" rows, see qce_check_heavy).
//
// What differs is where the decoder state lives.  Every edge of the codeword
// owns one float32 slot in the distributed shared memory of its cluster, in
// the CTA that owns the edge's 360-bit column: column g's circulant slots are
// contiguous 360-float blocks there, entry mm of slot i belongs to bit
// (g, mm).  The slot holds
//   * after the variable phase: q = tot - m, the variable-to-check value the
//     reference computes inside its check update (ldpc_kernel.c:120,
//     v = tot[j] - m[e]); the same rounded subtraction, done on the variable
//     side;
//   * after the check phase: m, the new check-to-variable message.
// The check phase therefore reads each edge's q with one 4-byte remote load
// (32 consecutive checks of a block row read 32 consecutive entries of a
// circulant slot), forms min1/min2/first/signs in registers, and writes the
// messages back into the same slots with posted remote stores.  A row's 360
// checks are 11 such warp items and an 8-check last chunk; a CTA's last
// chunks run four rows to a warp (8 lanes per row).  The variable
// phase is local: it sums its slots in the reference order, forms tot, and
// rewrites every slot as tot - m.  No per-check records are kept.
//
// Hard decisions for the syndrome (ldpc_kernel.c:95-101 evaluates it on
// tot before every update) live in a bitmap replicated in every CTA: 12
// 32-bit words per 360-bit column (bit mm of column g = word g*12 + mm/32,
// bit mm%32).  The variable phase writes each 32-bit ballot to every CTA of
// the cluster; the check phase looks up its bits locally.
//
// Shared memory per CTA: bitmap (nb*48 B) | syndrome exchange (256 B) |
// per-launch tables | the edge slots of the CTA's columns (1440 B per slot;
// 2880 B in the float64 build).
// For the 64800-bit codes (about 281k edges, 1.1 MB of slots) a 6-CTA
// cluster holds a codeword (about 215 KB per CTA).

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <type_traits>
#include <unordered_map>
#include <vector>

#include "../../include/atsc3_fec.h"
#include "common.cuh"

namespace atsc3 {

constexpr int EZ = 360;
constexpr int ECHUNK = 12;                // ceil(360 / 32) warps per row/column
constexpr int EMAXCL = 16;
constexpr int EWRAP = 1 << 8;
constexpr int EPART = 256;                // syndrome exchange bytes
constexpr int QBINS = 32;                 // variable-item bins per CTA (one per warp at 1024 threads)

// Compile-time slot counts per block row (NS >= the code's largest block-row
// degree; rows with fewer edges mask the rest) (the kernel templates).
__host__ __device__ constexpr int qce_ns(int dr) {
  return dr <= 8 ? 8 : dr <= 10 ? 10 : dr <= 11 ? 11 : dr <= 14 ? 14
       : dr <= 17 ? 17 : dr <= 22 ? 22 : dr <= 34 ? 34 : dr <= 56 ? 56 : 0;
}

// The same for the identity rows of a Type A code (3 to 7 edges in A/322):
// 4 and 6 slots keep the short rows unmasked.
__host__ __device__ constexpr int qce_ns_a(int dr) {
  return dr <= 4 ? 4 : dr <= 6 ? 6 : dr <= 8 ? 8 : 0;
}

struct QcePlan {
  int n = 0, K = 0, Q = 0, nb = 0;
  int qa = 0, qb = 0;           // accumulator / identity block rows
  int cluster = 1, smem = 0, part_off = 0, rt_off = 0, ri_off = 0, ct_off = 0;
  int ht_off = 0, buf_off = 0;
  int dr_max = 0, dr_light = 0, dc_max = 0, max_slots = 0, device = 0;
  int heavy = 0;                // rows above the compile-time slot count
  int vb = 4;                   // bytes per slot entry: 4 float32, 8 float64
  int64_t table_bytes = 0;
  int rb[EMAXCL + 1] = {0};     // block rows CTA c owns (column placement)
  int ci[EMAXCL + 1] = {0};     // check items (row*12 + chunk) of CTA c; with
                                // heavy rows: its light items only
  int hoff[EMAXCL + 1] = {0};   // heavy items of CTA c: hitems[hoff[c] .. hoff[c+1])
  int nhrows = 0;               // heavy rows (the accumulator rows) or 0
  int hsplit = 1;               // parts per heavy item (warps sharing it)
  int hpb_off = 0;              // shared-memory offset of the heavy partials
  int vbin_lo = 0, vbin_hi = 0; // least / most loaded variable-item bin (estimated cost)
  int ib[EMAXCL + 1] = {0};     // variable-phase items of CTA c in d_itab
  int cb[EMAXCL + 1] = {0};     // CTA c owns columns ccols[cb[c] .. cb[c+1])
  int4 *d_rdesc = nullptr;      // per row edge slot
  int32_t *d_ccols = nullptr;   // (nb) columns grouped by owner CTA
  int4 *d_itab = nullptr;       // variable-phase items, grouped by CTA
  int32_t *d_wbin = nullptr;    // (cluster, QBINS+1) bin offsets into each CTA's items
  int32_t *d_rptr = nullptr;    // (Q+1)
  int4 *d_cdesc = nullptr;      // per column
  uint8_t *d_s0 = nullptr;      // (nb*360) rotation start (zone A / only zone)
  uint8_t *d_s0b = nullptr;     // (nb*360) rotation start in zone B
  int16_t *d_hitems = nullptr;  // heavy check items, grouped by CTA
};

// Block rows: rows 0 .. qa-1 are the accumulator rows (check r + qa*k, the
// dual-diagonal parity part), rows qa .. qa+qb-1 the identity rows of a Type A
// code (check 360*qa + (r - qa) + qb*k, one parity bit each); a Type B code
// has qb = 0.
// Row slot (block row r, position j):  x = owner CTA | WRAP << 8 | j << 16,
// y = byte offset of the edge's circulant slot in the owner's shared memory,
// z = circulant shift u, w = byte offset of the column's bitmap words.
// Check (r, k) reads entry (k - u) mod 360 of the slot.
// Column descriptor (column g): x = slots d, y = byte offset of slot 0 in
// the owner's shared memory (slots follow at 1440-byte steps, sorted by
// (zone, u, row)), z = index of the dual-diagonal wrap slot (absent for bit
// 359) or -1, w = owner CTA | zone-A slots << 8.  ccols lists each CTA's
// columns (cb[c] .. cb[c+1]).
struct QceTables {
  std::vector<int4> rdesc;
  std::vector<int32_t> rptr;
  std::vector<int4> cdesc;
  std::vector<int32_t> ccols;
  std::vector<int4> itab;
  std::vector<int32_t> wbin;    // (cluster, QBINS+1) bin offsets, relative to ib[c]
  std::vector<uint8_t> s0, s0b;
  std::vector<int16_t> hitems;
};

// variable-phase item modes (bits 25-26 of the item's z word)
constexpr int VM_PAIR = 0;     // dual-diagonal parity column, 2 slots in check order
constexpr int VM_EXACT = 1;    // 1..4 slots of one zone, rotated in registers
constexpr int VM_GEN = 2;      // any slots of one zone, rotated by offsets
constexpr int VM_GEN2 = 3;     // slots in both zones: two rotated segments
constexpr uint32_t VNOWRAP = 0xFFu;

int qce_build(int n, int K, int QA, int QB, const int32_t *rowptr,
              const int32_t *addr, int cluster, QcePlan *p, QceTables *t,
              int vb = 4) {
  // vb: bytes per slot entry (4: float32 decoder, 8: float64 decoder)
  const int slotb = EZ * vb;
  const int Q = QA + QB;
  if (n % EZ || K % EZ || QA <= 0 || QB < 0 || (n - K) != Q * EZ) {
    set_error("invalid argument: not a 360-circulant Type A/B code");
    return -3;
  }
  if (cluster < 1 || cluster > EMAXCL) {
    set_error("invalid argument: cluster must be in 1..16");
    return -3;
  }
  const int nbi = K / EZ, nb = n / EZ, MA = QA * EZ;
  struct Slot { int col, row, u, pos, wrap, idx; };
  std::vector<std::vector<Slot>> rows(Q), cols(nb);
  // address-table rows: one per information column group and, for a Type A
  // code, one per accumulator parity column (its bits feed the identity
  // rows, A/322 6.1.3.1 step vii); accumulator address x -> (row, shift)
  const int ntab = nbi + (QB > 0 ? QA : 0);
  if (rowptr[0] != 0) {
    set_error("invalid argument: rowptr[0] must be 0");
    return -3;
  }
  for (int g = 0; g < ntab; ++g)
    if (rowptr[g + 1] < rowptr[g]) {
      set_error("invalid argument: rowptr must not decrease");
      return -3;
    }
  for (int g = 0; g < ntab; ++g)
    for (int e = rowptr[g]; e < rowptr[g + 1]; ++e) {
      const int x = addr[e];
      if (x < 0 || x >= n - K) {
        set_error("invalid argument: address outside the parity range");
        return -3;
      }
      if (x < MA) rows[x % QA].push_back(Slot{g, x % QA, x / QA, 0, 0, 0});
      else rows[QA + (x - MA) % QB].push_back(Slot{g, QA + (x - MA) % QB, (x - MA) / QB, 0, 0, 0});
    }
  int drm = 0, drb = 0;
  for (int r = 0; r < Q; ++r) {
    auto &R = rows[r];
    std::sort(R.begin(), R.end(),
              [](const Slot &a, const Slot &b) {
                return a.col != b.col ? a.col < b.col : a.u < b.u;
              });
    // Two circulants may share a block (the 16200-bit Type B codes of rates
    // 6/15, 8/15, 10/15, 12/15 and 13/15 have such blocks): they are two
    // slots of the same column with different shifts.  Within a check their
    // edges' order follows the bit index, which depends on the check, while
    // the slots keep one order; the check update does not depend on the
    // order of a check's edges (the first minimum matters only through min2,
    // and min2 == min1 when the minimum is shared), so one slot order serves
    // every check.  A repeated address cancels in GF(2)
    // (lab/m3_ldpc.py:199-211): both copies are dropped.
    {
      std::vector<Slot> keep;
      for (size_t i = 0; i < R.size(); ++i) {
        if (i + 1 < R.size() && R[i + 1].col == R[i].col && R[i + 1].u == R[i].u) {
          ++i;
          continue;
        }
        keep.push_back(R[i]);
      }
      R.swap(keep);
    }
    if (r < QA) {
      // dual diagonal: bits K+360(r-1)+k and K+360r+k (r >= 1); K+k and
      // K+360(QA-1)+k-1 (r = 0, absent for k = 0)
      if (r >= 1) {
        R.push_back(Slot{nbi + r - 1, r, 0, 0, 0, 0});
        R.push_back(Slot{nbi + r, r, 0, 0, 0, 0});
      } else {
        R.push_back(Slot{nbi, 0, 0, 0, 0, 0});
        R.push_back(Slot{nbi + QA - 1, 0, 1, 0, EWRAP, 0});
      }
    } else {
      // identity part of a Type A code: bit K + 360*QA + 360*(r-QA) + k
      R.push_back(Slot{nbi + r, r, 0, 0, 0, 0});
    }
    std::stable_sort(R.begin(), R.end(),
                     [](const Slot &a, const Slot &b) { return a.col < b.col; });
    for (int i = 0; i < (int)R.size(); ++i) R[i].pos = i;
    drm = std::max(drm, (int)R.size());
    if (r >= QA) drb = std::max(drb, (int)R.size());
  }
  // compile-time slots per row: the largest row for a Type B code; the
  // largest identity row for a Type A code, whose few accumulator rows of
  // higher degree take the kernel's loop path ("heavy" rows)
  const int dlight = QB > 0 ? drb : drm;
  const int ns = QB > 0 ? qce_ns_a(dlight) : qce_ns(dlight);
  if (ns == 0) {
    set_error(QB > 0 ? "unsupported: identity rows of more than 8 edges"
                     : "unsupported: block-row degree above 56");
    return -4;
  }
  std::vector<int> rdeg(Q);
  int heavy = 0;
  for (int r = 0; r < Q; ++r) {
    rdeg[r] = (int)rows[r].size();
    if (rdeg[r] > ns) heavy = 1;
  }
  if (drm > 250) {
    set_error("unsupported: block-row degree above 250");
    return -4;
  }
  for (int r = 0; r < Q; ++r)
    for (auto &sl : rows[r]) cols[sl.col].push_back(sl);
  int dcm = 0, total = 0;
  std::vector<int> dzA(nb, 0);
  for (int g = 0; g < nb; ++g) {
    auto &Cc = cols[g];
    std::sort(Cc.begin(), Cc.end(), [QA](const Slot &a, const Slot &c) {
      const int za = a.row >= QA, zc = c.row >= QA;
      if (za != zc) return za < zc;
      return a.u != c.u ? a.u < c.u : a.row < c.row;
    });
    for (int i = 0; i < (int)Cc.size(); ++i) {
      Cc[i].idx = i;
      if (Cc[i].row < QA) ++dzA[g];
      for (auto &rs : rows[Cc[i].row])      // back-reference row slot -> idx
        if (rs.col == g && rs.u == Cc[i].u) rs.idx = i;
    }
    dcm = std::max(dcm, (int)Cc.size());
    total += (int)Cc.size();
  }
  if (dcm > 250) {
    set_error("unsupported: column degree above 250");
    return -4;
  }
  // Check items (row*12 + chunk) per CTA.  Without heavy rows: contiguous
  // equal row ranges.  With heavy rows (the accumulator rows of a Type A
  // code, all of them): their items are dealt round-robin over the cluster
  // (a heavy item is long and runs in one warp, so no CTA should hold many),
  // then each CTA takes a contiguous range of the light items that evens out
  // the estimated work (a heavy item ~ 35 instructions per edge over two
  // passes, a light item ~ 25 per compile-time slot + 30).
  const int per = (Q + cluster - 1) / cluster;
  t->hitems.clear();
  p->hoff[0] = 0;
  p->nhrows = 0;
  if (!heavy) {
    for (int c = 0; c <= cluster; ++c) p->ci[c] = std::min(Q, c * per) * ECHUNK;
    for (int c = 1; c <= EMAXCL; ++c) p->hoff[c] = 0;
  } else {
    for (int r = 0; r < Q; ++r)
      if ((rdeg[r] > ns) != (r < QA)) {
        set_error("unsupported: heavy rows other than the accumulator rows");
        return -4;
      }
    if (ns < 6) {
      set_error("unsupported: heavy rows with identity rows of at most 4 edges");
      return -4;
    }
    p->nhrows = QA;
    // a heavy item's slots are cut into hsplit contiguous parts of about 24
    // edges, each pass taken by its own warp (partial minima merged in
    // shared memory between the two passes)
    // (only for rows above 64 edges -- 64800 7/15: parts pay an extra CTA
    // barrier and a partials buffer, which lighter heavy rows do not earn
    // back; those take one warp per item)
    int hdmax = 0;
    for (int r = 0; r < QA; ++r) hdmax = std::max(hdmax, rdeg[r]);
    p->hsplit = (hdmax > 64 && vb == 4) ? (hdmax + 23) / 24 : 1;
    std::vector<int64_t> hc(cluster, 0);
    std::vector<std::vector<int>> hl(cluster);
    for (int i = 0; i < QA * ECHUNK; ++i) {
      hl[i % cluster].push_back(i);
      hc[i % cluster] += 35 * rdeg[i / ECHUNK];
    }
    for (int c = 0; c < cluster; ++c) {
      for (int i : hl[c]) t->hitems.push_back((int16_t)i);
      p->hoff[c + 1] = (int)t->hitems.size();
    }
    for (int c = cluster + 1; c <= EMAXCL; ++c) p->hoff[c] = p->hoff[cluster];
    const int64_t cl = 25 * ns + 30;
    const int L0 = QA * ECHUNK, L1 = Q * ECHUNK;
    int64_t total = (int64_t)(L1 - L0) * cl;
    for (int c = 0; c < cluster; ++c) total += hc[c];
    const double target = (double)total / cluster;
    double acc = 0.0;
    p->ci[0] = L0;
    for (int c = 0; c < cluster; ++c) {
      acc += std::max(0.0, target - (double)hc[c]);
      int b = L0 + (int)(acc / (double)cl + 0.5);
      p->ci[c + 1] = std::min(L1, std::max(p->ci[c], b));
    }
    p->ci[cluster] = L1;
  }
  for (int c = cluster + 1; c <= EMAXCL; ++c) p->ci[c] = p->ci[cluster];
  // the row's owner for column placement: the CTA holding its chunk 0
  std::vector<int> rowown(Q, 0);
  for (int c = 0; c < cluster; ++c)
    for (int r = (p->ci[c] + ECHUNK - 1) / ECHUNK; r * ECHUNK < p->ci[c + 1]; ++r)
      rowown[r] = c;
  for (int r = 0; r < p->nhrows; ++r) rowown[r] = (r * ECHUNK) % cluster;
  // Column -> CTA assignment.  An edge is local when its column lives in the
  // CTA that owns its row, and a local edge saves the check phase a remote
  // load and a remote store.  Parity column j of the accumulator (edges in
  // rows j and j+1) goes to the owner of row j, an identity parity column to
  // the owner of its row, which makes nearly all parity edges local.  The
  // information columns follow in decreasing degree (stable), each to the
  // CTA that owns most of their rows among the CTAs that stay within the
  // balanced share ceil(slots / cluster), ties to the CTA holding fewer
  // slots; a column no CTA can take within the share goes to the CTA holding
  // the fewest.
  std::vector<int> order, load(cluster, 0), who(nb), mine(cluster);
  for (int j = 0; j < Q; ++j) {
    const int c = rowown[j];
    who[nbi + j] = c;
    load[c] += (int)cols[nbi + j].size();
  }
  const int share = (total + cluster - 1) / cluster;
  for (int g = 0; g < nbi; ++g) order.push_back(g);
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
    return cols[x].size() > cols[y].size();
  });
  for (int g : order) {
    const int d = (int)cols[g].size();
    std::fill(mine.begin(), mine.end(), 0);
    for (auto &sl : cols[g]) ++mine[rowown[sl.row]];
    int c = -1;
    for (int q = 0; q < cluster; ++q) {
      if (load[q] + d > share) continue;
      if (c < 0 || mine[q] > mine[c] || (mine[q] == mine[c] && load[q] < load[c])) c = q;
    }
    if (c < 0) {
      c = 0;
      for (int q = 1; q < cluster; ++q)
        if (load[q] < load[c]) c = q;
    }
    who[g] = c;
    load[c] += d;
  }
  t->ccols.clear();
  p->cb[0] = 0;
  for (int c = 0; c < cluster; ++c) {
    for (int g = 0; g < nb; ++g)
      if (who[g] == c) t->ccols.push_back(g);
    p->cb[c + 1] = (int)t->ccols.size();
  }
  for (int c = cluster + 1; c <= EMAXCL; ++c) p->cb[c] = nb;
  for (int c = 0; c <= cluster; ++c)
    p->rb[c] = std::min(Q, (p->ci[c] + ECHUNK - 1) / ECHUNK);
  for (int c = cluster + 1; c <= EMAXCL; ++c) p->rb[c] = Q;
  // wrap slot and item mode per column
  std::vector<int> wrapi(nb, -1), vmode(nb, VM_GEN);
  for (int g = 0; g < nb; ++g) {
    auto &Cc = cols[g];
    const int d = (int)Cc.size();
    for (auto &sl : Cc)
      if (sl.wrap) wrapi[g] = sl.idx;
    const bool one_zone = dzA[g] == 0 || dzA[g] == d;
    const bool acc_parity = g >= nbi && g < nbi + QA;
    if (acc_parity && d == 2 && (wrapi[g] < 0 || wrapi[g] == 1) && Cc[0].u == 0 &&
        (Cc[1].u == 0 || wrapi[g] == 1))
      vmode[g] = VM_PAIR;
    else if (d <= 4 && one_zone && wrapi[g] < 0)
      vmode[g] = VM_EXACT;
    else
      vmode[g] = one_zone ? VM_GEN : VM_GEN2;
  }
  // variable-phase items per CTA: every column is cut into six 64-bit
  // items (lane L takes bits 64p + L and 64p + 32 + L: two independent
  // sums a lane)
  auto items_of = [&](int g) { (void)g; return 6; };
  int maxitems = 0;
  for (int c = 0; c < cluster; ++c) {
    int ni = 0;
    for (int q = p->cb[c]; q < p->cb[c + 1]; ++q) ni += items_of(t->ccols[q]);
    maxitems = std::max(maxitems, ni);
  }
  // per CTA: rows touched by its check items (all 12 chunks get row-slot
  // entries) and heavy-row slot entries
  int maxrows = 0;
  for (int c = 0; c < cluster; ++c) {
    if (p->ci[c + 1] <= p->ci[c]) continue;
    const int r0 = p->ci[c] / ECHUNK, r1 = (p->ci[c + 1] - 1) / ECHUNK;
    maxrows = std::max(maxrows, r1 - r0 + 1);
  }
  // every CTA holds all heavy rows: an int4 of row info each, then 8 B per slot
  int heavy_bytes = 16 * p->nhrows;
  for (int r = 0; r < p->nhrows; ++r) heavy_bytes += 8 * rdeg[r];
  heavy_bytes = (heavy_bytes + 15) & ~15;
  const int hpb_rel = heavy_bytes;        // partials: 16 B per lane per part
  int maxnh = 0;
  for (int c = 0; c < cluster; ++c) maxnh = std::max(maxnh, p->hoff[c + 1] - p->hoff[c]);
  if (p->nhrows && p->hsplit > 1) heavy_bytes += maxnh * p->hsplit * 32 * 16;
  // shared memory: bitmap | syndrome exchange | row-slot table (per row,
  // chunk and slot, 8 B) | row info (3 words per row) | variable-phase item
  // table (16 B per item) | heavy rows (info + slots) | slots
  const int bm_bytes = (nb * ECHUNK * 4 + 15) & ~15;
  const int part_off = bm_bytes;
  const int rt_off = part_off + EPART;
  const int ri_off = rt_off + maxrows * ECHUNK * ns * 8;
  const int ct_off = ri_off + ((maxrows * 3 * (ns > 32 ? 8 : 4) + 15) & ~15);
  const int ht_off = ct_off + maxitems * 16;
  const int buf_off = ht_off + ((heavy_bytes + 15) & ~15);
  std::vector<int> owner(nb), base(nb);
  int maxs = 0;
  for (int c = 0; c < cluster; ++c) {
    int s = 0;
    for (int q = p->cb[c]; q < p->cb[c + 1]; ++q) {
      const int g = t->ccols[q];
      owner[g] = c;
      base[g] = buf_off + s * slotb;
      s += (int)cols[g].size();
    }
    maxs = std::max(maxs, s);
  }
  p->n = n; p->K = K; p->Q = Q; p->nb = nb;
  p->qa = QA; p->qb = QB;
  p->vb = vb;
  p->cluster = cluster;
  p->dr_max = drm;
  p->dr_light = dlight;
  p->heavy = heavy;
  p->dc_max = dcm;
  p->max_slots = maxs;
  p->part_off = part_off;
  p->rt_off = rt_off;
  p->ri_off = ri_off;
  p->ct_off = ct_off;
  p->ht_off = ht_off;
  p->hpb_off = ht_off + hpb_rel;
  p->buf_off = buf_off;
  p->smem = buf_off + maxs * slotb;
  t->rptr.assign(Q + 1, 0);
  t->rdesc.clear();
  for (int r = 0; r < Q; ++r) {
    for (auto &sl : rows[r])
      t->rdesc.push_back(make_int4(owner[sl.col] | sl.wrap | (sl.pos << 16),
                                   base[sl.col] + sl.idx * slotb, sl.u,
                                   sl.col * ECHUNK * 4));
    t->rptr[r + 1] = (int)t->rdesc.size();
  }
  t->cdesc.assign(nb, make_int4(0, 0, -1, 0));
  t->s0.assign((size_t)nb * EZ, 0);
  t->s0b.assign((size_t)nb * EZ, 0);
  for (int g = 0; g < nb; ++g) {
    auto &Cc = cols[g];
    t->cdesc[g] = make_int4((int)Cc.size(), base[g], wrapi[g], owner[g] | (dzA[g] << 8));
    // a bit's checks in ascending index: zone A (index r + QA*k) before zone
    // B, inside a zone by (k, r) = the slots sorted by (u, row), rotated to
    // start at the first slot whose k = mm + u wrapped past 359
    for (int mm = 0; mm < EZ; ++mm) {
      int sa = 0, sb = 0;
      for (auto &sl : Cc) {
        if (sl.u + mm >= EZ) continue;
        if (sl.row < QA) ++sa;
        else ++sb;
      }
      // a column of one zone keeps its rotation in s0 (zone B only: the
      // identity parity columns)
      t->s0[(size_t)g * EZ + mm] = (uint8_t)(dzA[g] == 0 ? sb : sa);
      t->s0b[(size_t)g * EZ + mm] = (uint8_t)(dzA[g] == 0 ? 0 : sb);
    }
  }
  // item {byte offset of slot 0's entry of the item's first bit, lam index
  // of that bit, slots | valid lanes of sub-chunk 0 << 8 | of sub-chunk 1
  // << 16 | absent wrap entry << 24 | mode << 25, bitmap word of sub-chunk 0
  // | zone-A slots << 16 | wrap slot << 24 (0xFF: none)}
  t->itab.clear();
  t->wbin.assign((size_t)cluster * (QBINS + 1), 0);
  p->ib[0] = 0;
  p->vbin_lo = 1 << 30;
  p->vbin_hi = 0;
  for (int c = 0; c < cluster; ++c) {
    std::vector<int4> items;
    for (int q = p->cb[c]; q < p->cb[c + 1]; ++q) {
      const int g = t->ccols[q];
      const int d = (int)cols[g].size();
      const int wrap = wrapi[g];
      const int step = items_of(g) == 6 ? 64 : 32;
      for (int mm0 = 0; mm0 < EZ; mm0 += step) {
        const int v0 = std::min(32, EZ - mm0);
        const int v1 = step == 64 ? std::max(0, std::min(32, EZ - mm0 - 32)) : 0;
        const int absent = (wrap >= 0 && mm0 + step >= EZ) ? 1 : 0;
        const uint32_t w = (uint32_t)(g * ECHUNK + mm0 / 32) | ((uint32_t)dzA[g] << 16) |
                           ((wrap >= 0 ? (uint32_t)wrap : VNOWRAP) << 24);
        items.push_back(make_int4(base[g] + vb * mm0, g * EZ + mm0,
                                  d | (v0 << 8) | (v1 << 16) | (absent << 24) |
                                      (vmode[g] << 25),
                                  (int)w));
      }
    }
    // Deal the CTA's items to QBINS bins, the most expensive first, each to
    // the least-loaded bin (longest-processing-time rule), so that every
    // warp walking its own bin has about the same work; a bin keeps its
    // items in column order.  Estimated cost (cycles per item of a
    // 1024-thread CTA under full load, fitted to per-warp phase times of
    // 64800-bit 6/15, 8/15 and 10/15 codewords): pair 840, 1-4 slots in
    // registers 280 + 240 d, any slots 1330 + 140 d (two zones: + 200).
    std::vector<int> cost(items.size()), order(items.size());
    for (size_t i = 0; i < items.size(); ++i) {
      const int d = items[i].z & 0xFF, mode = (items[i].z >> 25) & 3;
      cost[i] = mode == VM_PAIR ? 840 : mode == VM_EXACT ? 280 + 240 * d
              : mode == VM_GEN ? 1330 + 140 * d : 1530 + 140 * d;
      order[i] = (int)i;
    }
    std::stable_sort(order.begin(), order.end(),
                     [&](int x, int y) { return cost[x] > cost[y]; });
    std::vector<std::vector<int>> bins(QBINS);
    std::vector<int> load(QBINS, 0);
    for (int i : order) {
      const int b = (int)(std::min_element(load.begin(), load.end()) - load.begin());
      bins[b].push_back(i);
      load[b] += cost[i];
    }
    const int first = (int)t->itab.size();
    for (int b = 0; b < QBINS; ++b) {
      std::sort(bins[b].begin(), bins[b].end());
      t->wbin[(size_t)c * (QBINS + 1) + b] = (int)t->itab.size() - first;
      for (int i : bins[b]) t->itab.push_back(items[i]);
      p->vbin_lo = std::min(p->vbin_lo, load[b]);
      p->vbin_hi = std::max(p->vbin_hi, load[b]);
    }
    t->wbin[(size_t)c * (QBINS + 1) + QBINS] = (int)t->itab.size() - first;
    p->ib[c + 1] = (int)t->itab.size();
  }
  for (int c = cluster + 1; c <= EMAXCL; ++c) p->ib[c] = p->ib[cluster];
  return 0;
}

struct QceArgs {
  const void *llr;              // float or double (the kernel's value type)
  int64_t ld_llr;
  int nblk, n, iters;
  float alpha;
  double alpha_d;               // the scale of the float64 kernels
  // shared-memory layout (byte offsets): syndrome exchange words, per-chunk
  // row-slot table, per-row info, variable-phase items, heavy-row slots; the
  // bitmap sits at 0
  int part_off, rt_off, ri_off, ct_off, ht_off;
  int ci[EMAXCL + 1];
  int cb[EMAXCL + 1];
  int ib[EMAXCL + 1];
  int hoff[EMAXCL + 1];         // heavy items of CTA c: hitems[hoff[c] .. hoff[c+1])
  int nhrows;                   // heavy rows = block rows 0 .. nhrows-1
  int hsplit, hpb_off;          // parts per heavy item, partials' offset
  const int16_t *hitems;
  const int32_t *ccols;
  const int4 *itab;
  const int32_t *wbin;          // (cluster, QBINS+1) item-bin offsets per CTA
  const int4 *rdesc;
  const int32_t *rptr;
  const int4 *cdesc;
  const uint8_t *s0;
  const uint8_t *s0b;
  // optional learned weights, as ldpc_qc.cu: minima become
  // relu(min*w_a - w_b), (w_a, w_b) = (walpha, wbeta)[min(it, wT-1)][
  // dbucket[check degree]]; null -> (alpha, 0), bit-identical to min*alpha
  const float *walpha;
  const float *wbeta;
  const int8_t *dbucket;
  int wT, wnb;
  int wrow;          // 1: dbucket is indexed by the check's block row, not its degree
  uint8_t *bits;
  int64_t ld_bits;
  uint8_t *hard;
  int64_t ld_hard;
  uint8_t *conv;
  int32_t *its;
  int32_t *bad;
};


// Variable phase of one bit for a column of exactly D edges: the D slot
// entries are loaded in storage order, the sum is formed in the reference
// order (slots s0 .. D-1, then 0 .. s0-1) by selecting the rotated value for
// each position, and every slot is rewritten as tot - m.
template <typename V, bool TORCH, int D>
__device__ __forceinline__ V qce_var_exact(V *col, int s0, V li, bool mv) {
  V m[D];
#pragma unroll
  for (int i = 0; i < D; ++i) m[i] = col[i * EZ];
  const int s = s0 >= D ? s0 - D : s0;
  V acc = TORCH ? li : V(0);
#pragma unroll
  for (int t = 0; t < D; ++t) {
    V v = m[t];
#pragma unroll
    for (int c = 1; c < D; ++c) v = (s == c) ? m[(c + t) % D] : v;
    acc = add_rn(acc, v);
  }
  // torch semantics: + 0.0 turns a -0.0 sum into +0.0 (the only way a
  // slot could receive -0.0; the sign is the same for the hard decision)
  const V tot = TORCH ? add_rn(acc, V(0)) : add_rn(li, acc);
  if (mv) {
#pragma unroll
    for (int i = 0; i < D; ++i) col[i * EZ] = sub_rn(tot, m[i]);
  }
  return tot;
}



// Sums of one zone's slots of a column (`c0`, `c1` = the first slot of the
// two bits a lane takes in a 64-bit item, d slots) in each bit's reference
// order: slots s0 .. d-1, then 0 .. s0-1.  The two sums run interleaved, so
// a warp advances two independent chains of additions.  Inside a warp the
// bits' s0 differ little, so with lo/hi = the least/greatest s0 of both
// bits over the warp the common parts [hi, d) and [0, lo) are summed
// unconditionally and only [lo, hi) needs a per-bit choice (adding -0.0
// leaves a float sum unchanged).  The order of additions is each bit's own,
// so the sums are exact.
template <typename V>
__device__ __forceinline__ void qce_seg_sum2(V &acc0, V &acc1, const V *c0,
                                             const V *c1, int d, int s00,
                                             int s01) {
  // s0 runs 0 .. d (d: no slot wrapped, the same order as 0)
  const int lo = (int)__reduce_min_sync(0xffffffffu, (uint32_t)min(s00, s01));
  const int hi = (int)__reduce_max_sync(0xffffffffu, (uint32_t)max(s00, s01));
  if (hi - lo <= 2 && d > 0) {
    // the common case: at most two slots whose place differs between the
    // warp's bits, loaded once and held in registers for both passes
    const int i0 = min(lo, d - 1), i1 = min(lo + 1, d - 1);
    const bool h0 = lo < hi, h1 = lo + 1 < hi;
    const V w00 = c0[i0 * EZ], w01 = c0[i1 * EZ];
    const V w10 = c1[i0 * EZ], w11 = c1[i1 * EZ];
    acc0 = add_rn(acc0, h0 && lo >= s00 ? w00 : V(-0.0));
    acc1 = add_rn(acc1, h0 && lo >= s01 ? w10 : V(-0.0));
    acc0 = add_rn(acc0, h1 && lo + 1 >= s00 ? w01 : V(-0.0));
    acc1 = add_rn(acc1, h1 && lo + 1 >= s01 ? w11 : V(-0.0));
#pragma unroll 4
    for (int i = hi; i < d; ++i) {
      acc0 = add_rn(acc0, c0[i * EZ]);
      acc1 = add_rn(acc1, c1[i * EZ]);
    }
#pragma unroll 4
    for (int i = 0; i < lo; ++i) {
      acc0 = add_rn(acc0, c0[i * EZ]);
      acc1 = add_rn(acc1, c1[i * EZ]);
    }
    acc0 = add_rn(acc0, h0 && lo < s00 ? w00 : V(-0.0));
    acc1 = add_rn(acc1, h0 && lo < s01 ? w10 : V(-0.0));
    acc0 = add_rn(acc0, h1 && lo + 1 < s00 ? w01 : V(-0.0));
    acc1 = add_rn(acc1, h1 && lo + 1 < s01 ? w11 : V(-0.0));
    return;
  }
  for (int i = lo; i < hi; ++i) {
    const V m0 = c0[i * EZ], m1 = c1[i * EZ];
    acc0 = add_rn(acc0, i >= s00 ? m0 : V(-0.0));
    acc1 = add_rn(acc1, i >= s01 ? m1 : V(-0.0));
  }
#pragma unroll 4
  for (int i = hi; i < d; ++i) {
    acc0 = add_rn(acc0, c0[i * EZ]);
    acc1 = add_rn(acc1, c1[i * EZ]);
  }
#pragma unroll 4
  for (int i = 0; i < lo; ++i) {
    acc0 = add_rn(acc0, c0[i * EZ]);
    acc1 = add_rn(acc1, c1[i * EZ]);
  }
  for (int i = lo; i < hi; ++i) {
    const V m0 = c0[i * EZ], m1 = c1[i * EZ];
    acc0 = add_rn(acc0, i < s00 ? m0 : V(-0.0));
    acc1 = add_rn(acc1, i < s01 ? m1 : V(-0.0));
  }
}

// Variable phase of the two bits a lane takes in a 64-bit item, for a column
// of d edges (any d >= 1) whose first dA slots lie in the accumulator rows
// and the rest in the identity rows (dA == d for one zone): per bit the
// reference order is zone A rotated at s0, then zone B rotated at s0b;
// every slot of a bit that is live (mv) is rewritten as tot - m.  Returns
// the two posteriors.
template <typename V, bool TORCH>
__device__ __forceinline__ void qce_var_generic2(V *c0, V *c1, int d, int dA,
                                                 int s00, int s01, int s0b0,
                                                 int s0b1, V li0, V li1,
                                                 bool mv0, bool mv1, V &t0,
                                                 V &t1) {
  V a0 = TORCH ? li0 : V(0), a1 = TORCH ? li1 : V(0);
  qce_seg_sum2(a0, a1, c0, c1, dA, s00, s01);
  if (dA < d) qce_seg_sum2(a0, a1, c0 + dA * EZ, c1 + dA * EZ, d - dA, s0b0, s0b1);
  // torch semantics: + 0.0 turns a -0.0 sum into +0.0 (see qce_var_exact)
  t0 = TORCH ? add_rn(a0, V(0)) : add_rn(li0, a0);
  t1 = TORCH ? add_rn(a1, V(0)) : add_rn(li1, a1);
  int i = 0;
  for (; i + 2 <= d; i += 2) {
    const V m00 = c0[i * EZ], m01 = c0[(i + 1) * EZ];
    const V m10 = c1[i * EZ], m11 = c1[(i + 1) * EZ];
    if (mv0) {
      c0[i * EZ] = sub_rn(t0, m00);
      c0[(i + 1) * EZ] = sub_rn(t0, m01);
    }
    if (mv1) {
      c1[i * EZ] = sub_rn(t1, m10);
      c1[(i + 1) * EZ] = sub_rn(t1, m11);
    }
  }
  if (i < d) {
    const V m0 = c0[i * EZ], m1 = c1[i * EZ];
    if (mv0) c0[i * EZ] = sub_rn(t0, m0);
    if (mv1) c1[i * EZ] = sub_rn(t1, m1);
  }
}

// One check item: block row rl, chunk ch (32 consecutive checks), D slots.
// FULL: every slot is an edge of every lane's check and all 32 lanes are
// checks (no masking at all); otherwise `live` masks absent slots (rows of
// lower degree, the missing wrap edge of check (0, 0), lanes past 359), whose
// loads and stores go to a junk word.  SYN: also form the lane's syndrome
// bit from the hard-decision bitmap (else 0 is returned: the caller already
// knows that this iteration's syndrome is not zero).
//
// Signs are taken from the sign bits of the slot values: no slot that a
// check reads holds -0.0 (the prologue and the torch-semantics variable
// phase add +0.0, which turns -0.0 into +0.0 and changes nothing else; the
// other sums never produce -0.0), so the sign bit of t is exactly the
// reference's (v < 0).  Rows of up to 11 edges (their values stay in
// registers to the end) take the parity as the XOR of the sign bits and a
// message's sign bit as parity ^ sign(t): one XOR onto the magnitude that
// already carries the parity.  Longer rows keep a mask of the signs so the
// values can die early.
template <typename V, bool TORCH, int D, bool FULL, bool SYN, typename MASK>
__device__ __forceinline__ int qce_check_item(const uint2 *te, MASK live,
                                              uint32_t lane,
                                              const uint32_t *bm,
                                              uint32_t dummy, bool upd,
                                              const QceArgs &a, int it, int row) {
  // per slot: address, remote load (its value is first used by the update
  // below, so the syndrome lookup overlaps its latency), syndrome bit; the
  // syndrome-only final pass loads too (valid addresses, values unused)
  constexpr uint32_t VB = sizeof(V);
  using UB = decltype(vbits(V(0)));
  constexpr UB SIGN = (UB)1 << (8 * sizeof(UB) - 1);
  uint32_t ad[D];
  V t[D];
  uint32_t synw = 0;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    const uint2 e = te[j];
    const uint32_t x = (e.y >> 16) + lane;
    const uint32_t o = min(x, x - (uint32_t)EZ);    // (b + lane) mod 360
    if constexpr (FULL) {
      ad[j] = e.x + VB * o;
    } else {
      const uint32_t on = (uint32_t)(live >> j) & 1u;
      ad[j] = on ? e.x + VB * o : dummy;
    }
    t[j] = dsmem_ld<V>(ad[j]);
    if constexpr (SYN) {
      const uint32_t hw = bm[(e.y & 0xFFFFu) + (o >> 5)];
      if constexpr (FULL) {
        synw ^= hw >> (o & 31);
      } else {
        synw ^= (hw >> (o & 31)) & ((uint32_t)(live >> j) & 1u);
      }
    }
  }
  if (upd) {
    const V inf = vinf<V>();
    // min1/min2 with min/max only: the reference's strict-< update
    // (ldpc_kernel.c:121-126) gives min2 = min(min2, max(min1, mag)),
    // min1 = min(min1, mag), including ties
    // Rows of up to 11 edges keep their values to the end and pick each
    // message by comparing |t| with min1; longer rows track the first
    // minimum's position instead, so the values can die early (registers).
    constexpr bool BY_VALUE = D <= 11;
    constexpr bool WIDE = sizeof(MASK) > 4;
    V min1 = inf, min2 = inf;
    uint32_t first = 0;
    UB pw = 0;                                       // XOR of the sign bits
    MASK sv = 0;                                     // sign mask (long rows)
#pragma unroll
    for (int j = 0; j < D; ++j) {
      V mag = vabs(t[j]);
      UB tb = vbits(t[j]);
      if constexpr (!FULL) {
        const bool on = (live >> j) & 1;
        mag = on ? mag : inf;
        tb = on ? tb : (UB)0;
      }
      if constexpr (BY_VALUE) {
        pw ^= tb;
      } else {
        sv |= (tb & SIGN) ? ((MASK)1 << j) : (MASK)0;
        first = mag < min1 ? (uint32_t)j : first;
      }
      min2 = vmin(min2, vmax(min1, mag));
      min1 = vmin(min1, mag);
    }
    // float32: scale a.alpha or the learned (scale, offset); float64: the
    // scale a.alpha_d (no learned weights)
    V wa, wb = V(0);
    if constexpr (sizeof(V) == 8) wa = a.alpha_d;
    else wa = a.alpha;
    if (sizeof(V) == 4 && a.walpha) {
      int nl = D;
      if constexpr (!FULL) {
        if constexpr (WIDE) nl = __popcll((unsigned long long)live);
        else nl = __popc((uint32_t)live);
      }
      const int wi = min(it, a.wT - 1) * a.wnb + __ldg(a.dbucket + (a.wrow ? row : nl));
      wa = __ldg(a.walpha + wi);
      wb = __ldg(a.wbeta + wi);
    }
    V A = sub_rn(mul_rn(min1, wa), wb);
    V B = sub_rn(mul_rn(min2, wa), wb);
    A = A > V(0) ? A : V(0);
    B = B > V(0) ? B : V(0);
    // the edge holding the first minimum gets min2, every other min1; an
    // edge whose magnitude equals min1 but is not the first one has
    // min2 == min1, so testing |t| == min1 picks the same value
    if constexpr (BY_VALUE) {
      // magnitudes with the check's parity in the sign bit
      const UB psign = pw & SIGN;
      const UB ua = vbits(A) | psign, ub = vbits(B) | psign;
#pragma unroll
      for (int j = 0; j < D; ++j) {
        const bool take2 = vabs(t[j]) == min1;
        dsmem_st_bits(ad[j], (take2 ? ub : ua) ^ (vbits(t[j]) & SIGN));
      }
    } else {
      int par;
      if constexpr (WIDE) par = __popcll((unsigned long long)sv) & 1;
      else par = __popc((uint32_t)sv) & 1;
      const auto ua = vbits(A), ub = vbits(B);
      MASK all;
      if constexpr (FULL) all = (D >= 8 * (int)sizeof(MASK)) ? ~(MASK)0 : (((MASK)1 << D) - 1);
      else all = live;
      const MASK neg = par ? (sv ^ all) : sv;        // message signs
#pragma unroll
      for (int j = 0; j < D; ++j)
        dsmem_st_msg(ad[j], (uint32_t)j == first ? ub : ua, (uint32_t)(neg >> j) & 1u);
    }
  }
  return (int)(synw & 1u);
}

// One light check item (check-phase item wl of this CTA): chunks 0 ..
// ECHUNK-2 of a row on the unmasked paths where the row allows it, else the
// masked path; the rows' last chunks packed TAILG rows to a warp.  Returns
// the lane's syndrome bit (0 without SYN, and for lanes past the tails).
template <typename V, bool TORCH, int NS, bool SYN, typename MASK>
__device__ __forceinline__ int qce_light_item(int wl, int nlead, int coff,
                                              int ntail, const uint2 *rtab,
                                              const MASK *rinfo, uint32_t lane,
                                              const uint32_t *bm, uint32_t dummy,
                                              bool upd, const QceArgs &a, int it,
                                              int r0) {
  constexpr int TAILW = EZ - 32 * (ECHUNK - 1);
  constexpr int TAILG = 32 / TAILW;
  if (wl < nlead) {                              // chunks 0 .. ECHUNK-2 of a row
    const int u = wl + coff;
    const int rl = u / (ECHUNK - 1);
    const int ch = u - rl * (ECHUNK - 1);
    const MASK wm = rinfo[3 * rl + 1];
    const int deg = (int)rinfo[3 * rl + 2];
    const uint2 *te = rtab + (rl * ECHUNK + ch) * NS;
    if (wm == 0 && deg == NS)
      return qce_check_item<V, TORCH, NS, true, SYN, MASK>(te, (MASK)0, lane, bm, dummy,
                                                          upd, a, it, r0 + rl);
    if (wm == 0 && deg == NS - 1)
      return qce_check_item<V, TORCH, NS - 1, true, SYN, MASK>(te, (MASK)0, lane, bm,
                                                              dummy, upd, a, it, r0 + rl);
    if constexpr (NS >= 10) {                    // rows two short of the template
      if (wm == 0 && deg == NS - 2)
        return qce_check_item<V, TORCH, NS - 2, true, SYN, MASK>(te, (MASK)0, lane, bm,
                                                                dummy, upd, a, it, r0 + rl);
    }
    MASK live = rinfo[3 * rl];
    if (ch == 0 && lane == 0) live &= ~wm;       // check (0, 0): no wrap edge
    return qce_check_item<V, TORCH, NS, false, SYN, MASK>(te, live, lane, bm, dummy, upd,
                                                         a, it, r0 + rl);
  }
  const int t = (wl - nlead) * TAILG + (int)lane / TAILW;   // last chunks
  const bool valid = t < ntail;
  const int rl = valid ? t : 0;
  const uint2 *te = rtab + (rl * ECHUNK + ECHUNK - 1) * NS;
  const MASK live = valid ? rinfo[3 * rl] : (MASK)0;
  const int syn = qce_check_item<V, TORCH, NS, false, SYN, MASK>(
      te, live, lane % TAILW, bm, dummy, upd, a, it, r0 + rl);
  return valid ? syn : 0;
}

// Heavy rows (more edges than the compile-time slot count; the accumulator
// rows of the Type A codes): an item = 32 consecutive checks of the row, its
// deg slots cut into parts [j0, j1) that different warps walk.  he[j] =
// {shared::cluster address of slot j's block, shift u << 16 | bitmap word
// index}; wrapj = the slot that check (0, 0) lacks, or -1.
struct HeavyPart {               // one lane's partial state over [j0, j1)
  float min1, min2;
  int first;                     // absolute slot index of the first minimum
  uint32_t bits;                 // sign parity | syndrome bit << 1
};

__device__ __forceinline__ uint32_t heavy_addr(const uint2 &e, int ch, uint32_t lane,
                                               uint32_t *o) {
  int bb = ch * 32 - (int)(e.y >> 16);
  bb += bb < 0 ? EZ : 0;
  const uint32_t x = (uint32_t)bb + lane;
  *o = min(x, x - (uint32_t)EZ);
  return e.x + 4u * *o;
}

// Pass 1 over [j0, j1): min1/min2/first (strict <, ldpc_kernel.c:121-126),
// sign parity and syndrome bit of the loaded edge values.
__device__ __forceinline__ HeavyPart qce_heavy_pass1(const uint2 *he, int j0, int j1,
                                                     int wrapj, uint32_t lane, int ch,
                                                     const uint32_t *bm, uint32_t dummy) {
  const int k0 = ch * 32 + (int)lane;
  const bool lv = k0 < EZ;
  const float inf = __int_as_float(0x7f800000);
  HeavyPart r{inf, inf, j0, 0u};
  uint32_t synw = 0;
  for (int j = j0; j < j1; ++j) {
    const uint2 e = he[j];
    uint32_t o;
    const uint32_t ad = heavy_addr(e, ch, lane, &o);
    const bool on = lv && !(k0 == 0 && j == wrapj);
    const float t = dsmem_ld_f32(on ? ad : dummy);
    if (on) {
      const uint32_t hw = bm[(e.y & 0xFFFFu) + (o >> 5)];
      synw ^= hw >> (o & 31);
      const float mag = fabsf(t);
      r.bits ^= t < 0.f ? 1u : 0u;
      r.first = mag < r.min1 ? j : r.first;
      r.min2 = fminf(r.min2, fmaxf(r.min1, mag));
      r.min1 = fminf(r.min1, mag);
    }
  }
  r.bits |= (synw & 1u) << 1;
  return r;
}

// Pass 2 over [j0, j1): reload each value (this lane alone writes it, after
// reading) and store its message.
__device__ __forceinline__ void qce_heavy_pass2(const uint2 *he, int j0, int j1, int wrapj,
                                                uint32_t lane, int ch, uint32_t ua,
                                                uint32_t ub, int first, uint32_t par) {
  const int k0 = ch * 32 + (int)lane;
  const bool lv = k0 < EZ;
  for (int j = j0; j < j1; ++j) {
    const uint2 e = he[j];
    uint32_t o;
    const uint32_t ad = heavy_addr(e, ch, lane, &o);
    if (lv && !(k0 == 0 && j == wrapj)) {
      const float t = dsmem_ld_f32(ad);
      const uint32_t sg = par ^ (t < 0.f ? 1u : 0u);
      dsmem_st_u32(ad, (j == first ? ub : ua) | (sg << 31));
    }
  }
}

// Check item of a heavy row (more edges than the compile-time slot count;
// the accumulator rows of the Type A codes): 32 consecutive checks of the
// row, its deg slots walked in a loop.  he[j] = {shared::cluster address of
// slot j's block, shift u << 16 | bitmap word index}; wrapj = the slot that
// check (0, 0) lacks, or -1.  Pass 1 loads every edge value, forms the
// syndrome bit, min1/min2/first (strict <, ldpc_kernel.c:121-126) and the
// sign parity; pass 2 loads each value again (this lane alone writes it,
// after reading) and stores the message.  Returns the lane's syndrome bit.
template <typename V, bool TORCH>
__device__ __forceinline__ int qce_check_heavy(const uint2 *he, int deg, int wrapj,
                                            uint32_t lane, int ch,
                                            const uint32_t *bm, uint32_t dummy,
                                            bool upd, const QceArgs &a, int it, int row) {
  const int k0 = ch * 32 + (int)lane;
  const bool lv = k0 < EZ;
  constexpr uint32_t VB = sizeof(V);
  const V inf = vinf<V>();
  V min1 = inf, min2 = inf;
  int first = 0;
  uint32_t par = 0, synw = 0;
  for (int j = 0; j < deg; ++j) {
    const uint2 e = he[j];
    int bb = ch * 32 - (int)(e.y >> 16);
    bb += bb < 0 ? EZ : 0;
    const uint32_t x = (uint32_t)bb + lane;
    const uint32_t o = min(x, x - (uint32_t)EZ);
    const bool on = lv && !(k0 == 0 && j == wrapj);
    const V t = dsmem_ld<V>(on ? e.x + VB * o : dummy);
    if (on) {
      const uint32_t hw = bm[(e.y & 0xFFFFu) + (o >> 5)];
      synw ^= hw >> (o & 31);
      const V mag = vabs(t);
      par ^= t < V(0) ? 1u : 0u;
      first = mag < min1 ? j : first;
      min2 = vmin(min2, vmax(min1, mag));
      min1 = vmin(min1, mag);
    }
  }
  if (upd) {
    V wa, wb = V(0);
    if constexpr (sizeof(V) == 8) wa = a.alpha_d;
    else wa = a.alpha;
    if (sizeof(V) == 4 && a.walpha) {
      const int nl = deg - ((k0 == 0 && wrapj >= 0) ? 1 : 0);
      const int wi = min(it, a.wT - 1) * a.wnb + __ldg(a.dbucket + (a.wrow ? row : nl));
      wa = __ldg(a.walpha + wi);
      wb = __ldg(a.wbeta + wi);
    }
    V A = sub_rn(mul_rn(min1, wa), wb);
    V B = sub_rn(mul_rn(min2, wa), wb);
    A = A > V(0) ? A : V(0);
    B = B > V(0) ? B : V(0);
    const auto ua = vbits(A), ub = vbits(B);
    for (int j = 0; j < deg; ++j) {
      const uint2 e = he[j];
      int bb = ch * 32 - (int)(e.y >> 16);
      bb += bb < 0 ? EZ : 0;
      const uint32_t x = (uint32_t)bb + lane;
      const uint32_t o = min(x, x - (uint32_t)EZ);
      const bool on = lv && !(k0 == 0 && j == wrapj);
      if (on) {
        const uint32_t ad = e.x + VB * o;
        const V t = dsmem_ld<V>(ad);
        dsmem_st_msg(ad, j == first ? ub : ua, par ^ (t < V(0) ? 1u : 0u));
      }
    }
  }
  return lv ? (int)(synw & 1u) : 0;
}

// NS: compile-time slots per block row (qce_ns); NT: threads per CTA; TA:
// the Type A paths (rows above NS, columns in both zones) are compiled in.
// A variable item's inputs that the slots do not hold: its table entry, the
// channel LLRs of the lane's two bits (lane L takes bits y + L and y + 32 + L;
// lanes past the item's bit count read bit y) and their first-slot indices.
// None of them changes during a codeword, so the variable phase can fetch the
// next item's while it works on the current one.
template <typename V>
struct QceVarIn {
  uint4 iw;
  V li0, li1;
  int s00, s01;
};

template <typename V>
__device__ __forceinline__ void qce_var_fetch(QceVarIn<V> &f, const uint4 *itab, int w,
                                              int lane, const V *lam, const uint8_t *s0) {
  f.iw = itab[w];
  const uint32_t nv0 = (f.iw.z >> 8) & 0xFFu, nv1 = (f.iw.z >> 16) & 0xFFu;
  const int x0 = (int)f.iw.y + ((uint32_t)lane < nv0 ? lane : 0);
  const int x1 = (int)f.iw.y + ((uint32_t)lane < nv1 ? 32 + lane : 0);
  f.li0 = lam[x0];
  f.li1 = lam[x1];
  f.s00 = __ldg(s0 + x0);
  f.s01 = __ldg(s0 + x1);
}

template <typename V, bool TORCH, int NS, int NT, bool TA>
__global__ void __launch_bounds__(NT, 1) ldpc_qce_kernel(const QceArgs a) {
  using MASK = typename std::conditional<(NS > 32), unsigned long long,
                                         uint32_t>::type;
  extern __shared__ __align__(16) unsigned char smem[];
  const int rank = (int)cluster_ctarank();
  const int CL = (int)cluster_nctarank();
  const uint32_t *bm = reinterpret_cast<const uint32_t *>(smem);
  // syndrome counters (2, alternating iterations); junk word at [40]
  int *part = reinterpret_cast<int *>(smem + a.part_off);
  uint2 *rtab = reinterpret_cast<uint2 *>(smem + a.rt_off);
  MASK *rinfo = reinterpret_cast<MASK *>(smem + a.ri_off);
  uint4 *itab = reinterpret_cast<uint4 *>(smem + a.ct_off);
  const uint32_t sm_sa = smem_u32(smem);
  const uint32_t part_sa = smem_u32(part);
  const uint32_t dummy = part_sa + 40 * 4;   // junk word for masked slots
  // "an unsatisfied check was seen" flags (2, alternating iterations),
  // written into every CTA of the cluster by the first warps that see one
  volatile int *seen = part + 2;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nwarps = blockDim.x >> 5;
  // check items g = row*12 + chunk in [c0, c0 + ncitems); rows r0 .. r0+nr-1
  const int c0 = a.ci[rank], ncitems = a.ci[rank + 1] - c0;
  const int r0 = c0 / ECHUNK;
  const int nr = ncitems > 0 ? (c0 + ncitems + ECHUNK - 1) / ECHUNK - r0 : 0;
  // the check items run as: chunks 0 .. ECHUNK-2 of these rows in row order
  // (nlead of them, from chunk coff of row r0), then the rows' last chunks
  // (TAILW checks each; the rows whose last chunk is this CTA's) packed
  // TAILG to a warp, lane group g taking tail t = TAILG * item + g
  constexpr int TAILW = EZ - 32 * (ECHUNK - 1);
  constexpr int TAILG = 32 / TAILW;
  static_assert(TAILW > 0 && 32 % TAILW == 0, "tail chunk must divide a warp");
  const int coff = c0 - r0 * ECHUNK;
  const int ntail = max(0, min(nr, (c0 + ncitems) / ECHUNK - r0));
  const int nlead = ncitems - ntail;
  const int ncpk = nlead + (ntail + TAILG - 1) / TAILG;
  const int i0 = a.ib[rank], nvitems = a.ib[rank + 1] - i0;
  // heavy rows are compiled into the Type A kernels of 6 and 8 slots (the
  // builder refuses them with 4)
  constexpr bool HV = TA && NS >= 6;
  const int h0 = a.hoff[rank], nhi = HV ? a.hoff[rank + 1] - h0 : 0;
  // this lane's cluster address of CTA `lane`'s bitmap (ballot broadcast)
  const uint32_t bm_peer = lane < CL ? dsmem_map(sm_sa, (uint32_t)lane) : 0u;
  // this lane's cluster address of CTA `lane`'s seen flags
  const uint32_t seen_peer = lane < CL ? dsmem_map(part_sa + 8u, (uint32_t)lane) : 0u;

  // ---- per-launch tables ---------------------------------------------------
  // row slot (rl, chunk, j): {shared::cluster address of the slot block in
  // its owner, (first entry index b = (32*chunk - u) mod 360) << 16 | bitmap
  // word index of the column}; slots past the row degree repeat the last one.
  // Heavy rows (the accumulator rows of a Type A code, above NS edges; every
  // CTA holds all of them): hinfo[r] = {slot entries' offset in htab, wrap
  // slot + 1 (0: none), degree}, one htab entry per slot.
  int4 *hinfo = reinterpret_cast<int4 *>(smem + a.ht_off);
  uint2 *htab = reinterpret_cast<uint2 *>(smem + a.ht_off + 16 * a.nhrows);
  if (HV) {
    if (tid == 0) {
      int off = 0;
      for (int r = 0; r < a.nhrows; ++r) {
        const int rp = __ldg(a.rptr + r);
        const int deg = __ldg(a.rptr + r + 1) - rp;
        int wj = 0;
        for (int q = 0; q < deg; ++q)
          if (__ldg(a.rdesc + rp + q).x & EWRAP) wj = q + 1;
        hinfo[r] = make_int4(off, wj, deg, 0);
        off += deg;
      }
    }
    __syncthreads();
    for (int r = warp; r < a.nhrows; r += nwarps) {
      const int rp = __ldg(a.rptr + r);
      const int deg = __ldg(a.rptr + r + 1) - rp;
      const int off = hinfo[r].x;
      for (int j = lane; j < deg; j += 32) {
        const int4 d = __ldg(a.rdesc + rp + j);
        htab[off + j] = make_uint2(dsmem_map(sm_sa + (uint32_t)d.y, (uint32_t)(d.x & 0xFF)),
                                   ((uint32_t)d.z << 16) | ((uint32_t)d.w >> 2));
      }
    }
  }
  for (int e = tid; e < nr * NS; e += blockDim.x) {
    const int rl = e / NS;
    const int j = e - rl * NS;
    const int rp = __ldg(a.rptr + r0 + rl);
    const int deg = __ldg(a.rptr + r0 + rl + 1) - rp;
    const int4 d = __ldg(a.rdesc + rp + min(j, deg - 1));
    const uint32_t base = dsmem_map(sm_sa + (uint32_t)d.y, (uint32_t)(d.x & 0xFF));
    const uint32_t wb = (uint32_t)d.w >> 2;
#pragma unroll 1
    for (int ch = 0; ch < ECHUNK; ++ch) {
      int bb = ch * 32 - d.z;
      bb += bb < 0 ? EZ : 0;
      rtab[(rl * ECHUNK + ch) * NS + j] = make_uint2(base, ((uint32_t)bb << 16) | wb);
    }
    if (j == 0) {
      MASK wm = 0;
      for (int q = 0; q < deg; ++q)
        if (__ldg(a.rdesc + rp + q).x & EWRAP) wm |= (MASK)1 << q;
      rinfo[3 * rl] = deg >= (int)(8 * sizeof(MASK)) ? ~(MASK)0
                                                      : (((MASK)1 << deg) - 1);
      rinfo[3 * rl + 1] = wm;
      rinfo[3 * rl + 2] = (MASK)deg;
    }
  }
  // variable-phase items of this CTA (built on the host), and the bins the
  // host dealt them into (part[4 .. 4 + QBINS]): warp w walks bins
  // w*bpw .. (w+1)*bpw - 1, contiguous in the item list
  int *vbin = part + 4;
  for (int q = tid; q <= QBINS; q += blockDim.x) vbin[q] = __ldg(a.wbin + rank * (QBINS + 1) + q);
  for (int q = tid; q < nvitems; q += blockDim.x) {
    const int4 v = __ldg(a.itab + i0 + q);
    itab[q] = make_uint4((uint32_t)v.x, (uint32_t)v.y, (uint32_t)v.z, (uint32_t)v.w);
  }
  if (tid == 0) {
    part[0] = 0;
    part[1] = 0;
    part[2] = 0;
    part[3] = 0;
  }
  __syncthreads();

  // the absent wrap entry (last parity column, bit 359, its wrap slot) is
  // lane 7 of sub-chunk 1 of that column's last item, slot 1 of the column
  constexpr int ABSENT_LANE = EZ - 32 * (ECHUNK - 1) - 1;
  // this warp's variable items: bins warp*BPW .. (warp+1)*BPW - 1 (NT is
  // 512 or 1024), their offsets read from shared memory at each phase
  // (volatile: not kept in registers across the codeword loop)
  constexpr int BPW = QBINS / (NT / 32);
  static_assert(BPW >= 1 && QBINS % (NT / 32) == 0, "512 or 1024 threads");
  // the variable phase fetches item k+1's inputs while it works on item k
  // (their global loads leave the item's chain) where the registers allow:
  // float32 kernels of up to 8 slots (Type B) at 1024 threads, up to 22 at 512
  constexpr bool VPF = sizeof(V) == 4 && (NT >= 1024 ? (NS <= 8 && !TA) : NS <= 22);

  for (int b = (int)cluster_id_x(); b < a.nblk; b += (int)ncluster_x()) {
    const V *lam = reinterpret_cast<const V *>(a.llr) + (size_t)b * a.ld_llr;
    // ---- prologue: q = lam - 0 = lam on every slot, hard bits of lam; the
    // absent entry holds -0.0 (adding it is exact) ---------------------------
    for (int w = ((volatile int *)part)[4 + warp * BPW],
             we = ((volatile int *)part)[4 + (warp + 1) * BPW]; w < we; ++w) {
      const uint4 iw = itab[w];
      const int d = (int)(iw.z & 0xFFu);
      // the absent entry: bit 359 = lane 7 of the item's last sub-chunk
      const int asub = ((iw.z >> 16) & 0xFFu) ? 1 : 0;
      const int wrapi = (int)(iw.w >> 24);
#pragma unroll
      for (int sub = 0; sub < 2; ++sub) {
        const uint32_t nval = (iw.z >> (8 + 8 * sub)) & 0xFFu;
        if (nval == 0) break;                         // 32-bit item
        const bool mv = (uint32_t)lane < nval;
        const bool absent = sub == asub && ((iw.z >> 24) & 1u) && lane == ABSENT_LANE;
        const V li = mv ? lam[iw.y + 32 * sub + lane] : V(0);
        V *col = reinterpret_cast<V *>(smem + iw.x) + 32 * sub + lane;
        // q = lam - 0; stored as lam + 0 (+0.0 for a -0.0 LLR, which the
        // check phase's sign-bit tests then read like the reference's v < 0)
        const V lq = add_rn(li, V(0));
        if (mv)
          for (int i = 0; i < d; ++i) col[i * EZ] = (absent && i == wrapi) ? V(-0.0) : lq;
        const uint32_t hb = __ballot_sync(0xffffffffu, mv && li < V(0));
        if (lane < CL) dsmem_st_u32(bm_peer + ((iw.w & 0xFFFFu) + sub) * 4u, hb);
      }
    }
    cluster_sync_all();      // (a cluster barrier also orders this CTA)

    for (int it = 0;; ++it) {
      const bool upd = it < a.iters;   // the last pass only needs the syndrome
      // the count of the previous iteration has been read by every thread
      // (a barrier ago); its slot is reused two iterations later
      if (tid == 0 && it > 0) {
        part[(it - 1) & 1] = 0;
        part[2 + ((it - 1) & 1)] = 0;
      }
      // ---------------- check phase ----------------------------------------
      int mybad = 0;
      // Type A with heavy rows: this CTA's heavy items first, one warp each,
      // then its light items.  With hsplit > 1 (very heavy rows): phase A =
      // pass 1 of every heavy item part (one warp each; partials to shared
      // memory) and the light items; phase B (after a CTA barrier) = merge
      // each item's partials and pass 2 of every part.
      // (the parts path is float32 only; float64 plans keep one warp per item)
      const bool split = HV && sizeof(V) == 4 && a.nhrows && a.hsplit > 1;
      const int nhp = (HV && a.nhrows) ? (split ? nhi * a.hsplit : nhi) : 0;
      for (int w = warp; w < nhp + ncpk; w += nwarps) {
        int syn;
        if (HV && w < nhp && !split) {             // one warp per heavy item
          const int hi = __ldg(a.hitems + h0 + w);
          const int row = hi / ECHUNK;
          const int4 hf = hinfo[row];
          mybad += qce_check_heavy<V, TORCH>(htab + hf.x, hf.z, hf.y - 1, (uint32_t)lane,
                                          hi - row * ECHUNK, bm, dummy, upd, a, it, row);
          continue;
        }
        if (HV && w < nhp) {
          const int i = w / a.hsplit, part = w - i * a.hsplit;
          const int hi = __ldg(a.hitems + h0 + i);
          const int row = hi / ECHUNK;
          const int4 hf = hinfo[row];
          const int j0 = part * hf.z / a.hsplit, j1 = (part + 1) * hf.z / a.hsplit;
          const HeavyPart r = qce_heavy_pass1(htab + hf.x, j0, j1, hf.y - 1, (uint32_t)lane,
                                              hi - row * ECHUNK, bm, dummy);
          reinterpret_cast<float4 *>(smem + a.hpb_off)[w * 32 + lane] =
              make_float4(r.min1, r.min2, __int_as_float(r.first), __uint_as_float(r.bits));
          continue;
        }
        // Light items form their syndrome bits only while no warp of the
        // cluster has reported an unsatisfied check in this iteration: once
        // one has, the iteration's syndrome is known to be nonzero, which is
        // all an updating iteration needs (the count itself is only output
        // by the final, update-free pass, which always forms every bit).
        // Rows of more than 14 slots always form them: a second copy of
        // their unrolled item code would cost those kernels registers.
        const int wl = w - nhp;
        if (NS > 14 || !upd || seen[it & 1] == 0) {
          syn = qce_light_item<V, TORCH, NS, true, MASK>(wl, nlead, coff, ntail, rtab, rinfo,
                                                         (uint32_t)lane, bm, dummy, upd, a, it, r0);
          mybad += syn;
          if (NS <= 14 && upd && __any_sync(0xffffffffu, syn != 0) && lane < CL)
            dsmem_st_u32(seen_peer + (uint32_t)((it & 1) * 4), 1u);
        } else if constexpr (NS <= 14) {
          qce_light_item<V, TORCH, NS, false, MASK>(wl, nlead, coff, ntail, rtab, rinfo,
                                                    (uint32_t)lane, bm, dummy, upd, a, it, r0);
        }
      }
      if (split) {
        __syncthreads();
        const float4 *pb = reinterpret_cast<const float4 *>(smem + a.hpb_off);
        for (int w = warp; w < nhp; w += nwarps) {
          const int i = w / a.hsplit, part = w - i * a.hsplit;
          const int hi = __ldg(a.hitems + h0 + i);
          const int row = hi / ECHUNK;
          const int ch = hi - row * ECHUNK;
          const int4 hf = hinfo[row];
          const int k0 = ch * 32 + lane;
          // merge the parts in slot order: the first minimum is the lowest
          // part's on ties; min2 = the second order statistic
          const float inf = __int_as_float(0x7f800000);
          float min1 = inf, min2 = inf;
          int first = 0;
          uint32_t bits = 0;
          for (int q = 0; q < a.hsplit; ++q) {
            const float4 v = pb[(i * a.hsplit + q) * 32 + lane];
            if (v.x < min1) {
              min2 = fminf(min1, v.y);
              min1 = v.x;
              first = __float_as_int(v.z);
            } else {
              min2 = fminf(min2, v.x);
            }
            min2 = fminf(min2, v.y);
            bits ^= __float_as_uint(v.w);
          }
          if (part == 0 && k0 < EZ) mybad += (int)((bits >> 1) & 1u);
          if (upd) {
            float wa = a.alpha, wb = 0.f;
            if (a.walpha) {
              const int nl = hf.z - ((k0 == 0 && hf.y > 0) ? 1 : 0);
              const int wi = min(it, a.wT - 1) * a.wnb + __ldg(a.dbucket + (a.wrow ? row : nl));
              wa = __ldg(a.walpha + wi);
              wb = __ldg(a.wbeta + wi);
            }
            float A = __fsub_rn(__fmul_rn(min1, wa), wb);
            float B = __fsub_rn(__fmul_rn(min2, wa), wb);
            A = A > 0.f ? A : 0.f;
            B = B > 0.f ? B : 0.f;
            const int j0 = part * hf.z / a.hsplit, j1 = (part + 1) * hf.z / a.hsplit;
            qce_heavy_pass2(htab + hf.x, j0, j1, hf.y - 1, (uint32_t)lane, ch,
                            __float_as_uint(A), __float_as_uint(B), first, bits & 1u);
          }
        }
      }
      // unsatisfied checks: every warp adds its count into the counter of
      // every CTA of the cluster, so after the barrier each CTA holds the total
      mybad = __reduce_add_sync(0xffffffffu, mybad);
      if (lane < CL && mybad)
        dsmem_red_add_u32(dsmem_map(part_sa + (uint32_t)((it & 1) * 4), (uint32_t)lane),
                          (uint32_t)mybad);
      cluster_sync_all();
      const int badct = part[it & 1];
      const bool done = (badct == 0) && (!TORCH || it > 0);
      if (done || it >= a.iters) {
        // outputs from this CTA's bitmap replica (complete in every CTA):
        // CTA `rank` writes its share of the codeword's bytes / bits
        const int nby = a.n >> 3;
        const int by0 = (int)((int64_t)nby * rank / CL);
        const int by1 = (int)((int64_t)nby * (rank + 1) / CL);
        if (a.hard) {
          uint8_t *ho = a.hard + (size_t)b * a.ld_hard;
          for (int by = by0 + tid; by < by1; by += blockDim.x) {
            const int g = by / 45;
            const int bb = (by - g * 45) * 8;
            const uint32_t v = (bm[g * ECHUNK + (bb >> 5)] >> (bb & 31)) & 0xFFu;
            ho[by] = (uint8_t)(__brev(v) >> 24);
          }
        }
        if (a.bits) {
          uint8_t *bo = a.bits + (size_t)b * a.ld_bits;
          for (int i = by0 * 8 + tid; i < by1 * 8; i += blockDim.x) {
            const int g = i / EZ;
            const int mm = i - g * EZ;
            bo[i] = (uint8_t)((bm[g * ECHUNK + (mm >> 5)] >> (mm & 31)) & 1u);
          }
        }
        if (rank == 0 && tid == 0) {
          a.conv[b] = done ? 1 : 0;
          a.its[b] = it;
          a.bad[b] = done ? 0 : badct;
        }
        // every CTA has read its replica before the next codeword's prologue
        // writes the replicas of the whole cluster; both counters start at 0
        cluster_sync_all();
        if (tid == 0) {
          part[0] = 0;
          part[1] = 0;
          part[2] = 0;
          part[3] = 0;
        }
        break;
      }
      // ---------------- variable phase (local) -----------------------------
      // (the first item's inputs are fetched after the barrier: its release
      // would wait for loads issued before it)
      const int vw0 = ((volatile int *)part)[4 + warp * BPW];
      const int vwe = ((volatile int *)part)[4 + (warp + 1) * BPW];
      QceVarIn<V> nx;
      if (VPF && vw0 < vwe) qce_var_fetch(nx, itab, vw0, lane, lam, a.s0);
      for (int vw = vw0; vw < vwe; ++vw) {
        QceVarIn<V> cur;
        if constexpr (VPF) {
          cur = nx;
          if (vw + 1 < vwe) qce_var_fetch(nx, itab, vw + 1, lane, lam, a.s0);
        } else {
          qce_var_fetch(cur, itab, vw, lane, lam, a.s0);
        }
        const uint4 iw = cur.iw;
        const int d = (int)(iw.z & 0xFFu);
        const int mode = (int)((iw.z >> 25) & 3u);
        const uint32_t bw = iw.w & 0xFFFFu;            // bitmap word
        if (mode <= VM_EXACT) {
          // 64-bit item: lane L takes bits y + L and y + 32 + L
          const uint32_t nv0 = (iw.z >> 8) & 0xFFu, nv1 = (iw.z >> 16) & 0xFFu;
          const bool mv0 = (uint32_t)lane < nv0, mv1 = (uint32_t)lane < nv1;
          const int l0 = mv0 ? lane : 0, l1 = mv1 ? 32 + lane : 0;
          const V li0 = cur.li0, li1 = cur.li1;
          V *col0 = reinterpret_cast<V *>(smem + iw.x) + l0;
          V *col1 = reinterpret_cast<V *>(smem + iw.x) + l1;
          V t0, t1;
          if (mode == VM_PAIR) {
            // dual-diagonal parity column: slots in check order for every
            // bit (u = 0 twice, or u = 0, 1 for the last column, whose wrap
            // entry of bit 359 is absent and holds -0.0)
            const V a0 = col0[0], b0 = col0[EZ], a1 = col1[0], b1 = col1[EZ];
            V s0 = TORCH ? li0 : V(0), s1 = TORCH ? li1 : V(0);
            s0 = add_rn(add_rn(s0, a0), b0);
            s1 = add_rn(add_rn(s1, a1), b1);
            t0 = TORCH ? add_rn(s0, V(0)) : add_rn(li0, s0);   // no -0.0 (see
            t1 = TORCH ? add_rn(s1, V(0)) : add_rn(li1, s1);   // qce_var_exact)
            const bool absent = ((iw.z >> 24) & 1u) && lane == ABSENT_LANE;
            if (mv0) {
              col0[0] = sub_rn(t0, a0);
              col0[EZ] = sub_rn(t0, b0);
            }
            if (mv1) {
              col1[0] = sub_rn(t1, a1);
              col1[EZ] = absent ? V(-0.0) : sub_rn(t1, b1);
            }
          } else {
            const int r0s = cur.s00, r1s = cur.s01;
            if (d == 3) {
              t0 = qce_var_exact<V, TORCH, 3>(col0, r0s, li0, mv0);
              t1 = qce_var_exact<V, TORCH, 3>(col1, r1s, li1, mv1);
            } else if (d == 4) {
              t0 = qce_var_exact<V, TORCH, 4>(col0, r0s, li0, mv0);
              t1 = qce_var_exact<V, TORCH, 4>(col1, r1s, li1, mv1);
            } else if (d == 2) {
              t0 = qce_var_exact<V, TORCH, 2>(col0, r0s, li0, mv0);
              t1 = qce_var_exact<V, TORCH, 2>(col1, r1s, li1, mv1);
            } else {
              t0 = qce_var_exact<V, TORCH, 1>(col0, r0s, li0, mv0);
              t1 = qce_var_exact<V, TORCH, 1>(col1, r1s, li1, mv1);
            }
          }
          const uint32_t h0 = __ballot_sync(0xffffffffu, mv0 && t0 < V(0));
          const uint32_t h1 = __ballot_sync(0xffffffffu, mv1 && t1 < V(0));
          if (lane < CL) {
            dsmem_st_u32(bm_peer + bw * 4u, h0);
            if (nv1) dsmem_st_u32(bm_peer + (bw + 1) * 4u, h1);
          }
        } else {
          // 64-bit item of any degree, one zone or both: lane L takes bits
          // y + L and y + 32 + L (lanes past 359 read bit y)
          const uint32_t nv0 = (iw.z >> 8) & 0xFFu, nv1 = (iw.z >> 16) & 0xFFu;
          const bool mv0 = (uint32_t)lane < nv0, mv1 = (uint32_t)lane < nv1;
          const int x0 = (int)iw.y + (mv0 ? lane : 0);
          const int x1 = (int)iw.y + (mv1 ? 32 + lane : 0);
          const V li0 = cur.li0, li1 = cur.li1;
          V *c0 = reinterpret_cast<V *>(smem + iw.x) + (x0 - (int)iw.y);
          V *c1 = reinterpret_cast<V *>(smem + iw.x) + (x1 - (int)iw.y);
          const int s00 = cur.s00, s01 = cur.s01;
          int dA = d, s0b0 = 0, s0b1 = 0;
          if (TA && mode == VM_GEN2) {
            dA = (int)((iw.w >> 16) & 0xFFu);
            s0b0 = __ldg(a.s0b + x0);
            s0b1 = __ldg(a.s0b + x1);
          }
          V t0, t1;
          qce_var_generic2<V, TORCH>(c0, c1, d, dA, s00, s01, s0b0, s0b1, li0, li1,
                                     mv0, mv1, t0, t1);
          // the absent wrap entry (bit 359 = lane 7 of the column's last
          // item's last sub-chunk) stays -0.0
          if (((iw.z >> 24) & 1u) && lane == ABSENT_LANE)
            (nv1 ? c1 : c0)[(int)(iw.w >> 24) * EZ] = V(-0.0);
          const uint32_t h0 = __ballot_sync(0xffffffffu, mv0 && t0 < V(0));
          const uint32_t h1 = __ballot_sync(0xffffffffu, mv1 && t1 < V(0));
          if (lane < CL) {
            dsmem_st_u32(bm_peer + bw * 4u, h0);
            if (nv1) dsmem_st_u32(bm_peer + (bw + 1) * 4u, h1);
          }
        }
      }
      cluster_sync_all();
    }
  }
  cluster_sync_all();
}

typedef void (*QceFn)(const QceArgs);

// NS <= 17 keeps a check's slot addresses and values in the 64 registers of
// the 1024-thread build; larger NS run 512 threads (128 registers) only.
template <int NS, bool TA>
static QceFn qce_pick(int semantics, bool big, bool f64) {
  if (f64)       // float64 slots and values: 512 threads (128 registers)
    return semantics ? ldpc_qce_kernel<double, true, NS, 512, TA>
                     : ldpc_qce_kernel<double, false, NS, 512, TA>;
  if constexpr (NS <= 17) {
    if (big)
      return semantics ? ldpc_qce_kernel<float, true, NS, 1024, TA>
                       : ldpc_qce_kernel<float, false, NS, 1024, TA>;
  }
  return semantics ? ldpc_qce_kernel<float, true, NS, 512, TA>
                   : ldpc_qce_kernel<float, false, NS, 512, TA>;
}

// ta: the plan has identity rows (a Type A code); its kernels carry the
// Type A paths and take 4, 6 or 8 slots (qce_ns_a of the identity rows).
// f64: the float64 build (the plan's slots hold doubles).
static QceFn qce_fn(int semantics, int dr, int threads, bool ta, bool f64 = false) {
  const bool big = threads > 512 && !f64;
  if (ta) {
    switch (qce_ns_a(dr)) {
      case 4: return qce_pick<4, true>(semantics, big, f64);
      case 6: return qce_pick<6, true>(semantics, big, f64);
      case 8: return qce_pick<8, true>(semantics, big, f64);
      default: return nullptr;
    }
  }
  switch (qce_ns(dr)) {
    case 8: return qce_pick<8, false>(semantics, big, f64);
    case 10: return qce_pick<10, false>(semantics, big, f64);
    case 11: return qce_pick<11, false>(semantics, big, f64);
    case 14: return qce_pick<14, false>(semantics, big, f64);
    case 17: return qce_pick<17, false>(semantics, big, f64);
    case 22: return qce_pick<22, false>(semantics, big, f64);
    case 34: return qce_pick<34, false>(semantics, big, f64);
    case 56: return f64 ? nullptr : qce_pick<56, false>(semantics, big, false);
    default: return nullptr;
  }
}

// default CTA size: 1024 threads while a check's slot addresses and values
// fit the 64-register budget (NS <= 17), else 512
static int qce_default_threads(int dr) { return qce_ns(dr) <= 17 ? 1024 : 512; }

static std::mutex g_qce_mu;
static std::unordered_map<uint64_t, int> g_qce_occ;
static std::unordered_map<uint64_t, int> g_qce_attr;

static int32_t qce_prepare(QceFn fn, int dev) {
  const uint64_t key = (uint64_t)(uintptr_t)fn ^ ((uint64_t)dev << 56);
  {
    std::lock_guard<std::mutex> g(g_qce_mu);
    if (g_qce_attr.count(key)) return 0;
  }
  int smax = 0;
  ATSC3_CUDA(cudaDeviceGetAttribute(&smax, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  ATSC3_CUDA(cudaFuncSetAttribute((const void *)fn,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  ATSC3_CUDA(cudaFuncSetAttribute(
      (const void *)fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  std::lock_guard<std::mutex> g(g_qce_mu);
  g_qce_attr[key] = 1;
  return 0;
}

static int32_t qce_max_clusters(QceFn fn, int cl, int smem, int threads, int dev,
                                int *out) {
  const uint64_t key = ((uint64_t)(uintptr_t)fn * 1315423911ull) ^
                       ((uint64_t)cl << 1) ^ ((uint64_t)smem << 8) ^
                       ((uint64_t)threads << 30) ^ ((uint64_t)dev << 44);
  {
    std::lock_guard<std::mutex> g(g_qce_mu);
    auto it = g_qce_occ.find(key);
    if (it != g_qce_occ.end()) {
      *out = it->second;
      return 0;
    }
  }
  int32_t rc = qce_prepare(fn, dev);
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
  std::lock_guard<std::mutex> g(g_qce_mu);
  g_qce_occ[key] = n;
  *out = n;
  return 0;
}

}  // namespace atsc3

struct atsc3_ldpc_qce_plan {
  atsc3::QcePlan p;
};

extern "C" {

static int32_t qce_plan_create_vb(int32_t n, int32_t kldpc, int32_t qa, int32_t qb,
                                  const int32_t *rowptr, const int32_t *addr,
                                  int32_t cluster, int vb, atsc3_ldpc_qce_plan **out) {
  using namespace atsc3;
  ATSC3_ARG(out && rowptr && addr, "null argument");
  *out = nullptr;
  int dev = 0;
  ATSC3_CUDA(cudaGetDevice(&dev));
  int smax = 0;
  ATSC3_CUDA(cudaDeviceGetAttribute(&smax, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  auto *h = new atsc3_ldpc_qce_plan();
  QceTables t;
  int rc = -4;
  if (cluster == 0) {
    // smallest cluster whose per-CTA shared memory fits; a structural
    // rejection (-3, -4 from the build) ends the search with its message
    bool fits = false;
    for (int cl = 1; cl <= EMAXCL; ++cl) {
      rc = qce_build(n, kldpc, qa, qb, rowptr, addr, cl, &h->p, &t, vb);
      if (rc) break;
      if (h->p.smem <= smax) {
        fits = true;
        break;
      }
    }
    if (rc == 0 && !fits) {
      set_error("unsupported: no cluster size fits");
      rc = -4;
    }
    // float64: every size from there up to 16 keeps about as many clusters
    // resident on a 64800-bit code (7 on B200), so the larger ones occupy
    // more SMs and decode faster (64800 6/15: 9.5 ms per frame at 11 CTAs,
    // 8.1 at 16).  Take the size that occupies the most SMs (resident
    // clusters x CTAs), the smaller one on a tie.
    if (rc == 0 && vb == 8) {
      const int cl0 = h->p.cluster;
      int best = cl0, best_sms = -1;
      for (int cl = cl0; cl <= EMAXCL; ++cl) {
        QcePlan pp;
        QceTables tt;
        if (qce_build(n, kldpc, qa, qb, rowptr, addr, cl, &pp, &tt, vb) || pp.smem > smax)
          continue;
        QceFn fn = qce_fn(1, pp.dr_light, 512, pp.qb > 0, true);
        int ncl = 0;
        if (!fn || qce_max_clusters(fn, cl, pp.smem, 512, dev, &ncl)) continue;
        if (ncl * cl > best_sms) {
          best_sms = ncl * cl;
          best = cl;
        }
      }
      if (best != cl0) {
        t = QceTables();
        rc = qce_build(n, kldpc, qa, qb, rowptr, addr, best, &h->p, &t, vb);
      }
    }
  } else {
    rc = qce_build(n, kldpc, qa, qb, rowptr, addr, cluster, &h->p, &t, vb);
    if (rc == 0 && h->p.smem > smax) {
      set_error("unsupported: per-CTA shared memory above the device limit");
      rc = -4;
    }
  }
  if (rc) {
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
  if (e == cudaSuccess) e = up((void **)&h->p.d_ccols, t.ccols.data(), t.ccols.size() * 4);
  if (e == cudaSuccess) e = up((void **)&h->p.d_itab, t.itab.data(), t.itab.size() * 16);
  if (e == cudaSuccess) e = up((void **)&h->p.d_wbin, t.wbin.data(), t.wbin.size() * 4);
  if (e == cudaSuccess) e = up((void **)&h->p.d_s0, t.s0.data(), t.s0.size());
  if (e == cudaSuccess) e = up((void **)&h->p.d_s0b, t.s0b.data(), t.s0b.size());
  if (e == cudaSuccess)
    e = up((void **)&h->p.d_hitems, t.hitems.data(), t.hitems.size() * sizeof(int16_t));
  if (e != cudaSuccess) {
    atsc3_ldpc_qce_plan_destroy(h);
    return cuda_fail(e, "qce plan upload");
  }
  *out = h;
  return 0;
}

int32_t atsc3_ldpc_qce_plan_create2(int32_t n, int32_t kldpc, int32_t qa,
                                    int32_t qb, const int32_t *rowptr,
                                    const int32_t *addr, int32_t cluster,
                                    atsc3_ldpc_qce_plan **out) {
  return qce_plan_create_vb(n, kldpc, qa, qb, rowptr, addr, cluster, 4, out);
}

int32_t atsc3_ldpc_qce_plan_create_f64(int32_t n, int32_t kldpc, int32_t qa,
                                       int32_t qb, const int32_t *rowptr,
                                       const int32_t *addr, int32_t cluster,
                                       atsc3_ldpc_qce_plan **out) {
  return qce_plan_create_vb(n, kldpc, qa, qb, rowptr, addr, cluster, 8, out);
}

int32_t atsc3_ldpc_qce_plan_create(int32_t n, int32_t kldpc, int32_t qldpc,
                                   const int32_t *rowptr, const int32_t *addr,
                                   int32_t cluster, atsc3_ldpc_qce_plan **out) {
  return atsc3_ldpc_qce_plan_create2(n, kldpc, qldpc, 0, rowptr, addr, cluster, out);
}

void atsc3_ldpc_qce_plan_destroy(atsc3_ldpc_qce_plan *h) {
  if (!h) return;
  cudaFree(h->p.d_rdesc);
  cudaFree(h->p.d_rptr);
  cudaFree(h->p.d_cdesc);
  cudaFree(h->p.d_ccols);
  cudaFree(h->p.d_itab);
  cudaFree(h->p.d_wbin);
  cudaFree(h->p.d_s0);
  cudaFree(h->p.d_s0b);
  cudaFree(h->p.d_hitems);
  delete h;
}

int32_t atsc3_ldpc_qce_plan_info(const atsc3_ldpc_qce_plan *h, int64_t *info) {
  ATSC3_ARG(h && info, "null argument");
  info[0] = h->p.n;
  info[1] = h->p.K;
  info[2] = h->p.Q;
  info[3] = h->p.cluster;
  info[4] = h->p.smem;
  info[5] = h->p.dr_max;
  info[6] = h->p.dc_max;
  info[7] = h->p.table_bytes;
  info[8] = h->p.max_slots;
  info[9] = h->p.cb[1] - h->p.cb[0];   // columns of CTA 0
  return 0;
}

int32_t atsc3_ldpc_qce_tables_host2(int32_t n, int32_t kldpc, int32_t qa,
                                    int32_t qb, const int32_t *rowptr,
                                    const int32_t *addr, int32_t cluster,
                                    int32_t *meta, int32_t *rdesc,
                                    int32_t *rptr, int32_t *cdesc,
                                    int32_t *ccols, uint8_t *s0,
                                    uint8_t *s0b, int32_t *itab,
                                    int32_t *hitems) {
  using namespace atsc3;
  ATSC3_ARG(meta && rowptr && addr, "null argument");
  QcePlan p;
  QceTables t;
  int rc = qce_build(n, kldpc, qa, qb, rowptr, addr, cluster, &p, &t);
  if (rc) return rc;
  meta[0] = (int32_t)t.rdesc.size();
  meta[1] = p.nb;
  meta[2] = p.smem;
  meta[3] = p.part_off;
  meta[4] = p.dr_max;
  meta[5] = p.dc_max;
  meta[6] = p.max_slots;
  meta[7] = p.buf_off;
  for (int c = 0; c <= EMAXCL; ++c) {
    meta[8 + c] = p.rb[c];
    meta[25 + c] = p.cb[c];
  }
  for (int c = 0; c <= EMAXCL; ++c) meta[42 + c] = p.ci[c];
  meta[59] = p.heavy;
  meta[60] = p.dr_light;
  meta[61] = (int32_t)t.itab.size();
  for (int c = 0; c <= EMAXCL; ++c) meta[62 + c] = p.hoff[c];
  meta[79] = p.nhrows;
  meta[80] = p.vbin_lo;
  meta[81] = p.vbin_hi;
  meta[82] = QBINS;
  if (rdesc) std::memcpy(rdesc, t.rdesc.data(), t.rdesc.size() * 16);
  if (rptr) std::memcpy(rptr, t.rptr.data(), t.rptr.size() * 4);
  if (cdesc) std::memcpy(cdesc, t.cdesc.data(), t.cdesc.size() * 16);
  if (ccols) std::memcpy(ccols, t.ccols.data(), t.ccols.size() * 4);
  if (s0) std::memcpy(s0, t.s0.data(), t.s0.size());
  if (s0b) std::memcpy(s0b, t.s0b.data(), t.s0b.size());
  if (itab) std::memcpy(itab, t.itab.data(), t.itab.size() * 16);
  if (hitems)
    for (size_t i = 0; i < t.hitems.size(); ++i) hitems[i] = t.hitems[i];
  return 0;
}

int32_t atsc3_ldpc_qce_bins_host(int32_t n, int32_t kldpc, int32_t qa, int32_t qb,
                                 const int32_t *rowptr, const int32_t *addr,
                                 int32_t cluster, int32_t *wbin) {
  using namespace atsc3;
  ATSC3_ARG(rowptr && addr && wbin, "null argument");
  QcePlan p;
  QceTables t;
  int rc = qce_build(n, kldpc, qa, qb, rowptr, addr, cluster, &p, &t);
  if (rc) return rc;
  std::memcpy(wbin, t.wbin.data(), t.wbin.size() * 4);
  return 0;
}

int32_t atsc3_ldpc_qce_tables_host(int32_t n, int32_t kldpc, int32_t qldpc,
                                   const int32_t *rowptr, const int32_t *addr,
                                   int32_t cluster, int32_t *meta,
                                   int32_t *rdesc, int32_t *rptr,
                                   int32_t *cdesc, int32_t *ccols,
                                   uint8_t *s0) {
  ATSC3_ARG(meta != nullptr, "null argument");
  int32_t m[96];
  const int32_t rc = atsc3_ldpc_qce_tables_host2(n, kldpc, qldpc, 0, rowptr, addr, cluster,
                                                 m, rdesc, rptr, cdesc, ccols, s0,
                                                 nullptr, nullptr, nullptr);
  if (rc == 0 && meta) std::memcpy(meta, m, 42 * sizeof(int32_t));
  return rc;
}

// Recognise an A/322 code (360-bit circulants; Type B: accumulator parity;
// Type A: accumulator rows plus identity rows) in CSR tables laid out as
// lab/m3_ldpc.py:459-482 builds them, and recover its address table.  The
// tables are accepted only if they are exactly that code's parity-check
// matrix in the reference's edge order, so the decoders built from the
// address table see the same edges in the same order:
//  * checks ascending, each check's columns strictly ascending;
//  * vedge = the stable argsort of cidx (each bit's edges by ascending check);
//  * qb identity block rows = the trailing degree-1 parity bits / 360 (0 for
//    Type B, whose last parity bit alone has degree 1); qa = nc/360 - qb;
//  * a table address x maps bit mm of its group to check (x + mm*qa) mod 360qa
//    (x < 360qa) or 360qa + (x - 360qa + mm*qb) mod 360qb
//    (lab/m3_ldpc.py:63-66); info bit 360g + mm is on the checks of bit 360g
//    mapped that way;
//  * accumulator parity bit K + 360j + k is on checks c = j + qa*k and c + 1
//    (c + 1 < 360qa) and, for Type A, on the identity-row checks of bit
//    K + 360j mapped as above (A/322 step vii); identity parity bit
//    K + 360qa + 360j + k on check 360qa + j + qb*k.
// Output: kq = {K, qa, qb}; rowptr (K/360 + 1 rows, + qa for Type A) and
// addr (each row's addresses, ascending), sized by the caller for n/360 + 1
// and nedges entries.  Returns 0, or -4 (not such a structure; nothing else
// is wrong with the tables).
int32_t atsc3_ldpc_qc_detect2(const int32_t *cptr, const int32_t *cidx,
                              const int32_t *vptr, const int32_t *vedge,
                              int32_t n, int32_t nc, int32_t nedges,
                              int32_t *kq, int32_t *rowptr, int32_t *addr) {
  using namespace atsc3;
  ATSC3_ARG(cptr && cidx && vptr && vedge && kq && rowptr && addr, "null argument");
  ATSC3_ARG(n > 0 && nc > 0 && nedges >= 0, "bad size");
  auto no = [](const char *why) {
    set_error(why);
    return (int32_t)-4;
  };
  if (n % EZ || nc % EZ || nc >= n) return no("not a 360-circulant code");
  const int K = n - nc, nbi = K / EZ;
  if (cptr[0] != 0 || cptr[nc] != nedges || vptr[0] != 0 || vptr[n] != nedges)
    return no("inconsistent CSR");
  std::vector<int32_t> chk((size_t)nedges);
  for (int c = 0; c < nc; ++c) {
    if (cptr[c + 1] < cptr[c]) return no("inconsistent CSR");
    for (int e = cptr[c]; e < cptr[c + 1]; ++e) {
      if (cidx[e] < 0 || cidx[e] >= n) return no("column out of range");
      if (e > cptr[c] && cidx[e] <= cidx[e - 1]) return no("columns not ascending");
      chk[e] = c;
    }
  }
  std::vector<int32_t> fill((size_t)n, 0);
  for (int v = 0; v < n; ++v)
    if (vptr[v + 1] < vptr[v]) return no("inconsistent CSR");
  for (int e = 0; e < nedges; ++e) {
    const int v = cidx[e];
    const int k = vptr[v] + fill[v]++;
    if (k >= vptr[v + 1] || vedge[k] != e) return no("vedge is not the stable argsort of cidx");
  }
  int tail = 0;                                  // trailing degree-1 parity bits
  while (tail < nc && vptr[n - tail] - vptr[n - tail - 1] == 1) ++tail;
  const int qb = (tail % EZ == 0 && tail < nc) ? tail / EZ : 0;
  const int qa = nc / EZ - qb, MA = qa * EZ, MB = qb * EZ;
  auto map = [&](int64_t x, int64_t mm) -> int64_t {
    return x < MA ? (x + mm * qa) % MA : MA + (x - MA + mm * qb) % MB;
  };
  auto col_is = [&](int v, std::vector<int64_t> &want) {
    std::sort(want.begin(), want.end());
    if ((int)want.size() != vptr[v + 1] - vptr[v]) return false;
    for (size_t i = 0; i < want.size(); ++i)
      if (chk[vedge[vptr[v] + (int)i]] != want[i]) return false;
    return true;
  };
  std::vector<int64_t> want;
  // table rows: info groups, then (Type A) the accumulator parity groups'
  // identity-row checks
  rowptr[0] = 0;
  const int nrows = nbi + (qb > 0 ? qa : 0);
  for (int g = 0; g < nrows; ++g) {
    const int v0 = g < nbi ? g * EZ : K + (g - nbi) * EZ;
    int w = rowptr[g];
    for (int i = vptr[v0]; i < vptr[v0 + 1]; ++i) {
      const int c = chk[vedge[i]];
      if (g >= nbi && c < MA) continue;          // the dual diagonal
      addr[w++] = c;
    }
    rowptr[g + 1] = w;
  }
  for (int g = 0; g < nbi; ++g)
    for (int mm = 0; mm < EZ; ++mm) {
      want.clear();
      for (int i = rowptr[g]; i < rowptr[g + 1]; ++i) want.push_back(map(addr[i], mm));
      if (!col_is(g * EZ + mm, want)) return no("info column not a circulant shift");
    }
  for (int j = 0; j < qa; ++j)
    for (int k = 0; k < EZ; ++k) {
      const int c = j + qa * k;
      want.clear();
      want.push_back(c);
      if (c + 1 < MA) want.push_back(c + 1);
      if (qb > 0)
        for (int i = rowptr[nbi + j]; i < rowptr[nbi + j + 1]; ++i)
          want.push_back(map(addr[i], k));
      if (!col_is(K + EZ * j + k, want)) return no("parity part is not the accumulator");
    }
  for (int j = 0; j < qb; ++j)
    for (int k = 0; k < EZ; ++k) {
      want.clear();
      want.push_back(MA + j + (int64_t)qb * k);
      if (!col_is(K + MA + EZ * j + k, want)) return no("parity part is not the identity");
    }
  kq[0] = K;
  kq[1] = qa;
  kq[2] = qb;
  return 0;
}

// Type B only (kq = {K, Q}); a Type A code returns -4.
int32_t atsc3_ldpc_qc_detect(const int32_t *cptr, const int32_t *cidx,
                             const int32_t *vptr, const int32_t *vedge,
                             int32_t n, int32_t nc, int32_t nedges,
                             int32_t *kq, int32_t *rowptr, int32_t *addr) {
  using namespace atsc3;
  ATSC3_ARG(kq != nullptr, "null argument");
  int32_t k3[3];
  const int32_t rc = atsc3_ldpc_qc_detect2(cptr, cidx, vptr, vedge, n, nc, nedges,
                                           k3, rowptr, addr);
  if (rc) return rc;
  if (k3[2] != 0) {
    set_error("a Type A code (use atsc3_ldpc_qc_detect2)");
    return -4;
  }
  kq[0] = k3[0];
  kq[1] = k3[1];
  return 0;
}

int32_t atsc3_ldpc_qce_config(const atsc3_ldpc_qce_plan *h, int32_t threads,
                              int32_t semantics, int32_t *out) {
  using namespace atsc3;
  ATSC3_ARG(h && out, "null argument");
  if (threads <= 0) threads = qce_default_threads(h->p.dr_light);
  if (qce_ns(h->p.dr_light) > 17 || h->p.vb == 8) threads = std::min(threads, 512);
  QceFn fn = qce_fn(semantics, h->p.dr_light, threads, h->p.qb > 0, h->p.vb == 8);
  ATSC3_ARG(fn != nullptr, "no kernel for this degree");
  int ncl = 0;
  int32_t rc = qce_max_clusters(fn, h->p.cluster, h->p.smem, threads, h->p.device, &ncl);
  if (rc) return rc;
  out[0] = ncl;
  out[1] = h->p.cluster;
  out[2] = h->p.smem;
  out[3] = threads;
  return 0;
}

static int32_t qce_decode_impl(
    const atsc3_ldpc_qce_plan *h, const void *llr, int64_t ld_llr,
    int32_t nblk, int32_t iters, double alpha, int32_t semantics,
    const float *walpha, const float *wbeta, int32_t wT, int32_t wnb,
    const int8_t *dbucket, uint8_t *bits, int64_t ld_bits, uint8_t *hard,
    int64_t ld_hard, uint8_t *conv, int32_t *its, int32_t *bad,
    int32_t threads, void *stream, bool f64, int wrow = 0) {
  using namespace atsc3;
  ATSC3_ARG(h != nullptr, "null plan");
  const QcePlan &p = h->p;
  ATSC3_ARG(p.vb == (f64 ? 8 : 4),
            f64 ? "not a float64 plan (atsc3_ldpc_qce_plan_create_f64)"
                : "a float64 plan needs atsc3_ldpc_qce_decode_f64");
  ATSC3_ARG(!(f64 && walpha), "learned weights are float32 only");
  ATSC3_ARG(nblk >= 0 && iters >= 0, "negative size");
  ATSC3_ARG(semantics == 0 || semantics == 1, "semantics must be 0 or 1");
  ATSC3_ARG(!(semantics == 1 && iters == 0), "semantics 1 needs iters >= 1");
  ATSC3_ARG(ld_llr >= p.n, "ld_llr < n");
  ATSC3_ARG(bits == nullptr || ld_bits >= p.n, "ld_bits < n");
  ATSC3_ARG(hard == nullptr || ld_hard >= (p.n + 7) / 8, "ld_hard < ceil(n/8)");
  if (nblk == 0) return 0;
  ATSC3_ARG(conv && its && bad, "null status output");
  ATSC3_ARG(llr != nullptr, "null llr");
  if (threads <= 0) threads = qce_default_threads(p.dr_light);
  ATSC3_ARG(threads == 512 || threads == 1024, "threads must be 512 or 1024");
  if (qce_ns(p.dr_light) > 17 || f64) threads = 512;   // only the 512-thread build
  QceFn fn = qce_fn(semantics, p.dr_light, threads, p.qb > 0, f64);
  if (!fn) {
    set_error("unsupported: block-row degree too high");
    return -4;
  }
  int ncl = 0;
  int32_t rc = qce_max_clusters(fn, p.cluster, p.smem, threads, p.device, &ncl);
  if (rc) return rc;
  if (ncl <= 0) {
    set_error("unsupported: cluster configuration cannot be resident");
    return -4;
  }
  ncl = std::min(ncl, nblk);
  QceArgs a;
  std::memset(&a, 0, sizeof(a));
  a.llr = llr;
  a.ld_llr = ld_llr;
  a.nblk = nblk;
  a.n = p.n;
  a.iters = iters;
  a.alpha = (float)alpha;
  a.alpha_d = alpha;
  a.part_off = p.part_off;
  a.rt_off = p.rt_off;
  a.ri_off = p.ri_off;
  a.ct_off = p.ct_off;
  a.ht_off = p.ht_off;
  for (int c = 0; c <= EMAXCL; ++c) {
    a.ci[c] = p.ci[c];
    a.cb[c] = p.cb[c];
    a.hoff[c] = p.hoff[c];
  }
  a.nhrows = p.nhrows;
  a.hsplit = p.hsplit;
  a.hpb_off = p.hpb_off;
  a.hitems = p.d_hitems;
  a.ccols = p.d_ccols;
  a.itab = p.d_itab;
  a.wbin = p.d_wbin;
  for (int c = 0; c <= EMAXCL; ++c) a.ib[c] = p.ib[c];
  a.rdesc = p.d_rdesc;
  a.rptr = p.d_rptr;
  a.cdesc = p.d_cdesc;
  a.s0 = p.d_s0;
  a.s0b = p.d_s0b;
  if (walpha) {
    ATSC3_ARG(wbeta && dbucket && wT > 0 && wnb > 0,
              "weights need wbeta, dbucket, wT > 0, wnb > 0");
    a.walpha = walpha;
    a.wbeta = wbeta;
    a.dbucket = dbucket;
    a.wT = wT;
    a.wnb = wnb;
    a.wrow = wrow;
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

int32_t atsc3_ldpc_qce_decode_weighted(
    const atsc3_ldpc_qce_plan *h, const float *llr, int64_t ld_llr,
    int32_t nblk, int32_t iters, float alpha, int32_t semantics,
    const float *walpha, const float *wbeta, int32_t wT, int32_t wnb,
    const int8_t *dbucket, uint8_t *bits, int64_t ld_bits, uint8_t *hard,
    int64_t ld_hard, uint8_t *conv, int32_t *its, int32_t *bad,
    int32_t threads, void *stream) {
  return qce_decode_impl(h, llr, ld_llr, nblk, iters, alpha, semantics, walpha, wbeta,
                         wT, wnb, dbucket, bits, ld_bits, hard, ld_hard, conv, its, bad,
                         threads, stream, false);
}

int32_t atsc3_ldpc_qce_decode_weighted_rows(
    const atsc3_ldpc_qce_plan *h, const float *llr, int64_t ld_llr,
    int32_t nblk, int32_t iters, float alpha, int32_t semantics,
    const float *walpha, const float *wbeta, int32_t wT, int32_t wnb,
    const int8_t *rbucket, uint8_t *bits, int64_t ld_bits, uint8_t *hard,
    int64_t ld_hard, uint8_t *conv, int32_t *its, int32_t *bad,
    int32_t threads, void *stream) {
  using namespace atsc3;
  ATSC3_ARG(walpha && rbucket, "row weights need walpha and rbucket");
  ATSC3_ARG(h && h->p.qa + h->p.qb <= 256, "null plan or more than 256 block rows");
  return qce_decode_impl(h, llr, ld_llr, nblk, iters, alpha, semantics, walpha, wbeta,
                         wT, wnb, rbucket, bits, ld_bits, hard, ld_hard, conv, its, bad,
                         threads, stream, false, 1);
}

int32_t atsc3_ldpc_qce_decode_f64(const atsc3_ldpc_qce_plan *h, const double *llr,
                                  int64_t ld_llr, int32_t nblk, int32_t iters,
                                  double alpha, int32_t semantics, uint8_t *bits,
                                  int64_t ld_bits, uint8_t *hard, int64_t ld_hard,
                                  uint8_t *conv, int32_t *its, int32_t *bad,
                                  int32_t threads, void *stream) {
  return qce_decode_impl(h, llr, ld_llr, nblk, iters, alpha, semantics, nullptr, nullptr,
                         0, 0, nullptr, bits, ld_bits, hard, ld_hard, conv, its, bad,
                         threads, stream, true);
}

int32_t atsc3_ldpc_qce_decode(const atsc3_ldpc_qce_plan *h, const float *llr,
                              int64_t ld_llr, int32_t nblk, int32_t iters,
                              float alpha, int32_t semantics, uint8_t *bits,
                              int64_t ld_bits, uint8_t *hard, int64_t ld_hard,
                              uint8_t *conv, int32_t *its, int32_t *bad,
                              int32_t threads, void *stream) {
  return atsc3_ldpc_qce_decode_weighted(h, llr, ld_llr, nblk, iters, alpha,
                                        semantics, nullptr, nullptr, 0, 0,
                                        nullptr, bits, ld_bits, hard, ld_hard,
                                        conv, its, bad, threads, stream);
}

}  // extern "C"

namespace atsc3 {
// Device the plan's tables were built on (internal; used by the
// allocation-free entry point to refuse a plan from another GPU).
int qce_plan_device(const atsc3_ldpc_qce_plan *h) { return h->p.device; }
}  // namespace atsc3
