// ldpc_layered.cu -- layered normalised min-sum for the quasi-cyclic A/322
// Type B codes (sm_100a).
//
// Schedule: the Q block rows of the code are the layers (360 checks each; a
// layer touches every bit at most once).  Per layer, every check k runs
//     v_e = P[var_e] - m_e                        (old message from its record)
//     min1 / min2 / first / parity over |v|, v<0  (lab/ldpc_kernel.c:116-134 rules)
//     m_e' = +-(e == first ? min2 : min1) * alpha, sign parity ^ (v_e < 0)
//     P[var_e] = v_e + m_e'
// with the posterior P updated in place.  The syndrome of sign(P) is taken
// before the first iteration (retire with its = 0) and after each full
// iteration.  This is not the reference's flooding schedule (which has no
// layered counterpart); oracle/ldpc_oracle.c:oracle_layered_f32 is its
// bit-exact CPU statement.
//
// Layout: one CTA per codeword (persistent CTAs stride over codewords).  P
// (n floats) and the per-check records (16 B: min1*alpha, min2*alpha, sign
// bits, first position) live in global memory -- per-CTA scratch that stays
// L2-resident.  A layer's column blocks (360 posteriors = 1440 B each) are
// staged into shared memory with bulk asynchronous copies
// (cp.async.bulk ... mbarrier::complete_tx, one copy per circulant, no
// multicast), updated there by the 360 check threads, and written back with
// coalesced stores.  A packed hard-decision bitmap of the whole codeword is
// kept in shared memory and refreshed at each write-back, so the per-
// iteration syndrome is a shared-memory gather.  Waits on the mbarrier are
// bounded: on timeout the kernel waits once more for its copies, records an
// error (1, or 2 when the second wait ran out too) and stops.

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "../../include/atsc3_fec.h"
#include "common.cuh"

namespace atsc3 {

constexpr int LZ = 360;
constexpr int LTHREADS = 384;
constexpr uint32_t LSPIN = 1u << 22;      // mbarrier polls before giving up

struct LayPlan {
  int n = 0, K = 0, Q = 0, nb = 0, dr_max = 0, device = 0;
  int4 *d_slots = nullptr;     // per row slot {column, shift, wrap, 0}
  int32_t *d_rptr = nullptr;   // (Q+1)
  int64_t table_bytes = 0;
};

struct LayArgs {
  const float *llr;
  int64_t ld_llr;
  int nblk, n, Q, iters;
  float alpha;
  const int4 *slots;
  const int32_t *rptr;
  float *P;          // scratch (gridDim.x, n)
  uint4 *rec;        // scratch (gridDim.x, Q*360)
  uint8_t *bits;
  int64_t ld_bits;
  uint8_t *hard;
  int64_t ld_hard;
  uint8_t *conv;
  int32_t *its;
  int32_t *bad;
  int32_t *err;
  int fail_layer;    // test hook: take the timeout path at this layer, or -1
};

__device__ __forceinline__ void mbar_init(uint32_t a, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(a), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t a, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
               :: "r"(a), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t a, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok) : "r"(a), "r"(parity) : "memory");
  return ok != 0;
}

// bounded wait: true when the phase completed
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t a, uint32_t parity) {
  for (uint32_t i = 0; i < LSPIN; ++i)
    if (mbar_try_wait(a, parity)) return true;
  return false;
}

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src,
                                         uint32_t bytes, uint32_t mbar) {
  uint64_t g;
  asm("cvta.to.global.u64 %0, %1;" : "=l"(g) : "l"(src));
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
      "[%0], [%1], %2, [%3];"
      :: "r"(dst), "l"(g), "r"(bytes), "r"(mbar) : "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.global;\n\tfence.proxy.async.shared::cta;" ::: "memory");
}

// DR: unroll bound of slots per block row (>= every row degree)
template <int DR>
__global__ void __launch_bounds__(LTHREADS, 2) ldpc_layered_kernel(const LayArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  float *stage = reinterpret_cast<float *>(smem);               // DR * 360
  uint8_t *hb = smem + (size_t)DR * LZ * 4;                     // n/8 bytes
  uint64_t *mbar = reinterpret_cast<uint64_t *>(hb + ((a.n / 8 + 15) & ~15));
  __shared__ int s_bad, s_fail;
  const int tid = threadIdx.x;
  const int k = tid;                                            // check row
  const bool act = k < LZ;
  const int nb8 = a.n / 8;
  const int nc = a.Q * LZ;
  const uint32_t mb = smem_u32(mbar);
  const uint32_t st_sa = smem_u32(stage);
  float *P = a.P + (size_t)blockIdx.x * a.n;
  uint4 *R = a.rec + (size_t)blockIdx.x * nc;
  uint32_t phase = 0;

  if (tid == 0) {
    mbar_init(mb, 1);
    s_fail = 0;
  }
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  __syncthreads();

  for (int b = blockIdx.x; b < a.nblk; b += gridDim.x) {
    const float *lam = a.llr + (size_t)b * a.ld_llr;
    for (int i = tid; i < a.n; i += blockDim.x) P[i] = lam[i];
    for (int q = tid; q < nb8; q += blockDim.x) {
      uint32_t v = 0;
#pragma unroll
      for (int t = 0; t < 8; ++t) v |= (lam[8 * q + t] < 0.f ? 1u : 0u) << (7 - t);
      hb[q] = (uint8_t)v;
    }
    fence_proxy_async();
    __syncthreads();
    int it = 0;
    bool done = false;
    int badct = 0;
    for (;; ++it) {
      // ---- syndrome of the hard decisions (bitmap) ----------------------
      if (tid == 0) s_bad = 0;
      __syncthreads();
      int mine = 0;
      if (act) {
        for (int r = 0; r < a.Q; ++r) {
          const int s0 = __ldg(a.rptr + r), s1 = __ldg(a.rptr + r + 1);
          uint32_t par = 0;
          for (int s = s0; s < s1; ++s) {
            const int4 sl = __ldg(a.slots + s);
            if (sl.z && k == 0) continue;
            int o = k - sl.y;
            o += o < 0 ? LZ : 0;
            const int bit = sl.x * LZ + o;
            par ^= (hb[bit >> 3] >> (7 - (bit & 7))) & 1u;
          }
          mine += (int)par;
        }
      }
      mine = __reduce_add_sync(0xffffffffu, mine);
      if ((tid & 31) == 0 && mine) atomicAdd(&s_bad, mine);
      __syncthreads();
      badct = s_bad;
      if (badct == 0) { done = true; break; }
      if (it >= a.iters) break;
      // ---- one iteration: every layer in order --------------------------
      for (int r = 0; r < a.Q; ++r) {
        const int s0 = __ldg(a.rptr + r);
        const int d = __ldg(a.rptr + r + 1) - s0;
        if (tid == 0) {
          mbar_expect_tx(mb, (uint32_t)(d * LZ * 4));
          for (int j = 0; j < d; ++j) {
            const int4 sl = __ldg(a.slots + s0 + j);
            bulk_g2s(st_sa + (uint32_t)(j * LZ * 4), P + (size_t)sl.x * LZ,
                     (uint32_t)(LZ * 4), mb);
          }
        }
        uint4 ro = make_uint4(0u, 0u, 0u, 0u);
        if (act && it > 0) ro = R[(size_t)r * LZ + k];
        bool ok = mbar_wait_bounded(mb, phase);
        // test hook: behave as if this (completed) wait had run out, so the
        // error path runs with no copy in flight
        if (it * a.Q + r == a.fail_layer) ok = false;
        phase ^= 1u;
        if (__syncthreads_or(!ok)) {
          // A wait ran out.  Copies may still be landing in this CTA's
          // shared memory: wait for the same phase once more (bounded).
          // *err = 1: the copies then completed and the CTA returned with
          // nothing in flight; *err = 2: the second wait ran out as well,
          // so copies may still have been in flight when the CTA returned
          // (the launch's outputs are void and the context is suspect).
          const bool drained = mbar_wait_bounded(mb, phase ^ 1u);
          if (tid == 0) {
            s_fail = 1;
            atomicMax(a.err, drained ? 1 : 2);
          }
          return;
        }
        if (act) {
          const float Ao = __uint_as_float(ro.x), Bo = __uint_as_float(ro.y);
          const uint32_t Fo = ro.w & 0xFFu;
          const uint64_t So = (uint64_t)ro.z | ((uint64_t)(ro.w >> 8) << 32);
          float v[DR];
          int oo[DR];
          float min1 = __int_as_float(0x7f800000), min2 = min1;
          uint32_t first = 0, par = 0;
          uint64_t live = 0;
#pragma unroll
          for (int j = 0; j < DR; ++j) {
            v[j] = 0.f;
            oo[j] = 0;
            if (j < d) {
              const int4 sl = __ldg(a.slots + s0 + j);
              if (!(sl.z && k == 0)) {
                int o = k - sl.y;
                o += o < 0 ? LZ : 0;
                oo[j] = j * LZ + o;
                float mo = ((uint32_t)j == Fo) ? Bo : Ao;
                if ((So >> j) & 1ull) mo = -mo;
                const float vv = __fsub_rn(stage[oo[j]], mo);
                v[j] = vv;
                live |= 1ull << j;
                par ^= vv < 0.f ? 1u : 0u;
                const float mag = fabsf(vv);
                if (mag < min1) { min2 = min1; min1 = mag; first = (uint32_t)j; }
                else if (mag < min2) { min2 = mag; }
              }
            }
          }
          const float A = __fmul_rn(min1, a.alpha), B = __fmul_rn(min2, a.alpha);
          uint64_t sg = 0;
#pragma unroll
          for (int j = 0; j < DR; ++j) {
            if ((live >> j) & 1ull) {
              float m = ((uint32_t)j == first) ? B : A;
              if (par ^ (v[j] < 0.f ? 1u : 0u)) {
                m = -m;
                sg |= 1ull << j;
              }
              stage[oo[j]] = __fadd_rn(v[j], m);
            }
          }
          R[(size_t)r * LZ + k] = make_uint4(__float_as_uint(A), __float_as_uint(B),
                                             (uint32_t)sg,
                                             first | ((uint32_t)(sg >> 32) << 8));
        }
        __syncthreads();
        // ---- write back the layer's columns; refresh the bitmap ---------
        for (int j = 0; j < d; ++j) {
          const int c = __ldg(a.slots + s0 + j).x;
          for (int i = tid; i < LZ; i += blockDim.x) P[(size_t)c * LZ + i] = stage[j * LZ + i];
          if (tid < LZ / 8) {
            uint32_t vb = 0;
#pragma unroll
            for (int t = 0; t < 8; ++t)
              vb |= (stage[j * LZ + 8 * tid + t] < 0.f ? 1u : 0u) << (7 - t);
            hb[c * (LZ / 8) + tid] = (uint8_t)vb;
          }
        }
        fence_proxy_async();
        __syncthreads();
      }
    }
    // ---- retire ----------------------------------------------------------
    if (a.bits) {
      uint8_t *bo = a.bits + (size_t)b * a.ld_bits;
      for (int i = tid; i < a.n; i += blockDim.x) bo[i] = P[i] < 0.f ? 1 : 0;
    }
    if (a.hard) {
      uint8_t *ho = a.hard + (size_t)b * a.ld_hard;
      for (int q = tid; q < nb8; q += blockDim.x) ho[q] = hb[q];
    }
    if (tid == 0) {
      a.conv[b] = done ? 1 : 0;
      a.its[b] = it;
      a.bad[b] = done ? 0 : badct;
    }
    __syncthreads();
  }
}

typedef void (*LayFn)(const LayArgs);

static LayFn lay_fn(int dr) {
  if (dr <= 8) return ldpc_layered_kernel<8>;
  if (dr <= 12) return ldpc_layered_kernel<12>;
  if (dr <= 16) return ldpc_layered_kernel<16>;
  if (dr <= 24) return ldpc_layered_kernel<24>;
  if (dr <= 34) return ldpc_layered_kernel<34>;
  return nullptr;
}

static int lay_smem(int dr_bucket, int n) {
  return dr_bucket * LZ * 4 + ((n / 8 + 15) & ~15) + 16;
}

static int dr_bucket(int dr) {
  return dr <= 8 ? 8 : dr <= 12 ? 12 : dr <= 16 ? 16 : dr <= 24 ? 24 : 34;
}

}  // namespace atsc3

struct atsc3_ldpc_layered_plan {
  atsc3::LayPlan p;
};

namespace atsc3 {
static std::atomic<int> g_lay_fail_layer{-1};
}  // namespace atsc3

extern "C" {

int32_t atsc3_ldpc_layered_plan_create(int32_t n, int32_t kldpc, int32_t qldpc,
                                       const int32_t *rowptr,
                                       const int32_t *addr,
                                       atsc3_ldpc_layered_plan **out) {
  using namespace atsc3;
  ATSC3_ARG(out && rowptr && addr, "null argument");
  *out = nullptr;
  ATSC3_ARG(n % LZ == 0 && kldpc % LZ == 0 && qldpc > 0 &&
                n - kldpc == qldpc * LZ,
            "not a 360-circulant Type B code");
  ATSC3_ARG(n <= 65535 * 8, "codeword too long");
  const int nbi = kldpc / LZ;
  struct Sl { int col, u, wrap; };
  std::vector<std::vector<Sl>> rows(qldpc);
  for (int g = 0; g < nbi; ++g)
    for (int e = rowptr[g]; e < rowptr[g + 1]; ++e) {
      const int x = addr[e];
      ATSC3_ARG(x >= 0 && x < n - kldpc, "address outside the parity range");
      rows[x % qldpc].push_back(Sl{g, x / qldpc, 0});
    }
  std::vector<int4> slots;
  std::vector<int32_t> rptr(qldpc + 1, 0);
  int dr = 0;
  for (int r = 0; r < qldpc; ++r) {
    auto &R = rows[r];
    std::sort(R.begin(), R.end(), [](const Sl &a, const Sl &b) { return a.col < b.col; });
    for (size_t i = 1; i < R.size(); ++i)
      if (R[i].col == R[i - 1].col) {
        set_error("unsupported: two circulants share a block (not layerable)");
        return -4;
      }
    if (r >= 1) {
      R.push_back(Sl{nbi + r - 1, 0, 0});
      R.push_back(Sl{nbi + r, 0, 0});
    } else {
      R.push_back(Sl{nbi, 0, 0});
      R.push_back(Sl{nbi + qldpc - 1, 1, 1});
    }
    for (auto &s : R) slots.push_back(make_int4(s.col, s.u, s.wrap, 0));
    rptr[r + 1] = (int)slots.size();
    dr = std::max(dr, (int)R.size());
  }
  if (!lay_fn(dr)) {
    set_error("unsupported: block-row degree above 34");
    return -4;
  }
  int dev = 0;
  ATSC3_CUDA(cudaGetDevice(&dev));
  auto *h = new atsc3_ldpc_layered_plan();
  h->p.n = n;
  h->p.K = kldpc;
  h->p.Q = qldpc;
  h->p.nb = n / LZ;
  h->p.dr_max = dr;
  h->p.device = dev;
  cudaError_t e = cudaMalloc(&h->p.d_slots, slots.size() * 16);
  if (e == cudaSuccess) e = cudaMemcpy(h->p.d_slots, slots.data(), slots.size() * 16, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMalloc(&h->p.d_rptr, rptr.size() * 4);
  if (e == cudaSuccess) e = cudaMemcpy(h->p.d_rptr, rptr.data(), rptr.size() * 4, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(h->p.d_slots);
    cudaFree(h->p.d_rptr);
    delete h;
    return cuda_fail(e, "layered plan upload");
  }
  h->p.table_bytes = (int64_t)(slots.size() * 16 + rptr.size() * 4);
  *out = h;
  return 0;
}

void atsc3_ldpc_layered_plan_destroy(atsc3_ldpc_layered_plan *h) {
  if (!h) return;
  cudaFree(h->p.d_slots);
  cudaFree(h->p.d_rptr);
  delete h;
}

int32_t atsc3_ldpc_layered_workspace(const atsc3_ldpc_layered_plan *h,
                                     int32_t ctas, int64_t *bytes) {
  ATSC3_ARG(h && bytes && ctas > 0, "bad argument");
  *bytes = (int64_t)ctas * ((int64_t)h->p.n * 4 + (int64_t)h->p.Q * atsc3::LZ * 16) + 256;
  return 0;
}

int32_t atsc3_ldpc_layered_decode(const atsc3_ldpc_layered_plan *h,
                                  const float *llr, int64_t ld_llr,
                                  int32_t nblk, int32_t iters, float alpha,
                                  uint8_t *bits, int64_t ld_bits, uint8_t *hard,
                                  int64_t ld_hard, uint8_t *conv, int32_t *its,
                                  int32_t *bad, void *workspace, int32_t ctas,
                                  int32_t *err, void *stream) {
  using namespace atsc3;
  ATSC3_ARG(h != nullptr, "null plan");
  const LayPlan &p = h->p;
  ATSC3_ARG(nblk >= 0 && iters >= 0, "negative size");
  if (nblk == 0) return 0;
  ATSC3_ARG(llr && conv && its && bad && workspace && err, "null pointer");
  ATSC3_ARG(ctas > 0, "ctas must be > 0 (the workspace is sized for it)");
  ATSC3_ARG(ld_llr >= p.n, "ld_llr < n");
  ATSC3_ARG(((uintptr_t)workspace & 255) == 0, "workspace must be 256-byte aligned");
  ATSC3_ARG(bits == nullptr || ld_bits >= p.n, "ld_bits < n");
  ATSC3_ARG(hard == nullptr || ld_hard >= p.n / 8, "ld_hard < n/8");
  LayFn fn = lay_fn(p.dr_max);
  const int smem = lay_smem(dr_bucket(p.dr_max), p.n);
  ATSC3_CUDA(cudaFuncSetAttribute((const void *)fn,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  LayArgs a;
  std::memset(&a, 0, sizeof(a));
  a.llr = llr;
  a.ld_llr = ld_llr;
  a.nblk = nblk;
  a.n = p.n;
  a.Q = p.Q;
  a.iters = iters;
  a.alpha = alpha;
  a.slots = p.d_slots;
  a.rptr = p.d_rptr;
  a.P = reinterpret_cast<float *>(workspace);
  a.rec = reinterpret_cast<uint4 *>(reinterpret_cast<char *>(workspace) +
                                    (((size_t)ctas * p.n * 4 + 255) & ~(size_t)255));
  a.bits = bits;
  a.ld_bits = ld_bits;
  a.hard = hard;
  a.ld_hard = ld_hard;
  a.conv = conv;
  a.its = its;
  a.bad = bad;
  a.err = err;
  a.fail_layer = g_lay_fail_layer.exchange(-1);
  const int grid = std::min(ctas, nblk);
  fn<<<grid, LTHREADS, smem, (cudaStream_t)stream>>>(a);
  ATSC3_CUDA(cudaGetLastError());
  return 0;
}

int32_t atsc3_ldpc_layered_inject_timeout(int32_t layer) {
  ATSC3_ARG(layer >= -1, "layer must be >= -1");
  atsc3::g_lay_fail_layer.store(layer);
  return 0;
}

}  // extern "C"
