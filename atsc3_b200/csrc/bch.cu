// bch.cu -- BCH zero-syndrome check (A/322 6.1.2.1) and Baseband Packet
// descramble for sm_100a.
//
// The syndrome of the K_ldpc-bit BCH codeword m (MSB first, bit 0 = x^(K-1))
// is m(x) mod g(x), deg g = 192 (Ninner 64800) or 168 (16200).  It is linear
// in the bits, so it is the XOR over the set bits of the precomputed rows
// R[pos] = x^(K-1-pos) mod g(x) -- the same GF(2) matrix product
// lab/m9_accel.py:169-236 evaluates with popcounts.  Zero syndrome = BCH OK.
//
// One CTA per codeword; each thread folds the rows of the bits it owns into
// six 32-bit words, then a warp-shuffle and shared-memory XOR reduction.
// The descrambled payload (lab/m9_fast.py:942-949: hard bits XOR the
// scrambling sequence, packed MSB-first) is written by the same CTA.

#include <cuda_runtime.h>

#include "../../include/atsc3_fec.h"
#include "common.cuh"

namespace atsc3 {

__device__ __forceinline__ void fold_row(uint32_t (&acc)[6],
                                         const uint32_t *__restrict__ rtab,
                                         int pos) {
  const uint2 *r = reinterpret_cast<const uint2 *>(rtab + (size_t)pos * 6);
  const uint2 a = __ldg(r), b = __ldg(r + 1), c = __ldg(r + 2);
  acc[0] ^= a.x; acc[1] ^= a.y; acc[2] ^= b.x;
  acc[3] ^= b.y; acc[4] ^= c.x; acc[5] ^= c.y;
}

__device__ __forceinline__ void reduce_store(uint32_t (&acc)[6], uint32_t *syn,
                                             uint8_t *ok) {
  __shared__ uint32_t red[32][6];
#pragma unroll
  for (int w = 0; w < 6; ++w)
    for (int o = 16; o > 0; o >>= 1)
      acc[w] ^= __shfl_xor_sync(0xffffffffu, acc[w], o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0)
#pragma unroll
    for (int w = 0; w < 6; ++w) red[warp][w] = acc[w];
  __syncthreads();
  if (threadIdx.x < 6) {
    uint32_t v = 0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) v ^= red[q][threadIdx.x];
    syn[threadIdx.x] = v;
    red[0][threadIdx.x] = v;   // safe: every warp's value already folded
  }
  __syncthreads();
  if (threadIdx.x == 0 && ok) {
    uint32_t any = 0;
    for (int w = 0; w < 6; ++w) any |= red[0][w];
    *ok = any == 0 ? 1 : 0;
  }
}

__global__ void __launch_bounds__(256) bch_packed_kernel(
    const uint8_t *__restrict__ hard, int64_t ld_hard, int kldpc,
    const uint32_t *__restrict__ rtab, uint32_t *__restrict__ syn,
    uint8_t *__restrict__ ok, const uint8_t *__restrict__ scr, int kpay,
    uint8_t *__restrict__ payload, int64_t ld_payload) {
  const int b = blockIdx.x;
  const uint8_t *h = hard + (size_t)b * ld_hard;
  uint32_t acc[6] = {0, 0, 0, 0, 0, 0};
  const int nword = kldpc >> 5;              // whole 32-bit words
  const uint32_t *hw = reinterpret_cast<const uint32_t *>(h);
  for (int w = threadIdx.x; w < nword; w += blockDim.x) {
    uint32_t v = __ldg(hw + w);              // bytes 4w..4w+3, LSB = byte 4w
    while (v) {
      const int t = __ffs(v) - 1;            // bit t: byte t>>3, bit t&7
      v &= v - 1;
      const int pos = 32 * w + 8 * (t >> 3) + (7 - (t & 7));
      fold_row(acc, rtab, pos);
    }
  }
  for (int pos = nword * 32 + threadIdx.x; pos < kldpc; pos += blockDim.x)
    if ((h[pos >> 3] >> (7 - (pos & 7))) & 1) fold_row(acc, rtab, pos);
  if (payload && scr) {
    uint8_t *po = payload + (size_t)b * ld_payload;
    for (int j = threadIdx.x; j < (kpay >> 3); j += blockDim.x)
      po[j] = h[j] ^ __ldg(scr + j);
  }
  reduce_store(acc, syn + (size_t)b * 6, ok ? ok + b : nullptr);
}

__global__ void __launch_bounds__(256) bch_bits_kernel(
    const uint8_t *__restrict__ bits, int64_t ld_bits, int kldpc,
    const uint32_t *__restrict__ rtab, uint32_t *__restrict__ syn) {
  const int b = blockIdx.x;
  const uint8_t *h = bits + (size_t)b * ld_bits;
  uint32_t acc[6] = {0, 0, 0, 0, 0, 0};
  for (int pos = threadIdx.x; pos < kldpc; pos += blockDim.x)
    if (h[pos] & 1) fold_row(acc, rtab, pos);
  reduce_store(acc, syn + (size_t)b * 6, nullptr);
}

int32_t bch_check_launch(const uint8_t *hard, int64_t ld_hard, int nblk,
                         int kldpc, const uint32_t *rtab, uint32_t *syn,
                         uint8_t *ok, const uint8_t *scr, int kpay,
                         uint8_t *payload, int64_t ld_payload,
                         cudaStream_t st) {
  ATSC3_ARG(nblk >= 0 && kldpc > 0, "bad size");
  if (nblk == 0) return 0;
  ATSC3_ARG(hard && rtab && syn, "null pointer");
  ATSC3_ARG(ld_hard * 8 >= kldpc, "ld_hard*8 < kldpc");
  ATSC3_ARG(ld_hard % 4 == 0 && ((uintptr_t)hard & 3) == 0,
            "hard must be 4-byte aligned with ld_hard a multiple of 4");
  ATSC3_ARG(((uintptr_t)rtab & 7) == 0, "rtab must be 8-byte aligned");
  if (payload) {
    ATSC3_ARG(scr != nullptr, "payload needs the scrambling bytes");
    ATSC3_ARG(kpay % 8 == 0 && kpay <= kldpc, "kpayload must be a multiple of 8");
    ATSC3_ARG(ld_payload >= kpay / 8, "ld_payload < kpayload/8");
  }
  bch_packed_kernel<<<nblk, 256, 0, st>>>(hard, ld_hard, kldpc, rtab, syn, ok,
                                          scr, kpay, payload, ld_payload);
  ATSC3_CUDA(cudaGetLastError());
  return 0;
}

int32_t bch_bits_launch(const uint8_t *bits, int64_t ld_bits, int nblk,
                        int kldpc, const uint32_t *rtab, uint32_t *syn,
                        cudaStream_t st) {
  ATSC3_ARG(nblk >= 0 && kldpc > 0, "bad size");
  if (nblk == 0) return 0;
  ATSC3_ARG(bits && rtab && syn, "null pointer");
  ATSC3_ARG(ld_bits >= kldpc, "ld_bits < kldpc");
  ATSC3_ARG(((uintptr_t)rtab & 7) == 0, "rtab must be 8-byte aligned");
  bch_bits_kernel<<<nblk, 256, 0, st>>>(bits, ld_bits, kldpc, rtab, syn);
  ATSC3_CUDA(cudaGetLastError());
  return 0;
}

// ---- uneven batches: per-block BCH length, tables and payload -------------
struct BchBatchArgs {
  const uint8_t *hard;
  const int64_t *hard_off;
  const int32_t *kldpc;
  const uint32_t *rtab;
  const int64_t *rtab_off;    // uint32 words
  const uint8_t *scr;         // scrambling bytes (longest payload)
  const int32_t *kpay;
  uint8_t *payload;
  const int64_t *pay_off;
  uint32_t *syn;
  uint8_t *ok;
};

__global__ void __launch_bounds__(256) bch_batch_kernel(const BchBatchArgs a) {
  const int b = blockIdx.x;
  const uint8_t *h = a.hard + a.hard_off[b];
  const int kldpc = a.kldpc[b];
  const uint32_t *rtab = a.rtab + a.rtab_off[b];
  uint32_t acc[6] = {0, 0, 0, 0, 0, 0};
  const int nword = kldpc >> 5;
  const uint32_t *hw = reinterpret_cast<const uint32_t *>(h);
  for (int w = threadIdx.x; w < nword; w += blockDim.x) {
    uint32_t v = __ldg(hw + w);
    while (v) {
      const int t = __ffs(v) - 1;
      v &= v - 1;
      fold_row(acc, rtab, 32 * w + 8 * (t >> 3) + (7 - (t & 7)));
    }
  }
  for (int pos = nword * 32 + threadIdx.x; pos < kldpc; pos += blockDim.x)
    if ((h[pos >> 3] >> (7 - (pos & 7))) & 1) fold_row(acc, rtab, pos);
  if (a.payload) {
    uint8_t *po = a.payload + a.pay_off[b];
    for (int j = threadIdx.x; j < (a.kpay[b] >> 3); j += blockDim.x)
      po[j] = h[j] ^ __ldg(a.scr + j);
  }
  reduce_store(acc, a.syn + (size_t)b * 6, a.ok + b);
}

}  // namespace atsc3

extern "C" {

int32_t atsc3_bch_batch(const uint8_t *hard, const int64_t *hard_off,
                        const int32_t *kldpc, const uint32_t *rtab,
                        const int64_t *rtab_off, const uint8_t *scr,
                        const int32_t *kpay, uint8_t *payload,
                        const int64_t *pay_off, uint32_t *syn, uint8_t *ok,
                        int32_t nblk, void *stream) {
  using namespace atsc3;
  ATSC3_ARG(nblk >= 0, "negative size");
  if (nblk == 0) return 0;
  ATSC3_ARG(hard && hard_off && kldpc && rtab && rtab_off && syn && ok, "null pointer");
  ATSC3_ARG(!payload || (scr && kpay && pay_off), "payload needs scr, kpay, pay_off");
  BchBatchArgs a{hard, hard_off, kldpc, rtab, rtab_off, scr, kpay, payload,
                 pay_off, syn, ok};
  bch_batch_kernel<<<nblk, 256, 0, (cudaStream_t)stream>>>(a);
  ATSC3_CUDA(cudaGetLastError());
  return 0;
}


int32_t atsc3_bch_check(const uint8_t *hard, int64_t ld_hard, int32_t nblk,
                        int32_t kldpc, const uint32_t *rtab, uint32_t *syn,
                        uint8_t *ok, const uint8_t *scr, int32_t kpayload,
                        uint8_t *payload, int64_t ld_payload, void *stream) {
  return atsc3::bch_check_launch(hard, ld_hard, nblk, kldpc, rtab, syn, ok,
                                 scr, kpayload, payload, ld_payload,
                                 (cudaStream_t)stream);
}

int32_t atsc3_bch_syndrome_bits(const uint8_t *bits, int64_t ld_bits,
                                int32_t nblk, int32_t kldpc,
                                const uint32_t *rtab, uint32_t *syn,
                                void *stream) {
  return atsc3::bch_bits_launch(bits, ld_bits, nblk, kldpc, rtab, syn,
                                (cudaStream_t)stream);
}

}  // extern "C"
