// noalloc.cu -- the whole FEC decode (demap + de-interleave, LDPC, BCH +
// descramble) for callers that must not allocate device memory.
//
// Who needs it: code that runs where cudaMalloc is not available or not
// allowed -- a real-time receive loop with a fixed memory budget that must
// never enter the allocator, a host process that hands the GPU only
// pre-reserved buffers, or a plugin host that forbids device allocation on
// its decode thread.  The regular path (atsc3_demap -> atsc3_ldpc_*_decode
// -> atsc3_bch_check) needs a caller-provided LLR buffer and hard-decision
// buffer between the three kernels; this entry point keeps those two
// intermediates in file-scope __device__ arrays instead, so the caller only
// passes inputs and outputs.
//
// Limits and rules:
//  * at most ATSC3_NOALLOC_MAX_BLOCKS codewords of at most
//    ATSC3_NOALLOC_MAX_N bits per call (about 4.3 MB of scratch, held on
//    every GPU that loads the library until the process exits); larger
//    requests are rejected with -3 and a message;
//  * the first call on a device looks up the scratch's device address
//    (cudaGetSymbolAddress, with that device current); make that first call
//    before any stream capture;
//  * all calls share the one scratch: calls that overlap on the GPU (other
//    streams, other threads) race and corrupt each other -- serialise them;
//  * every call writes all the scratch it reads, so nothing needs clearing
//    (kldpc <= ncell*nbits is enforced so BCH never reads past what the LDPC
//    step wrote);
//  * the plan must have been built on the current device (-3 otherwise);
//  * the LDPC plan is created beforehand (atsc3_ldpc_qce_plan_create /
//    _create2, atsc3_ldpc_qc_plan_create or atsc3_ldpc_plan_create, at
//    set-up; float32 plans); this entry point itself calls no allocator.

#include <cuda_runtime.h>

#include <mutex>

#include "../../include/atsc3_fec.h"
#include "common.cuh"
#include "ldpc_plan.h"

#define ATSC3_NOALLOC_MAX_BLOCKS 16
#define ATSC3_NOALLOC_MAX_N 64800
#define ATSC3_NOALLOC_HARD_LD 8100    // bytes per codeword, a multiple of 4

static __device__ __align__(256) float
    g_noalloc_llr[ATSC3_NOALLOC_MAX_BLOCKS * ATSC3_NOALLOC_MAX_N];
static __device__ __align__(256) uint8_t
    g_noalloc_hard[ATSC3_NOALLOC_MAX_BLOCKS * ATSC3_NOALLOC_HARD_LD];

namespace atsc3 {
int32_t demap_launch(const float *cells, int64_t ld_cells, int nblk, int ncell,
                     const float *pts, int nbits, int sigma_mode,
                     const float *sigma2, int64_t ld_sigma, float s2scalar,
                     const int32_t *lam_of_q, float *out, int64_t ld_out,
                     cudaStream_t st);
int32_t flood_launch(const atsc3_ldpc_plan *p, const void *llr, int64_t ld_llr,
                     int nblk, int iters, double alpha, int semantics,
                     uint8_t *bits, int64_t ld_bits, uint8_t *hard,
                     int64_t ld_hard, uint8_t *conv, int32_t *its,
                     int32_t *bad, int threads, cudaStream_t stream,
                     int max_clusters_cap);
int32_t bch_check_launch(const uint8_t *hard, int64_t ld_hard, int nblk,
                         int kldpc, const uint32_t *rtab, uint32_t *syn,
                         uint8_t *ok, const uint8_t *scr, int kpay,
                         uint8_t *payload, int64_t ld_payload,
                         cudaStream_t st);

int qce_plan_device(const atsc3_ldpc_qce_plan *h);
int qc_plan_device(const atsc3_ldpc_qc_plan *h);

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_mu;
float *g_llr_ptr[kMaxDevices] = {nullptr};
uint8_t *g_hard_ptr[kMaxDevices] = {nullptr};

// Device addresses of the scratch arrays for the current device, looked up
// once per device (host code cannot take the address of a __device__
// array directly: the host-side symbol is only a stand-in).
int32_t scratch_for_current_device(float **llr, uint8_t **hard) {
  int dev = 0;
  ATSC3_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("unsupported: device index above 63");
    return -4;
  }
  std::lock_guard<std::mutex> g(g_mu);
  if (!g_llr_ptr[dev]) {
    void *a = nullptr, *b = nullptr;
    ATSC3_CUDA(cudaGetSymbolAddress(&a, g_noalloc_llr));
    ATSC3_CUDA(cudaGetSymbolAddress(&b, g_noalloc_hard));
    g_llr_ptr[dev] = static_cast<float *>(a);
    g_hard_ptr[dev] = static_cast<uint8_t *>(b);
  }
  *llr = g_llr_ptr[dev];
  *hard = g_hard_ptr[dev];
  return 0;
}
}  // namespace
}  // namespace atsc3

extern "C" int32_t atsc3_fec_decode_noalloc(
    const void *plan, int32_t plan_kind, const float *cells, int64_t ld_cells,
    int32_t nblk, int32_t ncell, const float *pts, int32_t nbits,
    int32_t sigma_mode, const float *sigma2, int64_t ld_sigma,
    float sigma2_scalar, const int32_t *lam_of_q, int32_t iters, float alpha,
    const uint32_t *rtab, int32_t kldpc, const uint8_t *scr, int32_t kpayload,
    uint8_t *payload, int64_t ld_payload, uint8_t *conv, int32_t *its,
    int32_t *bad, uint32_t *syn, uint8_t *ok, void *stream) {
  using namespace atsc3;
  ATSC3_ARG(plan != nullptr, "null plan");
  ATSC3_ARG(plan_kind >= 0 && plan_kind <= 2,
            "plan_kind must be 0 (CSR), 1 (QC record layout) or 2 (QC edge buffer)");
  ATSC3_ARG(nblk >= 0 && ncell > 0 && nbits > 0, "bad size");
  const int64_t n = (int64_t)ncell * nbits;
  if (nblk > ATSC3_NOALLOC_MAX_BLOCKS || n > ATSC3_NOALLOC_MAX_N) {
    set_error("invalid argument: atsc3_fec_decode_noalloc serves at most 16 "
              "codewords of at most 64800 bits per call (fixed scratch); "
              "split the batch");
    return -3;
  }
  // BCH reads the first kldpc hard decisions of each scratch row, and the
  // LDPC step writes only the first n of them: a longer kldpc would read
  // bits another call left behind.
  ATSC3_ARG(kldpc > 0 && kldpc <= n, "kldpc must be in 1..ncell*nbits");
  ATSC3_ARG(kpayload >= 0 && kpayload <= kldpc, "kpayload must be in 0..kldpc");
  if (nblk == 0) return 0;
  ATSC3_ARG(lam_of_q != nullptr, "lam_of_q required (codeword order)");
  int plan_dev = 0;
  if (plan_kind == 1 || plan_kind == 2) {
    int64_t info[10];
    int32_t rc0 = plan_kind == 1
        ? atsc3_ldpc_qc_plan_info((const atsc3_ldpc_qc_plan *)plan, info)
        : atsc3_ldpc_qce_plan_info((const atsc3_ldpc_qce_plan *)plan, info);
    if (rc0) return rc0;
    ATSC3_ARG(info[0] == n, "ncell*nbits differs from the plan's codeword length");
    plan_dev = plan_kind == 1
        ? qc_plan_device((const atsc3_ldpc_qc_plan *)plan)
        : qce_plan_device((const atsc3_ldpc_qce_plan *)plan);
  } else {
    ATSC3_ARG(((const atsc3_ldpc_plan *)plan)->n == n,
              "ncell*nbits differs from the plan's codeword length");
    plan_dev = ((const atsc3_ldpc_plan *)plan)->device;
  }
  // the scratch is per device: the plan's tables and the scratch must be on
  // the same (current) GPU
  int cur_dev = 0;
  ATSC3_CUDA(cudaGetDevice(&cur_dev));
  ATSC3_ARG(plan_dev == cur_dev,
            "the plan was built on another device than the current one");
  float *llr = nullptr;
  uint8_t *hard = nullptr;
  int32_t rc = scratch_for_current_device(&llr, &hard);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  rc = demap_launch(cells, ld_cells, nblk, ncell, pts, nbits, sigma_mode,
                    sigma2, ld_sigma, sigma2_scalar, lam_of_q, llr, n, st);
  if (rc) return rc;
  if (plan_kind == 2) {
    // a float64 plan is refused here (-3): the scratch holds float32 LLRs
    rc = atsc3_ldpc_qce_decode((const atsc3_ldpc_qce_plan *)plan, llr, n, nblk,
                               iters, alpha, 0, nullptr, 0, hard,
                               ATSC3_NOALLOC_HARD_LD, conv, its, bad, 0, stream);
  } else if (plan_kind == 1) {
    rc = atsc3_ldpc_qc_decode((const atsc3_ldpc_qc_plan *)plan, llr, n, nblk,
                              iters, alpha, 0, nullptr, 0, hard,
                              ATSC3_NOALLOC_HARD_LD, conv, its, bad, 0, stream);
  } else {
    rc = flood_launch((const atsc3_ldpc_plan *)plan, llr, n, nblk, iters,
                      (double)alpha, 0, nullptr, 0, hard, ATSC3_NOALLOC_HARD_LD,
                      conv, its, bad, 0, st, 0);
  }
  if (rc) return rc;
  return bch_check_launch(hard, ATSC3_NOALLOC_HARD_LD, nblk, kldpc, rtab, syn,
                          ok, scr, kpayload, payload, ld_payload, st);
}
