// capi.cu -- error state and device facts of the C ABI.
#include <cuda_runtime.h>

#include <string>

#include "../../include/atsc3_fec.h"
#include "common.cuh"

#define ATSC3_VERSION 1

namespace atsc3 {

static thread_local std::string t_err;

void set_error(const std::string &msg) { t_err = msg; }
const char *get_error() { return t_err.c_str(); }

int32_t cuda_fail(cudaError_t e, const char *what) {
  set_error(std::string("CUDA error in ") + what + ": " +
            cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
  return -2;
}

}  // namespace atsc3

extern "C" {

const char *atsc3_last_error(void) { return atsc3::get_error(); }

int32_t atsc3_device_info(int32_t *info) {
  ATSC3_ARG(info != nullptr, "null info");
  int dev = 0;
  ATSC3_CUDA(cudaGetDevice(&dev));
  int sms = 0, smem = 0, maj = 0, mnr = 0;
  ATSC3_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  ATSC3_CUDA(cudaDeviceGetAttribute(&smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  ATSC3_CUDA(cudaDeviceGetAttribute(&maj, cudaDevAttrComputeCapabilityMajor, dev));
  ATSC3_CUDA(cudaDeviceGetAttribute(&mnr, cudaDevAttrComputeCapabilityMinor, dev));
  info[0] = sms;
  info[1] = smem;
  info[2] = maj * 10 + mnr;
  info[3] = ATSC3_VERSION;
  return 0;
}

}  // extern "C"
