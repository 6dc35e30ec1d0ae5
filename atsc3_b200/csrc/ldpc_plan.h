// ldpc_plan.h -- device tables of one LDPC code for the cluster decoders.
#pragma once

#include <stdint.h>

#include <vector>

struct atsc3_ldpc_plan {
  int n = 0, nc = 0, nedges = 0;
  int dmax_c = 0, dmax_v = 0;
  int cluster = 1;      // CTAs per codeword
  int dtype = 0;        // 0 float32, 1 float64
  int rec_bytes = 16;   // per-check record size in shared memory
  int ncp = 0;          // checks per CTA (multiple of 32)
  int nvlog2 = 0;       // log2(variables per CTA)
  int nslc = 0, nslv = 0;
  int smem_bytes = 0;   // dynamic shared memory per CTA
  int device = 0;
  int64_t table_bytes = 0;
  // device tables
  uint16_t *d_cent = nullptr;
  int32_t *d_cslice = nullptr;
  uint32_t *d_vent = nullptr;
  int32_t *d_vslice = nullptr;
};

namespace atsc3 {

// Host part of the table build (no CUDA calls).  Returns 0, -1 (degree),
// -3 (inconsistent tables) or -4 (unsupported size); fills the vectors.
int build_tables(const int32_t *cptr, const int32_t *cidx,
                 const int32_t *vptr, const int32_t *vedge, int n, int nc,
                 int nedges, int cluster, int *ncp, int *nvlog2,
                 std::vector<uint16_t> &cent, std::vector<int32_t> &cslice,
                 std::vector<uint32_t> &vent, std::vector<int32_t> &vslice,
                 int *dmax_c, int *dmax_v);

int record_bytes(int dtype, int dmax_c);  // 0 when unsupported
int plan_smem_bytes(int dtype, int rec_bytes, int ncp, int nvlog2);

}  // namespace atsc3
