// common.cuh -- shared helpers of the sm_100a FEC kernels: error state,
// cluster special registers and barriers, distributed-shared-memory access.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

namespace atsc3 {

// Per-thread message of the last failure, returned by atsc3_last_error().
void set_error(const std::string &msg);
const char *get_error();

int32_t cuda_fail(cudaError_t e, const char *what);

#define ATSC3_CUDA(call)                                                  \
  do {                                                                    \
    cudaError_t _e = (call);                                              \
    if (_e != cudaSuccess) return ::atsc3::cuda_fail(_e, #call);          \
  } while (0)

#define ATSC3_ARG(cond, msg)                                              \
  do {                                                                    \
    if (!(cond)) {                                                        \
      ::atsc3::set_error(std::string("invalid argument: ") + (msg));      \
      return -3;                                                          \
    }                                                                     \
  } while (0)

// ---------------------------------------------------------------------------
// device helpers
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint32_t cluster_ctarank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}

__device__ __forceinline__ uint32_t cluster_nctarank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
  return r;
}

__device__ __forceinline__ uint32_t cluster_id_x() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(r));
  return r;
}

__device__ __forceinline__ uint32_t ncluster_x() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%nclusterid.x;" : "=r"(r));
  return r;
}

// Full cluster barrier with release/acquire ordering of all memory
// operations (shared, distributed shared and global) of the cluster.
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile(
      "barrier.cluster.arrive.release.aligned;\n\t"
      "barrier.cluster.wait.acquire.aligned;" ::: "memory");
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// shared::cta address in this CTA -> shared::cluster address of the same
// offset in CTA `rank` of the cluster.
// mapa only translates an address (no memory access), so it is not
// volatile: the compiler may schedule and predicate it freely.
__device__ __forceinline__ uint32_t dsmem_map(uint32_t local, uint32_t rank) {
  uint32_t r;
  asm("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(local), "r"(rank));
  return r;
}

__device__ __forceinline__ float dsmem_ld_f32(uint32_t a) {
  float v;
  asm volatile("ld.shared::cluster.f32 %0, [%1];" : "=f"(v) : "r"(a));
  return v;
}

__device__ __forceinline__ double dsmem_ld_f64(uint32_t a) {
  double v;
  asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(v) : "r"(a));
  return v;
}

__device__ __forceinline__ uint4 dsmem_ld_v4(uint32_t a) {
  uint4 v;
  asm volatile("ld.shared::cluster.v4.u32 {%0, %1, %2, %3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "r"(a));
  return v;
}

__device__ __forceinline__ void dsmem_st_u32(uint32_t a, uint32_t v) {
  asm volatile("st.shared::cluster.u32 [%0], %1;" :: "r"(a), "r"(v)
               : "memory");
}

__device__ __forceinline__ void dsmem_st_u64(uint32_t a, unsigned long long v) {
  asm volatile("st.shared::cluster.u64 [%0], %1;" :: "r"(a), "l"(v)
               : "memory");
}

// atomic add into (possibly another CTA's) shared memory of the cluster
__device__ __forceinline__ void dsmem_red_add_u32(uint32_t a, uint32_t v) {
  asm volatile("red.shared::cluster.add.u32 [%0], %1;" :: "r"(a), "r"(v)
               : "memory");
}

template <typename T> __device__ __forceinline__ T dsmem_ld(uint32_t a);
template <> __device__ __forceinline__ float dsmem_ld<float>(uint32_t a) {
  return dsmem_ld_f32(a);
}
template <> __device__ __forceinline__ double dsmem_ld<double>(uint32_t a) {
  return dsmem_ld_f64(a);
}

// IEEE round-to-nearest arithmetic that the compiler may not contract into
// an FMA: the parity kernels must round every operation like the reference.
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float vabs(float a) { return fabsf(a); }
__device__ __forceinline__ double vabs(double a) { return fabs(a); }
__device__ __forceinline__ float vmin(float a, float b) { return fminf(a, b); }
__device__ __forceinline__ double vmin(double a, double b) { return fmin(a, b); }
__device__ __forceinline__ float vmax(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double vmax(double a, double b) { return fmax(a, b); }
template <typename V> __device__ __forceinline__ V vinf();
template <> __device__ __forceinline__ float vinf<float>() { return __int_as_float(0x7f800000); }
template <> __device__ __forceinline__ double vinf<double>() {
  return __longlong_as_double(0x7ff0000000000000ll);
}
// the raw bits of a message value and the store of a signed message
__device__ __forceinline__ uint32_t vbits(float a) { return __float_as_uint(a); }
__device__ __forceinline__ unsigned long long vbits(double a) {
  return (unsigned long long)__double_as_longlong(a);
}
__device__ __forceinline__ void dsmem_st_bits(uint32_t a, uint32_t bits) {
  dsmem_st_u32(a, bits);
}
__device__ __forceinline__ void dsmem_st_bits(uint32_t a, unsigned long long bits) {
  dsmem_st_u64(a, bits);
}
__device__ __forceinline__ void dsmem_st_msg(uint32_t a, uint32_t mag_bits, uint32_t neg) {
  dsmem_st_u32(a, mag_bits | (neg << 31));
}
__device__ __forceinline__ void dsmem_st_msg(uint32_t a, unsigned long long mag_bits,
                                             uint32_t neg) {
  dsmem_st_u64(a, mag_bits | ((unsigned long long)neg << 63));
}

}  // namespace atsc3
