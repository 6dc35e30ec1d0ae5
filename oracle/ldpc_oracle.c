/* ldpc_oracle.c -- TEST INFRASTRUCTURE ONLY (the parity oracle).
 *
 * CPU restatement of the Felbs/atsc3 min-sum decoders, used by the tests,
 * by smoke() and by the bench's CPU baseline as the checker.  Never linked
 * into the product.  Built with -O2 -ffp-contract=off so every float
 * operation is rounded separately, as in the reference build
 * (lab/build_ldpc_kernel.py:36).
 *
 * Messages are stored per edge here (the GPU keeps a compressed per-check
 * record instead), so the two implementations share no data layout.
 *
 * oracle_flood_f32 semantics 0 follows lab/ldpc_kernel.c:65-146 line by line:
 *   syndrome first (:95-113), first-minimum tie rule with strict < (:116-134),
 *   s = 0; s += m[vedge[k]]; tot = lam + s (:137-142).
 * semantics 1 follows lab/m9_gpu.py:168-220 and the float64 numpy decoder
 *   lab/m3_ldpc.py:560-630: update first, tot = lam; tot += m[e] in edge
 *   order (np.add.at), syndrome after the update, its = updates done.
 * oracle_flood_f64: semantics 1 in float64 (GpuMinSum dtype="float64").
 * oracle_layered_f32: the layered schedule the GPU layered decoder runs
 *   (no reference counterpart; see its comment).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define MAXDEG 128

#define DEFINE_FLOOD(NAME, T, FABS)                                           \
  int32_t NAME(const T *llr, int32_t nblk, int32_t n, int32_t nc,             \
               const int32_t *cptr, const int32_t *cidx, const int32_t *vptr, \
               const int32_t *vedge, int32_t iters, T alpha,                  \
               int32_t semantics, uint8_t *bits, uint8_t *conv, int32_t *its, \
               int32_t *bad) {                                                \
    int32_t ne = cptr[nc];                                                    \
    T *tot = (T *)malloc(sizeof(T) * (size_t)n);                              \
    T *m = (T *)malloc(sizeof(T) * (size_t)(ne ? ne : 1));                    \
    T v[MAXDEG];                                                              \
    if (!tot || !m) { free(tot); free(m); return -2; }                        \
    for (int32_t c = 0; c < nc; c++)                                          \
      if (cptr[c + 1] - cptr[c] > MAXDEG) { free(tot); free(m); return -1; }  \
    for (int32_t b = 0; b < nblk; b++) {                                      \
      const T *lam = llr + (size_t)b * n;                                     \
      uint8_t *bo = bits + (size_t)b * n;                                     \
      for (int32_t i = 0; i < n; i++) tot[i] = lam[i];                        \
      for (int32_t e = 0; e < ne; e++) m[e] = (T)0;                           \
      conv[b] = 0; its[b] = iters; bad[b] = -1;                               \
      for (int32_t it = 0; it <= iters; it++) {                               \
        int32_t badct = 0;                                                    \
        for (int32_t c = 0; c < nc; c++) {                                    \
          int par = 0;                                                        \
          for (int32_t e = cptr[c]; e < cptr[c + 1]; e++)                     \
            par ^= (tot[cidx[e]] < (T)0);                                     \
          badct += par;                                                       \
        }                                                                     \
        int may_retire = semantics == 0 || it > 0;                            \
        if (badct == 0 && may_retire) {                                       \
          for (int32_t i = 0; i < n; i++) bo[i] = tot[i] < (T)0;              \
          conv[b] = 1; its[b] = it; bad[b] = 0;                               \
          break;                                                              \
        }                                                                     \
        if (it == iters) {                                                    \
          for (int32_t i = 0; i < n; i++) bo[i] = tot[i] < (T)0;              \
          bad[b] = badct;                                                     \
          break;                                                              \
        }                                                                     \
        for (int32_t c = 0; c < nc; c++) {                                    \
          int32_t e0 = cptr[c], e1 = cptr[c + 1];                             \
          T min1 = (T)INFINITY, min2 = (T)INFINITY;                           \
          int32_t first = e0;                                                 \
          int par = 0;                                                        \
          for (int32_t e = e0; e < e1; e++) {                                 \
            T vv = tot[cidx[e]] - m[e];                                       \
            v[e - e0] = vv;                                                   \
            par ^= (vv < (T)0);                                               \
            T mag = FABS(vv);                                                 \
            if (mag < min1) { min2 = min1; min1 = mag; first = e; }           \
            else if (mag < min2) { min2 = mag; }                              \
          }                                                                   \
          for (int32_t e = e0; e < e1; e++) {                                 \
            T val = ((e == first) ? min2 : min1) * alpha;                     \
            if (par ^ (v[e - e0] < (T)0)) val = -val;                         \
            m[e] = val;                                                       \
          }                                                                   \
        }                                                                     \
        for (int32_t i = 0; i < n; i++) {                                     \
          if (semantics == 0) {                                               \
            T s = (T)0;                                                       \
            for (int32_t k = vptr[i]; k < vptr[i + 1]; k++) s += m[vedge[k]]; \
            tot[i] = lam[i] + s;                                              \
          } else {                                                            \
            T s = lam[i];                                                     \
            for (int32_t k = vptr[i]; k < vptr[i + 1]; k++) s += m[vedge[k]]; \
            tot[i] = s;                                                       \
          }                                                                   \
        }                                                                     \
      }                                                                       \
    }                                                                         \
    free(tot); free(m);                                                       \
    return 0;                                                                 \
  }

DEFINE_FLOOD(oracle_flood_f32, float, fabsf)
DEFINE_FLOOD(oracle_flood_f64, double, fabs)

int32_t oracle_abi(void) { return 3; }
