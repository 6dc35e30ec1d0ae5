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

/* Layered normalised min-sum over the block rows of a quasi-cyclic code --
 * the schedule the GPU layered decoder runs.  No reference counterpart (the
 * reference decodes flooding only); the arithmetic per check is that of
 * lab/ldpc_kernel.c:116-134 (first-minimum tie rule, strict <, messages
 * +-(first ? min2 : min1)*alpha with sign parity ^ (v < 0)), applied layer
 * by layer with the posterior updated in place:
 *   v_e = P[var_e] - m_e;   (update the check)   P[var_e] = v_e + m_e'.
 * Layers are the Q block rows in order; a layer touches each bit at most
 * once, so its checks are independent.  Row slots (position order): column
 * col[s], shift u[s], wrap[s]; check (r, k) reaches bit 360*col + (k-u) mod
 * 360, a wrap slot is absent for k == 0.  Checks are numbered a = Q*k + r.
 * Syndrome of sign(P) before the first iteration (retire with its = 0) and
 * after every full iteration (its = iterations done). */
int32_t oracle_layered_f32(const float *llr, int32_t nblk, int32_t n,
                           int32_t Q, const int32_t *rptr, const int32_t *col,
                           const int32_t *u, const int32_t *wrap,
                           int32_t iters, float alpha, uint8_t *bits,
                           uint8_t *conv, int32_t *its, int32_t *bad) {
  const int32_t Z = 360, nc = Q * Z;
  float *P = (float *)malloc(sizeof(float) * (size_t)n);
  float *A = (float *)malloc(sizeof(float) * (size_t)nc);
  float *B = (float *)malloc(sizeof(float) * (size_t)nc);
  int32_t *F = (int32_t *)malloc(sizeof(int32_t) * (size_t)nc);
  uint64_t *S = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)nc);
  if (!P || !A || !B || !F || !S) { free(P); free(A); free(B); free(F); free(S); return -2; }
  for (int32_t r = 0; r < Q; r++)
    if (rptr[r + 1] - rptr[r] > 64) { free(P); free(A); free(B); free(F); free(S); return -1; }
  for (int32_t b = 0; b < nblk; b++) {
    const float *lam = llr + (size_t)b * n;
    uint8_t *bo = bits + (size_t)b * n;
    for (int32_t i = 0; i < n; i++) P[i] = lam[i];
    for (int32_t c = 0; c < nc; c++) { A[c] = 0.f; B[c] = 0.f; F[c] = 0; S[c] = 0; }
    conv[b] = 0; its[b] = iters; bad[b] = -1;
    for (int32_t it = 0; it <= iters; it++) {
      int32_t badct = 0;
      for (int32_t r = 0; r < Q; r++)
        for (int32_t k = 0; k < Z; k++) {
          int par = 0;
          for (int32_t s = rptr[r]; s < rptr[r + 1]; s++) {
            if (wrap[s] && k == 0) continue;
            int32_t o = (k - u[s]) % Z; if (o < 0) o += Z;
            par ^= (P[col[s] * Z + o] < 0.0f);
          }
          badct += par;
        }
      if (badct == 0) {
        for (int32_t i = 0; i < n; i++) bo[i] = P[i] < 0.0f;
        conv[b] = 1; its[b] = it; bad[b] = 0;
        break;
      }
      if (it == iters) {
        for (int32_t i = 0; i < n; i++) bo[i] = P[i] < 0.0f;
        bad[b] = badct;
        break;
      }
      for (int32_t r = 0; r < Q; r++) {
        for (int32_t k = 0; k < Z; k++) {
          const int32_t c = Q * k + r;
          int32_t idx[64];
          float v[64];
          int32_t d = 0;
          float min1 = INFINITY, min2 = INFINITY;
          int32_t first = 0;
          int par = 0;
          for (int32_t s = rptr[r]; s < rptr[r + 1]; s++) {
            const int32_t j = s - rptr[r];
            if (wrap[s] && k == 0) continue;
            int32_t o = (k - u[s]) % Z; if (o < 0) o += Z;
            const int32_t vi = col[s] * Z + o;
            float mo = (j == F[c]) ? B[c] : A[c];
            if ((S[c] >> j) & 1u) mo = -mo;
            const float vv = P[vi] - mo;
            idx[d] = vi; v[d] = vv; d++;
            par ^= (vv < 0.0f);
            const float mag = fabsf(vv);
            if (mag < min1) { min2 = min1; min1 = mag; first = j; }
            else if (mag < min2) { min2 = mag; }
          }
          uint64_t sg = 0;
          const float a1 = min1 * alpha, a2 = min2 * alpha;
          for (int32_t t = 0, s = rptr[r]; s < rptr[r + 1]; s++) {
            const int32_t j = s - rptr[r];
            if (wrap[s] && k == 0) continue;
            float m = (j == first) ? a2 : a1;
            const int neg = par ^ (v[t] < 0.0f);
            if (neg) { m = -m; sg |= 1ull << j; }
            P[idx[t]] = v[t] + m;
            t++;
          }
          A[c] = a1; B[c] = a2; F[c] = first; S[c] = sg;
        }
      }
    }
  }
  free(P); free(A); free(B); free(F); free(S);
  return 0;
}
