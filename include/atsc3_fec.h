/* atsc3_fec.h -- C ABI of the B200 (sm_100a) ATSC 3.0 FEC back end.
 *
 * One shared library, libatsc3_fec.so, exports everything below.  Plain C
 * types only: pointers, sizes, and a cudaStream_t passed as void*.
 *
 * Two groups of entry points:
 *
 *  1. Drop-in for the Felbs/atsc3 compiled min-sum kernel
 *     (lab/ldpc_kernel.c:52-146, bound by ctypes in lab/m3_ldpc.py:425-456).
 *     Same symbol names, same argument order and meaning, HOST pointers.
 *
 *  2. Device-pointer entry points used by the Python host layer
 *     (atsc3_b200/) for the batched GPU path.  They replace the torch-eager
 *     GPU code of lab/m9_gpu.py (GpuMinSum.decode :138-220, GpuBicm.demap
 *     :301-316), the numpy demappers lab/m16_demap_fast.py:80-119 and
 *     lab/m44_ldm.py:2431-2494, and the BCH helpers lab/m9_accel.py:197-236.
 *     All pointers are device pointers unless stated; every launch goes to
 *     the given stream and nothing synchronises unless stated.
 *
 * Return codes: 0 ok; -1 a check degree above ATSC3_MAX_ROW_DEG (the
 * reference kernel's only error, lab/ldpc_kernel.c:78-80); -2 CUDA error;
 * -3 invalid argument; -4 configuration the kernels do not support (e.g.
 * shared memory needed above the device limit).  atsc3_last_error() returns
 * a message for the last failure on the calling thread.
 */
#ifndef ATSC3_FEC_H
#define ATSC3_FEC_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ATSC3_MAX_ROW_DEG 128

/* ---- 1. reference drop-in ------------------------------------------------ */

/* Returns 1.  Replaces ldpc_kernel_abi (lab/ldpc_kernel.c:52). */
int32_t ldpc_kernel_abi(void);

/* Replaces ldpc_minsum_f32 (lab/ldpc_kernel.c:65-146): flooding normalised
 * min-sum in float32, syndrome checked before each update, first-minimum tie
 * rule, variable sums in vedge order.  Bit-identical outputs (bits, conv,
 * its, bad).  All pointers are HOST pointers, C-contiguous.  The decode runs
 * on the GPU on a per-thread stream and the call returns when the outputs
 * are written.  `work` is accepted for ABI compatibility and not touched.
 * Device copies of the CSR tables are cached by content.  Thread-safe.
 * Returns 0, -1 (degree > 128, nothing written), -2 (CUDA error), -3. */
int32_t ldpc_minsum_f32(const float *llr, int32_t nblk, int32_t n,
                        int32_t nc, int32_t nedges,
                        const int32_t *cptr, const int32_t *cidx,
                        const int32_t *vptr, const int32_t *vedge,
                        int32_t iters, float alpha,
                        uint8_t *bits, uint8_t *conv, int32_t *its,
                        int32_t *bad, float *work);

/* ---- 2. device-pointer entry points --------------------------------------- */

const char *atsc3_last_error(void);

/* Library / device facts: info[0] = SM count, [1] = max dynamic shared
 * memory per block (bytes), [2] = compute capability major*10+minor,
 * [3] = library version. */
int32_t atsc3_device_info(int32_t *info);

typedef struct atsc3_ldpc_plan atsc3_ldpc_plan;

/* Build the device tables of one LDPC code for the flooding decoder.
 * cptr/cidx/vptr/vedge: HOST CSR tables (lab/m3_ldpc.py:459-482 layout).
 * dtype: 0 = float32 messages, 1 = float64 messages.
 * cluster: thread-block cluster size (1, 2, 4, 8, 16), 0 = smallest that
 * fits the per-codeword state in distributed shared memory.
 * Replaces GpuMinSum.__init__ (lab/m9_gpu.py:95-135). */
int32_t atsc3_ldpc_plan_create(const int32_t *cptr, const int32_t *cidx,
                               const int32_t *vptr, const int32_t *vedge,
                               int32_t n, int32_t nc, int32_t nedges,
                               int32_t dtype, int32_t cluster,
                               atsc3_ldpc_plan **out);
void atsc3_ldpc_plan_destroy(atsc3_ldpc_plan *plan);

/* info[0]=n [1]=nc [2]=nedges [3]=cluster [4]=shared bytes per CTA
 * [5]=record bytes [6]=max row degree [7]=max column degree
 * [8]=table bytes on device [9]=dtype */
int32_t atsc3_ldpc_plan_info(const atsc3_ldpc_plan *plan, int64_t *info);

/* Host-only table build used by the CPU tests: fills the check-phase and
 * variable-phase sliced-ELL tables for a given cluster size without touching
 * a GPU.  Call with null outputs to get the sizes in sizes[0..3] (entries of
 * cent, cslice, vent, vslice); sizes[4] = checks per CTA, sizes[5] = log2 of
 * variables per CTA. */
int32_t atsc3_ldpc_tables_host(const int32_t *cptr, const int32_t *cidx,
                               const int32_t *vptr, const int32_t *vedge,
                               int32_t n, int32_t nc, int32_t nedges,
                               int32_t cluster, int64_t *sizes,
                               uint16_t *cent, int32_t *cslice,
                               uint32_t *vent, int32_t *vslice);

/* Flooding normalised min-sum over nblk codewords, one thread-block cluster
 * per codeword, all iterations in one launch, per-codeword early stop.
 * llr: device (nblk, ld_llr) float32 or float64 (the plan's dtype).
 * semantics 0: lab/ldpc_kernel.c (syndrome before each update, its may be 0,
 *   variable sum from +0 then added to the channel LLR);
 * semantics 1: lab/m9_gpu.py:168-211 / lab/m3_ldpc.py:560-630 float64 path
 *   (update first, its >= 1, variable sum accumulated onto the channel LLR).
 * semantics 2 / 3 (float32 plans): semantics 1 as lab/m9_gpu.py runs it with
 *   dtype bfloat16 / float16 (lab/m9_gpu.py:100-101): every subtraction,
 *   scaled minimum (alpha itself rounded first) and partial variable sum is
 *   rounded to that type; llr must already hold values of that type.
 * bits (nullable): (nblk, ld_bits) uint8 hard decisions, 1 = negative LLR.
 * hard (nullable): (nblk, ld_hard) packed hard decisions, n/8 bytes, MSB
 *   first in each byte (numpy packbits order).
 * conv/its/bad: per codeword, as lab/ldpc_kernel.c:62.
 * threads: CTA size (0 = 1024). */
int32_t atsc3_ldpc_decode_flood(const atsc3_ldpc_plan *plan, const void *llr,
                                int64_t ld_llr, int32_t nblk, int32_t iters,
                                double alpha, int32_t semantics,
                                uint8_t *bits, int64_t ld_bits,
                                uint8_t *hard, int64_t ld_hard,
                                uint8_t *conv, int32_t *its, int32_t *bad,
                                int32_t threads, void *stream);

/* Launch facts of the flooding decoder for this plan: out[0] = clusters that
 * can be resident at once, [1] = CTAs per cluster, [2] = shared bytes per
 * CTA, [3] = threads per CTA. */
int32_t atsc3_ldpc_flood_config(const atsc3_ldpc_plan *plan, int32_t threads,
                                int32_t semantics, int32_t *out);

/* ---- quasi-cyclic decoder for the A/322 Type B codes ----------------------
 * Same decoding semantics and outputs as atsc3_ldpc_decode_flood (float32),
 * built from the Annex A address rows instead of CSR tables: the 360x360
 * circulant structure replaces per-edge tables (see csrc/ldpc_qc.cu).
 * Accepts Type B codes (Nldpc-Kldpc = 360*Qldpc) with at most one circulant
 * per block; returns -4 otherwise.  Replaces GpuMinSum.__init__/decode for
 * those codes. */
typedef struct atsc3_ldpc_qc_plan atsc3_ldpc_qc_plan;

int32_t atsc3_ldpc_qc_plan_create(int32_t n, int32_t kldpc, int32_t qldpc,
                                  const int32_t *rowptr, const int32_t *addr,
                                  int32_t cluster, atsc3_ldpc_qc_plan **out);
void atsc3_ldpc_qc_plan_destroy(atsc3_ldpc_qc_plan *plan);

/* info[0]=n [1]=K [2]=Q [3]=cluster [4]=shared bytes per CTA [5]=max
 * block-row degree [6]=max block-column degree [7]=table bytes [8]=block
 * rows per CTA [9]=360-bit columns per CTA */
int32_t atsc3_ldpc_qc_plan_info(const atsc3_ldpc_qc_plan *plan, int64_t *info);

/* Host-only descriptor build for the CPU tests (no CUDA call).  meta (42
 * ints): [0] row slots [1] column slots [2] 360-bit columns per CTA [3]
 * checks per CTA [4] block rows per CTA [5] max row degree [6] max column
 * degree [7] shared bytes [8..24] row split [25..41] variable-phase work
 * split.  rdesc/cdesc are int4 slots (rank | wrap<<8 | position<<16, byte
 * base, shift, 0).  Array outputs may be null. */
int32_t atsc3_ldpc_qc_tables_host(int32_t n, int32_t kldpc, int32_t qldpc,
                                  const int32_t *rowptr, const int32_t *addr,
                                  int32_t cluster, int32_t *meta,
                                  int32_t *rdesc, int32_t *rptr,
                                  int32_t *cdesc, int32_t *cptr, uint8_t *s0);

int32_t atsc3_ldpc_qc_config(const atsc3_ldpc_qc_plan *plan, int32_t threads,
                             int32_t semantics, int32_t *out);

int32_t atsc3_ldpc_qc_decode(const atsc3_ldpc_qc_plan *plan, const float *llr,
                             int64_t ld_llr, int32_t nblk, int32_t iters,
                             float alpha, int32_t semantics, uint8_t *bits,
                             int64_t ld_bits, uint8_t *hard, int64_t ld_hard,
                             uint8_t *conv, int32_t *its, int32_t *bad,
                             int32_t threads, void *stream);

/* As atsc3_ldpc_qc_decode with learned weights: each check's record minima
 * become relu(min*wa - wb), (wa, wb) = (walpha, wbeta)[min(it, wT-1)][
 * dbucket[check degree]] for the update of iteration it (0-based);
 * walpha/wbeta (wT, wnb) float32 and dbucket (64) int8 are device arrays.
 * With walpha == NULL it is atsc3_ldpc_qc_decode. */
int32_t atsc3_ldpc_qc_decode_weighted(
    const atsc3_ldpc_qc_plan *plan, const float *llr, int64_t ld_llr,
    int32_t nblk, int32_t iters, float alpha, int32_t semantics,
    const float *walpha, const float *wbeta, int32_t wT, int32_t wnb,
    const int8_t *dbucket, uint8_t *bits, int64_t ld_bits, uint8_t *hard,
    int64_t ld_hard, uint8_t *conv, int32_t *its, int32_t *bad,
    int32_t threads, void *stream);

/* ---- quasi-cyclic decoder, edge-buffer layout ------------------------------
 * Same semantics, arguments and outputs as the atsc3_ldpc_qc_* functions
 * above (they replace the same reference entry points:
 * lab/ldpc_kernel.c:65 ldpc_minsum_f32 and lab/m9_gpu.py:138-220
 * GpuMinSum.decode), for every A/322 code: Type B through
 * atsc3_ldpc_qce_plan_create, blocks holding two circulants included, and
 * Type A through atsc3_ldpc_qce_plan_create2.  Different state layout
 * (csrc/ldpc_qce.cu): one float32 slot per edge, owned by the edge's column,
 * holding the variable-to-check value after the variable phase and the
 * check-to-variable message after the check phase; hard decisions in a
 * bitmap replicated per CTA; no per-check records.  cluster: any size in
 * 1..16 (not only powers of two); 0 picks the smallest cluster whose per-CTA
 * shared memory fits (6 for the 64800-bit codes but 7/15, which takes 7;
 * 2 for the 16200-bit ones, 1 for 16200 2/15). */
typedef struct atsc3_ldpc_qce_plan atsc3_ldpc_qce_plan;

int32_t atsc3_ldpc_qce_plan_create(int32_t n, int32_t kldpc, int32_t qldpc,
                                   const int32_t *rowptr, const int32_t *addr,
                                   int32_t cluster, atsc3_ldpc_qce_plan **out);
void atsc3_ldpc_qce_plan_destroy(atsc3_ldpc_qce_plan *plan);

/* As atsc3_ldpc_qce_plan_create for both A/322 code types: qa accumulator
 * block rows (the dual-diagonal part; Q of a Type B code, Q1 of a Type A
 * code) and qb identity block rows (0 for Type B, Q2 for Type A, whose
 * address table then also holds the qa rows of the accumulator parity bits,
 * lab/m3_ldpc.py:119-159 step vii).  A Type A code's few accumulator rows
 * above the compile-time slot count take the kernel's loop path. */
int32_t atsc3_ldpc_qce_plan_create2(int32_t n, int32_t kldpc, int32_t qa,
                                    int32_t qb, const int32_t *rowptr,
                                    const int32_t *addr, int32_t cluster,
                                    atsc3_ldpc_qce_plan **out);

/* The float64 edge-buffer decoder (8-byte slots, float64 messages and
 * posteriors, 512 threads per CTA): the arithmetic of the float64 paths of
 * lab/m9_gpu.py:168-211 (torch semantics, GpuMinSum's default dtype) and
 * lab/m3_ldpc.py:560-630, bit for bit; semantics 0 (lab/ldpc_kernel.c
 * order) in float64 too.  A 64800-bit codeword needs at least 11 CTAs;
 * cluster 0 picks the size that occupies the most SMs (16 on B200).  Plans
 * from atsc3_ldpc_qce_plan_create_f64 decode only with
 * atsc3_ldpc_qce_decode_f64 (no learned weights); alpha is a double. */
int32_t atsc3_ldpc_qce_plan_create_f64(int32_t n, int32_t kldpc, int32_t qa,
                                       int32_t qb, const int32_t *rowptr,
                                       const int32_t *addr, int32_t cluster,
                                       atsc3_ldpc_qce_plan **out);
int32_t atsc3_ldpc_qce_decode_f64(const atsc3_ldpc_qce_plan *plan, const double *llr,
                                  int64_t ld_llr, int32_t nblk, int32_t iters,
                                  double alpha, int32_t semantics, uint8_t *bits,
                                  int64_t ld_bits, uint8_t *hard, int64_t ld_hard,
                                  uint8_t *conv, int32_t *its, int32_t *bad,
                                  int32_t threads, void *stream);

/* Host only.  Recognise an A/322 Type B code in CSR tables built as
 * lab/m3_ldpc.py:459-482 (_kernel_tables) builds them from
 * lab/m3_ldpc.py:166-212 (parity_check): 360-bit circulants, info bit
 * 360g+mm on checks (x + mm*Q) mod nc for the checks x of bit 360g,
 * accumulator parity through the column twist, vedge the stable argsort of
 * cidx.  On success kq = {K, Q}, rowptr (K/360 + 1 entries) and addr (the
 * checks of bit 360g, ascending; room for nedges) feed
 * atsc3_ldpc_qce_plan_create.  Returns 0, or -4 when the tables are not that
 * structure (a Type A code included: see atsc3_ldpc_qc_detect2). */
int32_t atsc3_ldpc_qc_detect(const int32_t *cptr, const int32_t *cidx,
                             const int32_t *vptr, const int32_t *vedge,
                             int32_t n, int32_t nc, int32_t nedges,
                             int32_t *kq, int32_t *rowptr, int32_t *addr);

/* As atsc3_ldpc_qc_detect for both code types: kq = {K, qa, qb} (qa
 * accumulator and qb identity block rows; qb = 0 for Type B), found from the
 * trailing degree-1 parity bits (the identity part of a Type A code).
 * rowptr has K/360 + 1 rows, plus qa rows for a Type A code (the identity-row
 * addresses of the accumulator parity bits, A/322 step vii); the outputs
 * feed atsc3_ldpc_qce_plan_create2.  ldpc_minsum_f32 uses it. */
int32_t atsc3_ldpc_qc_detect2(const int32_t *cptr, const int32_t *cidx,
                              const int32_t *vptr, const int32_t *vedge,
                              int32_t n, int32_t nc, int32_t nedges,
                              int32_t *kq, int32_t *rowptr, int32_t *addr);

/* info[0]=n [1]=K [2]=Q [3]=cluster [4]=shared bytes per CTA [5]=max
 * block-row degree [6]=max block-column degree [7]=table bytes [8]=most edge
 * slots (360 edges each) held by one CTA [9]=360-bit columns of CTA 0 */
int32_t atsc3_ldpc_qce_plan_info(const atsc3_ldpc_qce_plan *plan, int64_t *info);

/* Host-only descriptor build for the CPU tests (no CUDA call).  meta (42
 * ints): [0] row slots [1] 360-bit columns [2] shared bytes per CTA [3]
 * byte offset of the syndrome exchange words [4] max row degree [5] max
 * column degree [6] most slots per CTA [7] byte offset of the first slot
 * [8..24] block-row split [25..41]
 * CTA c owns columns ccols[meta[25+c] .. meta[26+c]).  rdesc: int4 per row
 * slot (owner | wrap<<8 | position<<16, slot byte offset in the owner,
 * shift, bitmap byte offset of the column); cdesc: int4 per column (slots,
 * byte offset of slot 0, wrap slot or -1, owner); ccols: the nb columns
 * grouped by owner.  Array outputs may be null. */
int32_t atsc3_ldpc_qce_tables_host(int32_t n, int32_t kldpc, int32_t qldpc,
                                   const int32_t *rowptr, const int32_t *addr,
                                   int32_t cluster, int32_t *meta,
                                   int32_t *rdesc, int32_t *rptr,
                                   int32_t *cdesc, int32_t *ccols,
                                   uint8_t *s0);

/* out[0] = clusters resident at once, [1] = CTAs per cluster, [2] = shared
 * bytes per CTA, [3] = threads per CTA (threads 0 = the default). */
/* atsc3_ldpc_qce_tables_host for both code types (qa, qb as in
 * atsc3_ldpc_qce_plan_create2).  meta (96 ints): [0..41] as
 * atsc3_ldpc_qce_tables_host, [42..58] check items (row*12 + chunk) of CTA
 * c from meta[42+c] to meta[43+c] (its light items when heavy rows exist),
 * [59] heavy rows present, [60] degree that sets the compile-time slot
 * count, [61] variable-phase items, [62..78] heavy items of CTA c:
 * hitems[meta[62+c] .. meta[63+c]), [79] heavy rows (block rows 0 ..),
 * [80] / [81] least / greatest estimated variable-item bin load, [82] bins
 * per CTA (QBINS).
 * s0b: (n) rotation start in the identity rows; itab: int4 per
 * variable-phase item; hitems: heavy check items, grouped by CTA.  Array
 * outputs may be null. */
int32_t atsc3_ldpc_qce_tables_host2(int32_t n, int32_t kldpc, int32_t qa,
                                    int32_t qb, const int32_t *rowptr,
                                    const int32_t *addr, int32_t cluster,
                                    int32_t *meta, int32_t *rdesc,
                                    int32_t *rptr, int32_t *cdesc,
                                    int32_t *ccols, uint8_t *s0,
                                    uint8_t *s0b, int32_t *itab,
                                    int32_t *hitems);

/* Variable-item bins of the edge-buffer plan (host only, no device work):
 * wbin = (cluster, QBINS + 1) offsets, relative to each CTA's first item in
 * the itab of atsc3_ldpc_qce_tables_host2; warp w of a CTA of T threads walks
 * bins w*QBINS/(T/32) .. (w+1)*QBINS/(T/32) - 1.  QBINS is meta[82] of
 * atsc3_ldpc_qce_tables_host2 (32). */
int32_t atsc3_ldpc_qce_bins_host(int32_t n, int32_t kldpc, int32_t qa, int32_t qb,
                                 const int32_t *rowptr, const int32_t *addr,
                                 int32_t cluster, int32_t *wbin);

int32_t atsc3_ldpc_qce_config(const atsc3_ldpc_qce_plan *plan, int32_t threads,
                              int32_t semantics, int32_t *out);

/* threads: 0 (default), 512 or 1024; codes with a block-row degree above
 * 17 always run 512 threads.  ld_hard >= ceil(n/8). */
int32_t atsc3_ldpc_qce_decode(const atsc3_ldpc_qce_plan *plan, const float *llr,
                              int64_t ld_llr, int32_t nblk, int32_t iters,
                              float alpha, int32_t semantics, uint8_t *bits,
                              int64_t ld_bits, uint8_t *hard, int64_t ld_hard,
                              uint8_t *conv, int32_t *its, int32_t *bad,
                              int32_t threads, void *stream);

/* As atsc3_ldpc_qce_decode with learned weights (the weighting of
 * atsc3_ldpc_qc_decode_weighted). */
int32_t atsc3_ldpc_qce_decode_weighted(
    const atsc3_ldpc_qce_plan *plan, const float *llr, int64_t ld_llr,
    int32_t nblk, int32_t iters, float alpha, int32_t semantics,
    const float *walpha, const float *wbeta, int32_t wT, int32_t wnb,
    const int8_t *dbucket, uint8_t *bits, int64_t ld_bits, uint8_t *hard,
    int64_t ld_hard, uint8_t *conv, int32_t *its, int32_t *bad,
    int32_t threads, void *stream);

/* As atsc3_ldpc_qce_decode_weighted with the weights indexed by the check's
 * block row instead of its degree: the minima of a check of block row r
 * become relu(min * walpha[i][rbucket[r]] - wbeta[i][rbucket[r]]), i =
 * min(it, wT - 1); rbucket (>= the code's block rows, at most 256) int8
 * device array.  No reference counterpart (a learned parameterisation). */
int32_t atsc3_ldpc_qce_decode_weighted_rows(
    const atsc3_ldpc_qce_plan *plan, const float *llr, int64_t ld_llr,
    int32_t nblk, int32_t iters, float alpha, int32_t semantics,
    const float *walpha, const float *wbeta, int32_t wT, int32_t wnb,
    const int8_t *rbucket, uint8_t *bits, int64_t ld_bits, uint8_t *hard,
    int64_t ld_hard, uint8_t *conv, int32_t *its, int32_t *bad,
    int32_t threads, void *stream);

/* ---- exact sum-product (near-miss rescue) ----------------------------------
 * Float64 log-tanh belief propagation over nblk codewords, replacing
 * lab/m16_margin.py:325-390 sum_product_decode_batch (the rescue
 * lab/m44_ldm.py:2527-2554 offers the blocks min-sum left a few checks
 * short).  Same stopping rule: syndrome before each update, its = the
 * iteration at which the syndrome is zero, else iters with bad = the
 * unsatisfied count.  cptr/cidx/vptr/vedge: DEVICE CSR tables
 * (lab/m3_ldpc.py:459-482 layout); llr (nblk, ld_llr) float64; bits (nblk,
 * ld_bits) uint8; conv/its/bad per block; work: atsc3_ldpc_sp_workspace
 * bytes, 8-byte aligned.  atsc3_ldpc_sp_decode runs to `iters`: it
 * launches 4*(iters+1)+1 kernels on `stream` and returns without
 * synchronising.  atsc3_ldpc_sp_step runs ONE iteration `it` (it = 0
 * initialises the work area first; steps run in order on one stream),
 * so a host can honour the reference's wall-clock deadline between
 * iterations (lab/m16_margin.py:364-371): `last` = 1 takes the syndrome at
 * `it` and retires every block still decoding with its current decisions
 * (conv 0 unless the syndrome is zero, its = it, bad = the unsatisfied
 * count), as iteration `iters` of a full decode does.  counts: device
 * int32[2] = {blocks still decoding after the step, blocks retired
 * unconverged by it}. */
int32_t atsc3_ldpc_sp_workspace(int32_t n, int32_t nedges, int32_t nblk,
                                int64_t *work_bytes);
int32_t atsc3_ldpc_sp_decode(const int32_t *cptr, const int32_t *cidx,
                             const int32_t *vptr, const int32_t *vedge,
                             int32_t n, int32_t nc, int32_t nedges,
                             const double *llr, int64_t ld_llr, int32_t nblk,
                             int32_t iters, uint8_t *bits, int64_t ld_bits,
                             uint8_t *conv, int32_t *its, int32_t *bad,
                             void *work, void *stream);
int32_t atsc3_ldpc_sp_step(const int32_t *cptr, const int32_t *cidx,
                           const int32_t *vptr, const int32_t *vedge,
                           int32_t n, int32_t nc, int32_t nedges,
                           const double *llr, int64_t ld_llr, int32_t nblk,
                           int32_t it, int32_t last, uint8_t *bits,
                           int64_t ld_bits, uint8_t *conv, int32_t *its,
                           int32_t *bad, void *work, int32_t *counts,
                           void *stream);

/* ---- common phase error correction ----------------------------------------
 * Replaces lab/m6_cells.py:176-209 cpe_correct (also lab/m9_gpu.py:283-299
 * GpuBicm.cpe): the pool (ncells complex128, interleaved re/im doubles) is
 * normalised to unit mean power, then per OFDM symbol s (cells
 * sym_ptr[s] .. sym_ptr[s+1]-1, contiguous) `iters` times: hard decisions
 * (region 0: nearest point of alphabet0, m0 points; region 1: alphabet1, m1
 * points; region 2: dummy[i], the known value; other values are ignored),
 * c = sum conj(hard) z / max(sum |hard|^2, 1e-12), z /= c.  out: the
 * corrected pool (complex128); gains: per-symbol total gain (complex128).
 * work: atsc3_cpe_workspace bytes.  Float64; agreement with the numpy
 * reference is to rounding (its sums run in other orders). */
int32_t atsc3_cpe_workspace(int64_t *work_bytes);
int32_t atsc3_cpe_correct(const double *pool, int64_t ncells,
                          const int32_t *sym_ptr, int32_t nsym,
                          const uint8_t *region, const double *alphabet0,
                          int32_t m0, const double *alphabet1, int32_t m1,
                          const double *dummy, int32_t iters, double *out,
                          double *gains, void *work, void *stream);

/* ---- layered decoder for the A/322 Type B codes ----------------------------
 * Layered normalised min-sum: the Q block rows are the layers, the posterior
 * is updated in place after each layer, syndrome before the first and after
 * every full iteration (csrc/ldpc_layered.cu; the bit-exact CPU statement is
 * oracle_layered_f32).  No reference counterpart: the reference decodes
 * flooding only.  One CTA per codeword; per-CTA scratch (posterior + check
 * records) lives in the caller's workspace, sized by
 * atsc3_ldpc_layered_workspace for `ctas` resident CTAs.  Bounded waits: a
 * copy wait that runs out makes the CTA wait once more for its copies and
 * return, setting *err (device int32, caller-zeroed) to 1 when the copies
 * then completed, or 2 when the second wait ran out too (copies may have
 * been in flight when the CTA returned: the outputs are void).
 * atsc3_ldpc_layered_inject_timeout(layer) is a test hook: the next decode
 * call takes that error path at global layer `layer` (iteration * Q + block
 * row) right after the layer's copies completed, so the path runs with
 * nothing in flight (-1 clears the hook). */
typedef struct atsc3_ldpc_layered_plan atsc3_ldpc_layered_plan;

int32_t atsc3_ldpc_layered_plan_create(int32_t n, int32_t kldpc, int32_t qldpc,
                                       const int32_t *rowptr,
                                       const int32_t *addr,
                                       atsc3_ldpc_layered_plan **out);
void atsc3_ldpc_layered_plan_destroy(atsc3_ldpc_layered_plan *plan);
int32_t atsc3_ldpc_layered_workspace(const atsc3_ldpc_layered_plan *plan,
                                     int32_t ctas, int64_t *bytes);
int32_t atsc3_ldpc_layered_decode(const atsc3_ldpc_layered_plan *plan,
                                  const float *llr, int64_t ld_llr,
                                  int32_t nblk, int32_t iters, float alpha,
                                  uint8_t *bits, int64_t ld_bits, uint8_t *hard,
                                  int64_t ld_hard, uint8_t *conv, int32_t *its,
                                  int32_t *bad, void *workspace, int32_t ctas,
                                  int32_t *err, void *stream);
int32_t atsc3_ldpc_layered_inject_timeout(int32_t layer);

/* ---- differentiable weighted min-sum ---------------------------------------
 * Unrolled flooding min-sum with per-iteration, per-check-degree scale and
 * offset: m = sgn * relu(alpha[t][d] * mu - beta[t][d]) (csrc/wms.cu).  No
 * reference counterpart.  Tables: device CSR (cptr, cidx, vptr, vedge), the
 * check and position of each variable-major edge (vchk, vpos), the bucket
 * of each check (int8, at most 127 buckets: its degree class, or its block
 * row for the per-row parameterisation).  records: (iters, nblk, nc) 16-byte per-check
 * checkpoints written by the forward and read by the backward.  Forward
 * writes tot_out = the posterior after `iters` iterations (no early stop).
 * Backward: gtot in = dL/dtot_out (overwritten), galpha/gbeta accumulate
 * (caller zeroes), work = nblk*n + 2*nblk*ne floats. */
int32_t atsc3_wms_forward(const int32_t *cptr, const int32_t *cidx,
                          const int32_t *vptr, const int32_t *vedge,
                          const int32_t *vchk, const int32_t *vpos,
                          const int8_t *cbucket, int32_t n, int32_t nc,
                          int32_t ne, int32_t nbucket, int32_t nblk,
                          int32_t iters, const float *llr, const float *alpha,
                          const float *beta, int32_t bf16, void *records,
                          float *tot_out, void *stream);
int32_t atsc3_wms_backward(const int32_t *cptr, const int32_t *cidx,
                           const int32_t *vptr, const int32_t *vedge,
                           const int32_t *vchk, const int32_t *vpos,
                           const int8_t *cbucket, int32_t n, int32_t nc,
                           int32_t ne, int32_t nbucket, int32_t nblk,
                           int32_t iters, const float *llr, const float *alpha,
                           const float *beta, const void *records, float *gtot,
                           float *galpha, float *gbeta, float *work,
                           void *stream);

/* NUC max-log soft demapper with the bit de-interleaver in its epilogue.
 * cells: (nblk, ld_cells) complex64 as interleaved float pairs.
 * pts: 3*M floats: Re p, Im p, |p|^2 (float32, |p|^2 rounded once from
 *   float64), M = 2^nbits, label order (y0 = MSB).
 * The point metric is |p|^2 - 2(Re z Re p + Im z Im p) in float32 in the
 * operation order of lab/m44_ldm.py:2431-2451, per-bit minima, then
 * (min_{b=1} - min_{b=0}) / sigma2 with IEEE division.
 * sigma_mode 0: one sigma2 for all cells (sigma2_scalar);
 *            1: one per cell, sigma2 = device (nblk, ld_sigma) float32
 *               (the lab/m9_fast.py:1096-1115 convention);
 *            2: one per block row, sigma2 = device (nblk,) float32;
 *            3: raw minima difference, no division.
 * lam_of_q (nullable, device int32 (ncell*nbits)): write the LLR of q_j to
 *   out[lam_of_q[j]] (codeword order); null writes q order.
 * out: (nblk, ld_out) float32. */
int32_t atsc3_demap(const float *cells, int64_t ld_cells, int32_t nblk,
                    int32_t ncell, const float *pts, int32_t nbits,
                    int32_t sigma_mode, const float *sigma2, int64_t ld_sigma,
                    float sigma2_scalar, const int32_t *lam_of_q, float *out,
                    int64_t ld_out, void *stream);

/* Time de-interleave fused into the demapper's load (csrc/timeint.cu):
 * demaps FEC Block b's cell s from the received PLP cell stream `cells`
 * (ncells complex64) at its source position, without writing the
 * de-interleaved cells; otherwise as atsc3_demap (bit de-interleaver through
 * lam_of_q, LLRs into out).  gather_mode:
 *   0: src_index (nblk, ncell) int32 source positions (-1: no cell) -- any
 *      map, e.g. a hybrid TI block with virtual FEC Blocks;
 *   1: hybrid TI, twisted block de-interleaver without virtual Blocks
 *      (replaces lab/m6_tbi.py:75-88 fec_block and its cached gather
 *      lab/m9_fast.py:1087-1093): p0 = stream offset, p1 = Nc (FEC Blocks
 *      per TI block), p2 = per_ti (cells per TI block); ncell = Nr;
 *      block b = TI block b / Nc, FEC Block b mod Nc;
 *   2: convolutional TI (replaces lab/m10_cti.py:126-141 deinterleave):
 *      p0 = C (pre-CTI position of the first FEC Block's first cell),
 *      p1 = Nrows, p2 = start_row.
 * sigma_mode: 0 scalar, 1 per received cell (indexed like cells), 2 per FEC
 * Block.  A cell whose source lies outside [0, ncells) is an erasure (LLR 0). */
int32_t atsc3_demap_gather(const float *cells, int64_t ncells, int32_t nblk,
                           int32_t ncell, const float *pts, int32_t nbits,
                           int32_t gather_mode, const int32_t *src_index,
                           int64_t p0, int64_t p1, int64_t p2,
                           int32_t sigma_mode, const float *sigma2,
                           float sigma2_scalar, const int32_t *lam_of_q,
                           float *out, int64_t ld_out, void *stream);

/* Per-row noise estimate of lab/m44_ldm.py:2480 / lab/m16_demap_fast.py:104:
 * sigma2[b] = max(mean_cells(|z|^2 + min_p metric), 1e-9), accumulated in
 * float64 (tolerance parity, not bit parity, with the numpy float32 mean). */
int32_t atsc3_demap_row_sigma2(const float *cells, int64_t ld_cells,
                               int32_t nblk, int32_t ncell, const float *pts,
                               int32_t nbits, float *sigma2, void *stream);

/* Float64 demapper: the same max-log LLRs in double arithmetic, replacing
 * the reference's default float64 `demap_llr_fast` (lab/m16_demap_fast.py:
 * 80-119: m = |p|^2 - 2 Re(y p*), per-bit minima, (a - b) / sigma2).
 * cells: (nblk, ld_cells) complex128 as (re, im) double pairs, 16-byte
 * aligned; pts: 3*M doubles (Re, Im, |p|^2); sigma_mode 0 scalar, 1 per
 * cell, 2 per row (sigma2 from atsc3_demap_row_sigma2_f64, the
 * lab/m16_demap_fast.py:104-106 estimate); lam_of_q nullable (q order). */
int32_t atsc3_demap_f64(const double *cells, int64_t ld_cells, int32_t nblk,
                        int32_t ncell, const double *pts, int32_t nbits,
                        int32_t sigma_mode, const double *sigma2,
                        int64_t ld_sigma, double sigma2_scalar,
                        const int32_t *lam_of_q, double *out, int64_t ld_out,
                        void *stream);
int32_t atsc3_demap_row_sigma2_f64(const double *cells, int64_t ld_cells,
                                   int32_t nblk, int32_t ncell,
                                   const double *pts, int32_t nbits,
                                   double *sigma2, void *stream);

/* BCH zero-syndrome check (A/322 6.1.2.1) plus descramble of the payload.
 * hard: (nblk, ld_hard) packed hard decisions (as atsc3_ldpc_decode_flood
 *   writes them); the first kldpc bits are the BCH codeword.
 * rtab: device (kldpc, 6) uint32, row pos = x^(kldpc-1-pos) mod g(x).
 * syn: (nblk, 6) uint32 remainder words (word w = coefficients 32w..).
 * ok: (nblk,) uint8, 1 when the syndrome is zero.
 * scr (nullable): kpayload/8 scrambling bytes; payload (nullable):
 *   (nblk, ld_payload) bytes = hard[:kpayload/8] XOR scr (descrambled
 *   Baseband Packet, lab/m9_fast.py:942-949). */
int32_t atsc3_bch_check(const uint8_t *hard, int64_t ld_hard, int32_t nblk,
                        int32_t kldpc, const uint32_t *rtab, uint32_t *syn,
                        uint8_t *ok, const uint8_t *scr, int32_t kpayload,
                        uint8_t *payload, int64_t ld_payload, void *stream);

/* Same syndrome from one byte per bit (lab/m9_accel.py:212-236 input). */
int32_t atsc3_bch_syndrome_bits(const uint8_t *bits, int64_t ld_bits,
                                int32_t nblk, int32_t kldpc,
                                const uint32_t *rtab, uint32_t *syn,
                                void *stream);

/* ---- uneven batches (one launch per stage over mixed codes) ---------------
 * Blocks of different code lengths, rates and constellations decoded
 * together; every per-block array is on the device.  Replaces the per-MODCOD
 * loops of lab/m9_fast.py:1117-1154 / lab/m44_ldm.py:2348-2390 when one
 * frame carries several PLPs.
 * atsc3_demap_batch: block b's cells at cells + 2*cell_off[b] floats, its
 *   alphabet (3*2^nbits[b] floats) at pts + pts_off[b], its de-interleaver
 *   at lq + lq_off[b], LLRs to llr + llr_off[b]; one sigma2 per block;
 *   chunk_blk/chunk_start: one entry per 256-cell chunk (the grid).
 * atsc3_ldpc_batch_prepare: device descriptors of float32 CSR plans built
 *   with one common cluster size (desc: atsc3_ldpc_batch_desc_bytes bytes);
 *   returns that cluster size and the shared bytes per CTA.
 * atsc3_ldpc_batch_decode: one persistent cluster launch; clusters take
 *   blocks from a device queue (counter zeroed before the launch, `order`
 *   lists blocks most-work-first); kernel semantics of ldpc_minsum_f32.
 * atsc3_bch_batch: per-block BCH length and remainder table (rtab +
 *   rtab_off[b] words), descrambled payload to payload + pay_off[b]. */
int32_t atsc3_demap_batch(const float *cells, const int64_t *cell_off,
                          const int32_t *ncell, const int32_t *nbits,
                          const float *pts, const int64_t *pts_off,
                          const float *sigma2, const int32_t *lq,
                          const int64_t *lq_off, float *llr,
                          const int64_t *llr_off, const int32_t *chunk_blk,
                          const int32_t *chunk_start, int32_t nchunks,
                          int32_t max_nbits, void *stream);
int32_t atsc3_ldpc_batch_desc_bytes(int32_t nplans, int64_t *bytes);
int32_t atsc3_ldpc_batch_prepare(const atsc3_ldpc_plan *const *plans,
                                 int32_t nplans, void *desc,
                                 int32_t *cluster_out, int32_t *smem_out);
int32_t atsc3_ldpc_batch_decode(const void *desc, int32_t cluster, int32_t smem,
                                const int32_t *bplan, const int32_t *order,
                                int32_t nblk, const float *llr,
                                const int64_t *llr_off, uint8_t *hard,
                                const int64_t *hard_off, uint8_t *conv,
                                int32_t *its, int32_t *bad, int32_t iters,
                                float alpha, int32_t *counter, int32_t threads,
                                int32_t max_clusters, void *stream);
int32_t atsc3_bch_batch(const uint8_t *hard, const int64_t *hard_off,
                        const int32_t *kldpc, const uint32_t *rtab,
                        const int64_t *rtab_off, const uint8_t *scr,
                        const int32_t *kpay, uint8_t *payload,
                        const int64_t *pay_off, uint32_t *syn, uint8_t *ok,
                        int32_t nblk, void *stream);

/* ---- decode without device allocation -------------------------------------
 * No counterpart in the reference (its decoders allocate through numpy and
 * torch).  For callers that must not allocate device memory on their decode
 * path -- a real-time loop with a fixed memory budget, or a host that only
 * lends the GPU pre-reserved buffers: the demap -> LDPC -> BCH chain of
 * atsc3_demap / atsc3_ldpc_qce_decode (plan_kind 2), atsc3_ldpc_qc_decode
 * (plan_kind 1) or atsc3_ldpc_decode_flood (plan_kind 0) / atsc3_bch_check
 * in one call, with its LLR and hard-decision intermediates in a fixed
 * file-scope device scratch (about 4.3 MB on every GPU that loads the
 * library) instead of caller buffers.  Limit: at most 16 codewords of at most 64800 bits per
 * call (-3 otherwise).  The first call on a device looks up the scratch
 * address: make it before any stream capture.  Calls that overlap on the GPU
 * share the scratch and race.  Arguments mean what they mean for the three
 * calls it chains (sigma_mode 0..2, lam_of_q required, float32 plans);
 * calls no allocator itself (the plan is made at set-up). */
int32_t atsc3_fec_decode_noalloc(
    const void *plan, int32_t plan_kind, const float *cells, int64_t ld_cells,
    int32_t nblk, int32_t ncell, const float *pts, int32_t nbits,
    int32_t sigma_mode, const float *sigma2, int64_t ld_sigma,
    float sigma2_scalar, const int32_t *lam_of_q, int32_t iters, float alpha,
    const uint32_t *rtab, int32_t kldpc, const uint8_t *scr, int32_t kpayload,
    uint8_t *payload, int64_t ld_payload, uint8_t *conv, int32_t *its,
    int32_t *bad, uint32_t *syn, uint8_t *ok, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* ATSC3_FEC_H */
