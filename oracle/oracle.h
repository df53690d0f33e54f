/*
 * CPU oracle for the GPU dictionary hot path.  TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load
 * this library.  It is the checker, never the product path: the CUDA library
 * in gpu-lsm-tree_b200/ has no CPU fallback.
 *
 * Two restatements of the reference's semantics, both kept as sorted arrays of
 * unique live keys (the std::map view of the structure):
 *
 *   orc_lsm_*   GPULSMOpt.cuh (class GPULSMOpt, :5599-5881): upsert where the
 *               newest batch and, inside a batch, the highest input index win;
 *               erase writes tombstones; lookups report the newest visible
 *               version; range sums wrap at 2^32; successor returns the first
 *               live key >= the query or 0xffffffff.
 *   orc_flix_*  FliX bucket layer (FliX/impl_cg_rtx_index_updates.cuh:1711-2677):
 *               insert-if-absent, physical delete, 32- or 64-bit keys, values
 *               are u32 "offsets", misses are not_found (0xffffffff), the
 *               successor miss is not_found zero-extended to the key width.
 *
 * Every batch operation applies the whole batch as the reference does; the
 * per-function comments in lsm_oracle.c / flix_oracle.c cite the reference
 * file:line each rule follows.
 */
#ifndef GPULSM_ORACLE_H
#define GPULSM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Threads used by the parallel loops (0 = all available). Returns the count in use. */
int orc_set_threads(int threads);
int orc_get_threads(void);

/* ---- GPULSMOpt semantics ---------------------------------------------- */
typedef struct orc_lsm orc_lsm;
orc_lsm *orc_lsm_create(void);
void orc_lsm_destroy(orc_lsm *d);
void orc_lsm_clear(orc_lsm *d);
uint64_t orc_lsm_size(const orc_lsm *d);
/* Copies the live (key, value) pairs in key order; returns the count. */
uint64_t orc_lsm_dump(const orc_lsm *d, uint32_t *keys, uint32_t *values);
void orc_lsm_bulk_build(orc_lsm *d, const uint32_t *keys, const uint32_t *values, uint64_t n);
void orc_lsm_insert(orc_lsm *d, const uint32_t *keys, const uint32_t *values, uint64_t n);
void orc_lsm_erase(orc_lsm *d, const uint32_t *keys, uint64_t n);
/* out_found may be NULL: misses then read 0xffffffff, else 0 with found=0. */
void orc_lsm_lookup(const orc_lsm *d, const uint32_t *queries, uint64_t n,
                    uint32_t *out_values, uint8_t *out_found);
void orc_lsm_range_sum(const orc_lsm *d, const uint32_t *lo, const uint32_t *hi,
                       uint64_t n, uint32_t *out_sums);
void orc_lsm_range_count(const orc_lsm *d, const uint32_t *lo, const uint32_t *hi,
                         uint64_t n, uint32_t *out_counts);
/* offsets[n+1] = exclusive scan of the per-query live counts (computed here). */
uint64_t orc_lsm_range_offsets(const orc_lsm *d, const uint32_t *lo, const uint32_t *hi,
                               uint64_t n, uint64_t *offsets);
void orc_lsm_range_pairs(const orc_lsm *d, const uint32_t *lo, const uint32_t *hi,
                         uint64_t n, const uint64_t *offsets, uint32_t *out_keys,
                         uint32_t *out_values);
void orc_lsm_successor(const orc_lsm *d, const uint32_t *queries, uint64_t n,
                       uint32_t *out_keys);

/* ---- FliX semantics ---------------------------------------------------- */
typedef struct orc_flix orc_flix;
/* key_bits is 32 or 64; keys are passed as u64 either way. */
orc_flix *orc_flix_create(int key_bits);
void orc_flix_destroy(orc_flix *f);
uint64_t orc_flix_size(const orc_flix *f);
uint64_t orc_flix_dump(const orc_flix *f, uint64_t *keys, uint32_t *values);
/* values = NULL means "value = input index" (build_bucket_layer_only). */
void orc_flix_build(orc_flix *f, const uint64_t *keys, const uint32_t *values, uint64_t n);
void orc_flix_insert(orc_flix *f, const uint64_t *keys, const uint32_t *values, uint64_t n);
void orc_flix_remove(orc_flix *f, const uint64_t *keys, uint64_t n);
void orc_flix_lookup(const orc_flix *f, const uint64_t *probes, uint64_t n, uint32_t *out);
void orc_flix_successor(const orc_flix *f, const uint64_t *probes, uint64_t n, uint64_t *out);

/* ---- learned position model (restated for gradient checks) ------------ */
void orc_model_gradients(const uint64_t *keys, uint64_t n, uint64_t kmin, uint32_t shift, uint32_t nseg,
                         const float *a, const float *b, double *ga, double *gb, double *loss);

#ifdef __cplusplus
}
#endif
#endif
