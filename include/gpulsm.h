/*
 * gpulsm.h - C ABI of the B200-native GPU dictionary.
 *
 * Drop-in boundary for the GPU dictionary hot path of the reference project:
 *   - gpulsm_dict_*  replaces class GPULSMOpt (GPULSMOpt.cuh:5599-5881) and
 *                    its adapter structs (gpu_dictionary_adapter.cuh:16-49);
 *   - gpulsm_flix_*  replaces the FliX bucket layer, class
 *                    cg_rtx_index_updates (FliX/impl_cg_rtx_index_updates.cuh:1711-2677).
 *
 * Conventions (same as the reference):
 *   - every key/value/output pointer is a DEVICE pointer owned by the caller;
 *     the library never frees it;
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default
 *     stream); calls enqueue work asynchronously and return;
 *   - operations on one handle are serialised internally (a mutex plus an
 *     event that orders work issued on different streams), as the reference
 *     does with operation_mutex_ / operation_done_ (GPULSMOpt.cuh:6852-6858);
 *   - every call returns a gpulsm_status; on failure gpulsm_last_error()
 *     returns the message (the reference throws instead).
 */
#ifndef GPULSM_H
#define GPULSM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum gpulsm_status {
  GPULSM_OK = 0,
  GPULSM_ERR_INVALID_ARGUMENT = 1, /* reference: std::invalid_argument */
  GPULSM_ERR_CAPACITY = 2,         /* reference: runtime_error "...capacity exhausted..." */
  GPULSM_ERR_PUBLICATION = 3,      /* reference: runtime_error "publication failed" */
  GPULSM_ERR_TIMEOUT = 4,          /* a bounded device wait gave up (no reference equivalent) */
  GPULSM_ERR_CUDA = 5,             /* reference: runtime_error from CUDA_CHECK */
  GPULSM_ERR_OUT_OF_MEMORY = 6,    /* reference: std::bad_alloc */
  GPULSM_ERR_LENGTH = 7            /* reference: std::length_error */
} gpulsm_status;

/* Status bits of gpulsm_dict_status(); bit 3 has the meaning of
 * kPublicationOutputOverflow (GPULSMOpt.cuh:535-541). */
#define GPULSM_STATUS_OUTPUT_OVERFLOW (1u << 3)
#define GPULSM_STATUS_WAIT_TIMEOUT (1u << 8)
#define GPULSM_STATUS_BAD_INPUT (1u << 9)

/* Search structure used inside each sorted level. */
#define GPULSM_SEARCH_DIRECTORY 0u /* radix directory over the level's key range */
#define GPULSM_SEARCH_LEARNED 1u   /* piecewise-linear position model + checked window */
#define GPULSM_SEARCH_BINARY 2u    /* plain binary search over each level (no auxiliary structure) */

/* Message of the last failed call on this thread. */
const char *gpulsm_last_error(void);
/* Library version string. */
const char *gpulsm_version(void);
/* Number of CUDA kernels this library has launched in this process (all
 * handles); a diagnostic so callers can attribute device work to it. */
uint64_t gpulsm_launch_count(void);

/* ===================== LSM dictionary (GPULSMOpt semantics) ============== */
typedef struct gpulsm_dict gpulsm_dict;

/* Mirrors DictionaryConfig (gpu_dictionary_adapter.cuh:16-23) plus tunables. */
typedef struct gpulsm_dict_config {
  uint64_t max_elements;        /* DictionaryConfig::max_elements (live rows incl. tombstones) */
  uint64_t batch_capacity;      /* DictionaryConfig::batch_capacity; 0 -> 2^20, max 2^20 */
  uint64_t level_zero_capacity; /* DictionaryConfig::level_zero_capacity; 0 -> batch * fan_in */
  uint32_t fan_in;              /* merge fan-in between levels, 2..16; 0 -> 4 */
  uint32_t rows_per_bucket_log2;/* directory density; 0 -> 3 (about 8 rows per bucket) */
  uint32_t search_mode;         /* GPULSM_SEARCH_* */
  uint32_t reserved;
} gpulsm_dict_config;

/* GPULSMOpt::GPULSMOpt(const DictionaryConfig&)  GPULSMOpt.cuh:5606 */
int gpulsm_dict_create(const gpulsm_dict_config *config, gpulsm_dict **out);
/* GPULSMOpt::~GPULSMOpt  GPULSMOpt.cuh:5689 */
int gpulsm_dict_destroy(gpulsm_dict *dict);
/* GPULSMOpt::clear  GPULSMOpt.cuh:5731 */
int gpulsm_dict_clear(gpulsm_dict *dict, void *stream);
/* No GPULSMOpt counterpart (its updates complete in the caller's stream):
 * makes `stream` wait until every update enqueued so far has been merged.
 * insert/erase return once their batch is admitted (its input has been read
 * in `stream`'s order); the merges run on the dictionary's own stream while
 * the next batch is admitted.  Every read operation joins by itself; join is
 * for callers that time or order updates against their own work. */
int gpulsm_dict_join(gpulsm_dict *dict, void *stream);
/* GPULSMOpt::bulk_build  GPULSMOpt.cuh:5738 (last duplicate wins) */
int gpulsm_dict_bulk_build(gpulsm_dict *dict, const uint32_t *keys, const uint32_t *values,
                           uint64_t count, void *stream);
/* GPULSMOpt::insert(DeviceKeyValueBatch)  GPULSMOpt.cuh:5836 (upsert, last input index wins) */
int gpulsm_dict_insert(gpulsm_dict *dict, const uint32_t *keys, const uint32_t *values,
                       uint64_t count, void *stream);
/* GPULSMOpt::erase(DeviceKeyBatch)  GPULSMOpt.cuh:5843 (tombstones) */
int gpulsm_dict_erase(gpulsm_dict *dict, const uint32_t *keys, uint64_t count, void *stream);
/* No GPULSMOpt counterpart (its batches are either inserts or erases): one
 * batch of both.  Row i erases keys[i] when erase[i] is nonzero, else inserts
 * (keys[i], values[i]); for a key given more than once the last row wins, as
 * within an insert or erase batch.  Equals inserting and erasing the rows one
 * at a time in input order. */
int gpulsm_dict_update(gpulsm_dict *dict, const uint32_t *keys, const uint32_t *values, const uint8_t *erase,
                       uint64_t count, void *stream);
/* GPULSMOpt::lookup(DeviceLookupBatch)  GPULSMOpt.cuh:5850; out_found may be NULL.
 * Miss: out_values = out_found ? 0 : 0xffffffff (GPULSMOpt.cuh:4742-4749). */
int gpulsm_dict_lookup(gpulsm_dict *dict, const uint32_t *queries, uint64_t count,
                       uint32_t *out_values, uint8_t *out_found, void *stream);
/* GPULSMOpt::range(DeviceRangeOutputBatch)  GPULSMOpt.cuh:5858: u32 sum of live
 * values with lo <= key <= hi, wrapping at 2^32; lo > hi gives 0. */
int gpulsm_dict_range_sum(gpulsm_dict *dict, const uint32_t *lo, const uint32_t *hi,
                          uint64_t count, uint32_t *out_sums, void *stream);
/* Live-key count per range (the "range count" of LSMu count, FliX/impl_lsm_tree.cuh:1208). */
int gpulsm_dict_range_count(gpulsm_dict *dict, const uint32_t *lo, const uint32_t *hi,
                            uint64_t count, uint32_t *out_counts, void *stream);
/* Range query returning pairs, step 1: offsets[count+1] (device, u64) = exclusive
 * scan of the live counts; offsets[count] is the total number of pairs. */
int gpulsm_dict_range_offsets(gpulsm_dict *dict, const uint32_t *lo, const uint32_t *hi,
                              uint64_t count, uint64_t *offsets, void *stream);
/* Step 2: writes each range's live (key, value) pairs in key order at
 * out_keys/out_values[offsets[i] ...]; offsets must come from step 1 with no
 * update in between. No counterpart in GPULSMOpt (it only sums). */
int gpulsm_dict_range_pairs(gpulsm_dict *dict, const uint32_t *lo, const uint32_t *hi,
                            uint64_t count, const uint64_t *offsets, uint32_t *out_keys,
                            uint32_t *out_values, void *stream);
/* GPULSMOpt::successor(DeviceSuccessorBatch)  GPULSMOpt.cuh:5865: smallest live
 * key >= query, else 0xffffffff. */
int gpulsm_dict_successor(gpulsm_dict *dict, const uint32_t *queries, uint64_t count,
                          uint32_t *out_keys, void *stream);
/* GPULSMOpt::canonical_carry_status  GPULSMOpt.cuh:5872 (synchronises). */
int gpulsm_dict_status(gpulsm_dict *dict, uint32_t *out_status);
/* GPULSMOpt::gpu_resident_bytes  GPULSMOpt.cuh:6341 */
int gpulsm_dict_resident_bytes(gpulsm_dict *dict, uint64_t *out_bytes);
/* LSMu cleanup  FliX/impl_lsm_tree.cuh:1256-1400 (no GPULSMOpt counterpart):
 * merges every level into one run that keeps only the newest live version of
 * each key (tombstones and shadowed versions dropped, as
 * lsm_mark_cleanup_survivors_kernel :485-500 keeps the first regular entry of
 * each key segment) and returns the live key count; synchronises.  Answers are
 * unchanged; later reads search one level. */
int gpulsm_dict_cleanup(gpulsm_dict *dict, void *stream, uint64_t *out_live_keys);
/* Number of live rows (synchronises; diagnostics). */
int gpulsm_dict_size(gpulsm_dict *dict, uint64_t *out_rows, uint32_t *out_levels);
/* Measurement hook (no reference counterpart): while enabled, every merge
 * kernel launch is bracketed by CUDA events on its stream and records the
 * rows it read and wrote.  _read (synchronises) returns, over the merges
 * timed since the previous read, the launch count, the summed device time in
 * ms and the algorithmic bytes (9 B per row read, 9 B per row written, 4 B
 * per directory entry written; the merges of an update that follows another
 * update leave their output's directory to the first read that needs it). */
int gpulsm_dict_kernel_timing(gpulsm_dict *dict, int enable);
int gpulsm_dict_kernel_timing_read(gpulsm_dict *dict, uint64_t *out_launches, double *out_ms,
                                   double *out_bytes);

/* ===================== FliX bucket layer ================================== */
typedef struct gpulsm_flix gpulsm_flix;

typedef struct gpulsm_flix_config {
  uint32_t key_bits;     /* 32 or 64 (key32 / key64, FliX/definitions.cuh:74-77) */
  uint32_t node_size;    /* entries per node; 0 -> 32 (NODESIZE=5) */
  uint32_t fill_percent; /* initial fill of build nodes; 0 -> 50 */
  uint32_t search_mode;  /* GPULSM_SEARCH_* for unsorted probes */
  uint64_t max_elements; /* capacity hint for the allocation region */
} gpulsm_flix_config;

int gpulsm_flix_create(const gpulsm_flix_config *config, gpulsm_flix **out);
int gpulsm_flix_destroy(gpulsm_flix *index);
/* build_bucket_layer_only  FliX/impl_cg_rtx_index_updates.cuh:1711; values NULL
 * -> value = input index (the reference's offsets). keys are u32 or u64 per key_bits. */
int gpulsm_flix_build(gpulsm_flix *index, const void *keys, const uint32_t *values,
                      uint64_t count, uint64_t max_count, void *stream);
/* insert  FliX/impl_cg_rtx_index_updates.cuh:2195 (insert if absent). Unlike the
 * reference, the batch may be unsorted and hold duplicates (first one applies). */
int gpulsm_flix_insert(gpulsm_flix *index, const void *keys, const uint32_t *values,
                       uint64_t count, void *stream);
/* remove  FliX/impl_cg_rtx_index_updates.cuh:2253 (physical delete, any order). */
int gpulsm_flix_remove(gpulsm_flix *index, const void *keys, uint64_t count, void *stream);
/* lookups_ordered  FliX/impl_cg_rtx_index_updates.cuh:2485: probes sorted
 * ascending; out[i] = value or 0xffffffff. */
int gpulsm_flix_lookups_ordered(gpulsm_flix *index, const void *sorted_probes, uint64_t count,
                                uint32_t *out_values, void *stream);
/* lookups_successor  FliX/impl_cg_rtx_index_updates.cuh:2647: probes sorted;
 * out = first stored key >= probe, else 0xffffffff zero-extended. */
int gpulsm_flix_lookups_successor(gpulsm_flix *index, const void *sorted_probes, uint64_t count,
                                  void *out_keys, void *stream);
/* Unsorted probes: sort with a permutation, ordered walk, scatter back
 * (the driver protocol of FliX/benchmarks_updates.cuh:252-360 in one call). */
int gpulsm_flix_lookup(gpulsm_flix *index, const void *probes, uint64_t count,
                       uint32_t *out_values, void *stream);
int gpulsm_flix_successor(gpulsm_flix *index, const void *probes, uint64_t count,
                          void *out_keys, void *stream);
/* rebuild_bucket_layer_only  FliX/impl_cg_rtx_index_updates.cuh:1821 */
int gpulsm_flix_rebuild(gpulsm_flix *index, void *stream);
int gpulsm_flix_resident_bytes(gpulsm_flix *index, uint64_t *out_bytes);
int gpulsm_flix_size(gpulsm_flix *index, uint64_t *out_keys);
int gpulsm_flix_status(gpulsm_flix *index, uint32_t *out_status);
/* allocation_buffer_next_free / allocation_buffer_total_nodes
 * FliX/impl_cg_rtx_index_updates.cuh:1690-1700 (synchronises): allocation-region
 * nodes taken by splits, nodes the region holds, head buckets, and how many
 * times the region was grown by a rebuild before a batch that could exhaust it. */
int gpulsm_flix_allocation_state(gpulsm_flix *index, uint64_t *out_used_nodes, uint64_t *out_region_nodes,
                                 uint64_t *out_buckets, uint32_t *out_grows);

/* ===================== multi-tenant batched dictionary ==================== */
/* Many independent u32 dictionaries (GPULSMOpt upsert semantics, inserts and
 * lookups) updated in rounds.  No reference counterpart: the reference would
 * need one GPULSMOpt per tenant, each with its fixed directories
 * (GPULSMOpt.cuh:5640-5702).  A round passes one batch per tenant as CSR:
 * keys/values concatenated in tenant order and offsets[tenants + 1] (u64), all
 * device memory; per-tenant answers equal one GPULSMOpt per tenant. */
typedef struct gpulsm_tenants gpulsm_tenants;
/* capacities: HOST array of per-tenant maximum live keys; max_round_keys bounds
 * one round's total batch; tile (256..4096), fan_in (1..16: rounds gathered in
 * a tenant's delta run before it merges into its main run) and fanout (8, 16,
 * 32: B-ary fence tree) are the tunables, 0 = defaults 2048 / 4 / 16. */
int gpulsm_tenants_create(uint32_t tenants, const uint64_t *capacities, uint64_t max_round_keys, uint32_t tile,
                          uint32_t fan_in, uint32_t fanout, gpulsm_tenants **out);
int gpulsm_tenants_destroy(gpulsm_tenants *pool);
int gpulsm_tenants_set_tuning(gpulsm_tenants *pool, uint32_t tile, uint32_t fan_in, uint32_t fanout);
/* One round: everything sized on the device, no host wait. */
int gpulsm_tenants_insert_round(gpulsm_tenants *pool, const uint32_t *keys, const uint32_t *values,
                                const uint64_t *offsets, void *stream);
/* The same round replayed from a CUDA graph captured once per (buffers, round
 * kind); stream must not be the legacy default stream. */
int gpulsm_tenants_round_graph(gpulsm_tenants *pool, const uint32_t *keys, const uint32_t *values,
                               const uint64_t *offsets, void *stream);
/* (tenant, key) lookups; out_found may be NULL (misses then read 0xffffffff). */
int gpulsm_tenants_lookup(gpulsm_tenants *pool, const uint32_t *tenant_ids, const uint32_t *keys, uint64_t count,
                          uint32_t *out_values, uint8_t *out_found, void *stream);
/* Rows held per tenant (main + delta runs; a key may appear in both), host array. */
int gpulsm_tenants_sizes(gpulsm_tenants *pool, uint64_t *out_rows);
int gpulsm_tenants_status(gpulsm_tenants *pool, uint32_t *out_status);
int gpulsm_tenants_resident_bytes(gpulsm_tenants *pool, uint64_t *out_bytes);

/* ===================== serving loop ======================================== */
/* No reference counterpart: GPULSMOpt serialises every call behind a mutex and
 * an operation event (GPULSMOpt.cuh:6852-6858) and leaves batching to the
 * caller.  A server owns one LSM dictionary and serves lookup / insert / erase
 * / range-sum requests submitted from any host thread with HOST buffers
 * (unlike the dict calls): a worker thread takes what has queued, in arrival
 * order, into a round of at most three dictionary calls (every insert and
 * erase of the round as one update batch, then every lookup and every range
 * sum, the two reads running concurrently), admits updates while the
 * dictionary's resident bytes plus the rounds in flight fit the device
 * budget (an update that cannot fit fails with
 * GPULSM_ERR_CAPACITY), and pipelines rounds through `depth` staging slots.
 * Submit copies the request's keys and values / upper bounds into a pinned
 * ring of the server before it returns (waiting while the ring is full); the
 * output buffers stay the caller's until the request is done.
 * Results equal applying the rounds in order and, inside a round, its updates
 * one at a time in submission order, then its reads - a linearization, since
 * every request of a round is in flight while the round runs
 * (gpulsm_server_wait_round reports each request's round). */
typedef struct gpulsm_server gpulsm_server;

#define GPULSM_SERVE_LOOKUP 0u    /* keys -> out values (miss 0xffffffff), found flags optional */
#define GPULSM_SERVE_INSERT 1u    /* keys, aux = values */
#define GPULSM_SERVE_ERASE 2u     /* keys */
#define GPULSM_SERVE_RANGE_SUM 3u /* keys = lower bounds, aux = upper bounds -> out u32 sums */

typedef struct gpulsm_serve_stats {
  uint64_t completed, rejected, rounds, keys;
  double p50_us, p99_us, max_us, mean_us; /* submit -> results in the caller's buffers */
  double mean_round_keys, wall_s;
  double gpu_busy_s, host_launch_s; /* device time of the rounds; worker time staging + launching */
  uint64_t graph_rounds;            /* lookup-only rounds replayed from a captured CUDA graph */
  double kind_gpu_s[4];             /* device time of each request kind's calls (updates: merges included;
                                       a round's update batch counts as insert, or erase when it only erases;
                                       a round's lookups and range sums run concurrently and count as lookup),
                                       timed on every eighth round and scaled by eight */
  double host_copy_s;               /* submitters' time copying request data into the server's pinned ring */
  double host_scatter_s;            /* completion time copying results into the requests' buffers */
  uint64_t graph_updates;           /* update batches replayed from a captured CUDA graph (staged admission) */
  uint64_t stage_flushes;           /* merges of the staged runs into the levels */
  double max_round_gpu_us;          /* the longest round's device time */
  double max_launch_us;             /* the worker's longest time staging and launching one round */
} gpulsm_serve_stats;

/* Open-loop load: Poisson arrivals at rate_per_s (0 = closed loop with
 * max_outstanding requests in flight) for `seconds`; kind mix (lookup, insert,
 * erase, range-sum); sizes log-uniform in [min_keys, max_keys]; keys drawn by
 * Zipf(zipf_s) rank over `universe` (host array); range widths log-uniform in
 * [1, range_width_max]. */
typedef struct gpulsm_load_spec {
  double rate_per_s, seconds;
  double mix[4];
  double zipf_s;
  uint32_t max_outstanding, min_keys, max_keys, range_width_max;
  uint64_t seed;
  const uint32_t *universe;
  uint64_t universe_n;
} gpulsm_load_spec;

/* budget_bytes: device bytes the dictionary and in-flight rounds may hold;
 * max_round_keys: keys per round (also the largest request), 0 -> 2^20;
 * depth: pipeline slots, 0 -> 3. */
int gpulsm_server_create(const gpulsm_dict_config *config, uint64_t budget_bytes, uint32_t max_round_keys,
                         uint32_t depth, gpulsm_server **out);
int gpulsm_server_destroy(gpulsm_server *server);
/* Preload (device buffers, as gpulsm_dict_bulk_build). */
int gpulsm_server_bulk_build(gpulsm_server *server, const uint32_t *keys, const uint32_t *values, uint64_t count,
                             void *stream);
int gpulsm_server_submit(gpulsm_server *server, uint32_t kind, const uint32_t *keys, const uint32_t *aux,
                         uint64_t count, uint32_t *out, uint8_t *out_found, uint64_t *out_ticket);
/* *out_state: 0 pending, 1 done, -status failed; a finished ticket is collected by this call. */
int gpulsm_server_poll(gpulsm_server *server, uint64_t ticket, int32_t *out_state);
int gpulsm_server_wait(gpulsm_server *server, uint64_t ticket, int32_t *out_state);
/* As wait; *out_round = the request's round, numbered from 1 in execution
 * order (0: completed without one - an empty or rejected request). */
int gpulsm_server_wait_round(gpulsm_server *server, uint64_t ticket, int32_t *out_state, uint64_t *out_round);
int gpulsm_server_drain(gpulsm_server *server);
int gpulsm_server_stats(gpulsm_server *server, gpulsm_serve_stats *out);
int gpulsm_server_reset_stats(gpulsm_server *server);
int gpulsm_server_run_load(gpulsm_server *server, const gpulsm_load_spec *spec, gpulsm_serve_stats *out);
int gpulsm_server_resident_bytes(gpulsm_server *server, uint64_t *out_bytes);
/* How update requests run (no reference counterpart).  0 (the default):
 * direct - each round's update batch is admitted and merged at once and the
 * round waits for the merges.  1: staged - each update batch is admitted into a staging run
 * by one replay of a captured CUDA graph and completes without waiting for
 * merges; the staged runs are the newest levels of point reads and range sums
 * and merge into the levels when the staging slots are full (or before a
 * non-graph update, a range count or a build).  Staged needs max_round_keys
 * <= 2^20.  Waits for the requests in flight; switching to direct merges the
 * staged runs first. */
int gpulsm_server_set_staged_updates(gpulsm_server *server, int staged);

/* ===================== learned position model ============================ */
/* A piecewise-linear CDF over one sorted key array (no reference counterpart:
 * the reference narrows searches with 128-cell rank directories,
 * GPULSMOpt.cuh:4605-4646).  Equal-width key segments (count rounded up to a
 * power of two), fp32 slope/intercept per segment trained on the GPU by
 * forward/backward kernels, exact through a per-segment maximum error.
 * `model` is caller-owned device memory of gpulsm_model_bytes(segments). */
uint64_t gpulsm_model_bytes(uint32_t segments);
/* Fit: interpolation init, `iters` preconditioned gradient steps, error bounds.
 * loss_history (device, iters + 1 floats, may be NULL) = mean squared error. */
int gpulsm_model_fit(const void *sorted_keys, uint64_t count, uint32_t key_bits, uint32_t segments,
                     uint32_t iters, void *model, float *loss_history, void *stream);
/* Gradients of the mean squared error for the current parameters:
 * grad[2s] = dL/da_s, grad[2s+1] = dL/db_s (device, 2 * segments floats). */
int gpulsm_model_gradients(const void *sorted_keys, uint64_t count, uint32_t key_bits, uint32_t segments,
                           void *model, float *grad, float *loss, void *stream);
/* Exact lower bounds (first index with key >= query) through the model. */
int gpulsm_model_lower_bound(const void *sorted_keys, uint64_t count, uint32_t key_bits, uint32_t segments,
                             const void *model, const void *queries, uint64_t query_count, uint64_t *out,
                             void *stream);
/* The same lower bounds by plain binary search (the method without the model). */
int gpulsm_binary_lower_bound(const void *sorted_keys, uint64_t count, uint32_t key_bits, const void *queries,
                              uint64_t query_count, uint64_t *out, void *stream);

/* ===================== building blocks ==================================== */
/* Stable LSD radix sort of (key, u32 value) pairs by key bits [begin_bit, end_bit)
 * (bits outside the range do not affect the order).  key_bits 32 or 64; values
 * may be NULL.  keys_out/values_out receive the result; keys_out may equal
 * keys_in (values_out values_in), a partial overlap of any two buffers is
 * rejected with GPULSM_ERR_INVALID_ARGUMENT.  Allocates its scratch on the
 * stream.  Returns once the sort has finished (it reads the passes' status
 * word back); a device look-back wait that gave up gives GPULSM_ERR_TIMEOUT. */
int gpulsm_sort_pairs(const void *keys_in, const uint32_t *values_in, void *keys_out,
                      uint32_t *values_out, uint64_t count, uint32_t key_bits, uint32_t begin_bit,
                      uint32_t end_bit, void *stream);
/* No counterpart in the reference.  The same sort for callers that must not
 * allocate device memory (e.g. a process whose device memory is owned by
 * another allocator under a fixed budget, or a latency-critical path that
 * cannot risk a blocking or failing allocation): it calls no cudaMalloc,
 * cudaFree or allocating library routine.  Its scratch is one static device
 * array (about 14 MiB, see gpulsm_sort_noalloc_scratch_bytes) that every GPU
 * loading the library holds until exit.  At most 2^20 keys per call; more
 * gives GPULSM_ERR_LENGTH.  All calls on a device share that array, which keeps
 * the previous call's contents (each call clears what must start at zero):
 * calls that overlap on the GPU race, so serialise them.  The first call on a
 * device resolves the array's address - make it before any stream capture.
 * Aliasing, the bit range and the status read-back (the call returns once the
 * sort has finished; GPULSM_ERR_TIMEOUT if a look-back wait gave up) are as
 * for gpulsm_sort_pairs. */
int gpulsm_sort_pairs_noalloc(const void *keys_in, const uint32_t *values_in, void *keys_out,
                              uint32_t *values_out, uint64_t count, uint32_t key_bits, uint32_t begin_bit,
                              uint32_t end_bit, void *stream);
uint64_t gpulsm_sort_noalloc_scratch_bytes(void);

#ifdef __cplusplus
}
#endif
#endif /* GPULSM_H */
