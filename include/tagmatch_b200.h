/*
 * TagMatch B200 engine: C ABI.
 *
 * Subset matching of 192-bit Bloom filters: every stored filter f carries a
 * set of uint32 keys; a query q returns the keys of every stored f with
 * f & ~q == 0.  Filters and queries are passed as 6 uint32 words; bit p of
 * the filter is bit (p % 32) of word p / 32, i.e. the little-endian image of
 * the reference's 24-byte binary record (bitvector.hh:210-212,
 * test_io.cc:50-68).
 *
 * The reference's interface is the static C++ class in tagmatch.hh:11-37 (a
 * process-wide singleton).  Here the same operations act on an engine
 * handle, and each entry point below names the reference member it
 * replaces.  A C++ facade with the reference's own class and header names
 * (include/tagmatch/tagmatch.hh) is built on top of these calls.
 *
 * Every call returns TM_OK (0) or a negative status; tm_last_error() gives
 * the message of the last failure on that handle.  No call ends the process
 * on a CUDA error (the reference prints and exits, gpu.cu:14-24).
 */
#ifndef TAGMATCH_B200_H
#define TAGMATCH_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TM_OK 0
#define TM_ERR_INVALID (-1)  /* bad argument */
#define TM_ERR_CUDA (-2)     /* CUDA runtime failure */
#define TM_ERR_STATE (-3)    /* call not valid in the current state */
#define TM_ERR_CAPACITY (-4) /* output buffer too small; required size reported */
#define TM_ERR_NOMEM (-5)    /* device or pinned allocation failed */
#define TM_ERR_IO (-6)       /* database file error */
#define TM_ERR_TIMEOUT (-7)  /* a bounded device-side wait expired */
#define TM_ERR_INTERNAL (-8)

#define TM_FILTER_WORDS 6

typedef struct tm_engine tm_engine;

/* Asynchronous completion callback (match_handler::match_done,
 * match_handler.hh:15-22): called exactly once per request on an engine
 * thread.  keys is valid only during the call. */
typedef void (*tm_match_callback)(void *user, uint64_t tag, const uint32_t *keys, uint64_t n_keys);

/* Creates / destroys an engine (the reference's static state).  The
 * engine's first device is the calling thread's current CUDA device at
 * tm_create (one process per GPU: set the device first); device work
 * starts at the first consolidate. */
int tm_create(tm_engine **out);
void tm_destroy(tm_engine *e);
const char *tm_last_error(const tm_engine *e);
const char *tm_version(void);

/* tagmatch::add(const filter_t &, const std::vector<tagmatch_key_t> &) and
 * tagmatch::add(const filter_t &, tagmatch_key_t) -- tagmatch.cc:66-77.
 * Stages keys for a filter until the next consolidate. */
int tm_add(tm_engine *e, const uint32_t filter[TM_FILTER_WORDS], const uint32_t *keys, uint32_t n_keys);
/* Bulk form: n filters [n][6] with keys in CSR form (key_offsets[n + 1]). */
int tm_add_many(tm_engine *e, const uint32_t *filters, uint64_t n, const uint32_t *key_offsets, const uint32_t *keys);
/* tagmatch::remove(const filter_t &, tagmatch_key_t) -- tagmatch.cc:62-64. */
int tm_remove(tm_engine *e, const uint32_t filter[TM_FILTER_WORDS], uint32_t key);

/* tagmatch::get/set_database_filename -- tagmatch.hh:22-23, tagmatch.cc:79-87. */
int tm_set_database_filename(tm_engine *e, const char *name);
const char *tm_get_database_filename(const tm_engine *e);
/* Keep the database in memory instead of the file (default: file, as the
 * reference).  No reference counterpart. */
int tm_set_persistence(tm_engine *e, int on);

/* tagmatch::consolidate(unsigned partition_size, unsigned threads) --
 * tagmatch.cc:92-165.  Merges staged updates into the table, rewrites the
 * database file, runs the GPU partitioner and builds the device table.
 * threads is kept for interface parity (the partitioner runs on the GPU). */
int tm_consolidate(tm_engine *e, uint32_t partition_size, uint32_t threads);
/* tagmatch::consolidate() with the stored parameters (default 1000, 1). */
int tm_consolidate_default(tm_engine *e);

/* tagmatch::start(unsigned threads, unsigned gpu_count) -- tagmatch.cc:179-186.
 * Replicates the table on gpu_count devices and starts the asynchronous
 * matcher.  Re-entrant. */
int tm_start(tm_engine *e, uint32_t threads, uint32_t gpu_count);
/* tagmatch::stop() -- tagmatch.cc:188-191, front_end.cc:693-771.  Flushes
 * every pending asynchronous request (all callbacks have fired on return).
 * Re-entrant. */
int tm_stop(tm_engine *e);
/* tagmatch::clear() -- tagmatch.cc:193-198. */
int tm_clear(tm_engine *e);
/* tagmatch::get/set_latency_limit_ms -- tagmatch.cc:166-168,
 * front_end.cc:555-561: a pending asynchronous batch older than this is
 * flushed; 0 means batches go out only when full or at stop(). */
int tm_set_latency_limit_ms(tm_engine *e, uint32_t ms);
uint32_t tm_get_latency_limit_ms(const tm_engine *e);
/* Largest number of queries per device batch (default 65536).  tm_match_batch
 * uses smaller batches when their results would exceed about 2^30 keys (from
 * the keys per query of its previous batch), so result copies keep pace. */
int tm_set_batch_limit(tm_engine *e, uint32_t queries);

/* tagmatch::match / tagmatch::match_unique (tagmatch.cc:200-210) for a
 * whole batch, synchronously.  queries: n [n][6] words.  out_offsets:
 * n + 1 entries; the keys of query i are out_keys[out_offsets[i] ..
 * out_offsets[i + 1]).  unique = 0: every key of every matching filter
 * (test_matcher.cc:74-81 order is not kept; the multiset is); unique != 0:
 * each query's keys sorted ascending without duplicates
 * (tagmatch_query.hh:99-119).  If capacity is too small, returns
 * TM_ERR_CAPACITY with the required key count in *n_keys (offsets are
 * complete).  Requires a consolidated table.  Host buffers may be pageable;
 * a pinned out_keys (cudaHostAlloc / cudaHostRegister) also receives part of
 * the keys by direct DMA. */
int tm_match_batch(tm_engine *e, const uint32_t *queries, uint64_t n, int unique, uint64_t *out_offsets,
                   uint32_t *out_keys, uint64_t capacity, uint64_t *n_keys);

/* Device-resident form on the engine's first device (the CUDA device that
 * was current at tm_create): queries, results and stream are device
 * objects.  *d_offsets / *d_keys point into engine-owned device memory
 * valid until the next match call on this engine. */
int tm_match_batch_device(tm_engine *e, const uint32_t *d_queries, uint32_t n, int unique, const uint64_t **d_offsets,
                          const uint32_t **d_keys, uint64_t *n_keys, void *stream);

/* No counterpart in the reference.  tm_match_batch_device without any device
 * allocation, for callers that cannot call cudaMalloc while matching (a
 * pool allocator owns the device memory, a serving thread cannot afford the
 * device synchronisation an allocation may cause, or the CUDA allocator may
 * not be entered where they run).  Every scratch buffer comes from one
 * static device array of 64 MiB that each GPU loading this library holds
 * until exit.  d_queries, d_out_offsets (n + 1 entries) and d_out_keys
 * (capacity keys) are device memory owned by the caller; results are as in
 * tm_match_batch.  Limits: n <= 4096 queries, tables of <= 16384
 * partitions, and the call's scratch within the array -- otherwise
 * TM_ERR_INVALID or TM_ERR_CAPACITY with a message saying what to split.
 * The array is shared by all calls and keeps the last call's contents:
 * calls whose work overlaps on the GPU (other threads, unordered streams)
 * race.  The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress); make it before any stream capture. */
int tm_match_batch_device_noalloc(tm_engine *e, const uint32_t *d_queries, uint32_t n, int unique,
                                  uint64_t *d_out_offsets, uint32_t *d_out_keys, uint64_t capacity, uint64_t *n_keys,
                                  void *stream);

/* tagmatch::match / match_unique with a handler (tagmatch.cc:200-210,
 * front_end.cc:540-551): queues one query; cb(user, tag, keys, n) fires
 * once, on an engine thread, after the query's batch completes. */
int tm_match_async(tm_engine *e, const uint32_t query[TM_FILTER_WORDS], int unique, uint64_t tag, tm_match_callback cb,
                   void *user);

/* Serving: a request of n queries [n][6] matched asynchronously; cb fires
 * once, on an engine thread, with the request's results (offsets[n + 1]
 * relative to keys) and a status.  Requests pending together are matched
 * in shared device batches (see tm_set_flush_mode).  Extends tm_match_async
 * (front_end.cc:540-551) from one query to a request. */
typedef void (*tm_request_callback)(void *user, uint64_t tag, const uint64_t *offsets, const uint32_t *keys,
                                    uint32_t n_queries, int status);
int tm_submit(tm_engine *e, const uint32_t *queries, uint32_t n, int unique, uint64_t tag, tm_request_callback cb,
              void *user);

/* When pending asynchronous work goes to the device:
 * TM_FLUSH_FULL_OR_LATENCY (default): a full batch (tm_set_batch_limit),
 *   the latency limit, or stop() -- the reference front end's rule
 *   (front_end.cc:325-376, 563-598);
 * TM_FLUSH_IMMEDIATE: whenever one of the device's two lanes is free, all
 *   pending requests (up to the batch limit and the memory budget) form the
 *   next batch -- continuous batching;
 * TM_FLUSH_SINGLE: one request per device batch on one lane (the plain
 *   batched path, for comparison);
 * TM_FLUSH_LEARNED: continuous batching whose flush points come from the
 *   learned cost model (tm_sched_train): a free lane takes the pending
 *   requests once they make a batch that keeps up with the measured
 *   arrival rate (the two lanes' queries over the batch's predicted time
 *   >= 1.25 x the rate), or once the oldest one's wait plus the batch's predicted time
 *   reaches half the latency target (tm_set_latency_target_ms); each batch
 *   also runs at the tiles per work item with the lowest predicted time
 *   (32 .. 8,192), so the model should be trained on samples recorded at
 *   several of those values; before training it behaves as
 *   TM_FLUSH_IMMEDIATE. */
#define TM_FLUSH_FULL_OR_LATENCY 0
#define TM_FLUSH_IMMEDIATE 1
#define TM_FLUSH_SINGLE 2
#define TM_FLUSH_LEARNED 3
int tm_set_flush_mode(tm_engine *e, int mode);
/* Where tm_submit's results go (no reference counterpart; the reference
 * always returns keys to the host, back_end.cc:288-302):
 * TM_RESULTS_HOST (default): offsets and keys in host memory;
 * TM_RESULTS_DEVICE: offsets in host memory, keys left in device memory --
 *   the callback's keys argument is a device pointer on the engine's first
 *   device, valid only until the callback returns (copy or consume it
 *   before returning).  Only whole requests with a request callback; a
 *   request split over batches still gets host keys. */
#define TM_RESULTS_HOST 0
#define TM_RESULTS_DEVICE 1
int tm_set_serving_results(tm_engine *e, int where);
/* Device-memory budget per lane for a batch's queues, hit records and keys; the
 * number of queries admitted into one batch is capped by it (estimated
 * from the bytes per query of recent batches).  Default 16 GiB. */
int tm_set_memory_budget(tm_engine *e, uint64_t bytes);

/* partitioning::balanced_partitioning(fib, masks) -- partitioning.cc:361-411,
 * run by the GPU partitioner.  filters: n unique filters [n][6].
 * partition_of[i] receives filter i's partition id; masks[p][6] the AND of
 * partition p's members (all ones for an empty partition); sizes[p] its
 * member count.  Partition ids follow the filters' position after the
 * splits.  Returns TM_ERR_CAPACITY with the count in *n_partitions when
 * capacity partitions do not fit. */
int tm_balanced_partitioning(const uint32_t *filters, uint64_t n, uint32_t max_p, uint32_t *partition_of,
                             uint32_t *masks, uint32_t *sizes, uint64_t capacity, uint64_t *n_partitions);

/* Autotuner (no reference counterpart): matches the n sample queries
 * [n][6] on the engine's first device with each candidate number of tiles per work item
 * (32..8,192) and device batch size (8,192..262,144, at most n), timed with
 * CUDA events, and keeps the fastest for this engine.  Reports the chosen
 * values and the sample's queries/s.  Results do not depend on either. */
int tm_autotune(tm_engine *e, const uint32_t *queries, uint32_t n, uint32_t *seg_tiles, uint32_t *batch_limit,
                double *queries_per_s);

/* Learned scheduler (no reference counterpart; the reference flushes a
 * partition queue when it is full or older than the latency limit,
 * front_end.cc:325-376, 563-598).  A cost model, an 8 -> 64 -> 64 -> 1 fp32
 * MLP trained on the GPU by the library's own kernels, predicts the log of a
 * subset-test work item's warp-cycles from: partition size, partition mask
 * popcount, queries queued for the partition, queries in the item, tiles in
 * the item, recent match density of the partition, filters per tile, tiles
 * per work item.
 *
 * tm_sched_record: while on, every batch the engine matches records its
 *   work items' timings as samples (features [8] + log warp-cycles).
 * tm_sched_samples: copies up to capacity samples (features [n][8],
 *   log_cycles [n]; either may be null) and reports the count in *n.
 * tm_sched_train: trains the model on all samples (mini-batch Adam, 90/10
 *   train/validation split), then derives its decisions: the partition
 *   order of the work queue and the predicted batch times that set the
 *   learned flush points.  Errors are on standardised log-cycles.
 * tm_sched_use_order: on = work queue in descending predicted item cost;
 *   off = partition id order (the static fallback).  Results never depend on
 *   the order.
 * tm_sched_predict_batch_ms: predicted device time of a batch of n queries.
 * tm_set_latency_target_ms: the p99 latency the learned flush points aim
 *   at (default 25 ms). */
typedef struct {
    uint64_t samples, steps;
    double train_mse, val_mse, val_r2, mean_mse, ms;
} tm_sched_report;
int tm_sched_record(tm_engine *e, int on);
int tm_sched_samples(tm_engine *e, float *features, float *log_cycles, uint64_t capacity, uint64_t *n);
int tm_sched_train(tm_engine *e, uint32_t epochs, tm_sched_report *report);
int tm_sched_use_order(tm_engine *e, int on);
int tm_sched_predict_batch_ms(tm_engine *e, uint32_t queries, double *ms);
int tm_set_latency_target_ms(tm_engine *e, uint32_t ms);
/* The cost model's kernels on caller data (for checking them): outputs
 * [n], the gradient of the mean squared error over the n samples with
 * respect to all tm_mlp_param_count() parameters (layout: W1 [64][8], b1
 * [64], W2 [64][64], b2 [64], W3 [64], b3), and the loss.  Runs on the
 * current CUDA device. */
uint32_t tm_mlp_param_count(void);
int tm_mlp_loss_grad(const float *params, const float *features, const float *targets, uint32_t n, float *outputs,
                     float *grad, float *loss);

/* Tiles per work item of the subset test (what tm_autotune chooses;
 * default 128): each work item is a group of four consecutive 256-query
 * chunks of a partition against this many of its tiles (up to 32 filters
 * each).  No reference counterpart.  Results do not depend on it. */
int tm_set_tiles_per_item(tm_engine *e, uint32_t seg_tiles);
uint32_t tm_get_tiles_per_item(const tm_engine *e);

/* Table statistics after consolidate. */
typedef struct {
    uint64_t filters;
    uint64_t keys;
    uint64_t partitions;
    uint64_t tiles;
    uint64_t device_bytes;
    uint32_t max_key;
} tm_table_info;
int tm_get_table_info(tm_engine *e, tm_table_info *info);

/* Cumulative statistics of the synchronous matcher: batches, queries,
 * routed (query, partition) pairs, work items, matching (query, filter)
 * pairs, output keys, hit-record buffer regrowths; with profiling on, the
 * subset-test kernel's launches and total time from CUDA events recorded
 * on its stream.  No reference counterpart (front_end::print_statistics,
 * front_end.cc:781-789, is the closest). */
typedef struct {
    uint64_t batches, queries, routed, items, pairs, keys;
    uint64_t pair_retries;
    uint64_t match_kernel_launches;
    double match_kernel_ms;
    uint64_t dense_tests; /* sum over batches and partitions of routed queries x partition size */
    uint64_t kernel_launches; /* all kernels launched by the matcher */
    uint64_t h2d_bytes, d2h_bytes; /* bytes copied by tm_match_batch (keys travel as 16 bits
                                      when every key of the table is below 65,536) */
    uint64_t records; /* hit records written by the subset test: one per (query, tile of up to
                         32 filters) with at least one match, 16 bytes each */
} tm_match_stats;
int tm_get_match_stats(tm_engine *e, tm_match_stats *st);
int tm_reset_match_stats(tm_engine *e);
/* Turns CUDA-event timing of the subset-test kernel on or off. */
int tm_set_profiling(tm_engine *e, int on);

#ifdef __cplusplus
}
#endif

#endif /* TAGMATCH_B200_H */
