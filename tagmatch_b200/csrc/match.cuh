// Batched matching on one device: routing, per-partition queues, the
// subset-test kernel, key gather and match_unique de-duplication.
#pragma once
#include <cstdint>
#include "partition.cuh"

namespace tmb {

constexpr int kSegTiles = 128;  // default tiles per work item (tm_autotune may change it)

// Device scratch for one in-flight batch (grow-only).
struct MatchScratch {
    DevBuf<uint32_t> queries;     // [nq][6] staged host input
    DevBuf<uint32_t> part_count;  // [P]
    DevBuf<uint32_t> part_off;    // [P + 1]
    DevBuf<uint32_t> part_cursor; // [P]
    DevBuf<uint32_t> queue;       // [routed][8]
    DevBuf<uint32_t> item_off;    // [P + 1] work items per partition (prefix)
    DevBuf<uint32_t> chunk_off;   // [P + 1] 256-query chunks per partition (prefix)
    DevBuf<uint32_t> slices;      // [chunks][192][8] bit-sliced "lacks bit" masks
    DevBuf<unsigned long long> work;  // optional kernel work counters
    DevBuf<uint16_t> keys16;          // keys narrowed for the host transfer
    DevBuf<unsigned long long> counters;  // [0] work item, [1] hit records, [2] error flags, [3] pairs
    DevBuf<HitRec> recs;          // hit records of the subset test
    DevBuf<uint32_t> qkeys;       // [nq]
    DevBuf<uint64_t> qoff;        // [nq + 1]
    DevBuf<uint32_t> qcursor;     // [nq]
    DevBuf<uint32_t> keys;        // [total keys] grouped by query
    DevBuf<uint32_t> ucount;      // [nq]
    DevBuf<uint64_t> uoff;        // [nq + 1]
    DevBuf<uint32_t> ukeys;       // [total unique] (also radix temp)
    MappedBuf<uint32_t> readback; // small device results read by the host (k_readback)
    std::vector<uint32_t> h_part_count, h_chunk_off, h_item_off;
    // work-queue order of the partitions (empty: id order); set by the
    // engine from the learned cost model
    std::vector<uint32_t> part_order;
    DevBuf<uint32_t> d_part_order;
    // per-item timing record of the subset test (for the cost model):
    // [2 item] warp-cycles, [2 item + 1] hit records, item = queue position
    bool record_items = false;
    DevBuf<unsigned long long> item_stats;
    std::vector<unsigned long long> h_item_stats;
    ScanScratch scr;
    int sm_count = 0;
    size_t rec_cap_hint = 0;
    uint32_t seg_tiles = kSegTiles;  // tiles per work item
    // optional CUDA-event timing of the subset-test kernel
    bool profile = false;
    cudaEvent_t ev_begin = nullptr, ev_end = nullptr;
    MatchScratch() = default;
    MatchScratch(const MatchScratch &) = delete;
    MatchScratch &operator=(const MatchScratch &) = delete;
    MatchScratch &operator=(MatchScratch &&o) noexcept;
    ~MatchScratch();
};

// Per-batch statistics (for the bench and the scheduler).
struct BatchStats {
    uint64_t routed = 0;   // (query, partition) pairs
    uint64_t items = 0;    // work items
    uint64_t pairs = 0;    // matching (query, filter) pairs
    uint64_t records = 0;  // hit records ((query, tile) with at least one match)
    uint64_t keys = 0;     // output keys
    int retries = 0;       // pair-buffer regrowths
    float match_ms = 0.f;  // subset-test kernel time (profiling on)
    uint64_t dense = 0;    // sum over partitions of routed queries x partition size
    uint32_t launches = 0; // kernels launched for the batch
};

// Matches nq queries already on the device (d_queries [nq][6]).  On return
// (stream synchronized) *d_offsets points to nq + 1 offsets and *d_keys to
// the keys of every query, both in scratch memory.  unique != 0 gives each
// query's keys sorted ascending without duplicates (match_unique).
void match_batch(const DevTable &t, const uint32_t *d_queries, uint32_t nq, bool unique, MatchScratch &s,
                 const uint64_t **d_offsets, const uint32_t **d_keys, uint64_t *n_keys, BatchStats *stats,
                 cudaStream_t st, cudaEvent_t match_begin = nullptr, cudaEvent_t match_end = nullptr);

// The subset test's path-choice constant (see match.cu).
uint32_t fpl_trip_cost();

// Narrows n keys (all < 65,536) to 16 bits into s.keys16 on stream st.
const uint16_t *narrow_keys(const uint32_t *d_keys, uint64_t n, MatchScratch &s, cudaStream_t st);

// The same pipeline with all scratch in a static device array (noalloc.cu):
// scratch is that array's device address on the current device, as
// returned by noalloc_scratch_address().
void match_batch_noalloc(const DevTable &t, const uint32_t *d_queries, uint32_t nq, bool unique, uint32_t seg_tiles,
                         void *scratch, uint64_t *d_out_offsets, uint32_t *d_out_keys, uint64_t capacity,
                         uint64_t *n_keys, cudaStream_t st);
// Device address of the no-allocation array on the current device.
void *noalloc_scratch_address();

}  // namespace tmb
