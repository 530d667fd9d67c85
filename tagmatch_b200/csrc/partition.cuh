// GPU balanced partitioner and table builder.
#pragma once
#include <cstdint>
#include <vector>
#include "tm_device.cuh"
#include "tm_host.hpp"
#include "scan.cuh"

namespace tmb {

// One contiguous range of the working filter order with its split state.
struct __align__(16) Seg {
    uint32_t begin, end;
    uint32_t used[kWords];  // pivot bits used on the path to this range
    uint32_t flags;         // kPhase* | kMaskEmpty
    uint32_t pad;
};
constexpr uint32_t kPhaseBalance = 0;   // size > max_p: balancing_pivot split
constexpr uint32_t kPhasePeel = 1;      // size <= max_p, empty pivot mask: peel most frequent bit
constexpr uint32_t kPhaseTile = 2;      // inside a partition: split down to <= 32 filters
constexpr uint32_t kPhaseMask = 3;
constexpr uint32_t kMaskEmpty = 4;

struct Range {
    uint32_t begin, end;
};

// Result of a partitioning run, all on the device except the partition list.
struct PartitionResult {
    uint32_t n = 0;                  // filters
    std::vector<Range> parts;        // partitions in id order (sorted by position)
    DevBuf<uint32_t> words;          // [n][6] filters in partition order
    DevBuf<uint32_t> order;          // [n] original index of each position
    DevBuf<uint32_t> tile_mark;      // [n] 1 where a tile starts (with_tiles only)
    std::vector<uint32_t> bit_freq;  // [192] bit frequencies over the whole table
};

// Device table used by the matcher.
struct DevTable {
    uint32_t n_filters = 0, n_parts = 0, n_tiles = 0;
    uint64_t n_keys = 0;
    uint32_t max_key = 0;
    DevBuf<uint32_t> tile_words;      // [n_tiles][6][32]
    DevBuf<TileInfo> tile_info;       // [n_tiles]
    DevBuf<uint32_t> tile_and;        // [n_tiles][8]: AND of the members (6 words), pad
    DevBuf<uint32_t> part_tile_begin; // [n_parts + 1]
    DevBuf<uint32_t> part_mask;       // [n_parts][8]: 6 mask words, tile count, pad
    DevBuf<uint32_t> slot_key_off;    // [n_tiles * 32 + 1]
    DevBuf<TileKeys> tile_keys;       // [n_tiles] key counts per lane as bit planes
    DevBuf<uint32_t> keys;            // [n_keys]
    DevBuf<uint32_t> slot_filter;     // [n_tiles * 32] original filter index (0xFFFFFFFF for empty lanes)
    std::vector<uint32_t> h_part_mask;  // host copy of the masks [n_parts][8]
    std::vector<uint32_t> h_part_tiles; // host copy of part_tile_begin
    std::vector<uint32_t> h_part_size;  // filters per partition
    size_t device_bytes() const;
};

// Runs the partitioner on filters already on the device (d_filters [n][6]).
// with_tiles also splits every partition into tiles of <= 32 filters.
void gpu_partition(const uint32_t *d_filters, uint32_t n, uint32_t max_p, bool with_tiles, PartitionResult &out,
                   cudaStream_t st);

// Builds the matcher table from a partitioning run (with_tiles) and the
// per-filter keys (CSR over the original filter order, on the device).
void build_table(const PartitionResult &pr, const uint32_t *d_key_off, const uint32_t *d_keys, uint64_t n_keys,
                 DevTable &t, cudaStream_t st);

}  // namespace tmb
