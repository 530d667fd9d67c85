// Shared device-side definitions for the TagMatch B200 engine.
//
// Filters and queries are 192-bit Bloom filters held as 6 x uint32 words in
// the reference's 32-bit view (bitvector.hh:210-212): bit p is bit (p % 32)
// of word p / 32.  f matches q when f is a subset of q, f & ~q == 0
// (bitvector.hh:282-296).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace tmb {

constexpr int kWords = 6;          // 32-bit words per filter
constexpr int kBits = 192;         // filter width
constexpr int kTile = 32;          // filters per tile (one per lane of a warp)
constexpr int kChunk = 256;        // queries per partition batch (QUERIES_BATCH_SIZE, parameters.hh:13)
constexpr int kItemChunks = 4;     // 256-query chunks of one partition that a subset-test work item covers
constexpr int kItemQueries = kItemChunks * kChunk;
constexpr int kQueueWords = 8;     // queued query record: 6 filter words, query id, pad (32 bytes)
constexpr unsigned kFull = 0xFFFFFFFFu;

// Tile descriptor (16 bytes): the positions of up to 8 bits that every
// member of the tile holds, most selective (rarest in the table) first,
// padded with kNoBit; member count; owning partition.  A query lacking any
// of these bits matches no filter of the tile.
constexpr int kSelBits = 8;
constexpr uint32_t kNoBit = 192;  // selects the all-zero slice row
struct __align__(16) TileInfo {
    uint32_t sel[2];  // 8 bit positions, one per byte
    uint32_t count;
    uint32_t partition;
};

// One candidate query's hits in one tile: bit l of mask is set when the
// tile's filter in lane l (slot tile * 32 + l) matches the query; nkeys is
// the number of keys of those filters.
struct __align__(16) HitRec {
    uint32_t query;
    uint32_t tile;
    uint32_t mask;
    uint32_t nkeys;
};

// Key counts of a tile's filters as bit planes, so that the keys of any
// hit mask m are popc(m & p[0]) + 2 popc(m & p[1]) + 4 popc(m & p[2]):
// bit l of p[b] is bit b of the key count of the filter in lane l, for
// counts below 8.  Bit l of wide is set when that filter has 8 keys or
// more; masks that touch such lanes are counted from the slot offsets.
struct __align__(16) TileKeys {
    uint32_t p[3];
    uint32_t wide;
};

__device__ __forceinline__ uint32_t keys_of_mask(const TileKeys &tk, uint32_t m) {
    return __popc(m & tk.p[0]) + 2u * __popc(m & tk.p[1]) + 4u * __popc(m & tk.p[2]);
}

__device__ __forceinline__ uint32_t andnot_or(uint32_t f, uint32_t q, uint32_t acc) {
    return (f & ~q) | acc;  // one LOP3
}

__device__ __forceinline__ bool subset6(const uint32_t *f, const uint32_t *q) {
    uint32_t a = f[0] & ~q[0];
    a = andnot_or(f[1], q[1], a);
    a = andnot_or(f[2], q[2], a);
    a = andnot_or(f[3], q[3], a);
    a = andnot_or(f[4], q[4], a);
    a = andnot_or(f[5], q[5], a);
    return a == 0;
}

__device__ __forceinline__ int bit_of(const uint32_t *f, unsigned b) {
    return (f[b >> 5] >> (b & 31)) & 1;
}

}  // namespace tmb

// Status codes (TM_OK, TM_ERR_*) come from the C ABI header.
#include "../../include/tagmatch_b200.h"
