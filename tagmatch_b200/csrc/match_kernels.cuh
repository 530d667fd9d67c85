// Device kernels of the batched matcher (routing, slices, subset test, key
// gather, match_unique).  Included by match.cu (the engine's pipeline) and
// noalloc.cu (the pipeline over caller-free static scratch); each
// translation unit gets its own internal copy.
#pragma once
#include <algorithm>
#include "match.cuh"

namespace tmb {
namespace {

constexpr int kRouteThreads = 256;
constexpr int kMatchThreads = 256;
constexpr int kMatchWarps = kMatchThreads / 32;
constexpr int kWarpRecs = 64;  // staged hit records per warp (1 KB)
constexpr int kQuad = 1;       // tiles a warp selects candidates for at once (for all chunks of its item)
constexpr int kTileLanes = 32 / kQuad;  // lanes per tile in the selection: 8 words x kItemChunks chunks
static_assert(kTileLanes == 8 * kItemChunks, "selection lanes");
constexpr uint32_t kMaxRouteParts = 1536;  // partition masks per routing window (48 KB of shared memory)
constexpr unsigned long long kSpinLimit = 1ull << 26;

inline unsigned blocks_for(size_t n, unsigned t) { return unsigned((n + t - 1) / t); }

// ---------------------------------------------------------------------------
// Routing
// ---------------------------------------------------------------------------
template <bool FILL>
__global__ void __launch_bounds__(kRouteThreads) k_route(const uint32_t *__restrict__ queries, uint32_t nq,
                                                         const uint32_t *__restrict__ part_mask, uint32_t p0, uint32_t pw,
                                                         uint32_t *__restrict__ part_count, const uint32_t *__restrict__ part_off,
                                                         uint32_t *__restrict__ part_cursor, uint32_t *__restrict__ queue) {
    extern __shared__ uint32_t sm[];
    uint32_t *s_mask = sm;                          // [pw][6]
    uint32_t *s_cnt = sm + size_t(pw) * kWords;     // [pw]
    uint32_t *s_base = s_cnt + pw;                  // [pw] (FILL)
    for (uint32_t i = threadIdx.x; i < pw; i += blockDim.x) {
#pragma unroll
        for (int k = 0; k < kWords; ++k) s_mask[i * kWords + k] = part_mask[size_t(p0 + i) * 8 + k];
        s_cnt[i] = 0;
    }
    __syncthreads();
    const uint32_t qi = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = qi < nq;
    uint32_t q[kWords];
#pragma unroll
    for (int k = 0; k < kWords; ++k) q[k] = valid ? queries[size_t(qi) * kWords + k] : 0u;
    if (valid) {
        for (uint32_t i = 0; i < pw; ++i)
            if (subset6(s_mask + i * kWords, q)) atomicAdd(&s_cnt[i], 1u);
    }
    __syncthreads();
    if constexpr (!FILL) {
        for (uint32_t i = threadIdx.x; i < pw; i += blockDim.x)
            if (s_cnt[i]) atomicAdd(&part_count[p0 + i], s_cnt[i]);
    } else {
    for (uint32_t i = threadIdx.x; i < pw; i += blockDim.x) {
        const uint32_t c = s_cnt[i];
        s_base[i] = c ? part_off[p0 + i] + atomicAdd(&part_cursor[p0 + i], c) : 0u;
        s_cnt[i] = 0;
    }
    __syncthreads();
    if (valid) {
        for (uint32_t i = 0; i < pw; ++i) {
            if (subset6(s_mask + i * kWords, q)) {
                const uint32_t pos = s_base[i] + atomicAdd(&s_cnt[i], 1u);
                uint4 *dst = reinterpret_cast<uint4 *>(queue + size_t(pos) * kQueueWords);
                dst[0] = make_uint4(q[0], q[1], q[2], q[3]);
                dst[1] = make_uint4(q[4], q[5], qi, 0u);
            }
        }
    }
    }
}

constexpr int kSliceRows = kBits + 1;  // 192 bit rows + the all-zero padding row

// Bit-sliced query masks of one 256-query chunk: z[b * 8 + w] bit l is set
// when query 32 w + l of the chunk lacks filter bit b, or does not exist
// (so an absent query is never a candidate).
__global__ void __launch_bounds__(kChunk) k_slices(const uint32_t *__restrict__ queue, const uint32_t *__restrict__ part_off,
                                                   const uint32_t *__restrict__ part_count,
                                                   const uint32_t *__restrict__ chunk_off, uint32_t n_parts,
                                                   uint32_t *__restrict__ slices) {
    const uint32_t c = blockIdx.x;
    uint32_t lo = 0, hi = n_parts;  // partition of this chunk: chunk_off[lo] <= c < chunk_off[lo + 1]
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (chunk_off[mid] <= c) lo = mid;
        else hi = mid;
    }
    const uint32_t p = lo;
    const uint32_t chunk = c - chunk_off[p];
    const uint32_t nq = min((uint32_t)kChunk, part_count[p] - chunk * kChunk);
    const unsigned lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t j = w * 32 + lane;
    uint32_t q[kWords];
    const bool valid = j < nq;
#pragma unroll
    for (int k = 0; k < kWords; ++k)
        q[k] = valid ? queue[size_t(part_off[p] + chunk * kChunk + j) * kQueueWords + k] : 0u;
    uint32_t mine[kWords];
#pragma unroll
    for (int k = 0; k < kWords; ++k) {
#pragma unroll
        for (int b = 0; b < 32; ++b) {
            const uint32_t z = __ballot_sync(kFull, !valid || !((q[k] >> b) & 1u));
            if (lane == (unsigned)b) mine[k] = z;
        }
    }
    uint32_t *zc = slices + size_t(c) * kSliceRows * 8;
#pragma unroll
    for (int k = 0; k < kWords; ++k) zc[(k * 32 + lane) * 8 + w] = mine[k];
    if (lane == 0) zc[kNoBit * 8 + w] = 0u;  // the padding row: no query lacks it
}

// ---------------------------------------------------------------------------
// Matching
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// One bulk (non-tensor, non-multicast) TMA copy global -> shared memory.
__device__ __forceinline__ void tma_bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Bounded wait on an mbarrier phase; false when the limit expired.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    unsigned long long spins = 0;
    while (!mbar_try_wait(bar, parity)) {
        if (++spins > kSpinLimit) return false;
    }
    return true;
}

// Keys of the filters in a hit mask.  The table keeps keys in slot order, so
// a run of adjacent set bits [lo, hi) is the one key range [o[lo], o[hi])
// (o: the tile's slot key offsets, 33 of them).  Calls f(begin, end) per run.
template <class F>
__device__ __forceinline__ void for_each_key_run(const uint32_t *__restrict__ o, uint32_t mask, F f) {
    uint64_t m = mask;
    while (m) {
        const int lo = __ffsll(m) - 1;
        const uint64_t filled = m + (1ull << lo);  // the carry clears the run and sets bit hi
        const int hi = __ffsll(filled & ~m) - 1;
        f(o[lo], o[hi]);
        m &= filled;
    }
}

// Keys of hit mask m of tile t: from the tile's key-count bit planes, or,
// when m touches a filter with 8 keys or more, from the slot offsets.
__device__ __forceinline__ uint32_t mask_keys(const TileKeys &tk, uint32_t m, const uint32_t *__restrict__ slot_key_off,
                                              uint32_t t) {
    if (!(m & tk.wide)) return keys_of_mask(tk, m);
    uint32_t nk = 0;
    for_each_key_run(slot_key_off + size_t(t) * kTile, m, [&](uint32_t b, uint32_t e) { nk += e - b; });
    return nk;
}

struct MatchArgs {
    const uint32_t *tile_words;
    const TileInfo *tile_info;
    const TileKeys *tile_keys;
    const uint32_t *slot_key_off;
    const uint32_t *part_tile_begin;
    const uint32_t *part_count;
    const uint32_t *part_off;
    const uint32_t *item_off;
    const uint32_t *chunk_off;
    const uint32_t *queue;
    const uint32_t *slices;
    uint32_t n_parts;
    uint32_t seg_tiles;            // tiles per work item
    // [0] next item, [1] hit records, [2] error flags, [3] matching
    // (query, filter) pairs
    unsigned long long *counters;
    HitRec *recs;
    unsigned long long rec_cap;
    uint32_t *qkeys;               // [batch queries] key totals, zeroed by the caller
    uint32_t fpl_trip_cost;        // path choice: estimated cost of one 4-candidate trip of the lane-per-filter loop
    // work-queue order: item_off runs over positions, part_order[pos] is the
    // partition at that position (null: partition id order)
    const uint32_t *part_order;
    // optional timing record per item: [2 item] warp-cycles summed over the
    // CTA's warps, [2 item + 1] hit records; null when off
    unsigned long long *item_stats;
    // optional work counters (diagnostics): [0] tile visits, [1] passes of
    // the lane-per-query path, [2] candidate (query, tile) pairs, [3] trips
    // of the lane-per-filter path, [4] items, [5] 4-filter groups tested by
    // the lane-per-query path, [6] its busy lanes summed over passes, [7]
    // its tile visits with at most 16 candidates; null when off
    unsigned long long *work;
};

constexpr int kSliceWords = kSliceRows * 8;  // 193 x 256 bits

// A chunk's staged query records (8 KB).  kPadQuery marks the gather's
// padding records (no query).
constexpr uint32_t kPadQuery = 0xFFFFFFFFu;
constexpr int kStageWords = kChunk * kQueueWords;

// Shared memory of one matcher CTA (dynamic; ~54 KB, 4 CTAs per SM).
struct MatchSmem {
    uint32_t q[kItemChunks][kStageWords];                // the item's chunks' query records
    HitRec rec[kMatchWarps][kWarpRecs];                  // staged hit records per warp
    // candidate lists per warp and tile: the chunks' candidates in chunk
    // order (query index in its chunk), padded to a multiple of 4
    uint8_t list[kMatchWarps][kQuad][kItemQueries + 8];
    TileKeys tk[kMatchWarps][kQuad];                     // key-count planes of the warp's tiles
    uint4 tf[kMatchWarps][kWords][kTile / 4];            // a warp's tile: word k of filters 4 g .. 4 g + 3
    uint64_t full, empty;
    uint32_t item;
    int fail;
    // thread 0's record of a copy in flight, with the parity of the phase
    // that completes it
    uint32_t inflight, inflight_par;
};

// 4 CTAs per SM: 228 KB of shared memory per SM, 1 KB of it reserved per CTA
static_assert(4 * (sizeof(MatchSmem) + 1024) <= 228 * 1024, "the matcher's shared memory must fit 4 CTAs per SM");

// Moves a warp's n staged records to the global record buffer (one atomic
// reserves their place; past the capacity they are only counted, and the
// host re-runs the batch with a larger buffer).
__device__ __forceinline__ void flush_recs(HitRec *buf, uint32_t n, const MatchArgs &a, unsigned lane) {
    __syncwarp();
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(&a.counters[1], (unsigned long long)n);
    base = __shfl_sync(kFull, base, 0);
    if (base + n <= a.rec_cap) {
        for (uint32_t i = lane; i < n; i += 32) a.recs[base + i] = buf[i];
    }
    __syncwarp();
}

// A work item: kItemChunks consecutive 256-query chunks of one partition
// (nq[c] queries in chunk c, 0 past the partition's last chunk) against one
// segment of its tiles.
struct ItemRef {
    uint32_t p, qbase, nq[kItemChunks], tb, te, zchunk;
};

__device__ __forceinline__ ItemRef locate(const MatchArgs &a, uint32_t item) {
    uint32_t lo = 0, hi = a.n_parts;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (a.item_off[mid] <= item) lo = mid;
        else hi = mid;
    }
    const uint32_t local = item - a.item_off[lo];
    if (a.part_order) lo = a.part_order[lo];
    ItemRef r;
    r.p = lo;
    const uint32_t pq = a.part_count[lo];
    const uint32_t nchunks = (pq + kChunk - 1) / kChunk;
    const uint32_t ngroups = (nchunks + kItemChunks - 1) / kItemChunks;
    const uint32_t group = local % ngroups, seg = local / ngroups;
    const uint32_t c0 = group * kItemChunks;
    r.qbase = a.part_off[lo] + c0 * kChunk;
#pragma unroll
    for (int c = 0; c < kItemChunks; ++c)
        r.nq[c] = c0 + c < nchunks ? min((uint32_t)kChunk, pq - (c0 + c) * kChunk) : 0u;
    r.tb = a.part_tile_begin[lo] + seg * a.seg_tiles;
    r.te = min(r.tb + a.seg_tiles, a.part_tile_begin[lo + 1]);
    r.zchunk = a.chunk_off[lo] + c0;
    return r;
}

// Thread 0: claim the next item and start the copies of its chunks' query
// records; the item id is published through the full barrier's phase
// completion.  Returns whether copies are in flight.
__device__ __forceinline__ bool produce(const MatchArgs &a, uint32_t total, MatchSmem &S) {
    const uint32_t item = uint32_t(atomicAdd(&a.counters[0], 1ull));
    S.item = item;
    if (item < total) {
        const ItemRef r = locate(a, item);
        uint32_t bytes = 0;
#pragma unroll
        for (int c = 0; c < kItemChunks; ++c) bytes += r.nq[c] * kQueueWords * sizeof(uint32_t);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(&S.full, bytes);
#pragma unroll
        for (int c = 0; c < kItemChunks; ++c) {
            if (!r.nq[c]) continue;
            tma_bulk_g2s(S.q[c], a.queue + (size_t(r.qbase) + size_t(c) * kChunk) * kQueueWords,
                         r.nq[c] * kQueueWords * sizeof(uint32_t), &S.full);
        }
        return true;
    }
    mbar_arrive(&S.full);  // nothing to copy: complete the phase so consumers see the end
    return false;
}

// The subset test.  Persistent CTAs take work items (partition, two
// consecutive 256-query chunks of its queue, segment of its tiles) from an
// atomic counter; thread 0 stages the item's query records and slices with
// bulk TMA copies into the CTA's two chunk buffers.  Each warp takes two
// tiles (<= 32 filters each) at a time:
//  * selection, for both tiles and both chunks at once: the tile's 8
//    selector bits (bits every member holds); lane l ORs the "lacks bit"
//    slices of 32-query word l & 7 of chunk (l >> 3) & 1 for tile l >> 4,
//    so a query that lacks any of them is dropped; the remaining candidates
//    go to the tile's list (one byte per query: the first chunk's, then the
//    second's, placed by a prefix sum over the tile's 16 words);
// then, tile by tile, over the candidates of both chunks together (one pass
// over the tile's filters for 512 queries: fuller passes and trips):
//  * many candidates: one candidate query per lane, the tile's filters read
//    from shared memory (one broadcast 128-bit load gives word k of four
//    filters): 6 LOP3 per (query, filter), the lane's hit mask over the tile
//    built bit by bit; one pass per 32 candidates;
//  * few candidates: one filter per lane (the tile in registers), four
//    candidates per trip, one ballot per candidate for its hit mask;
//  * each (query, tile) with a hit becomes a 16-byte record (query, tile,
//    hit mask, key count from the tile's key-count bit planes), staged in a
//    per-warp buffer and flushed with one atomic; the query's key total is
//    added to qkeys[query] (for the prefix sum that places its keys).
// The path per tile is chosen from the candidate count and the tile size
// (estimated instruction costs; the choice does not change results).
// COUNT: diagnostics instantiation that also tallies its work (a.work);
// TIMED: records each item's warp-cycles and hit records (a.item_stats).
template <bool COUNT, bool TIMED>
__global__ void __launch_bounds__(kMatchThreads, 4) k_match(MatchArgs a) {  // 4 CTAs per SM: up to 64 registers
    extern __shared__ __align__(128) unsigned char smem_raw[];
    MatchSmem &S = *reinterpret_cast<MatchSmem *>(smem_raw);
    const unsigned tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t total = a.item_off[a.n_parts];
    if (tid == 0) {
        mbar_init(&S.full, 1);
        mbar_init(&S.empty, kMatchWarps);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        S.fail = 0;
        S.inflight = 0;
        S.inflight_par = 0;
    }
    __syncthreads();
    uint32_t w_tiles = 0, w_passes = 0, w_cand = 0, w_trips = 0, w_items = 0, w_groups = 0, w_lanes = 0, w_small = 0;
    uint32_t wn = 0;      // records staged by this warp (warp-uniform)
    uint32_t w_recs = 0;  // records this warp has produced (warp-uniform)
    uint32_t pairs = 0;  // matching (query, filter) pairs found by this lane
    const uint32_t lane_lt = (1u << lane) - 1u;
    uint32_t *tfw = reinterpret_cast<uint32_t *>(S.tf[warp]);
    for (uint32_t it = 0;; ++it) {
        // stage the next item once every warp has released the buffers
        // (they held item it - 1); thread 0 keeps track of the copies in
        // flight, so that none still targets this CTA's shared memory when
        // it exits
        if (tid == 0) {
            bool ok = true;
            if (it >= 1) ok = mbar_wait(&S.empty, (it - 1) & 1);
            if (ok) {
                S.inflight = produce(a, total, S) ? 1u : 0u;
                S.inflight_par = it & 1;
            } else {
                atomicOr(&a.counters[2], 1ull);
                S.fail = 1;
            }
        }
        // every exit is taken by whole warps (record flushes use the full warp)
        const bool got = mbar_wait(&S.full, it & 1);
        if (tid == 0 && got) S.inflight = 0;
        if (!__all_sync(kFull, got)) {
            if (lane == 0) atomicOr(&a.counters[2], 2ull);
            break;
        }
        const uint32_t item = S.item;
        if (__any_sync(kFull, item >= total || S.fail)) break;
        const ItemRef r = locate(a, item);
        if (COUNT) ++w_items;
        long long item_c0 = 0;
        uint32_t item_recs0 = 0;
        if (TIMED) {
            item_c0 = clock64();
            item_recs0 = w_recs;
        }
        for (uint32_t t0 = r.tb + warp * kQuad; t0 < r.te; t0 += kMatchWarps * kQuad) {
            // selection for the warp's tiles and all chunks of the item at
            // once: lane l serves word l & 7 of chunk (l >> 3) % kItemChunks
            // for tile t0 + l / kTileLanes; the tile's 8 selector bits OR the
            // "lacks" slices of the lane's 32 queries (read through L1: the
            // item's slices are shared by all its tiles)
            const uint32_t gi = lane / kTileLanes, tl = lane % kTileLanes, ch = tl >> 3, w = lane & 7;
            const uint32_t tq = t0 + gi;
            uint32_t nqc = r.nq[0];  // queries in the lane's chunk (no dynamic index into r)
#pragma unroll
            for (int c = 1; c < kItemChunks; ++c)
                if (ch == (uint32_t)c) nqc = r.nq[c];
            uint32_t cand = 0, tcount = 0;
            if (tq < r.te) {
                const TileInfo ti = a.tile_info[tq];
                tcount = ti.count;
                if (nqc) {  // chunks past the partition's last have no slices
                    const uint32_t *zl = a.slices + (size_t(r.zchunk) + ch) * kSliceWords + w;
                    const uint32_t lack =
                        __ldg(&zl[(ti.sel[0] & 0xFFu) * 8]) | __ldg(&zl[((ti.sel[0] >> 8) & 0xFFu) * 8]) |
                        __ldg(&zl[((ti.sel[0] >> 16) & 0xFFu) * 8]) | __ldg(&zl[(ti.sel[0] >> 24) * 8]) |
                        __ldg(&zl[(ti.sel[1] & 0xFFu) * 8]) | __ldg(&zl[((ti.sel[1] >> 8) & 0xFFu) * 8]) |
                        __ldg(&zl[((ti.sel[1] >> 16) & 0xFFu) * 8]) | __ldg(&zl[(ti.sel[1] >> 24) * 8]);
                    cand = ~lack;
                    if (w * 32 + 32 > nqc) cand &= w * 32 >= nqc ? 0u : ((1u << (nqc - w * 32)) - 1u);
                }
                if (tl == 0) S.tk[warp][gi] = a.tile_keys[tq];
            }
            if (COUNT) w_tiles += __popc(__ballot_sync(kFull, tq < r.te && tl == 0));  // lane 0 reports
            // candidate lists (query index in its chunk, one byte each): a
            // prefix sum over each tile's words (chunk by chunk) places every
            // lane's queries
            const uint32_t cnt = __popc(cand);
            uint32_t incl = cnt;
#pragma unroll
            for (int o = 1; o < kTileLanes; o <<= 1) {
                const uint32_t v = __shfl_up_sync(kFull, incl, o);
                if (tl >= (unsigned)o) incl += v;
            }
            {
                uint8_t *lst = S.list[warp][gi];
                uint32_t pos = incl - cnt;
                while (cand) {
                    lst[pos++] = uint8_t(w * 32 + __ffs(cand) - 1);
                    cand &= cand - 1;
                }
                const uint32_t nt = __shfl_sync(kFull, incl, lane | (kTileLanes - 1));
                if (tl < 4) lst[nt + tl] = 0;  // pad to a multiple of 4 (its hits are dropped)
            }
            __syncwarp();
            for (int i = 0; i < kQuad; ++i) {
                const uint32_t n = __shfl_sync(kFull, incl, kTileLanes * i + kTileLanes - 1);
                // list positions where chunks 1 .. kItemChunks - 1 begin: the
                // candidate at position x is in chunk sum_c (x >= cb[c])
                uint32_t cb[kItemChunks - 1];
#pragma unroll
                for (int c = 0; c + 1 < kItemChunks; ++c) cb[c] = __shfl_sync(kFull, incl, kTileLanes * i + 8 * c + 7);
                auto chunk_of = [&](uint32_t x) {
                    uint32_t c = 0;
#pragma unroll
                    for (int k = 0; k + 1 < kItemChunks; ++k) c += x >= cb[k] ? 1u : 0u;
                    return c;
                };
                if (COUNT) w_cand += n;  // the warp's candidates (lane 0 reports)
                if (n == 0) continue;
                const uint32_t t = t0 + i;
                const uint32_t count = __shfl_sync(kFull, tcount, kTileLanes * i);
                const uint8_t *lst = S.list[warp][i];
                uint32_t f[kWords];
#pragma unroll
                for (int k = 0; k < kWords; ++k) f[k] = __ldg(&a.tile_words[(size_t(t) * kWords + k) * kTile + lane]);
                const uint32_t vm = count >= 32u ? kFull : (1u << count) - 1u;  // lanes holding a filter
                const uint32_t groups = (count + 3) >> 2;
                const bool per_query = ((n + 31) >> 5) * (16u + 40u * groups) < ((n + 3) >> 2) * a.fpl_trip_cost;
                if (per_query) {
#pragma unroll
                    for (int k = 0; k < kWords; ++k) tfw[k * kTile + lane] = f[k];
                    __syncwarp();
                    for (uint32_t p0 = 0; p0 < n; p0 += 32) {
                        if (COUNT) {
                            ++w_passes;
                            w_groups += groups;
                            w_lanes += min(32u, n - p0);
                            if (p0 == 0 && n <= 16) ++w_small;
                        }
                        const uint32_t j = p0 + lane;
                        const uint4 *sq = reinterpret_cast<const uint4 *>(S.q[chunk_of(j)]);
                        const uint32_t c2 = j < n ? 2u * lst[j] : 0u;
                        const uint4 qa = sq[c2], qb = sq[c2 + 1];
                        uint32_t m = 0;
#pragma unroll
                        for (int g = 0; g < kTile / 4; ++g) {
                            if (g >= (int)groups) break;
                            const uint4 w0 = S.tf[warp][0][g], w1 = S.tf[warp][1][g], w2 = S.tf[warp][2][g];
                            const uint4 w3 = S.tf[warp][3][g], w4 = S.tf[warp][4][g], w5 = S.tf[warp][5][g];
                            uint32_t x0 = w0.x & ~qa.x, x1 = w0.y & ~qa.x, x2 = w0.z & ~qa.x, x3 = w0.w & ~qa.x;
                            x0 = andnot_or(w1.x, qa.y, x0);
                            x1 = andnot_or(w1.y, qa.y, x1);
                            x2 = andnot_or(w1.z, qa.y, x2);
                            x3 = andnot_or(w1.w, qa.y, x3);
                            x0 = andnot_or(w2.x, qa.z, x0);
                            x1 = andnot_or(w2.y, qa.z, x1);
                            x2 = andnot_or(w2.z, qa.z, x2);
                            x3 = andnot_or(w2.w, qa.z, x3);
                            x0 = andnot_or(w3.x, qa.w, x0);
                            x1 = andnot_or(w3.y, qa.w, x1);
                            x2 = andnot_or(w3.z, qa.w, x2);
                            x3 = andnot_or(w3.w, qa.w, x3);
                            x0 = andnot_or(w4.x, qb.x, x0);
                            x1 = andnot_or(w4.y, qb.x, x1);
                            x2 = andnot_or(w4.z, qb.x, x2);
                            x3 = andnot_or(w4.w, qb.x, x3);
                            x0 = andnot_or(w5.x, qb.y, x0);
                            x1 = andnot_or(w5.y, qb.y, x1);
                            x2 = andnot_or(w5.z, qb.y, x2);
                            x3 = andnot_or(w5.w, qb.y, x3);
                            if (x0 == 0) m |= 1u << (4 * g);
                            if (x1 == 0) m |= 2u << (4 * g);
                            if (x2 == 0) m |= 4u << (4 * g);
                            if (x3 == 0) m |= 8u << (4 * g);
                        }
                        m &= vm;
                        if (j >= n) m = 0;
                        const uint32_t wm = __ballot_sync(kFull, m != 0);
                        if (wm == 0) continue;
                        if (wn + 32 > (uint32_t)kWarpRecs) {
                            flush_recs(S.rec[warp], wn, a, lane);
                            wn = 0;
                        }
                        if (m) {
                            const uint32_t nk = mask_keys(S.tk[warp][i], m, a.slot_key_off, t);
                            S.rec[warp][wn + __popc(wm & lane_lt)] = HitRec{qb.z, t, m, nk};
                            atomicAdd(&a.qkeys[qb.z], nk);
                            pairs += __popc(m);
                        }
                        wn += __popc(wm);
                        if (TIMED) w_recs += __popc(wm);
                    }
                } else {
                    const bool lane_valid = lane < count;
                    for (uint32_t j = 0; j < n; j += 4) {
                        if (COUNT) ++w_trips;
                        const uint32_t idx4 = *reinterpret_cast<const uint32_t *>(lst + j);
                        const uint32_t ia = (idx4 & 0xFFu) * 2, ib = ((idx4 >> 8) & 0xFFu) * 2;
                        const uint32_t ic = ((idx4 >> 16) & 0xFFu) * 2, id = (idx4 >> 24) * 2;
                        const uint4 *sa = reinterpret_cast<const uint4 *>(S.q[chunk_of(j)]);
                        const uint4 *sb = reinterpret_cast<const uint4 *>(S.q[chunk_of(j + 1)]);
                        const uint4 *sc = reinterpret_cast<const uint4 *>(S.q[chunk_of(j + 2)]);
                        const uint4 *sd = reinterpret_cast<const uint4 *>(S.q[chunk_of(j + 3)]);
                        const uint4 p0 = sa[ia], p1 = sa[ia + 1];
                        const uint4 q0 = sb[ib], q1 = sb[ib + 1];
                        const uint4 r0 = sc[ic], r1 = sc[ic + 1];
                        const uint4 u0 = sd[id], u1 = sd[id + 1];
                        uint32_t x0 = f[0] & ~p0.x, x1 = f[0] & ~q0.x, x2 = f[0] & ~r0.x, x3 = f[0] & ~u0.x;
                        x0 = andnot_or(f[1], p0.y, x0);
                        x1 = andnot_or(f[1], q0.y, x1);
                        x2 = andnot_or(f[1], r0.y, x2);
                        x3 = andnot_or(f[1], u0.y, x3);
                        x0 = andnot_or(f[2], p0.z, x0);
                        x1 = andnot_or(f[2], q0.z, x1);
                        x2 = andnot_or(f[2], r0.z, x2);
                        x3 = andnot_or(f[2], u0.z, x3);
                        x0 = andnot_or(f[3], p0.w, x0);
                        x1 = andnot_or(f[3], q0.w, x1);
                        x2 = andnot_or(f[3], r0.w, x2);
                        x3 = andnot_or(f[3], u0.w, x3);
                        x0 = andnot_or(f[4], p1.x, x0);
                        x1 = andnot_or(f[4], q1.x, x1);
                        x2 = andnot_or(f[4], r1.x, x2);
                        x3 = andnot_or(f[4], u1.x, x3);
                        x0 = andnot_or(f[5], p1.y, x0);
                        x1 = andnot_or(f[5], q1.y, x1);
                        x2 = andnot_or(f[5], r1.y, x2);
                        x3 = andnot_or(f[5], u1.y, x3);
                        // common case: no hit among the four (one min chain, one vote)
                        if (!__any_sync(kFull, lane_valid && min(min(x0, x1), min(x2, x3)) == 0)) continue;
                        // warp-uniform from here: one ballot per candidate gives the
                        // tile's hit mask for that query; lane k < 4 stages record k
                        // (list padding repeats query 0 and is dropped)
                        const uint32_t b0 = __ballot_sync(kFull, x0 == 0) & vm;
                        const uint32_t b1 = __ballot_sync(kFull, x1 == 0) & vm;
                        const uint32_t b2 = __ballot_sync(kFull, x2 == 0) & vm;
                        const uint32_t b3 = __ballot_sync(kFull, x3 == 0) & vm;
                        const uint32_t mine = lane == 0 ? b0 : lane == 1 ? b1 : lane == 2 ? b2 : b3;
                        const uint32_t qid = lane == 0 ? p1.z : lane == 1 ? q1.z : lane == 2 ? r1.z : u1.z;
                        const bool wr = lane < 4 && mine != 0 && j + lane < n;
                        const uint32_t wm = __ballot_sync(kFull, wr);
                        if (wm == 0) continue;
                        if (wn + 4 > (uint32_t)kWarpRecs) {
                            flush_recs(S.rec[warp], wn, a, lane);
                            wn = 0;
                        }
                        if (wr) {
                            const uint32_t nk = mask_keys(S.tk[warp][i], mine, a.slot_key_off, t);
                            S.rec[warp][wn + __popc(wm & lane_lt)] = HitRec{qid, t, mine, nk};
                            atomicAdd(&a.qkeys[qid], nk);
                            pairs += __popc(mine);
                        }
                        wn += __popc(wm);
                        if (TIMED) w_recs += __popc(wm);
                    }
                }
                __syncwarp();  // the tile buffer is rebuilt for the next tile
            }
            __syncwarp();  // the lists are rebuilt for the next tiles
        }
        __syncwarp();
        if (TIMED && lane == 0) {
            atomicAdd(&a.item_stats[2 * size_t(item)], (unsigned long long)(clock64() - item_c0));
            atomicAdd(&a.item_stats[2 * size_t(item) + 1], (unsigned long long)(w_recs - item_recs0));
        }
        if (lane == 0) mbar_arrive(&S.empty);
    }
    if (wn) flush_recs(S.rec[warp], wn, a, lane);
    pairs = __reduce_add_sync(kFull, pairs);
    if (lane == 0 && pairs) atomicAdd(&a.counters[3], (unsigned long long)pairs);
    if (COUNT && lane == 0) {
        atomicAdd(&a.work[0], (unsigned long long)w_tiles);
        atomicAdd(&a.work[1], (unsigned long long)w_passes);
        atomicAdd(&a.work[2], (unsigned long long)w_cand);
        atomicAdd(&a.work[3], (unsigned long long)w_trips);
        atomicAdd(&a.work[5], (unsigned long long)w_groups);
        atomicAdd(&a.work[6], (unsigned long long)w_lanes);
        atomicAdd(&a.work[7], (unsigned long long)w_small);
        if (warp == 0) atomicAdd(&a.work[4], (unsigned long long)w_items);
    }
    // no copy may still target this CTA's shared memory when it exits: after
    // a failed wait, wait (bounded) for the copies still in flight
    if (tid == 0 && S.inflight && !mbar_wait(&S.full, S.inflight_par)) atomicOr(&a.counters[2], 4ull);
}

// Launches the subset test on grid CTAs (its shared memory is above the
// 48 KB static limit, so the size is set on the kernel first).
template <bool COUNT, bool TIMED>
inline void launch_match_t(const MatchArgs &a, unsigned grid, cudaStream_t st) {
    TM_CUDA(cudaFuncSetAttribute(k_match<COUNT, TIMED>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(sizeof(MatchSmem))));
    TM_CUDA(cudaFuncSetAttribute(k_match<COUNT, TIMED>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 int(cudaSharedmemCarveoutMaxShared)));
    k_match<COUNT, TIMED><<<grid, kMatchThreads, sizeof(MatchSmem), st>>>(a);
}

template <bool COUNT>
inline void launch_match(const MatchArgs &a, unsigned grid, cudaStream_t st) {
    if (a.item_stats) launch_match_t<COUNT, true>(a, grid, st);
    else launch_match_t<COUNT, false>(a, grid, st);
}

// ---------------------------------------------------------------------------
// Key gather
// ---------------------------------------------------------------------------
// records per lane per warp step (loads in flight) and the gather's
// minimum resident CTAs per SM (register budget); build-time tunables
#ifndef TM_FILL_PER_LANE
#define TM_FILL_PER_LANE 2
#endif
#ifndef TM_FILL_MIN_CTAS
#define TM_FILL_MIN_CTAS 6
#endif
constexpr int kFillPerLane = TM_FILL_PER_LANE;

constexpr int kFillThreads = 256;
constexpr int kFillWarps = kFillThreads / 32;
constexpr int kFillStep = 32 * kFillPerLane;  // records per warp step

// Position of the k-th set bit (k from 0) of x, which has more than k set
// bits: halving popcounts.
__device__ __forceinline__ uint32_t nth_set_bit(uint32_t x, uint32_t k) {
    uint32_t pos = 0;
#pragma unroll
    for (int s = 16; s >= 1; s >>= 1) {
        const uint32_t lowc = __popc(x & ((1u << s) - 1u));
        if (k >= lowc) {
            k -= lowc;
            x >>= s;
            pos += s;
        }
    }
    return pos;
}

// Copies every record's keys into its query's range (qoff).  Each record's
// keys are reserved with one atomic on the query's cursor (qcursor, zeroed
// by the caller).  The table keeps keys in slot order, so each run of
// adjacent hit bits [lo, hi) of a record's mask is the key range
// [o[lo], o[hi]) of the tile's slot offsets o.  A warp takes 32 x
// kFillPerLane records per step and numbers all their runs (a prefix sum
// over the lanes' run counts); lane i of a batch then takes run 32 b + i:
// a 5-step shuffle search for the lane whose records hold it, the record
// from shared memory, the run's first bit by halving popcounts, its key
// range from the slot offsets, and its place in the record's output from
// the keys of the hit bits below it (the tile's key-count planes).  The
// warp copies the batch's runs together, 32 keys per step (a prefix sum
// over the run lengths and, for key j, a 5-step search for the run that
// owns it), so the stores coalesce and a record with several runs costs no
// extra pass over the warp.
__global__ void __launch_bounds__(kFillThreads, TM_FILL_MIN_CTAS) k_key_fill(
    const HitRec *__restrict__ recs, const unsigned long long *__restrict__ counters,
    const uint32_t *__restrict__ slot_key_off, const TileKeys *__restrict__ tile_keys, const uint32_t *__restrict__ tkeys,
    const uint64_t *__restrict__ qoff, uint32_t *__restrict__ qcursor, uint32_t *__restrict__ out) {
    // per warp and record of the step: tile, hit mask, keys, runs of the
    // lane's earlier records; and the record's first output position
    __shared__ uint4 s_rec[kFillWarps][kFillStep];
    __shared__ unsigned long long s_dst[kFillWarps][kFillStep];
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned long long n = counters[1];
    const unsigned long long warps = (unsigned long long)gridDim.x * kFillWarps;
    const unsigned long long wid = (unsigned long long)blockIdx.x * kFillWarps + warp;
    for (unsigned long long base = wid * kFillStep; base < n; base += warps * kFillStep) {
        HitRec r[kFillPerLane];
#pragma unroll
        for (int j = 0; j < kFillPerLane; ++j) {
            const unsigned long long i = base + j * 32 + lane;
            r[j] = i < n ? recs[i] : HitRec{kPadQuery, 0u, 0u, 0u};
        }
        uint32_t nruns = 0;
        unsigned long long dst[kFillPerLane];
#pragma unroll
        for (int j = 0; j < kFillPerLane; ++j) {
            const bool live = r[j].query != kPadQuery && r[j].nkeys != 0;
            const uint32_t m = live ? r[j].mask : 0u;
            dst[j] = live ? qoff[r[j].query] + atomicAdd(&qcursor[r[j].query], r[j].nkeys) : 0ull;
            s_rec[warp][j * 32 + lane] = make_uint4(r[j].tile, m, live ? r[j].nkeys : 0u, nruns);
            nruns += __popc(m & ~(m << 1));  // run starts
        }
        uint32_t incl = nruns;
#pragma unroll
        for (int s = 1; s < 32; s <<= 1) {
            const uint32_t v = __shfl_up_sync(kFull, incl, s);
            if (lane >= (unsigned)s) incl += v;
        }
        const uint32_t total = __shfl_sync(kFull, incl, 31);
        const uint32_t excl = incl - nruns;
        __syncwarp();
        for (uint32_t rb = 0; rb < total; rb += 32) {
            const uint32_t ri = rb + lane;
            uint32_t owner = 0;  // first lane whose inclusive run count exceeds ri
#pragma unroll
            for (int s = 16; s >= 1; s >>= 1) {
                const uint32_t v = __shfl_sync(kFull, incl, owner + s - 1);
                if (v <= ri) owner += s;
            }
            const uint32_t oexcl = __shfl_sync(kFull, excl, owner);
            const bool have = ri < total;
            uint32_t slot = owner, src = 0, end = 0, below = 0, t = 0, nk = 0;
            bool last = true;
            TileKeys tk{{0u, 0u, 0u}, 0u};
            if (have) {
                const uint32_t k = ri - oexcl;  // run number within the owner lane's records
                // its record: the last whose earlier-run count is <= k
#pragma unroll
                for (int jj = 1; jj < kFillPerLane; ++jj)
                    if (s_rec[warp][jj * 32 + owner].w <= k) slot = jj * 32 + owner;
                const uint4 rc = s_rec[warp][slot];
                const uint32_t m = rc.y;
                t = rc.x;
                nk = rc.z;
                const uint32_t lo = nth_set_bit(m & ~(m << 1), k - rc.w);
                const uint32_t hi = lo + uint32_t(__ffsll(~((unsigned long long)m >> lo))) - 1u;
                const uint32_t *o = slot_key_off + size_t(t) * kTile;
                below = m & ((1u << lo) - 1u);  // hit bits of the earlier runs
                last = hi >= 32u || (m >> hi) == 0u;
                src = o[lo];
                if (!last) end = o[hi];
                if (below) tk = tile_keys[t];
            }
            if (rb == 0) {
                // the cursor atomics' results, published once the first
                // batch's offset loads are in flight
#pragma unroll
                for (int j = 0; j < kFillPerLane; ++j) s_dst[warp][j * 32 + lane] = dst[j];
                __syncwarp();
            }
            uint32_t len = 0;
            unsigned long long d = 0;
            if (have) {
                const uint32_t bk = below ? mask_keys(tk, below, slot_key_off, t) : 0u;
                len = last ? nk - bk : end - src;
                d = s_dst[warp][slot] + bk;
            }
            // the batch's runs, copied together
            uint32_t kin = len;
#pragma unroll
            for (int s = 1; s < 32; s <<= 1) {
                const uint32_t v = __shfl_up_sync(kFull, kin, s);
                if (lane >= (unsigned)s) kin += v;
            }
            const uint32_t keys = __shfl_sync(kFull, kin, 31);
            const uint32_t start = kin - len;
            for (uint32_t j0 = 0; j0 < keys; j0 += 32) {
                const uint32_t kk = j0 + lane;
                uint32_t ro = 0;  // first lane whose inclusive key count exceeds kk
#pragma unroll
                for (int s = 16; s >= 1; s >>= 1) {
                    const uint32_t v = __shfl_sync(kFull, kin, ro + s - 1);
                    if (v <= kk) ro += s;
                }
                const uint32_t ostart = __shfl_sync(kFull, start, ro);
                const uint32_t osrc = __shfl_sync(kFull, src, ro);
                const unsigned long long odst = __shfl_sync(kFull, d, ro);
                if (kk < keys) out[odst + (kk - ostart)] = tkeys[osrc + (kk - ostart)];
            }
        }
        __syncwarp();  // the shared entries are rewritten by the next step
    }
}

// ---------------------------------------------------------------------------
// match_unique
// ---------------------------------------------------------------------------
constexpr int kUniqThreads = 256;

// Key space [0, 32 * words): a bitmap per query in shared memory; the set
// bits read in order are the sorted unique keys.
__global__ void __launch_bounds__(kUniqThreads) k_unique_bitmap(const uint32_t *__restrict__ keys, const uint64_t *__restrict__ qoff,
                                                                uint32_t words, uint32_t *__restrict__ ukeys,
                                                                uint32_t *__restrict__ ucount) {
    extern __shared__ uint32_t bm[];
    const uint32_t q = blockIdx.x;
    const uint64_t b = qoff[q], e = qoff[q + 1];
    if (e == b) {
        if (threadIdx.x == 0) ucount[q] = 0;
        return;
    }
    for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) bm[i] = 0;
    __syncthreads();
    // four key loads in flight per thread
    constexpr uint32_t kU = 4;
    uint64_t i = b + threadIdx.x;
    for (; i + (kU - 1) * blockDim.x < e; i += kU * blockDim.x) {
        uint32_t k[kU];
#pragma unroll
        for (uint32_t u = 0; u < kU; ++u) k[u] = keys[i + u * blockDim.x];
#pragma unroll
        for (uint32_t u = 0; u < kU; ++u) atomicOr(&bm[k[u] >> 5], 1u << (k[u] & 31));
    }
    for (; i < e; i += blockDim.x) {
        const uint32_t k = keys[i];
        atomicOr(&bm[k >> 5], 1u << (k & 31));
    }
    __syncthreads();
    // read-out in order: warp w takes words [w * per, (w + 1) * per), 32 at
    // a time (lane l word l); a prefix sum over the lanes' popcounts places
    // the round's keys, which the warp then writes 32 consecutive keys per
    // step (each lane finds the word holding its key by a 5-step shuffle
    // search, then the bit by halving popcounts), so the stores coalesce
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const uint32_t per = ((words + nwarps - 1) / nwarps + 31) & ~31u;
    const uint32_t w0 = min(words, warp * per), w1 = min(words, w0 + per);
    uint32_t c = 0;
    for (uint32_t w = w0 + lane; w < w1; w += 32) c += __popc(bm[w]);
    c = __reduce_add_sync(kFull, c);
    uint32_t tot;
    uint32_t pos = block_excl_scan<uint32_t>(lane == 0 ? c : 0u, tot);
    pos = __shfl_sync(kFull, pos, 0);  // this warp's first output position
    uint64_t d = b + pos;
    for (uint32_t r0 = w0; r0 < w1; r0 += 32) {
        const uint32_t w = r0 + lane;
        const uint32_t x = w < w1 ? bm[w] : 0u;
        const uint32_t cnt = __popc(x);
        uint32_t incl = cnt;
#pragma unroll
        for (int s = 1; s < 32; s <<= 1) {
            const uint32_t v = __shfl_up_sync(kFull, incl, s);
            if (lane >= (unsigned)s) incl += v;
        }
        const uint32_t total = __shfl_sync(kFull, incl, 31);
        for (uint32_t j0 = 0; j0 < total; j0 += 32) {
            const uint32_t j = j0 + lane;
            uint32_t owner = 0;
#pragma unroll
            for (int step = 16; step >= 1; step >>= 1) {
                const uint32_t v = __shfl_sync(kFull, incl, owner + step - 1);
                if (v <= j) owner += step;
            }
            const uint32_t oincl = __shfl_sync(kFull, incl, owner), ocnt = __shfl_sync(kFull, cnt, owner);
            uint32_t ox = __shfl_sync(kFull, x, owner);
            if (j < total) {
                uint32_t rk = j - (oincl - ocnt), bit = 0;  // rank of the key's bit within the word
#pragma unroll
                for (int s = 16; s >= 1; s >>= 1) {
                    const uint32_t lowc = __popc(ox & ((1u << s) - 1u));
                    if (rk >= lowc) {
                        rk -= lowc;
                        ox >>= s;
                        bit += s;
                    }
                }
                ukeys[d + j] = (r0 + owner) * 32 + bit;
            }
        }
        d += total;
    }
    if (threadIdx.x == 0) ucount[q] = tot;
}

// General key space: block LSD radix sort of the query's keys (4-bit digits,
// stable per-thread ranges) through ukeys as the ping-pong buffer, then
// unique.  Sorted keys end in ukeys[b..e); the unique prefix is compacted in
// place.
constexpr int kRadixBits = 4;
constexpr int kRadixBuckets = 1 << kRadixBits;

__global__ void __launch_bounds__(kUniqThreads) k_unique_sort(uint32_t *__restrict__ keys, const uint64_t *__restrict__ qoff,
                                                              uint32_t *__restrict__ ukeys, uint32_t *__restrict__ ucount) {
    __shared__ uint32_t s_hist[kRadixBuckets * kUniqThreads];
    const uint32_t q = blockIdx.x;
    const uint64_t b = qoff[q], e = qoff[q + 1];
    const uint64_t n = e - b;
    if (n == 0) {
        if (threadIdx.x == 0) ucount[q] = 0;
        return;
    }
    const uint64_t per = (n + blockDim.x - 1) / blockDim.x;
    const uint64_t r0 = min(n, threadIdx.x * per), r1 = min(n, r0 + per);
    uint32_t *src = keys + b, *dst = ukeys + b;
    for (int shift = 0; shift < 32; shift += kRadixBits) {
        uint32_t h[kRadixBuckets];
#pragma unroll
        for (int d = 0; d < kRadixBuckets; ++d) h[d] = 0;
        for (uint64_t i = r0; i < r1; ++i) h[(src[i] >> shift) & (kRadixBuckets - 1)]++;
#pragma unroll
        for (int d = 0; d < kRadixBuckets; ++d) s_hist[d * kUniqThreads + threadIdx.x] = h[d];
        __syncthreads();
        // exclusive scan over (digit, thread) order: each thread scans a
        // contiguous run of kRadixBuckets entries
        uint32_t run[kRadixBuckets];
        uint32_t sum = 0;
#pragma unroll
        for (int d = 0; d < kRadixBuckets; ++d) {
            run[d] = s_hist[threadIdx.x * kRadixBuckets + d];
            sum += run[d];
        }
        uint32_t tot;
        uint32_t pre = block_excl_scan<uint32_t>(sum, tot);
#pragma unroll
        for (int d = 0; d < kRadixBuckets; ++d) {
            s_hist[threadIdx.x * kRadixBuckets + d] = pre;
            pre += run[d];
        }
        __syncthreads();
#pragma unroll
        for (int d = 0; d < kRadixBuckets; ++d) h[d] = s_hist[d * kUniqThreads + threadIdx.x];
        for (uint64_t i = r0; i < r1; ++i) {
            const uint32_t k = src[i];
            dst[h[(k >> shift) & (kRadixBuckets - 1)]++] = k;
        }
        __syncthreads();
        uint32_t *tmp = src;
        src = dst;
        dst = tmp;
    }
    // 8 passes: the sorted keys are back in keys[b..e); unique into ukeys.
    uint32_t c = 0;
    for (uint64_t i = r0; i < r1; ++i) c += (i == 0 || src[i] != src[i - 1]);
    uint32_t tot;
    uint32_t pos = block_excl_scan<uint32_t>(c, tot);
    for (uint64_t i = r0; i < r1; ++i)
        if (i == 0 || src[i] != src[i - 1]) ukeys[b + pos++] = src[i];
    if (threadIdx.x == 0) ucount[q] = tot;
}

__global__ void k_compact(const uint32_t *__restrict__ ukeys, const uint64_t *__restrict__ qoff,
                          const uint64_t *__restrict__ uoff, uint32_t nq, uint32_t *__restrict__ out) {
    const uint32_t q = blockIdx.x;
    if (q >= nq) return;
    const uint64_t src = qoff[q], dst = uoff[q], n = uoff[q + 1] - uoff[q];
    // four loads in flight per thread
    uint64_t i = threadIdx.x;
    for (; i + 3 * blockDim.x < n; i += 4 * blockDim.x) {
        uint32_t v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) v[u] = ukeys[src + i + u * blockDim.x];
#pragma unroll
        for (int u = 0; u < 4; ++u) out[dst + i + u * blockDim.x] = v[u];
    }
    for (; i < n; i += blockDim.x) out[dst + i] = ukeys[src + i];
}

// Copies na words at a, then nb words at b, into mapped pinned host memory
// (dst is its device view).  Used for the few numbers the host needs in the
// middle of a batch (queue sizes, pair and key totals).
__global__ void k_readback(const uint32_t *__restrict__ a, uint32_t na, const uint32_t *__restrict__ b, uint32_t nb,
                           uint32_t *__restrict__ dst) {
    const uint32_t n = na + nb;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        dst[i] = i < na ? a[i] : b[i - na];
}

// Keys narrowed to 16 bits for the trip to the host (tables whose largest
// key is below 65,536); the host widens them back.
__global__ void k_narrow16(const uint32_t *__restrict__ in, uint64_t n, uint16_t *__restrict__ out) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i * 4 < n; i += stride) {
        if (i * 4 + 4 <= n && (reinterpret_cast<uintptr_t>(in) & 15) == 0) {
            const uint4 v = reinterpret_cast<const uint4 *>(in)[i];
            uint2 w;
            w.x = (v.x & 0xFFFFu) | (v.y << 16);
            w.y = (v.z & 0xFFFFu) | (v.w << 16);
            reinterpret_cast<uint2 *>(out)[i] = w;
        } else {
            for (uint64_t k = i * 4; k < n && k < i * 4 + 4; ++k) out[k] = uint16_t(in[k]);
        }
    }
}

}  // namespace
}  // namespace tmb
