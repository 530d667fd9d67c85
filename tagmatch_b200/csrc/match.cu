// Batched subset matching on one device.
//
// The reference routes each query on CPU threads to every partition whose
// mask is a subset of the query (front_end.cc:465-477), queues it per
// partition, ships full queues of 256 queries to the GPU
// (front_end.cc:350-376, back_end.cc:243-302) where three_phase_matching
// (gpu.cu:60-607) tests one filter per thread against the batch held in
// constant memory and appends every hit with a global atomic
// (gpu.cu:53-58); the host then turns (query, filter) hits into keys
// (back_end.cc:288-302) and sorts/uniques them for match_unique
// (tagmatch_query.hh:99-119).
//
// Here the whole path runs on the device for a batch of queries:
//   k_route      one thread per query tests the partition masks (held in
//                shared memory); CTA-local counts reserve queue space with
//                one global atomic per (CTA, partition); queue records are
//                32 bytes (6 query words, query id, pad);
//   host plan    work items = (partition, group of four 256-query chunks,
//                segment of the partition's tiles), offsets computed on the
//                host from the per-partition counts, partitions in id order
//                or in the order the learned cost model gives;
//   k_slices     per 256-query chunk, bit-sliced "lacks bit b" masks:
//                Z[b] bit j set when query j of the chunk lacks bit b
//                (192 x 256 bits, ballot per bit);
//   k_match      persistent CTAs take items from an atomic counter.  Each
//                item's query records are staged into shared memory by bulk
//                TMA copies (cp.async.bulk + mbarrier), one per chunk; the
//                buffers are released by per-warp mbarrier arrivals.  A warp
//                takes one tile of <= 32 filters at a time; the tile's AND
//                mask selects candidate queries of all four chunks by
//                OR-ing the slices of its bits (one 32-query word per lane);
//                the candidates are tested either one per lane against the
//                tile's filters broadcast from shared memory, or, when they
//                are few, four at a time against the tile held one filter
//                per lane (6 LOP3s per (query, filter) either way); each
//                (query, tile) with a hit becomes a (query, tile, hit mask,
//                key count) record, staged per warp in shared memory and
//                flushed with one global atomic, and its key count is added
//                to the query's total;
//   k_key_fill   after a prefix sum of the query totals: one cursor atomic
//                per record; the runs of adjacent hit bits of a warp's 64
//                records (one key range each) are numbered and copied 32 at
//                a time by the whole warp;
//   k_unique_*   match_unique: per-query bitmap (small key spaces, output
//                comes out sorted) or per-query block radix sort + unique.
// Result overflow is exact: the record buffer is regrown and the batch re-run
// (the reference truncates silently at 4,194,304 hits, gpu.cu:55).
#include "match_kernels.cuh"
#include <cstdio>
#include <cstring>
#include <cstdlib>

namespace tmb {

MatchScratch &MatchScratch::operator=(MatchScratch &&o) noexcept {
    if (this == &o) return *this;
    queries = std::move(o.queries);
    part_count = std::move(o.part_count);
    part_off = std::move(o.part_off);
    part_cursor = std::move(o.part_cursor);
    queue = std::move(o.queue);
    item_off = std::move(o.item_off);
    chunk_off = std::move(o.chunk_off);
    slices = std::move(o.slices);
    work = std::move(o.work);
    keys16 = std::move(o.keys16);
    counters = std::move(o.counters);
    recs = std::move(o.recs);
    qkeys = std::move(o.qkeys);
    qoff = std::move(o.qoff);
    qcursor = std::move(o.qcursor);
    keys = std::move(o.keys);
    ucount = std::move(o.ucount);
    uoff = std::move(o.uoff);
    ukeys = std::move(o.ukeys);
    readback = std::move(o.readback);
    part_order = std::move(o.part_order);
    d_part_order = std::move(o.d_part_order);
    record_items = o.record_items;
    item_stats = std::move(o.item_stats);
    h_item_stats = std::move(o.h_item_stats);
    for (int i = 0; i < 2 * ScanScratch::kLevels; ++i) scr.levels[i] = std::move(o.scr.levels[i]);
    sm_count = o.sm_count;
    rec_cap_hint = o.rec_cap_hint;
    seg_tiles = o.seg_tiles;
    profile = o.profile;
    if (ev_begin) cudaEventDestroy(ev_begin);
    if (ev_end) cudaEventDestroy(ev_end);
    ev_begin = o.ev_begin;
    ev_end = o.ev_end;
    o.ev_begin = o.ev_end = nullptr;
    return *this;
}

// Estimated cost of one 4-candidate trip of the subset test's
// lane-per-filter loop, against which the lane-per-query pass is weighed
// for each tile (TM_FPL_TRIP_COST overrides it; results do not depend on
// it).  Measured on the config-1 step with 1,024-query work items: flat
// from 75 to 150, worse below (45: +9%).
uint32_t fpl_trip_cost() {
    static const uint32_t v = [] {
        const char *e = std::getenv("TM_FPL_TRIP_COST");
        return e ? uint32_t(std::strtoul(e, nullptr, 10)) : 90u;
    }();
    return v;
}

const uint16_t *narrow_keys(const uint32_t *d_keys, uint64_t n, MatchScratch &s, cudaStream_t st) {
    s.keys16.reserve(std::max<uint64_t>(n, 1) + 8);
    if (n) {
        const unsigned blocks = unsigned(std::min<uint64_t>((n / 4 + 255) / 256 + 1, 148 * 16));
        k_narrow16<<<blocks, 256, 0, st>>>(d_keys, n, s.keys16.p);
        TM_CHECK_LAUNCH();
    }
    return s.keys16.p;
}

// Reads na words at a and nb words at b (device memory) into s.readback
// and waits for them: a kernel writes them to mapped host memory, so the
// read does not wait for copies that other streams have queued on the copy
// engines (the host pipeline keeps multi-GB result copies in flight while
// the next batch is matched).
const uint32_t *read_back(MatchScratch &s, const void *a, uint32_t na, const void *b, uint32_t nb, cudaStream_t st) {
    s.readback.reserve(size_t(na) + nb);
    const unsigned blocks = std::min(64u, (na + nb + 255) / 256);
    k_readback<<<std::max(blocks, 1u), 256, 0, st>>>(static_cast<const uint32_t *>(a), na,
                                                     static_cast<const uint32_t *>(b), nb, s.readback.d);
    TM_CHECK_LAUNCH();
    TM_CUDA(cudaStreamSynchronize(st));
    return s.readback.h;
}

MatchScratch::~MatchScratch() {
    if (ev_begin) cudaEventDestroy(ev_begin);
    if (ev_end) cudaEventDestroy(ev_end);
}

void match_batch(const DevTable &t, const uint32_t *d_queries, uint32_t nq, bool unique, MatchScratch &s,
                 const uint64_t **d_offsets, const uint32_t **d_keys, uint64_t *n_keys, BatchStats *stats,
                 cudaStream_t st, cudaEvent_t match_begin, cudaEvent_t match_end) {
    if (s.sm_count == 0) {
        int dev;
        TM_CUDA(cudaGetDevice(&dev));
        TM_CUDA(cudaDeviceGetAttribute(&s.sm_count, cudaDevAttrMultiProcessorCount, dev));
    }
    const uint32_t P = t.n_parts;
    BatchStats bs;
    s.qkeys.reserve(std::max<uint32_t>(nq, 1));
    s.qoff.reserve(size_t(nq) + 1);
    s.counters.reserve(4);
    if (nq == 0 || P == 0 || t.n_tiles == 0) {
        TM_CUDA(cudaMemsetAsync(s.qoff.p, 0, (size_t(nq) + 1) * sizeof(uint64_t), st));
        TM_CUDA(cudaStreamSynchronize(st));
        *d_offsets = s.qoff.p;
        *d_keys = s.keys.p;
        *n_keys = 0;
        if (match_begin) TM_CUDA(cudaEventRecord(match_begin, st));
        if (match_end) TM_CUDA(cudaEventRecord(match_end, st));
        if (stats) *stats = bs;
        return;
    }
    // ---- routing ----
    s.part_count.reserve(P);
    s.part_off.reserve(size_t(P) + 1);
    s.part_cursor.reserve(P);
    TM_CUDA(cudaMemsetAsync(s.part_count.p, 0, P * sizeof(uint32_t), st));
    TM_CUDA(cudaMemsetAsync(s.part_cursor.p, 0, P * sizeof(uint32_t), st));
    const unsigned rblocks = blocks_for(nq, kRouteThreads);
    for (uint32_t p0 = 0; p0 < P; p0 += kMaxRouteParts) {
        const uint32_t pw = std::min(kMaxRouteParts, P - p0);
        const size_t smem = size_t(pw) * (kWords + 2) * sizeof(uint32_t);
        k_route<false><<<rblocks, kRouteThreads, smem, st>>>(d_queries, nq, t.part_mask.p, p0, pw, s.part_count.p, nullptr,
                                                            nullptr, nullptr);
        TM_CHECK_LAUNCH();
    }
    exclusive_scan<uint32_t, uint32_t>(s.part_count.p, s.part_off.p, P, s.scr, st);
    s.h_part_count.resize(P);
    const uint32_t *rb = read_back(s, s.part_count.p, P, s.part_off.p + P, 1, st);
    std::copy(rb, rb + P, s.h_part_count.begin());
    const uint32_t routed = rb[P];
    bs.routed = routed;
    for (uint32_t p = 0; p < P; ++p) bs.dense += uint64_t(s.h_part_count[p]) * t.h_part_size[p];
    const uint32_t windows = (P + kMaxRouteParts - 1) / kMaxRouteParts;
    bs.launches += 2 * windows + 3 + scan_launches(P);  // route x2, readback, slices, match, scan
    s.queue.reserve(size_t(std::max<uint32_t>(routed, 1)) * kQueueWords + kChunk * kQueueWords);
    for (uint32_t p0 = 0; p0 < P; p0 += kMaxRouteParts) {
        const uint32_t pw = std::min(kMaxRouteParts, P - p0);
        const size_t smem = size_t(pw) * (kWords + 2) * sizeof(uint32_t);
        k_route<true><<<rblocks, kRouteThreads, smem, st>>>(d_queries, nq, t.part_mask.p, p0, pw, nullptr, s.part_off.p,
                                                           s.part_cursor.p, s.queue.p);
        TM_CHECK_LAUNCH();
    }
    // ---- plan: chunks and work items per partition (host, from the counts) ----
    s.h_chunk_off.resize(size_t(P) + 1);
    s.h_item_off.resize(size_t(P) + 1);
    uint32_t chunks = 0, items = 0;
    for (uint32_t p = 0; p < P; ++p) {
        s.h_chunk_off[p] = chunks;
        chunks += (s.h_part_count[p] + kChunk - 1) / kChunk;
    }
    // work items in the queue order: partition id order, or the order the
    // learned cost model gives (most expensive items first)
    const bool ordered = s.part_order.size() == P;
    for (uint32_t pos = 0; pos < P; ++pos) {
        const uint32_t p = ordered ? s.part_order[pos] : pos;
        s.h_item_off[pos] = items;
        // an item: kItemChunks chunks of the partition x one tile segment
        const uint32_t ng = (s.h_part_count[p] + kItemQueries - 1) / kItemQueries;
        const uint32_t nt = t.h_part_tiles[p + 1] - t.h_part_tiles[p];
        items += ng * ((nt + s.seg_tiles - 1) / s.seg_tiles);
    }
    s.h_chunk_off[P] = chunks;
    s.h_item_off[P] = items;
    if (ordered) {
        s.d_part_order.reserve(P);
        TM_CUDA(cudaMemcpyAsync(s.d_part_order.p, s.part_order.data(), size_t(P) * 4, cudaMemcpyHostToDevice, st));
    }
    s.item_off.reserve(size_t(P) + 1);
    s.chunk_off.reserve(size_t(P) + 1);
    TM_CUDA(cudaMemcpyAsync(s.item_off.p, s.h_item_off.data(), (size_t(P) + 1) * 4, cudaMemcpyHostToDevice, st));
    TM_CUDA(cudaMemcpyAsync(s.chunk_off.p, s.h_chunk_off.data(), (size_t(P) + 1) * 4, cudaMemcpyHostToDevice, st));
    s.slices.reserve(size_t(std::max<uint32_t>(chunks, 1)) * kSliceWords);
    if (chunks) {
        k_slices<<<chunks, kChunk, 0, st>>>(s.queue.p, s.part_off.p, s.part_count.p, s.chunk_off.p, P, s.slices.p);
        TM_CHECK_LAUNCH();
    }
    bs.items = items;
    // ---- match (regrow and re-run on pair overflow) ----
    if (s.rec_cap_hint == 0) s.rec_cap_hint = size_t(nq) * 512 + (1u << 20);
    s.recs.reserve(s.rec_cap_hint);
    unsigned long long hc[4] = {0, 0, 0, 0};
    for (int attempt = 0;; ++attempt) {
        TM_CUDA(cudaMemsetAsync(s.counters.p, 0, 4 * sizeof(unsigned long long), st));
        static const bool work_counters = std::getenv("TM_WORK_COUNTERS") != nullptr;
        if (work_counters) {
            s.work.reserve(8);
            TM_CUDA(cudaMemsetAsync(s.work.p, 0, 8 * sizeof(unsigned long long), st));
        }
        // per-query key totals are summed by the subset test itself
        TM_CUDA(cudaMemsetAsync(s.qkeys.p, 0, nq * sizeof(uint32_t), st));
        if (s.record_items) {
            s.item_stats.reserve(2 * size_t(std::max<uint32_t>(items, 1)));
            TM_CUDA(cudaMemsetAsync(s.item_stats.p, 0, 2 * size_t(items) * sizeof(unsigned long long), st));
        }
        MatchArgs a{t.tile_words.p, t.tile_info.p, t.tile_keys.p, t.slot_key_off.p, t.part_tile_begin.p, s.part_count.p,
                    s.part_off.p, s.item_off.p, s.chunk_off.p, s.queue.p, s.slices.p, P, s.seg_tiles, s.counters.p,
                    s.recs.p, (unsigned long long)s.recs.cap, s.qkeys.p, fpl_trip_cost(),
                    ordered ? s.d_part_order.p : nullptr, s.record_items ? s.item_stats.p : nullptr,
                    work_counters ? s.work.p : nullptr};
        if (match_begin && attempt == 0) TM_CUDA(cudaEventRecord(match_begin, st));
        if (s.profile) {
            if (!s.ev_begin) {
                TM_CUDA(cudaEventCreate(&s.ev_begin));
                TM_CUDA(cudaEventCreate(&s.ev_end));
            }
            TM_CUDA(cudaEventRecord(s.ev_begin, st));
        }
        if (work_counters) launch_match<true>(a, unsigned(s.sm_count) * 4, st);
        else launch_match<false>(a, unsigned(s.sm_count) * 4, st);
        TM_CHECK_LAUNCH();
        if (s.profile) TM_CUDA(cudaEventRecord(s.ev_end, st));
        if (match_end) TM_CUDA(cudaEventRecord(match_end, st));
        std::memcpy(hc, read_back(s, s.counters.p, 8, nullptr, 0, st), 4 * sizeof(unsigned long long));
        if (hc[2]) throw Error(TM_ERR_TIMEOUT, "match kernel: bounded wait for the query copy expired");
        if (work_counters) {
            unsigned long long w[8];
            TM_CUDA(cudaMemcpy(w, s.work.p, sizeof(w), cudaMemcpyDeviceToHost));
            std::fprintf(stderr,
                         "[tm work] queries %u tile_visits %llu query_passes %llu candidates %llu filter_trips %llu "
                         "items %llu query_groups %llu query_lanes %llu small_query_visits %llu records %llu pairs %llu\n",
                         nq, w[0], w[1], w[2], w[3], w[4], w[5], w[6], w[7], hc[1], hc[3]);
        }
        if (s.profile) {
            float ms = 0.f;
            TM_CUDA(cudaEventElapsedTime(&ms, s.ev_begin, s.ev_end));
            bs.match_ms += ms;
        }
        if (hc[1] <= s.recs.cap) break;
        if (attempt >= 3) throw Error(TM_ERR_INTERNAL, "hit record buffer regrowth did not converge");
        s.rec_cap_hint = size_t(hc[1] + hc[1] / 4 + 1024);
        s.recs.reserve(s.rec_cap_hint);
        bs.retries++;
    }
    bs.records = hc[1];
    if (s.record_items) {
        s.h_item_stats.resize(2 * size_t(items));
        if (items)
            TM_CUDA(cudaMemcpyAsync(s.h_item_stats.data(), s.item_stats.p, 2 * size_t(items) * sizeof(unsigned long long),
                                    cudaMemcpyDeviceToHost, st));
    }
    // ---- keys ----
    const unsigned gblocks = std::max(1u, std::min(blocks_for(hc[1], kFillThreads * kFillPerLane), unsigned(s.sm_count) * 16));
    // record-count readback, fill, key-total readback; each retry: match + readback
    bs.launches += 3 + scan_launches(nq) + 2 * uint32_t(bs.retries);
    exclusive_scan<uint32_t, uint64_t>(s.qkeys.p, s.qoff.p, nq, s.scr, st);
    uint64_t total = 0;
    std::memcpy(&total, read_back(s, s.qoff.p + nq, 2, nullptr, 0, st), sizeof(uint64_t));
    bs.pairs = hc[3];
    s.keys.reserve(std::max<uint64_t>(total, 1));
    s.qcursor.reserve(nq);
    TM_CUDA(cudaMemsetAsync(s.qcursor.p, 0, nq * sizeof(uint32_t), st));
    k_key_fill<<<gblocks, kFillThreads, 0, st>>>(s.recs.p, s.counters.p, t.slot_key_off.p, t.tile_keys.p, t.keys.p, s.qoff.p, s.qcursor.p, s.keys.p);
    TM_CHECK_LAUNCH();
    if (!unique) {
        TM_CUDA(cudaStreamSynchronize(st));
        *d_offsets = s.qoff.p;
        *d_keys = s.keys.p;
        *n_keys = total;
        bs.keys = total;
        if (stats) *stats = bs;
        return;
    }
    // ---- match_unique ----
    s.ucount.reserve(nq);
    s.uoff.reserve(size_t(nq) + 1);
    s.ukeys.reserve(std::max<uint64_t>(total, 1));
    const uint64_t bitmap_words = (uint64_t(t.max_key) >> 5) + 1;
    if (bitmap_words * 4 <= 48 * 1024) {
        k_unique_bitmap<<<nq, kUniqThreads, bitmap_words * 4, st>>>(s.keys.p, s.qoff.p, uint32_t(bitmap_words), s.ukeys.p,
                                                                     s.ucount.p);
    } else {
        k_unique_sort<<<nq, kUniqThreads, 0, st>>>(s.keys.p, s.qoff.p, s.ukeys.p, s.ucount.p);
    }
    TM_CHECK_LAUNCH();
    exclusive_scan<uint32_t, uint64_t>(s.ucount.p, s.uoff.p, nq, s.scr, st);
    // compact into s.keys (unique prefix of every segment is <= its length)
    k_compact<<<nq, 256, 0, st>>>(s.ukeys.p, s.qoff.p, s.uoff.p, nq, s.keys.p);
    bs.launches += 3 + scan_launches(nq);  // unique, compact, readback, scan
    TM_CHECK_LAUNCH();
    uint64_t utotal = 0;
    std::memcpy(&utotal, read_back(s, s.uoff.p + nq, 2, nullptr, 0, st), sizeof(uint64_t));
    *d_offsets = s.uoff.p;
    *d_keys = s.keys.p;
    *n_keys = utotal;
    bs.keys = utotal;
    if (stats) *stats = bs;
}

}  // namespace tmb
