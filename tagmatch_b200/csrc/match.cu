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
//   host plan    work items = (partition, 256-query chunk, 128-tile segment),
//                offsets computed on the host from the per-partition counts;
//   k_slices     per 256-query chunk, bit-sliced "lacks bit b" masks:
//                Z[b] bit j set when query j of the chunk lacks bit b
//                (192 x 256 bits, ballot per bit);
//   k_match      persistent CTAs take items from an atomic counter.  Each
//                item's queries and slices are staged into shared memory by
//                bulk TMA copies (cp.async.bulk + mbarrier), double-buffered:
//                the next item loads while this one is matched, and the
//                buffer is released by per-warp mbarrier arrivals instead of
//                a CTA barrier.  Each warp takes one tile of <= 32 filters in
//                registers; the tile's AND mask selects candidate queries by
//                OR-ing the slices of its bits (8 lanes, one 32-query word
//                each); each candidate is tested against the 32 filters with
//                6 LOP3s; hits are compacted with ballot/popc into a
//                per-warp shared-memory buffer flushed with one global atomic;
//   k_key_count / k_key_fill   per-query key counts (warp-aggregated atomics
//                over lanes holding the same query), prefix sums, key copy;
//   k_unique_*   match_unique: per-query bitmap (small key spaces, output
//                comes out sorted) or per-query block radix sort + unique.
// Result overflow is exact: the pair buffer is regrown and the batch re-run
// (the reference truncates silently at 4,194,304 hits, gpu.cu:55).
#include "match.cuh"
#include <algorithm>

namespace tmb {
namespace {

constexpr int kRouteThreads = 256;
constexpr int kMatchThreads = 256;
constexpr int kMatchWarps = kMatchThreads / 32;
constexpr int kWarpBuf = 256;  // staged pairs per warp
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
    uint32_t *zc = slices + size_t(c) * kBits * 8;
#pragma unroll
    for (int k = 0; k < kWords; ++k) zc[(k * 32 + lane) * 8 + w] = mine[k];
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

struct MatchArgs {
    const uint32_t *tile_words;
    const TileInfo *tile_info;
    const uint32_t *part_tile_begin;
    const uint32_t *part_count;
    const uint32_t *part_off;
    const uint32_t *item_off;
    const uint32_t *chunk_off;
    const uint32_t *queue;
    const uint32_t *slices;
    uint32_t n_parts;
    unsigned long long *counters;  // [0] next item, [1] pairs, [2] error flags
    Pair *pairs;
    unsigned long long pair_cap;
};

constexpr int kSliceWords = kBits * 8;  // 192 x 256 bits

// One staging buffer: a chunk's query records and slices.
struct __align__(128) Stage {
    uint32_t q[kChunk * kQueueWords];  // 8 KB
    uint32_t z[kSliceWords];           // 6 KB
};

__device__ __forceinline__ void flush_warp(Pair *buf, uint32_t n, const MatchArgs &a, unsigned lane) {
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(&a.counters[1], (unsigned long long)n);
    base = __shfl_sync(kFull, base, 0);
    if (base + n <= a.pair_cap) {
        for (uint32_t i = lane; i < n; i += 32) a.pairs[base + i] = buf[i];
    }
    __syncwarp();
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

struct ItemRef {
    uint32_t p, qbase, nq, tb, te, zchunk;
};

__device__ __forceinline__ ItemRef locate(const MatchArgs &a, uint32_t item) {
    uint32_t lo = 0, hi = a.n_parts;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (a.item_off[mid] <= item) lo = mid;
        else hi = mid;
    }
    ItemRef r;
    r.p = lo;
    const uint32_t local = item - a.item_off[lo];
    const uint32_t pq = a.part_count[lo];
    const uint32_t nchunks = (pq + kChunk - 1) / kChunk;
    const uint32_t chunk = local % nchunks, seg = local / nchunks;
    r.qbase = a.part_off[lo] + chunk * kChunk;
    r.nq = min((uint32_t)kChunk, pq - chunk * kChunk);
    r.tb = a.part_tile_begin[lo] + seg * kSegTiles;
    r.te = min(r.tb + (uint32_t)kSegTiles, a.part_tile_begin[lo + 1]);
    r.zchunk = a.chunk_off[lo] + chunk;
    return r;
}

// Thread 0: claim the next item and start its copy into stage `buf`; the
// item id is published through the full barrier's phase completion.
__device__ __forceinline__ void produce(const MatchArgs &a, uint32_t total, Stage *st, uint64_t *full, uint32_t *s_item,
                                        int buf) {
    const uint32_t item = uint32_t(atomicAdd(&a.counters[0], 1ull));
    s_item[buf] = item;
    if (item < total) {
        const ItemRef r = locate(a, item);
        const uint32_t qbytes = r.nq * kQueueWords * sizeof(uint32_t);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(&full[buf], qbytes + kSliceWords * sizeof(uint32_t));
        tma_bulk_g2s(st[buf].q, a.queue + size_t(r.qbase) * kQueueWords, qbytes, &full[buf]);
        tma_bulk_g2s(st[buf].z, a.slices + size_t(r.zchunk) * kSliceWords, kSliceWords * sizeof(uint32_t), &full[buf]);
    } else {
        mbar_arrive(&full[buf]);  // nothing to copy: complete the phase so consumers see the end
    }
}

__global__ void __launch_bounds__(kMatchThreads) k_match(MatchArgs a) {
    __shared__ Stage st[2];
    __shared__ __align__(16) Pair s_out[kMatchWarps][kWarpBuf];
    __shared__ __align__(8) uint64_t full[2], empty[2];
    __shared__ uint32_t s_item[2];
    __shared__ int s_fail;
    const unsigned tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t total = a.item_off[a.n_parts];
    if (tid == 0) {
        mbar_init(&full[0], 1);
        mbar_init(&full[1], 1);
        mbar_init(&empty[0], kMatchWarps);
        mbar_init(&empty[1], kMatchWarps);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_fail = 0;
    }
    __syncthreads();
    if (tid == 0) produce(a, total, st, full, s_item, 0);
    uint32_t nout = 0;  // staged pairs in this warp's buffer
    for (uint32_t it = 0;; ++it) {
        const int b = it & 1;
        // prefetch the next item into the other stage once every warp has
        // released it (it held item it - 1)
        if (tid == 0) {
            bool ok = true;
            if (it >= 1) ok = mbar_wait(&empty[b ^ 1], ((it - 1) >> 1) & 1);
            if (ok) produce(a, total, st, full, s_item, b ^ 1);
            else { atomicOr(&a.counters[2], 1ull); s_fail = 1; }
        }
        if (!mbar_wait(&full[b], (it >> 1) & 1)) {
            atomicOr(&a.counters[2], 2ull);
            break;
        }
        const uint32_t item = s_item[b];
        if (item >= total || s_fail) break;
        const ItemRef r = locate(a, item);
        const uint4 *sq = reinterpret_cast<const uint4 *>(st[b].q);
        const uint32_t *sz = st[b].z;
        for (uint32_t t = r.tb + warp; t < r.te; t += kMatchWarps) {
            uint32_t f[kWords];
#pragma unroll
            for (int k = 0; k < kWords; ++k) f[k] = __ldg(&a.tile_words[(size_t(t) * kWords + k) * kTile + lane]);
            const TileInfo ti = a.tile_info[t];
            const bool lane_valid = lane < ti.count;
            // candidates: queries holding every bit of the tile's AND mask;
            // lane w < 8 builds the word for queries 32 w .. 32 w + 31
            uint32_t lack = 0;
#pragma unroll
            for (int k = 0; k < kWords; ++k) {
                uint32_t m = ti.and_mask[k];
                while (m) {
                    const uint32_t bit = k * 32 + __ffs(m) - 1;
                    m &= m - 1;
                    if (lane < 8) lack |= sz[bit * 8 + lane];
                }
            }
            uint32_t cand_word = lane < 8 ? ~lack : 0u;
            if (lane < 8 && lane * 32 + 32 > r.nq) cand_word &= lane * 32 >= r.nq ? 0u : ((1u << (r.nq - lane * 32)) - 1u);
            for (uint32_t g = 0; g < 8; ++g) {
                uint32_t c = __shfl_sync(kFull, cand_word, g);
                while (c) {
                    const uint32_t j0 = g * 32 + __ffs(c) - 1;
                    c &= c - 1;
                    const bool two = c != 0;
                    const uint32_t j1 = two ? g * 32 + __ffs(c) - 1 : j0;
                    c &= c - 1;
                    const uint4 a0 = sq[j0 * 2], a1 = sq[j0 * 2 + 1];
                    const uint4 b0 = sq[j1 * 2], b1 = sq[j1 * 2 + 1];
                    uint32_t x = f[0] & ~a0.x, y = f[0] & ~b0.x;
                    x = andnot_or(f[1], a0.y, x);
                    y = andnot_or(f[1], b0.y, y);
                    x = andnot_or(f[2], a0.z, x);
                    y = andnot_or(f[2], b0.z, y);
                    x = andnot_or(f[3], a0.w, x);
                    y = andnot_or(f[3], b0.w, y);
                    x = andnot_or(f[4], a1.x, x);
                    y = andnot_or(f[4], b1.x, y);
                    x = andnot_or(f[5], a1.y, x);
                    y = andnot_or(f[5], b1.y, y);
                    const bool h0 = lane_valid && x == 0;
                    const bool h1 = two && lane_valid && y == 0;
                    const uint32_t m0 = __ballot_sync(kFull, h0), m1 = __ballot_sync(kFull, h1);
                    if (m0 | m1) {
                        const uint32_t n0 = __popc(m0), n1 = __popc(m1);
                        if (nout + n0 + n1 > (uint32_t)kWarpBuf) {
                            flush_warp(s_out[warp], nout, a, lane);
                            nout = 0;
                        }
                        const uint32_t below = (1u << lane) - 1u;
                        if (h0) s_out[warp][nout + __popc(m0 & below)] = Pair{a1.z, t * kTile + lane};
                        if (h1) s_out[warp][nout + n0 + __popc(m1 & below)] = Pair{b1.z, t * kTile + lane};
                        nout += n0 + n1;
                        __syncwarp();
                    }
                }
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[b]);
    }
    if (nout) flush_warp(s_out[warp], nout, a, lane);
}

// ---------------------------------------------------------------------------
// Key gather
// ---------------------------------------------------------------------------
// Lanes of a warp that hold pairs of the same query form one group
// (__match_any_sync); each lane gets the sum of its group's key counts and
// the part of it held by lower lanes, so a group needs one atomic.
__device__ __forceinline__ void group_sums(uint32_t peers, uint32_t nk, unsigned lane, uint32_t &excl, uint32_t &tot) {
    excl = 0;
    tot = 0;
#pragma unroll
    for (int l = 0; l < 32; ++l) {
        const uint32_t v = __shfl_sync(kFull, nk, l);
        if ((peers >> l) & 1u) {
            tot += v;
            if ((unsigned)l < lane) excl += v;
        }
    }
}

__global__ void k_key_count(const Pair *__restrict__ pairs, const unsigned long long *__restrict__ counters,
                            const uint32_t *__restrict__ slot_key_off, uint32_t *__restrict__ qkeys) {
    const unsigned long long n = counters[1];
    const unsigned lane = threadIdx.x & 31;
    const unsigned long long warps = (unsigned long long)gridDim.x * (blockDim.x >> 5);
    for (unsigned long long base = ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x - lane); base < n;
         base += warps * 32) {
        const unsigned long long i = base + lane;
        const bool valid = i < n;
        Pair pr{0xFFFFFFFFu, 0u};
        uint32_t nk = 0;
        if (valid) {
            pr = pairs[i];
            nk = slot_key_off[pr.slot + 1] - slot_key_off[pr.slot];
        }
        const uint32_t peers = __match_any_sync(kFull, pr.query);
        uint32_t excl, tot;
        group_sums(peers, nk, lane, excl, tot);
        if (valid && lane == (unsigned)(__ffs(peers) - 1) && tot) atomicAdd(&qkeys[pr.query], tot);
    }
}

__global__ void k_key_fill(const Pair *__restrict__ pairs, const unsigned long long *__restrict__ counters,
                           const uint32_t *__restrict__ slot_key_off, const uint32_t *__restrict__ tkeys,
                           const uint64_t *__restrict__ qoff, uint32_t *__restrict__ qcursor, uint32_t *__restrict__ out) {
    const unsigned long long n = counters[1];
    const unsigned lane = threadIdx.x & 31;
    const unsigned long long warps = (unsigned long long)gridDim.x * (blockDim.x >> 5);
    for (unsigned long long base = ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x - lane); base < n;
         base += warps * 32) {
        const unsigned long long i = base + lane;
        const bool valid = i < n;
        Pair pr{0xFFFFFFFFu, 0u};
        uint32_t b = 0, e = 0;
        if (valid) {
            pr = pairs[i];
            b = slot_key_off[pr.slot];
            e = slot_key_off[pr.slot + 1];
        }
        const uint32_t peers = __match_any_sync(kFull, pr.query);
        uint32_t excl, tot;
        group_sums(peers, e - b, lane, excl, tot);
        const unsigned leader = __ffs(peers) - 1;
        uint64_t pos = 0;
        if (valid && lane == leader && tot) pos = qoff[pr.query] + atomicAdd(&qcursor[pr.query], tot);
        pos = __shfl_sync(kFull, pos, leader) + excl;
        for (uint32_t k = b; k < e; ++k) out[pos++] = tkeys[k];
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
    for (uint64_t i = b + threadIdx.x; i < e; i += blockDim.x) {
        const uint32_t k = keys[i];
        atomicOr(&bm[k >> 5], 1u << (k & 31));
    }
    __syncthreads();
    const uint32_t per = (words + blockDim.x - 1) / blockDim.x;
    const uint32_t w0 = threadIdx.x * per, w1 = min(w0 + per, words);
    uint32_t c = 0;
    for (uint32_t w = w0; w < w1; ++w) c += __popc(bm[w]);
    uint32_t tot;
    uint32_t pos = block_excl_scan<uint32_t>(c, tot);
    uint64_t d = b + pos;
    for (uint32_t w = w0; w < w1; ++w) {
        uint32_t x = bm[w];
        while (x) {
            const uint32_t bit = __ffs(x) - 1;
            x &= x - 1;
            ukeys[d++] = w * 32 + bit;
        }
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
    for (uint64_t i = threadIdx.x; i < n; i += blockDim.x) out[dst + i] = ukeys[src + i];
}

}  // namespace

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
    counters = std::move(o.counters);
    pairs = std::move(o.pairs);
    qkeys = std::move(o.qkeys);
    qoff = std::move(o.qoff);
    qcursor = std::move(o.qcursor);
    keys = std::move(o.keys);
    ucount = std::move(o.ucount);
    uoff = std::move(o.uoff);
    ukeys = std::move(o.ukeys);
    for (int i = 0; i < 2 * ScanScratch::kLevels; ++i) scr.levels[i] = std::move(o.scr.levels[i]);
    sm_count = o.sm_count;
    pair_cap_hint = o.pair_cap_hint;
    profile = o.profile;
    if (ev_begin) cudaEventDestroy(ev_begin);
    if (ev_end) cudaEventDestroy(ev_end);
    ev_begin = o.ev_begin;
    ev_end = o.ev_end;
    o.ev_begin = o.ev_end = nullptr;
    return *this;
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
    uint32_t routed = 0;
    s.h_part_count.resize(P);
    TM_CUDA(cudaMemcpyAsync(&routed, s.part_off.p + P, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    TM_CUDA(cudaMemcpyAsync(s.h_part_count.data(), s.part_count.p, P * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    TM_CUDA(cudaStreamSynchronize(st));
    bs.routed = routed;
    for (uint32_t p = 0; p < P; ++p) bs.dense += uint64_t(s.h_part_count[p]) * t.h_part_size[p];
    const uint32_t windows = (P + kMaxRouteParts - 1) / kMaxRouteParts;
    bs.launches += 2 * windows + 2 + scan_launches(P);  // route x2, slices, match, scan
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
        s.h_item_off[p] = items;
        const uint32_t nc = (s.h_part_count[p] + kChunk - 1) / kChunk;
        const uint32_t nt = t.h_part_tiles[p + 1] - t.h_part_tiles[p];
        chunks += nc;
        items += nc * ((nt + kSegTiles - 1) / kSegTiles);
    }
    s.h_chunk_off[P] = chunks;
    s.h_item_off[P] = items;
    s.item_off.reserve(size_t(P) + 1);
    s.chunk_off.reserve(size_t(P) + 1);
    TM_CUDA(cudaMemcpyAsync(s.item_off.p, s.h_item_off.data(), (size_t(P) + 1) * 4, cudaMemcpyHostToDevice, st));
    TM_CUDA(cudaMemcpyAsync(s.chunk_off.p, s.h_chunk_off.data(), (size_t(P) + 1) * 4, cudaMemcpyHostToDevice, st));
    s.slices.reserve(size_t(std::max<uint32_t>(chunks, 1)) * kBits * 8);
    if (chunks) {
        k_slices<<<chunks, kChunk, 0, st>>>(s.queue.p, s.part_off.p, s.part_count.p, s.chunk_off.p, P, s.slices.p);
        TM_CHECK_LAUNCH();
    }
    bs.items = items;
    // ---- match (regrow and re-run on pair overflow) ----
    if (s.pair_cap_hint == 0) s.pair_cap_hint = size_t(nq) * 1024 + (1u << 20);
    s.pairs.reserve(s.pair_cap_hint);
    unsigned long long hc[4] = {0, 0, 0, 0};
    for (int attempt = 0;; ++attempt) {
        TM_CUDA(cudaMemsetAsync(s.counters.p, 0, 4 * sizeof(unsigned long long), st));
        MatchArgs a{t.tile_words.p, t.tile_info.p, t.part_tile_begin.p, s.part_count.p, s.part_off.p, s.item_off.p,
                    s.chunk_off.p, s.queue.p, s.slices.p, P, s.counters.p, s.pairs.p, (unsigned long long)s.pairs.cap};
        if (match_begin && attempt == 0) TM_CUDA(cudaEventRecord(match_begin, st));
        if (s.profile) {
            if (!s.ev_begin) {
                TM_CUDA(cudaEventCreate(&s.ev_begin));
                TM_CUDA(cudaEventCreate(&s.ev_end));
            }
            TM_CUDA(cudaEventRecord(s.ev_begin, st));
        }
        k_match<<<unsigned(s.sm_count) * 4, kMatchThreads, 0, st>>>(a);
        TM_CHECK_LAUNCH();
        if (s.profile) TM_CUDA(cudaEventRecord(s.ev_end, st));
        if (match_end) TM_CUDA(cudaEventRecord(match_end, st));
        TM_CUDA(cudaMemcpyAsync(hc, s.counters.p, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
        TM_CUDA(cudaStreamSynchronize(st));
        if (hc[2]) throw Error(TM_ERR_TIMEOUT, "match kernel: bounded wait for the query copy expired");
        if (s.profile) {
            float ms = 0.f;
            TM_CUDA(cudaEventElapsedTime(&ms, s.ev_begin, s.ev_end));
            bs.match_ms += ms;
        }
        if (hc[1] <= s.pairs.cap) break;
        if (attempt >= 3) throw Error(TM_ERR_INTERNAL, "pair buffer regrowth did not converge");
        s.pair_cap_hint = size_t(hc[1] + hc[1] / 4 + 1024);
        s.pairs.reserve(s.pair_cap_hint);
        bs.retries++;
    }
    bs.pairs = hc[1];
    // ---- keys ----
    TM_CUDA(cudaMemsetAsync(s.qkeys.p, 0, nq * sizeof(uint32_t), st));
    const unsigned gblocks = std::max(1u, std::min(blocks_for(hc[1], 256), unsigned(s.sm_count) * 16));
    bs.launches += 2 + scan_launches(nq) + uint32_t(bs.retries);
    k_key_count<<<gblocks, 256, 0, st>>>(s.pairs.p, s.counters.p, t.slot_key_off.p, s.qkeys.p);
    TM_CHECK_LAUNCH();
    exclusive_scan<uint32_t, uint64_t>(s.qkeys.p, s.qoff.p, nq, s.scr, st);
    uint64_t total = 0;
    TM_CUDA(cudaMemcpyAsync(&total, s.qoff.p + nq, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
    TM_CUDA(cudaStreamSynchronize(st));
    s.keys.reserve(std::max<uint64_t>(total, 1));
    s.qcursor.reserve(nq);
    TM_CUDA(cudaMemsetAsync(s.qcursor.p, 0, nq * sizeof(uint32_t), st));
    k_key_fill<<<gblocks, 256, 0, st>>>(s.pairs.p, s.counters.p, t.slot_key_off.p, t.keys.p, s.qoff.p, s.qcursor.p, s.keys.p);
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
    uint64_t utotal = 0;
    TM_CUDA(cudaMemcpyAsync(&utotal, s.uoff.p + nq, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
    // compact into s.keys (unique prefix of every segment is <= its length)
    k_compact<<<nq, 256, 0, st>>>(s.ukeys.p, s.qoff.p, s.uoff.p, nq, s.keys.p);
    bs.launches += 2 + scan_launches(nq);
    TM_CHECK_LAUNCH();
    TM_CUDA(cudaStreamSynchronize(st));
    *d_offsets = s.uoff.p;
    *d_keys = s.keys.p;
    *n_keys = utotal;
    bs.keys = utotal;
    if (stats) *stats = bs;
}

}  // namespace tmb
