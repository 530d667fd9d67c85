// GPU balanced partitioner and matcher-table builder.
//
// Partition semantics follow the reference's partitioner
// (partitioning.cc:230-411): every range larger than max_p is split, by a
// stable partition that keeps the zero side first (:133-148), on
// balancing_pivot (:262-278); leaves whose pivot mask is still empty go
// through nonzero_mask_partitioning (:230-250), which peels off the one side
// of the most frequent bit until every member shares a bit; each
// partition's mask is the AND of its members (:389-407).  The reference
// makes those choices on the host and only counts bit frequencies on the GPU
// (partitioner_gpu.cu:30-43, one global atomic per set bit).  Here every
// range that is active at one depth of the split tree is processed by the
// same launches:
//
//   k_freq     per-range 192-bin histograms, warp ballot + popc per bit,
//              shared-memory reduction, one global add per bin per CTA;
//   k_decide   one warp per range picks the pivot (warp argmin);
//   k_split_*  a stable two-way split by chunk counts + prefix sums + an
//              in-CTA stable rank (the reference's GPU mirror is unstable,
//              partitioner_gpu.cu:47-67);
//   k_children classifies the two sides into the next active list, the
//              partition list, or (table builds) the tile list.
//
// For the matcher table each partition is then split further, down to tiles
// of at most 32 filters.  The AND of a tile's members lets the matcher skip
// the whole tile for any query that lacks one of those bits, so these splits
// pick the bit (not yet used inside the partition) that maximises
// (members holding it) x (estimated chance that a query lacks it), the
// chance estimated from the bit's frequency over the whole table.
#include "partition.cuh"
#include <algorithm>
#include <cmath>
#include <cstring>

namespace tmb {
namespace {

constexpr int kPChunk = 1024;  // filters per partitioner chunk
constexpr int kPThreads = 256;
constexpr uint32_t kActFinal = 0x100;
constexpr uint32_t kActChop = 0x200;
// Exponent of the tile-split weight (1 - table frequency of the bit)^k.  A
// query is roughly the union of several stored tag sets, so a bit that is
// frequent in the table is very likely present in a query; k ~ 10-16
// minimised candidate (query, tile) pairs on the seeded workloads.
constexpr double kTileWeightExp = 12.0;

struct Counters {
    uint32_t next;
    uint32_t next_chunks;
    uint32_t finals;
    uint32_t leaves;
};

__device__ __forceinline__ uint32_t find_seg(const uint32_t *chunk_off, uint32_t n_act, uint32_t chunk) {
    uint32_t lo = 0, hi = n_act;  // chunk_off[lo] <= chunk < chunk_off[hi]
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (chunk_off[mid] <= chunk) lo = mid;
        else hi = mid;
    }
    return lo;
}

__global__ void k_nchunks(const Seg *segs, uint32_t n_act, uint32_t *nch) {
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n_act) nch[s] = (segs[s].end - segs[s].begin + kPChunk - 1) / kPChunk;
}

__global__ void __launch_bounds__(kPThreads) k_freq(const Seg *__restrict__ segs, const uint32_t *__restrict__ chunk_off,
                                                    uint32_t n_act, const uint32_t *__restrict__ words,
                                                    uint32_t *__restrict__ freq) {
    __shared__ uint32_t s_cnt[kBits];
    __shared__ uint32_t s_seg;
    const unsigned tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid < kBits) s_cnt[tid] = 0;
    if (tid == 0) s_seg = find_seg(chunk_off, n_act, blockIdx.x);
    __syncthreads();
    const uint32_t s = s_seg;
    const Seg seg = segs[s];
    const uint32_t cstart = seg.begin + (blockIdx.x - chunk_off[s]) * kPChunk;
    const uint32_t cend = min(cstart + (uint32_t)kPChunk, seg.end);
    uint32_t c[kWords] = {0, 0, 0, 0, 0, 0};
    for (uint32_t base = cstart + warp * 32; base < cend; base += kPThreads) {
        const uint32_t i = base + lane;
        uint32_t w[kWords] = {0, 0, 0, 0, 0, 0};
        if (i < cend) {
#pragma unroll
            for (int k = 0; k < kWords; ++k) w[k] = words[size_t(i) * kWords + k];
        }
#pragma unroll
        for (int k = 0; k < kWords; ++k) {
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                uint32_t bal = __ballot_sync(kFull, (w[k] >> j) & 1u);
                if (lane == (unsigned)j) c[k] += __popc(bal);
            }
        }
    }
#pragma unroll
    for (int k = 0; k < kWords; ++k)
        if (c[k]) atomicAdd(&s_cnt[k * 32 + lane], c[k]);
    __syncthreads();
    if (tid < kBits && s_cnt[tid]) atomicAdd(&freq[size_t(s) * kBits + tid], s_cnt[tid]);
}

__device__ __forceinline__ unsigned long long warp_min_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long u = __shfl_xor_sync(kFull, v, o);
        v = u < v ? u : v;
    }
    return v;
}

__global__ void k_decide(const Seg *__restrict__ segs, uint32_t n_act, const uint32_t *__restrict__ freq,
                         const float *__restrict__ tile_weight, uint32_t *__restrict__ action) {
    const uint32_t s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned lane = threadIdx.x & 31;
    if (s >= n_act) return;
    const Seg seg = segs[s];
    const uint32_t size = seg.end - seg.begin;
    const uint32_t half = size / 2;
    const uint32_t phase = seg.flags & kPhaseMask;
    const uint32_t *fr = freq + size_t(s) * kBits;
    // first unused bit (balancing_pivot's starting candidate)
    uint32_t u = kBits;
    for (int k = 0; k < kWords; ++k) {
        uint32_t free_bits = ~seg.used[k];
        if (free_bits) { u = k * 32 + __ffs(free_bits) - 1; break; }
    }
    unsigned long long best = ~0ull;
#pragma unroll
    for (int k = 0; k < kWords; ++k) {
        const uint32_t b = k * 32 + lane;
        const uint32_t f = fr[b];
        const uint32_t dist = f > half ? f - half : half - f;
        unsigned long long key = ~0ull;
        if (phase == kPhaseBalance) {
            // smallest distance among bits >= u, earliest bit on ties: the
            // reference scans every later bit, used or not (:268-276)
            if (b >= u) key = ((unsigned long long)dist << 8) | b;
        } else if (phase == kPhasePeel) {
            key = ((unsigned long long)(0xFFFFFFFFu - f) << 8) | b;  // first maximum
        } else {
            // tile phase: the bit whose one side prunes the most queries,
            // scored as (members holding it) x (weight: estimated chance
            // that a query lacks it); highest score, earliest bit
            const bool used = (seg.used[k] >> lane) & 1u;
            if (f > 0 && f < size && !used) {
                const float score = float(f) * tile_weight[b];
                key = ((unsigned long long)(~__float_as_uint(score)) << 8) | b;
            }
        }
        best = key < best ? key : best;
    }
    best = warp_min_u64(best);
    if (lane == 0) {
        uint32_t a;
        if (phase == kPhaseBalance) {
            a = (u >= kBits) ? kActFinal : uint32_t(best & 0xFF);
        } else if (phase == kPhasePeel) {
            const uint32_t maxf = 0xFFFFFFFFu - uint32_t(best >> 8);
            // maxf == 0 only for a range of all-zero filters, on which the
            // reference never terminates; it becomes its own partition.
            a = (maxf == size || maxf == 0) ? kActFinal : uint32_t(best & 0xFF);
        } else {
            a = (best == ~0ull) ? kActChop : uint32_t(best & 0xFF);
        }
        action[s] = a;
    }
}

__global__ void __launch_bounds__(kPThreads) k_split_count(const Seg *__restrict__ segs, const uint32_t *__restrict__ chunk_off,
                                                           uint32_t n_act, const uint32_t *__restrict__ action,
                                                           const uint32_t *__restrict__ words, uint32_t *__restrict__ zc) {
    __shared__ uint32_t s_seg, s_cnt;
    if (threadIdx.x == 0) { s_seg = find_seg(chunk_off, n_act, blockIdx.x); s_cnt = 0; }
    __syncthreads();
    const uint32_t s = s_seg;
    const uint32_t a = action[s];
    if (a >= kBits) {
        if (threadIdx.x == 0) zc[blockIdx.x] = 0;
        return;
    }
    const Seg seg = segs[s];
    const uint32_t cstart = seg.begin + (blockIdx.x - chunk_off[s]) * kPChunk;
    const uint32_t cend = min(cstart + (uint32_t)kPChunk, seg.end);
    uint32_t z = 0;
    for (uint32_t i = cstart + threadIdx.x; i < cend; i += kPThreads)
        z += !((words[size_t(i) * kWords + (a >> 5)] >> (a & 31)) & 1u);
    z = __reduce_add_sync(kFull, z);
    if ((threadIdx.x & 31) == 0 && z) atomicAdd(&s_cnt, z);
    __syncthreads();
    if (threadIdx.x == 0) zc[blockIdx.x] = s_cnt;
}

__global__ void __launch_bounds__(kPThreads) k_split_scatter(const Seg *__restrict__ segs, const uint32_t *__restrict__ chunk_off,
                                                             uint32_t n_act, const uint32_t *__restrict__ action,
                                                             const uint64_t *__restrict__ zoff,
                                                             const uint32_t *__restrict__ words, const uint32_t *__restrict__ order,
                                                             uint32_t *__restrict__ words_out, uint32_t *__restrict__ order_out) {
    __shared__ uint32_t s_seg;
    if (threadIdx.x == 0) s_seg = find_seg(chunk_off, n_act, blockIdx.x);
    __syncthreads();
    const uint32_t s = s_seg;
    const uint32_t a = action[s];
    const Seg seg = segs[s];
    const uint32_t cstart = seg.begin + (blockIdx.x - chunk_off[s]) * kPChunk;
    const uint32_t cend = min(cstart + (uint32_t)kPChunk, seg.end);
    const bool split = a < kBits;
    const uint32_t zb = split ? uint32_t(zoff[blockIdx.x] - zoff[chunk_off[s]]) : 0;        // zeros before this chunk
    const uint32_t zseg = split ? uint32_t(zoff[chunk_off[s + 1]] - zoff[chunk_off[s]]) : 0;  // zeros in the range
    const uint32_t local = cstart - seg.begin;
    uint32_t zrun = 0;
    for (uint32_t r = 0; r < (uint32_t)kPChunk; r += kPThreads) {
        const uint32_t i = cstart + r + threadIdx.x;
        const bool valid = i < cend;
        uint32_t w[kWords];
        uint32_t o = 0;
        if (valid) {
#pragma unroll
            for (int k = 0; k < kWords; ++k) w[k] = words[size_t(i) * kWords + k];
            o = order[i];
        }
        uint32_t z = (valid && split) ? !((w[a >> 5 & 7] >> (a & 31)) & 1u) : 0u;
        uint32_t tot;
        uint32_t zr = block_excl_scan<uint32_t>(z, tot);
        if (valid) {
            uint32_t dst;
            if (!split) {
                dst = i;
            } else {
                const uint32_t zero_rank = zrun + zr;
                const uint32_t pos_in_chunk = r + threadIdx.x;
                if (z) dst = seg.begin + zb + zero_rank;
                else dst = seg.begin + zseg + (local - zb) + (pos_in_chunk - zero_rank);
            }
#pragma unroll
            for (int k = 0; k < kWords; ++k) words_out[size_t(dst) * kWords + k] = w[k];
            order_out[dst] = o;
        }
        zrun += tot;
        if (r + kPThreads >= cend - cstart) break;
    }
}

__global__ void __launch_bounds__(kPThreads) k_copy_back(const Seg *__restrict__ segs, const uint32_t *__restrict__ chunk_off,
                                                         uint32_t n_act, const uint32_t *__restrict__ words_in,
                                                         const uint32_t *__restrict__ order_in, uint32_t *__restrict__ words,
                                                         uint32_t *__restrict__ order) {
    __shared__ uint32_t s_seg;
    if (threadIdx.x == 0) s_seg = find_seg(chunk_off, n_act, blockIdx.x);
    __syncthreads();
    const uint32_t s = s_seg;
    const Seg seg = segs[s];
    const uint32_t cstart = seg.begin + (blockIdx.x - chunk_off[s]) * kPChunk;
    const uint32_t cend = min(cstart + (uint32_t)kPChunk, seg.end);
    for (uint32_t i = cstart + threadIdx.x; i < cend; i += kPThreads) {
#pragma unroll
        for (int k = 0; k < kWords; ++k) words[size_t(i) * kWords + k] = words_in[size_t(i) * kWords + k];
        order[i] = order_in[i];
    }
}

struct ChildCtx {
    Seg *next;
    Range *finals;
    Range *leaves;
    Counters *cnt;
    uint32_t max_p;
    uint32_t finals_cap, leaves_cap;
    bool with_tiles;
};

__device__ void push_active(const ChildCtx &c, uint32_t b, uint32_t e, const uint32_t *used, uint32_t flags) {
    uint32_t k = atomicAdd(&c.cnt->next, 1u);
    Seg s;
    s.begin = b;
    s.end = e;
#pragma unroll
    for (int i = 0; i < kWords; ++i) s.used[i] = used ? used[i] : 0u;
    s.flags = flags;
    s.pad = 0;
    c.next[k] = s;
    atomicAdd(&c.cnt->next_chunks, (e - b + kPChunk - 1) / kPChunk);
}

__device__ void push_leaf(const ChildCtx &c, uint32_t b, uint32_t e) {
    uint32_t k = atomicAdd(&c.cnt->leaves, 1u);
    if (k < c.leaves_cap) c.leaves[k] = Range{b, e};
}

__device__ void push_final(const ChildCtx &c, uint32_t b, uint32_t e) {
    uint32_t k = atomicAdd(&c.cnt->finals, 1u);
    if (k < c.finals_cap) c.finals[k] = Range{b, e};
    if (c.with_tiles) {
        if (e - b > (uint32_t)kTile) push_active(c, b, e, nullptr, kPhaseTile);
        else if (e > b) push_leaf(c, b, e);
    }
}

// A side of a balancing split (the partition rules of do_balanced_partitioning).
__device__ void balance_child(const ChildCtx &c, uint32_t b, uint32_t e, const uint32_t *used, bool mask_empty) {
    const uint32_t size = e - b;
    if (size > c.max_p) push_active(c, b, e, used, kPhaseBalance | (mask_empty ? kMaskEmpty : 0u));
    else if (mask_empty && size > 0) push_active(c, b, e, nullptr, kPhasePeel);
    else push_final(c, b, e);
}

__device__ void tile_child(const ChildCtx &c, uint32_t b, uint32_t e, const uint32_t *used) {
    if (e - b > (uint32_t)kTile) push_active(c, b, e, used, kPhaseTile);
    else if (e > b) push_leaf(c, b, e);
}

__global__ void k_children(const Seg *__restrict__ segs, uint32_t n_act, const uint32_t *__restrict__ action,
                           const uint32_t *__restrict__ chunk_off, const uint64_t *__restrict__ zoff, ChildCtx c) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_act) return;
    const Seg seg = segs[s];
    const uint32_t a = action[s];
    const uint32_t phase = seg.flags & kPhaseMask;
    if (a < kBits) {
        const uint32_t z = uint32_t(zoff[chunk_off[s + 1]] - zoff[chunk_off[s]]);
        const uint32_t m = seg.begin + z;
        uint32_t used[kWords];
#pragma unroll
        for (int k = 0; k < kWords; ++k) used[k] = seg.used[k];
        used[a >> 5] |= 1u << (a & 31);
        if (phase == kPhaseBalance) {
            balance_child(c, seg.begin, m, used, (seg.flags & kMaskEmpty) != 0);
            balance_child(c, m, seg.end, used, false);
        } else if (phase == kPhasePeel) {
            push_final(c, m, seg.end);
            push_active(c, seg.begin, m, nullptr, kPhasePeel);
        } else {
            tile_child(c, seg.begin, m, used);
            tile_child(c, m, seg.end, used);
        }
    } else if (a == kActFinal) {
        push_final(c, seg.begin, seg.end);
    } else {
        push_leaf(c, seg.begin, seg.end);  // cannot split further: chopped into tiles of 32
    }
}

__global__ void k_mark_tiles(const Range *__restrict__ leaves, uint32_t n_leaves, uint32_t *__restrict__ mark) {
    const uint32_t l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= n_leaves) return;
    const Range r = leaves[l];
    for (uint32_t p = r.begin; p < r.end; p += kTile) mark[p] = 1;
}

__global__ void k_init_order(uint32_t *order, uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) order[i] = i;
}

inline unsigned blocks_for(size_t n, unsigned t) { return unsigned((n + t - 1) / t); }

}  // namespace

void gpu_partition(const uint32_t *d_filters, uint32_t n, uint32_t max_p, bool with_tiles, PartitionResult &out,
                   cudaStream_t st) {
    if (max_p == 0) throw Error(TM_ERR_INVALID, "partition size must be at least 1");
    out.n = n;
    out.parts.clear();
    out.bit_freq.assign(kBits, 0);
    out.words.reserve(size_t(n) * kWords);
    out.order.reserve(n);
    if (with_tiles) out.tile_mark.reserve(n);
    if (n == 0) return;
    TM_CUDA(cudaMemcpyAsync(out.words.p, d_filters, size_t(n) * kWords * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
    k_init_order<<<blocks_for(n, 256), 256, 0, st>>>(out.order.p, n);
    TM_CHECK_LAUNCH();

    DevBuf<uint32_t> alt_words, alt_order;
    alt_words.reserve(size_t(n) * kWords);
    alt_order.reserve(n);
    DevBuf<Seg> segs[2];
    DevBuf<uint32_t> nch, chunk_off, freq, action, zc;
    DevBuf<uint64_t> zoff;
    DevBuf<Range> finals, leaves;
    DevBuf<Counters> cnt;
    DevBuf<float> weights;
    ScanScratch scr;
    cnt.reserve(1);
    weights.reserve(kBits);
    uint32_t finals_cap = n + 1024;
    uint32_t leaves_cap = with_tiles ? n + 1 : 1;
    finals.reserve(finals_cap);
    leaves.reserve(leaves_cap);

    // root
    Seg root;
    std::memset(&root, 0, sizeof(root));
    root.begin = 0;
    root.end = n;
    root.flags = n > max_p ? (kPhaseBalance | kMaskEmpty) : kPhasePeel;
    segs[0].reserve(1);
    TM_CUDA(cudaMemcpyAsync(segs[0].p, &root, sizeof(Seg), cudaMemcpyHostToDevice, st));
    uint32_t n_act = 1;
    uint32_t total_chunks = (n + kPChunk - 1) / kPChunk;
    int cur = 0;
    Counters hc;
    std::memset(&hc, 0, sizeof(hc));
    TM_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(Counters), st));
    int levels = 0;
    while (n_act > 0) {
        if (++levels > 100000) throw Error(TM_ERR_INTERNAL, "partitioner did not converge");
        nch.reserve(n_act);
        chunk_off.reserve(n_act + 1);
        k_nchunks<<<blocks_for(n_act, 256), 256, 0, st>>>(segs[cur].p, n_act, nch.p);
        TM_CHECK_LAUNCH();
        exclusive_scan<uint32_t, uint32_t>(nch.p, chunk_off.p, n_act, scr, st);
        freq.reserve(size_t(n_act) * kBits);
        TM_CUDA(cudaMemsetAsync(freq.p, 0, size_t(n_act) * kBits * sizeof(uint32_t), st));
        k_freq<<<total_chunks, kPThreads, 0, st>>>(segs[cur].p, chunk_off.p, n_act, out.words.p, freq.p);
        TM_CHECK_LAUNCH();
        action.reserve(n_act);
        if (levels == 1) {
            // bit frequencies of the whole table -> tile-split weights:
            // a query lacks bit b with estimated probability
            // (1 - freq_b / n)^kTileWeightExp
            std::vector<uint32_t> &rf = out.bit_freq;
            rf.assign(kBits, 0);
            TM_CUDA(cudaMemcpyAsync(rf.data(), freq.p, kBits * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
            TM_CUDA(cudaStreamSynchronize(st));
            std::vector<float> w(kBits);
            for (int b = 0; b < kBits; ++b) w[b] = float(std::pow(1.0 - double(rf[b]) / double(n), kTileWeightExp));
            weights.reserve(kBits);
            TM_CUDA(cudaMemcpyAsync(weights.p, w.data(), kBits * sizeof(float), cudaMemcpyHostToDevice, st));
        }
        k_decide<<<blocks_for(size_t(n_act) * 32, 256), 256, 0, st>>>(segs[cur].p, n_act, freq.p, weights.p, action.p);
        TM_CHECK_LAUNCH();
        zc.reserve(total_chunks);
        zoff.reserve(size_t(total_chunks) + 1);
        k_split_count<<<total_chunks, kPThreads, 0, st>>>(segs[cur].p, chunk_off.p, n_act, action.p, out.words.p, zc.p);
        TM_CHECK_LAUNCH();
        exclusive_scan<uint32_t, uint64_t>(zc.p, zoff.p, total_chunks, scr, st);
        k_split_scatter<<<total_chunks, kPThreads, 0, st>>>(segs[cur].p, chunk_off.p, n_act, action.p, zoff.p, out.words.p,
                                                           out.order.p, alt_words.p, alt_order.p);
        TM_CHECK_LAUNCH();
        k_copy_back<<<total_chunks, kPThreads, 0, st>>>(segs[cur].p, chunk_off.p, n_act, alt_words.p, alt_order.p, out.words.p,
                                                       out.order.p);
        TM_CHECK_LAUNCH();
        segs[cur ^ 1].reserve(size_t(n_act) * 2 + 2);
        TM_CUDA(cudaMemsetAsync(&cnt.p->next, 0, 2 * sizeof(uint32_t), st));
        ChildCtx c{segs[cur ^ 1].p, finals.p, leaves.p, cnt.p, max_p, finals_cap, leaves_cap, with_tiles};
        k_children<<<blocks_for(n_act, 128), 128, 0, st>>>(segs[cur].p, n_act, action.p, chunk_off.p, zoff.p, c);
        TM_CHECK_LAUNCH();
        TM_CUDA(cudaMemcpyAsync(&hc, cnt.p, sizeof(Counters), cudaMemcpyDeviceToHost, st));
        TM_CUDA(cudaStreamSynchronize(st));
        if (hc.finals > finals_cap || hc.leaves > leaves_cap) throw Error(TM_ERR_INTERNAL, "partitioner list overflow");
        n_act = hc.next;
        total_chunks = hc.next_chunks;
        cur ^= 1;
    }

    // partitions in position order
    std::vector<Range> h(hc.finals);
    if (hc.finals) TM_CUDA(cudaMemcpy(h.data(), finals.p, sizeof(Range) * hc.finals, cudaMemcpyDeviceToHost));
    std::sort(h.begin(), h.end(), [](const Range &x, const Range &y) {
        return x.begin != y.begin ? x.begin < y.begin : x.end < y.end;
    });
    out.parts = std::move(h);

    if (with_tiles) {
        TM_CUDA(cudaMemsetAsync(out.tile_mark.p, 0, size_t(n) * sizeof(uint32_t), st));
        if (hc.leaves) {
            k_mark_tiles<<<blocks_for(hc.leaves, 256), 256, 0, st>>>(leaves.p, hc.leaves, out.tile_mark.p);
            TM_CHECK_LAUNCH();
        }
    }
    TM_CUDA(cudaStreamSynchronize(st));
}

// ---------------------------------------------------------------------------
// Table build
// ---------------------------------------------------------------------------
namespace {

// One warp per tile: transposes the members into [6][32] words, ANDs them,
// records the original filter index of every lane, and picks the tile's
// selection bits: the first kSelBits bits of the AND in `bit_order` (rarest
// in the table first).
__global__ void k_build_tiles(const uint32_t *__restrict__ words, const uint32_t *__restrict__ order,
                              const uint32_t *__restrict__ tile_begin /* n_tiles + 1 */, uint32_t n_tiles,
                              const uint32_t *__restrict__ part_tile_begin, uint32_t n_parts,
                              const uint8_t *__restrict__ bit_order, uint32_t *__restrict__ tile_words,
                              TileInfo *__restrict__ info, uint32_t *__restrict__ tile_and,
                              uint32_t *__restrict__ slot_filter) {
    const uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned lane = threadIdx.x & 31;
    if (t >= n_tiles) return;
    const uint32_t b = tile_begin[t], e = tile_begin[t + 1];
    const uint32_t cnt = e - b;
    const bool valid = lane < cnt;
    uint32_t w[kWords];
#pragma unroll
    for (int k = 0; k < kWords; ++k) w[k] = valid ? words[size_t(b + lane) * kWords + k] : 0u;
#pragma unroll
    for (int k = 0; k < kWords; ++k) tile_words[(size_t(t) * kWords + k) * kTile + lane] = w[k];
    slot_filter[size_t(t) * kTile + lane] = valid ? order[b + lane] : 0xFFFFFFFFu;
    uint32_t am[kWords];
#pragma unroll
    for (int k = 0; k < kWords; ++k) am[k] = __reduce_and_sync(kFull, valid ? w[k] : 0xFFFFFFFFu);
    if (lane < 8) tile_and[size_t(t) * 8 + lane] = lane < kWords ? am[lane < kWords ? lane : 0] : 0u;
    if (lane == 0) {
        uint32_t lo = 0, hi = n_parts;  // owning partition: last p with part_tile_begin[p] <= t
        while (hi - lo > 1) {
            uint32_t mid = (lo + hi) >> 1;
            if (part_tile_begin[mid] <= t) lo = mid;
            else hi = mid;
        }
        uint32_t sel[2] = {0, 0};
        int k = 0;
        for (int i = 0; i < kBits && k < kSelBits; ++i) {
            const uint32_t bit = bit_order[i];
            if ((am[bit >> 5] >> (bit & 31)) & 1u) {
                sel[k >> 2] |= bit << (8 * (k & 3));
                ++k;
            }
        }
        for (; k < kSelBits; ++k) sel[k >> 2] |= kNoBit << (8 * (k & 3));
        TileInfo ti;
        ti.sel[0] = sel[0];
        ti.sel[1] = sel[1];
        ti.count = cnt;
        ti.partition = lo;
        info[t] = ti;
    }
}

__global__ void k_tile_begin(const uint32_t *__restrict__ mark, const uint32_t *__restrict__ mark_off, uint32_t n,
                             uint32_t *__restrict__ tile_begin) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && mark[i]) tile_begin[mark_off[i]] = i;
    if (i == 0) tile_begin[mark_off[n]] = n;
}

__global__ void k_part_tiles(const Range *__restrict__ parts, uint32_t n_parts, const uint32_t *__restrict__ mark_off,
                             uint32_t *__restrict__ part_tile_begin) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < n_parts) part_tile_begin[p] = mark_off[parts[p].begin];
    if (p == 0) part_tile_begin[n_parts] = n_parts ? mark_off[parts[n_parts - 1].end] : 0;
}

__global__ void k_part_mask(const uint32_t *__restrict__ tile_and, const uint32_t *__restrict__ part_tile_begin,
                            uint32_t n_parts, uint32_t *__restrict__ part_mask) {
    const uint32_t p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned lane = threadIdx.x & 31;
    if (p >= n_parts) return;
    const uint32_t tb = part_tile_begin[p], te = part_tile_begin[p + 1];
    uint32_t m[kWords];
#pragma unroll
    for (int k = 0; k < kWords; ++k) m[k] = 0xFFFFFFFFu;
    for (uint32_t t = tb + lane; t < te; t += 32) {
#pragma unroll
        for (int k = 0; k < kWords; ++k) m[k] &= tile_and[size_t(t) * 8 + k];
    }
#pragma unroll
    for (int k = 0; k < kWords; ++k) m[k] = __reduce_and_sync(kFull, m[k]);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < kWords; ++k) part_mask[size_t(p) * 8 + k] = m[k];
        part_mask[size_t(p) * 8 + 6] = te - tb;
        part_mask[size_t(p) * 8 + 7] = 0;
    }
}

__global__ void k_slot_nkeys(const uint32_t *__restrict__ slot_filter, size_t n_slots, const uint32_t *__restrict__ key_off,
                             uint32_t *__restrict__ nkeys) {
    const size_t s = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (s >= n_slots) return;
    const uint32_t f = slot_filter[s];
    nkeys[s] = f == 0xFFFFFFFFu ? 0u : key_off[f + 1] - key_off[f];
}

__global__ void k_slot_keys(const uint32_t *__restrict__ slot_filter, size_t n_slots, const uint32_t *__restrict__ key_off,
                            const uint32_t *__restrict__ keys, const uint32_t *__restrict__ slot_key_off,
                            uint32_t *__restrict__ out_keys) {
    const size_t s = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (s >= n_slots) return;
    const uint32_t f = slot_filter[s];
    if (f == 0xFFFFFFFFu) return;
    const uint32_t b = key_off[f], e = key_off[f + 1];
    uint32_t d = slot_key_off[s];
    for (uint32_t k = b; k < e; ++k) out_keys[d++] = keys[k];
}

// One warp per tile: the key counts of its lanes' filters as bit planes.
__global__ void k_tile_keys(const uint32_t *__restrict__ slot_key_off, uint32_t n_tiles, TileKeys *__restrict__ out) {
    const uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned lane = threadIdx.x & 31;
    if (t >= n_tiles) return;
    const size_t s = size_t(t) * kTile + lane;
    const uint32_t nk = slot_key_off[s + 1] - slot_key_off[s];
    TileKeys tk;
    tk.p[0] = __ballot_sync(kFull, nk < 8 && (nk & 1));
    tk.p[1] = __ballot_sync(kFull, nk < 8 && (nk & 2));
    tk.p[2] = __ballot_sync(kFull, nk < 8 && (nk & 4));
    tk.wide = __ballot_sync(kFull, nk >= 8);
    if (lane == 0) out[t] = tk;
}

__global__ void k_max_key(const uint32_t *__restrict__ keys, size_t n, uint32_t *__restrict__ out) {
    uint32_t m = 0;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        m = max(m, keys[i]);
    m = __reduce_max_sync(kFull, m);
    if ((threadIdx.x & 31) == 0 && m) atomicMax(out, m);
}

}  // namespace

size_t DevTable::device_bytes() const {
    return tile_words.cap * sizeof(uint32_t) + tile_info.cap * sizeof(TileInfo) + tile_and.cap * 4 + part_tile_begin.cap * 4 +
           part_mask.cap * 4 + slot_key_off.cap * 4 + tile_keys.cap * sizeof(TileKeys) + keys.cap * 4 +
           slot_filter.cap * 4;
}

void build_table(const PartitionResult &pr, const uint32_t *d_key_off, const uint32_t *d_keys, uint64_t n_keys, DevTable &t,
                 cudaStream_t st) {
    const uint32_t n = pr.n;
    t.n_filters = n;
    t.n_parts = uint32_t(pr.parts.size());
    t.n_keys = n_keys;
    ScanScratch scr;
    DevBuf<uint32_t> mark_off, tile_begin, nkeys;
    DevBuf<Range> parts;
    mark_off.reserve(size_t(n) + 1);
    if (n) {
        exclusive_scan<uint32_t, uint32_t>(pr.tile_mark.p, mark_off.p, n, scr, st);
        TM_CUDA(cudaMemcpyAsync(&t.n_tiles, mark_off.p + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        TM_CUDA(cudaStreamSynchronize(st));
    } else {
        t.n_tiles = 0;
        TM_CUDA(cudaMemsetAsync(mark_off.p, 0, sizeof(uint32_t), st));
    }
    const uint32_t nt = t.n_tiles;
    const size_t n_slots = size_t(nt) * kTile;
    tile_begin.reserve(size_t(nt) + 1);
    if (n) {
        k_tile_begin<<<blocks_for(n, 256), 256, 0, st>>>(pr.tile_mark.p, mark_off.p, n, tile_begin.p);
        TM_CHECK_LAUNCH();
    }
    t.part_tile_begin.reserve(size_t(t.n_parts) + 1);
    parts.reserve(std::max<size_t>(t.n_parts, 1));
    if (t.n_parts) {
        TM_CUDA(cudaMemcpyAsync(parts.p, pr.parts.data(), sizeof(Range) * t.n_parts, cudaMemcpyHostToDevice, st));
    }
    k_part_tiles<<<blocks_for(std::max<uint32_t>(t.n_parts, 1), 256), 256, 0, st>>>(parts.p, t.n_parts, mark_off.p,
                                                                                    t.part_tile_begin.p);
    TM_CHECK_LAUNCH();
    t.tile_words.reserve(n_slots * kWords);
    t.tile_info.reserve(nt);
    t.tile_and.reserve(size_t(std::max<uint32_t>(nt, 1)) * 8);
    t.slot_filter.reserve(n_slots);
    // selection bits are taken rarest-first over the whole table
    std::vector<uint8_t> order_h(kBits);
    for (int b = 0; b < kBits; ++b) order_h[b] = uint8_t(b);
    std::stable_sort(order_h.begin(), order_h.end(),
                     [&](uint8_t x, uint8_t y) { return pr.bit_freq[x] < pr.bit_freq[y]; });
    DevBuf<uint8_t> bit_order;
    bit_order.reserve(kBits);
    TM_CUDA(cudaMemcpyAsync(bit_order.p, order_h.data(), kBits, cudaMemcpyHostToDevice, st));
    if (nt) {
        k_build_tiles<<<blocks_for(size_t(nt) * 32, 256), 256, 0, st>>>(pr.words.p, pr.order.p, tile_begin.p, nt,
                                                                       t.part_tile_begin.p, t.n_parts, bit_order.p,
                                                                       t.tile_words.p, t.tile_info.p, t.tile_and.p,
                                                                       t.slot_filter.p);
        TM_CHECK_LAUNCH();
    }
    t.part_mask.reserve(size_t(std::max<uint32_t>(t.n_parts, 1)) * 8);
    if (t.n_parts) {
        k_part_mask<<<blocks_for(size_t(t.n_parts) * 32, 256), 256, 0, st>>>(t.tile_and.p, t.part_tile_begin.p, t.n_parts,
                                                                            t.part_mask.p);
        TM_CHECK_LAUNCH();
    }
    // keys in slot order
    nkeys.reserve(n_slots);
    t.slot_key_off.reserve(n_slots + 1);
    t.keys.reserve(std::max<uint64_t>(n_keys, 1));
    if (n_slots) {
        k_slot_nkeys<<<blocks_for(n_slots, 256), 256, 0, st>>>(t.slot_filter.p, n_slots, d_key_off, nkeys.p);
        TM_CHECK_LAUNCH();
    }
    exclusive_scan<uint32_t, uint32_t>(nkeys.p, t.slot_key_off.p, n_slots, scr, st);
    if (n_slots) {
        k_slot_keys<<<blocks_for(n_slots, 256), 256, 0, st>>>(t.slot_filter.p, n_slots, d_key_off, d_keys, t.slot_key_off.p,
                                                             t.keys.p);
        TM_CHECK_LAUNCH();
    }
    t.tile_keys.reserve(std::max<uint32_t>(nt, 1));
    if (nt) {
        k_tile_keys<<<blocks_for(size_t(nt) * 32, 256), 256, 0, st>>>(t.slot_key_off.p, nt, t.tile_keys.p);
        TM_CHECK_LAUNCH();
    }
    DevBuf<uint32_t> mk;
    mk.reserve(1);
    TM_CUDA(cudaMemsetAsync(mk.p, 0, sizeof(uint32_t), st));
    if (n_keys) {
        k_max_key<<<256, 256, 0, st>>>(t.keys.p, n_keys, mk.p);
        TM_CHECK_LAUNCH();
    }
    TM_CUDA(cudaMemcpyAsync(&t.max_key, mk.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    t.h_part_size.resize(t.n_parts);
    for (uint32_t p = 0; p < t.n_parts; ++p) t.h_part_size[p] = pr.parts[p].end - pr.parts[p].begin;
    t.h_part_mask.assign(size_t(t.n_parts) * 8, 0);
    t.h_part_tiles.assign(size_t(t.n_parts) + 1, 0);
    if (t.n_parts) {
        TM_CUDA(cudaMemcpyAsync(t.h_part_mask.data(), t.part_mask.p, sizeof(uint32_t) * 8 * t.n_parts, cudaMemcpyDeviceToHost, st));
    }
    TM_CUDA(cudaMemcpyAsync(t.h_part_tiles.data(), t.part_tile_begin.p, sizeof(uint32_t) * (t.n_parts + 1),
                            cudaMemcpyDeviceToHost, st));
    TM_CUDA(cudaStreamSynchronize(st));
}

}  // namespace tmb
