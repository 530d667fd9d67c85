// Batched matching that allocates nothing: tm_match_batch_device_noalloc.
//
// Who needs it: callers that must not allocate device memory while they
// match -- code that has handed all device memory to its own pool
// allocator, latency-critical serving threads that cannot afford a
// cudaMalloc (which may synchronise the device), or callers running in a
// context where the CUDA allocator may not be entered.  For them this entry
// point runs the same routing, subset-test, key-gather and match_unique
// kernels as tm_match_batch_device, but takes every scratch buffer from one
// file-scope device array of fixed size, so it never calls cudaMalloc,
// cudaFree or any allocating library routine.  The caller passes the
// queries and the output buffers; the table is the engine's (built by
// consolidate).
//
// Limits: at most kNoAllocMaxQueries queries per call, at most
// kNoAllocMaxPartitions partitions in the table, and all scratch of the
// call (partition queues, query slices, matching pairs, and for
// match_unique a key buffer) within kNoAllocScratchBytes; a batch that
// needs more is rejected with TM_ERR_CAPACITY and a message giving the
// bytes it needed -- split it and call again.
//
// The array is shared by every call in the process and keeps the contents
// of the last call (each call clears what must start at zero).  Calls whose
// work overlaps on the GPU -- concurrent calls from several threads, or
// calls on different streams that are not ordered -- race on the array.
//
// In host code the array's name is only a host-side stand-in, not a device
// address.  Each engine looks up the array's device address once per device
// (cudaGetSymbolAddress, below, with that device current) at its first call
// of this entry point, and keeps it with its device table; make that first
// call before any stream capture.  A cudaDeviceReset frees the engine's
// device table along with the module that holds the array, so after a reset
// the engine is unusable anyway: create a new one, which looks the address
// up again.
#include "../../include/tagmatch_b200.h"
#include "engine.cuh"
#include "match_kernels.cuh"
#include <string>

namespace tmb {
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(64) << 20;  // 64 MiB per device
constexpr uint32_t kNoAllocMaxQueries = 4096;
constexpr uint32_t kNoAllocMaxPartitions = 16384;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

}  // namespace

void *noalloc_scratch_address() {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
        throw Error(TM_ERR_CUDA, cuda_msg(e, "cudaGetSymbolAddress(g_noalloc_scratch)", __FILE__, __LINE__));
    return p;
}

namespace {

// Bump carving of the static array, 256-byte aligned pieces.
struct Arena {
    unsigned char *base;
    size_t used = 0;
    template <class T>
    T *take(size_t count, const char *what) {
        const size_t off = (used + 255) & ~size_t(255);
        const size_t bytes = count * sizeof(T);
        if (off + bytes > kNoAllocScratchBytes)
            throw Error(TM_ERR_CAPACITY, std::string("no-allocation scratch exhausted at ") + what + ": needs " +
                                             std::to_string(off + bytes) + " bytes, the array holds " +
                                             std::to_string(kNoAllocScratchBytes) + "; split the batch");
        used = off + bytes;
        return reinterpret_cast<T *>(base + off);
    }
    // gives back everything taken after end (end: one past the last byte kept)
    void trim(const void *end) { used = size_t(static_cast<const unsigned char *>(end) - base); }
    size_t left() const {
        const size_t off = (used + 255) & ~size_t(255);
        return off < kNoAllocScratchBytes ? kNoAllocScratchBytes - off : 0;
    }
};

// Work-plan counts per partition: 256-query chunks, and work items (groups
// of kItemChunks chunks x tile segments).
__global__ void k_plan_counts(const uint32_t *__restrict__ part_count, const uint32_t *__restrict__ part_tile_begin,
                              uint32_t n_parts, uint32_t seg_tiles, uint32_t *__restrict__ nchunks,
                              uint32_t *__restrict__ nitems) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n_parts) return;
    const uint32_t c = (part_count[p] + kChunk - 1) / kChunk;
    const uint32_t nt = part_tile_begin[p + 1] - part_tile_begin[p];
    nchunks[p] = c;
    nitems[p] = ((c + kItemChunks - 1) / kItemChunks) * ((nt + seg_tiles - 1) / seg_tiles);
}

// Exclusive scan with block sums held in the arena (up to 2048 x 2048 elements).
template <class Tin, class Tout>
void scan_fixed(const Tin *in, Tout *out, size_t n, uint64_t *sums, uint64_t *offs, cudaStream_t st) {
    const size_t nb = (n + kScanTile - 1) / kScanTile;
    if (nb <= 1) {
        k_scan_apply<Tin, Tout><<<1, kScanThreads, 0, st>>>(in, n, nullptr, out);
        TM_CHECK_LAUNCH();
        return;
    }
    if (nb > size_t(kScanTile)) throw Error(TM_ERR_INVALID, "no-allocation scan: too many elements");
    k_scan_reduce<Tin, uint64_t><<<(unsigned)nb, kScanThreads, 0, st>>>(in, n, sums);
    TM_CHECK_LAUNCH();
    k_scan_apply<uint64_t, uint64_t><<<1, kScanThreads, 0, st>>>(sums, nb, nullptr, offs);
    TM_CHECK_LAUNCH();
    k_scan_apply<Tin, Tout><<<(unsigned)nb, kScanThreads, 0, st>>>(in, n, offs, out);
    TM_CHECK_LAUNCH();
}

}  // namespace

// The whole pipeline over the static array.  d_out_offsets: n + 1 entries;
// d_out_keys: capacity keys; both device memory owned by the caller.
void match_batch_noalloc(const DevTable &t, const uint32_t *d_queries, uint32_t nq, bool unique, uint32_t seg_tiles,
                         void *scratch, uint64_t *d_out_offsets, uint32_t *d_out_keys, uint64_t capacity,
                         uint64_t *n_keys, cudaStream_t st) {
    if (nq > kNoAllocMaxQueries)
        throw Error(TM_ERR_INVALID, "tm_match_batch_device_noalloc: at most " + std::to_string(kNoAllocMaxQueries) +
                                        " queries per call, got " + std::to_string(nq));
    const uint32_t P = t.n_parts;
    if (P > kNoAllocMaxPartitions)
        throw Error(TM_ERR_INVALID, "tm_match_batch_device_noalloc: the table has " + std::to_string(P) +
                                        " partitions, at most " + std::to_string(kNoAllocMaxPartitions) + " supported");
    int dev = 0, sms = 0;
    TM_CUDA(cudaGetDevice(&dev));
    TM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (seg_tiles == 0) throw Error(TM_ERR_INVALID, "tiles per work item must be positive");
    Arena ar{static_cast<unsigned char *>(scratch)};
    *n_keys = 0;
    if (nq == 0 || P == 0 || t.n_tiles == 0) {
        TM_CUDA(cudaMemsetAsync(d_out_offsets, 0, (size_t(nq) + 1) * sizeof(uint64_t), st));
        TM_CUDA(cudaStreamSynchronize(st));
        return;
    }
    unsigned long long *counters = ar.take<unsigned long long>(4, "counters");
    uint32_t *part_count = ar.take<uint32_t>(P, "partition counts");
    uint32_t *part_cursor = ar.take<uint32_t>(P, "partition cursors");
    uint32_t *part_off = ar.take<uint32_t>(size_t(P) + 1, "partition offsets");
    uint32_t *nchunks = ar.take<uint32_t>(P, "plan");
    uint32_t *nitems = ar.take<uint32_t>(P, "plan");
    uint32_t *chunk_off = ar.take<uint32_t>(size_t(P) + 1, "plan");
    uint32_t *item_off = ar.take<uint32_t>(size_t(P) + 1, "plan");
    uint64_t *sums = ar.take<uint64_t>(kScanTile, "scan");
    uint64_t *offs = ar.take<uint64_t>(kScanTile + 1, "scan");
    uint32_t *qkeys = ar.take<uint32_t>(nq, "query key counts");
    uint32_t *qcursor = ar.take<uint32_t>(nq, "query cursors");
    uint64_t *qoff = ar.take<uint64_t>(size_t(nq) + 1, "query offsets");
    uint32_t *ucount = ar.take<uint32_t>(nq, "unique counts");
    TM_CUDA(cudaMemsetAsync(counters, 0, 4 * sizeof(unsigned long long), st));
    TM_CUDA(cudaMemsetAsync(part_count, 0, P * sizeof(uint32_t), st));
    TM_CUDA(cudaMemsetAsync(part_cursor, 0, P * sizeof(uint32_t), st));
    TM_CUDA(cudaMemsetAsync(qkeys, 0, nq * sizeof(uint32_t), st));
    TM_CUDA(cudaMemsetAsync(qcursor, 0, nq * sizeof(uint32_t), st));

    // routing counts and the work plan
    const unsigned rblocks = blocks_for(nq, kRouteThreads);
    for (uint32_t p0 = 0; p0 < P; p0 += kMaxRouteParts) {
        const uint32_t pw = std::min(kMaxRouteParts, P - p0);
        const size_t smem = size_t(pw) * (kWords + 2) * sizeof(uint32_t);
        k_route<false><<<rblocks, kRouteThreads, smem, st>>>(d_queries, nq, t.part_mask.p, p0, pw, part_count, nullptr,
                                                            nullptr, nullptr);
        TM_CHECK_LAUNCH();
    }
    scan_fixed<uint32_t, uint32_t>(part_count, part_off, P, sums, offs, st);
    k_plan_counts<<<blocks_for(P, 256), 256, 0, st>>>(part_count, t.part_tile_begin.p, P, seg_tiles, nchunks, nitems);
    TM_CHECK_LAUNCH();
    scan_fixed<uint32_t, uint32_t>(nchunks, chunk_off, P, sums, offs, st);
    scan_fixed<uint32_t, uint32_t>(nitems, item_off, P, sums, offs, st);
    uint32_t routed = 0, chunks = 0;
    TM_CUDA(cudaMemcpyAsync(&routed, part_off + P, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    TM_CUDA(cudaMemcpyAsync(&chunks, chunk_off + P, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    TM_CUDA(cudaStreamSynchronize(st));

    uint32_t *queue = ar.take<uint32_t>(size_t(std::max<uint32_t>(routed, 1)) * kQueueWords, "partition queues");
    uint32_t *slices = ar.take<uint32_t>(size_t(std::max<uint32_t>(chunks, 1)) * kSliceWords, "query slices");
    for (uint32_t p0 = 0; p0 < P; p0 += kMaxRouteParts) {
        const uint32_t pw = std::min(kMaxRouteParts, P - p0);
        const size_t smem = size_t(pw) * (kWords + 2) * sizeof(uint32_t);
        k_route<true><<<rblocks, kRouteThreads, smem, st>>>(d_queries, nq, t.part_mask.p, p0, pw, nullptr, part_off,
                                                           part_cursor, queue);
        TM_CHECK_LAUNCH();
    }
    if (chunks) {
        k_slices<<<chunks, kChunk, 0, st>>>(queue, part_off, part_count, chunk_off, P, slices);
        TM_CHECK_LAUNCH();
    }
    // hit records fill what is left of the array; after the match the part
    // they did not use goes to the keys
    const size_t rec_room = ar.left() / sizeof(HitRec);
    if (rec_room < 256) throw Error(TM_ERR_CAPACITY, "no-allocation scratch exhausted before the hit records; split the batch");
    HitRec *recs = ar.take<HitRec>(rec_room - 32, "hit records");
    MatchArgs a{t.tile_words.p, t.tile_info.p, t.tile_keys.p, t.slot_key_off.p, t.part_tile_begin.p, part_count, part_off,
                item_off, chunk_off, queue, slices, P, seg_tiles, counters, recs, (unsigned long long)(rec_room - 32), qkeys,
                fpl_trip_cost(), nullptr, nullptr, nullptr};
    launch_match<false>(a, unsigned(sms) * 4, st);
    TM_CHECK_LAUNCH();
    unsigned long long hc[3] = {0, 0, 0};
    TM_CUDA(cudaMemcpyAsync(hc, counters, sizeof(hc), cudaMemcpyDeviceToHost, st));
    TM_CUDA(cudaStreamSynchronize(st));
    if (hc[2]) throw Error(TM_ERR_TIMEOUT, "match kernel: bounded wait for the query copy expired");
    if (hc[1] > rec_room - 32)
        throw Error(TM_ERR_CAPACITY, "no-allocation scratch too small for the " + std::to_string(hc[1]) +
                                         " hit records of this batch; split the batch");

    // keys
    ar.trim(recs + hc[1]);
    const unsigned gblocks = std::max(1u, std::min(blocks_for(hc[1], kFillThreads * kFillPerLane), unsigned(sms) * 16));
    uint64_t *key_off = unique ? qoff : d_out_offsets;
    scan_fixed<uint32_t, uint64_t>(qkeys, key_off, nq, sums, offs, st);
    uint64_t total = 0;
    TM_CUDA(cudaMemcpyAsync(&total, key_off + nq, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
    TM_CUDA(cudaStreamSynchronize(st));
    if (!unique) {
        *n_keys = total;
        if (total > capacity)
            throw Error(TM_ERR_CAPACITY, "output key buffer too small: " + std::to_string(total) + " keys needed");
        k_key_fill<<<gblocks, kFillThreads, 0, st>>>(recs, counters, t.slot_key_off.p, t.tile_keys.p, t.keys.p, d_out_offsets, qcursor, d_out_keys);
        TM_CHECK_LAUNCH();
        TM_CUDA(cudaStreamSynchronize(st));
        return;
    }
    // match_unique: keys into one arena buffer, de-duplicated into a second
    // one (the hit records' space when it is large enough: they are no
    // longer read once the keys are filled), then compacted into the
    // caller's output
    const uint64_t bitmap_words = (uint64_t(t.max_key) >> 5) + 1;
    const bool bitmap = bitmap_words * 4 <= 48 * 1024;
    uint32_t *keys = ar.take<uint32_t>(std::max<uint64_t>(total, 1), "match_unique keys");
    uint32_t *ukeys = std::max<uint64_t>(total, 1) * sizeof(uint32_t) <= hc[1] * sizeof(HitRec)
                          ? reinterpret_cast<uint32_t *>(recs)
                          : ar.take<uint32_t>(std::max<uint64_t>(total, 1), "match_unique keys");
    k_key_fill<<<gblocks, kFillThreads, 0, st>>>(recs, counters, t.slot_key_off.p, t.tile_keys.p, t.keys.p, qoff, qcursor, keys);
    TM_CHECK_LAUNCH();
    if (bitmap) {
        k_unique_bitmap<<<nq, kUniqThreads, bitmap_words * 4, st>>>(keys, qoff, uint32_t(bitmap_words), ukeys, ucount);
    } else {
        k_unique_sort<<<nq, kUniqThreads, 0, st>>>(keys, qoff, ukeys, ucount);
    }
    TM_CHECK_LAUNCH();
    scan_fixed<uint32_t, uint64_t>(ucount, d_out_offsets, nq, sums, offs, st);
    uint64_t utotal = 0;
    TM_CUDA(cudaMemcpyAsync(&utotal, d_out_offsets + nq, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
    TM_CUDA(cudaStreamSynchronize(st));
    *n_keys = utotal;
    if (utotal > capacity)
        throw Error(TM_ERR_CAPACITY, "output key buffer too small: " + std::to_string(utotal) + " keys needed");
    k_compact<<<nq, 256, 0, st>>>(ukeys, qoff, d_out_offsets, nq, d_out_keys);
    TM_CHECK_LAUNCH();
    TM_CUDA(cudaStreamSynchronize(st));
}

}  // namespace tmb
