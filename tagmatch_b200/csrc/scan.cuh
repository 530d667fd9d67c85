// Device-wide exclusive prefix sum (reduce-then-scan), used to turn
// per-partition and per-query counts into offsets.  out has n + 1 entries;
// out[n] is the total.
#pragma once
#include <cstdint>
#include <vector>
#include "tm_host.hpp"

namespace tmb {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

template <class T>
__device__ __forceinline__ T warp_incl_scan(T v) {
    const unsigned lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T u = __shfl_up_sync(0xFFFFFFFFu, v, o);
        if (lane >= (unsigned)o) v += u;
    }
    return v;
}

// Block-wide exclusive scan of one value per thread; the block total is
// returned through `total` (same value in every thread).
template <class T>
__device__ __forceinline__ T block_excl_scan(T v, T &total) {
    constexpr int NW = kScanThreads / 32;
    __shared__ T warp_tot[NW];
    __shared__ T blk_total;
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T incl = warp_incl_scan(v);
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        T w = lane < (unsigned)NW ? warp_tot[lane] : T(0);
        T wi = warp_incl_scan(w);
        if (lane < (unsigned)NW) warp_tot[lane] = wi - w;
        if (lane == (unsigned)NW - 1) blk_total = wi;
    }
    __syncthreads();
    T r = incl - v + warp_tot[warp];
    total = blk_total;
    __syncthreads();
    return r;
}

template <class Tin, class Tout>
__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(const Tin *__restrict__ in, size_t n, Tout *__restrict__ sums) {
    size_t base = size_t(blockIdx.x) * kScanTile;
    Tout s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        size_t idx = base + size_t(i) * kScanThreads + threadIdx.x;
        if (idx < n) s += Tout(in[idx]);
    }
    Tout tot;
    block_excl_scan<Tout>(s, tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

template <class Tin, class Tout>
__global__ void __launch_bounds__(kScanThreads) k_scan_apply(const Tin *__restrict__ in, size_t n,
                                                             const uint64_t *__restrict__ block_off, Tout *__restrict__ out) {
    size_t base = size_t(blockIdx.x) * kScanTile + size_t(threadIdx.x) * kScanItems;
    Tout v[kScanItems];
    Tout s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        size_t idx = base + i;
        v[i] = idx < n ? Tout(in[idx]) : Tout(0);
        s += v[i];
    }
    Tout tot;
    Tout pre = block_excl_scan<Tout>(s, tot);
    Tout off = (block_off ? block_off[blockIdx.x] : Tout(0)) + pre;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        size_t idx = base + i;
        if (idx < n) out[idx] = off;
        off += v[i];
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) {
        out[n] = (block_off ? block_off[blockIdx.x] : Tout(0)) + tot;
    }
}

// Scratch for the recursive block-sum levels.
// Fixed number of levels: 2048^8 elements is far beyond any input.
struct ScanScratch {
    static constexpr int kLevels = 8;
    DevBuf<uint64_t> levels[2 * kLevels];
};

// Number of kernel launches exclusive_scan makes for n elements.
inline uint32_t scan_launches(size_t n) {
    size_t nb = (n + kScanTile - 1) / kScanTile;
    return nb <= 1 ? 1u : 2u + scan_launches(nb);
}

// out[0..n]: exclusive prefix sums of in[0..n), out[n] = total.
template <class Tin, class Tout>
void exclusive_scan(const Tin *in, Tout *out, size_t n, ScanScratch &scr, cudaStream_t st, int level = 0) {
    size_t nb = (n + kScanTile - 1) / kScanTile;
    if (nb <= 1) {
        k_scan_apply<Tin, Tout><<<1, kScanThreads, 0, st>>>(in, n, nullptr, out);
        TM_CHECK_LAUNCH();
        return;
    }
    if (level >= ScanScratch::kLevels) throw Error(-8, "scan: too many levels");
    DevBuf<uint64_t> &sums = scr.levels[2 * level];
    DevBuf<uint64_t> &offs = scr.levels[2 * level + 1];
    sums.reserve(nb);
    offs.reserve(nb + 1);
    k_scan_reduce<Tin, uint64_t><<<(unsigned)nb, kScanThreads, 0, st>>>(in, n, sums.p);
    TM_CHECK_LAUNCH();
    exclusive_scan<uint64_t, uint64_t>(sums.p, offs.p, nb, scr, st, level + 1);
    k_scan_apply<Tin, Tout><<<(unsigned)nb, kScanThreads, 0, st>>>(in, n, offs.p, out);
    TM_CHECK_LAUNCH();
}

}  // namespace tmb
