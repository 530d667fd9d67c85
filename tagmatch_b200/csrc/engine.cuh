// TagMatch engine: update staging, consolidation (GPU partitioner + device
// table), batched and asynchronous matching on one or more devices.
#pragma once
#include <array>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <string>
#include <thread>
#include <vector>
#include "match.cuh"
#include "sched.cuh"

namespace tmb {

// 192-bit filter as 6 words, ordered like bitvector<192>::operator<
// (bitvector.hh:389-397): the lowest differing bit of the first differing
// 64-bit block decides, the side holding a 1 is greater.
struct FilterKey {
    std::array<uint32_t, kWords> w;
    bool operator<(const FilterKey &o) const {
        for (int blk = 0; blk < 3; ++blk) {
            const uint64_t x = uint64_t(w[2 * blk]) | (uint64_t(w[2 * blk + 1]) << 32);
            const uint64_t y = uint64_t(o.w[2 * blk]) | (uint64_t(o.w[2 * blk + 1]) << 32);
            if (x != y) return (y >> __builtin_ctzll(x ^ y)) & 1;
        }
        return false;
    }
    bool operator==(const FilterKey &o) const { return w == o.w; }
};

// Pending key additions/removals for one filter (tagmatch.cc:22-34).
struct KeysetChange {
    std::set<uint32_t> to_add, to_remove;
    // Applies the change to an existing key vector: removed keys go, kept
    // keys keep their order, new keys follow in ascending order.  (The
    // reference's apply, tagmatch.cc:36-59, never shrinks the vector, so a
    // removal there only sticks when enough keys are added in the same
    // update; here removals always take effect.)
    void apply(std::vector<uint32_t> &keys) const;
};

typedef void (*MatchCallback)(void *user, uint64_t tag, const uint32_t *keys, uint64_t n_keys);
typedef void (*BatchCallback)(void *user, uint64_t tag, const uint64_t *offsets, const uint32_t *keys, uint32_t n_queries,
                              int status);

struct AsyncRequest {
    uint32_t words[kWords];
    bool unique;
    uint64_t tag;
    MatchCallback cb;
    void *user;
};

// A submitted request of n queries, completed either per query (qcb,
// match_handler semantics) or as a whole (bcb).
struct Request {
    std::vector<uint32_t> words;  // [n][6]
    uint32_t n = 0;
    bool unique = false;
    uint64_t tag = 0;
    MatchCallback qcb = nullptr;
    BatchCallback bcb = nullptr;
    void *user = nullptr;
    uint32_t taken = 0;  // queries placed in device batches (queue lock)
    std::chrono::steady_clock::time_point arrived;  // when it was queued
    // pieces of a request split over several device batches
    std::mutex mtx;
    uint32_t done = 0;
    int status = 0;
    std::vector<uint32_t> counts;             // keys per query
    std::vector<std::vector<uint32_t>> part;  // keys per piece, by first query
};
using RequestPtr = std::shared_ptr<Request>;

// When asynchronous batches go to the device.
enum FlushMode : int {
    kFlushFullOrLatency = 0,  // full batch, latency limit, or stop() (front_end.cc semantics)
    kFlushImmediate = 1,      // whenever a lane is free: continuous batching of all pending requests
    kFlushSingle = 2,         // one request per device batch, one lane (plain batched path)
    kFlushLearned = 3,        // continuous batching with flush points from the learned cost model
};

struct EngineStats {
    uint64_t batches = 0, queries = 0, routed = 0, items = 0, pairs = 0, keys = 0, records = 0;
    uint64_t pair_retries = 0;
    uint64_t match_launches = 0;
    double match_ms = 0.0;
    uint64_t dense = 0, launches = 0;
    uint64_t h2d_bytes = 0, d2h_bytes = 0;  // host API transfers
    void add(const BatchStats &b, uint32_t nq, bool profiled) {
        batches++;
        queries += nq;
        routed += b.routed;
        items += b.items;
        pairs += b.pairs;
        records += b.records;
        keys += b.keys;
        pair_retries += b.retries;
        dense += b.dense;
        launches += b.launches;
        if (profiled) {
            match_launches += 1 + b.retries;
            match_ms += b.match_ms;
        }
    }
};

class Engine {
public:
    Engine();
    ~Engine();

    // staging (tagmatch.cc:62-77)
    void add(const uint32_t *filter, const uint32_t *keys, uint32_t n);
    // n filters [n][6] with keys in CSR form; staged in bulk arrays and
    // merged at consolidate (same table as n calls of add)
    void add_many(const uint32_t *filters, uint64_t n, const uint32_t *key_off, const uint32_t *keys);
    void remove(const uint32_t *filter, uint32_t key);
    void set_db(const std::string &f) { db_filename_ = f; }
    const std::string &db() const { return db_filename_; }
    void set_persist(bool on) { persist_ = on; }

    // tagmatch.cc:92-165
    void consolidate(uint32_t partition_size, uint32_t threads);
    void consolidate() { consolidate(partition_size_, partitioning_threads_); }

    // tagmatch.cc:174-198
    void start(uint32_t threads, uint32_t gpus);
    void start() { start(threads_, gpus_); }
    void stop();
    void clear();
    void set_latency_limit_ms(uint32_t ms) { latency_ms_.store(ms); }
    uint32_t latency_limit_ms() const { return latency_ms_.load(); }
    void set_batch_limit(uint32_t q) { batch_limit_ = q ? q : 1; }

    // synchronous batch match with host buffers; returns TM_ERR_CAPACITY
    // through the exception when out_keys is too small (needed in *n_keys)
    void match_host(const uint32_t *queries, uint64_t nq, bool unique, uint64_t *out_offsets, uint32_t *out_keys,
                    uint64_t capacity, uint64_t *n_keys);
    // synchronous batch match with device buffers on the first device
    void match_device(const uint32_t *d_queries, uint32_t nq, bool unique, const uint64_t **d_offsets,
                      const uint32_t **d_keys, uint64_t *n_keys, cudaStream_t st, BatchStats *bs, cudaEvent_t ev0,
                      cudaEvent_t ev1);
    // same as match_device, with every scratch buffer taken from a static
    // device array (no allocation); outputs are caller-owned device memory
    void match_device_noalloc(const uint32_t *d_queries, uint32_t nq, bool unique, uint64_t *d_offsets, uint32_t *d_keys,
                              uint64_t capacity, uint64_t *n_keys, cudaStream_t st);
    // asynchronous match: cb fires exactly once per request, on an engine
    // thread, after start() (requests made earlier wait for it)
    void submit(const AsyncRequest &r);
    // request of n queries [n][6]; bcb fires once with all its results
    void submit_request(const uint32_t *queries, uint32_t n, bool unique, uint64_t tag, BatchCallback bcb, void *user);
    void set_flush_mode(int m) { flush_mode_.store(m); }
    void set_memory_budget(uint64_t bytes) { memory_budget_.store(bytes ? bytes : 1); }

    // table introspection
    uint32_t n_filters() const { return uint32_t(key_off_.size() ? key_off_.size() - 1 : 0); }
    uint32_t n_partitions() const;
    uint32_t n_tiles() const;
    size_t device_bytes() const;
    const DevTable *table(int dev = 0) const;
    const EngineStats &stats() const { return stats_; }
    void reset_stats() { stats_ = EngineStats(); }
    void set_profiling(bool on);
    // times the candidate tile segments per work item and device batch
    // sizes on a sample of queries (device timing, CUDA events) and keeps
    // the fastest; returns the chosen pair and its queries/s
    void autotune(const uint32_t *queries, uint32_t n, uint32_t *seg_tiles, uint32_t *batch, double *qps);
    // tiles per work item of the subset test (what autotune chooses)
    void set_seg_tiles(uint32_t seg);
    uint32_t seg_tiles() const { return seg_tiles_; }
    bool profiling() const { return profile_; }
    // learned scheduler (sched.cuh)
    Scheduler &scheduler() { return sched_; }
    TrainReport train_scheduler(uint32_t epochs);
    void set_learned_order(bool on) { learned_order_.store(on); }
    void set_latency_target_ms(uint32_t ms) { latency_target_ms_.store(ms ? ms : 1); }
    // serving results left in device memory (request callbacks get a device
    // pointer to their keys) instead of copied to the host
    void set_device_results(bool on) { device_results_.store(on); }
    bool started() const { return started_; }
    // host copy of the consolidated filters (table order) and keys
    const std::vector<uint32_t> &filters() const { return filters_; }
    const std::vector<uint32_t> &key_offsets() const { return key_off_; }
    const std::vector<uint32_t> &keys() const { return keys_; }

private:
    static constexpr int kLanes = 2;
    struct Lane {
        MatchScratch scratch;
        cudaStream_t stream = nullptr;
        HostBuf<uint32_t> h_queries;
        HostBuf<uint64_t> h_offsets;
        HostBuf<uint32_t> h_keys;
        std::thread th;
    };
    struct Piece {
        RequestPtr r;
        uint32_t q0, n;
    };
    // One stage of match_host's pipeline: device scratch, a stream, and the
    // pinned staging its results cross PCIe into.  Lane 0 borrows the
    // device's own scratch and stream (shared with match_device).
    static constexpr int kHostLanes = 3;
    struct HostLane {
        MatchScratch scratch;
        cudaStream_t stream = nullptr;
        cudaEvent_t staged = nullptr;
        cudaEvent_t trace_ev[3] = {nullptr, nullptr, nullptr};  // TM_HOST_TRACE: matched, narrow copied, direct copied
        cudaEvent_t copy_ev[2] = {nullptr, nullptr};            // around a batch's key copies (direct share)
        HostBuf<uint64_t> h_offsets;
        HostBuf<uint32_t> h_keys;
        HostBuf<uint16_t> h_keys16;
    };
    struct Device {
        int index = 0;  // position in devs_ (and dev_version_)
        int id = 0;     // CUDA device: base_device_ + index
        cudaStream_t stream = nullptr;
        DevTable table;
        MatchScratch scratch;
        bool table_ready = false;
        HostLane host[kHostLanes];  // synchronous host-buffer pipeline
        void *noalloc_scratch = nullptr;  // device address of the no-allocation array (looked up once)
        Lane lanes[kLanes];         // asynchronous matcher lanes
        int busy_lanes = 0;         // lanes with a batch on this device (under q_mtx_)
    };
    void build_device_table(Device &d);
    // before / after every batch: work-queue order and timing record
    void prepare(MatchScratch &s, uint32_t nq, bool serving);
    void observe(const DevTable &t, const MatchScratch &s, uint32_t nq, double ms, uint64_t keys);
    void apply_seg_tiles(uint32_t seg);
    void consolidate_bulk();
    void clear_bulk();
    Device &device(int i);
    void enqueue(RequestPtr r);
    void worker_loop(int dev, int lane);
    void run_pieces(Device &d, Lane &ln, std::vector<Piece> &pieces, bool unique);

    std::map<FilterKey, KeysetChange> updates_;
    // bulk adds since the last consolidate: filters [m][6], key offsets [m + 1], keys
    std::vector<uint32_t> bulk_words_;
    std::vector<uint64_t> bulk_koff_;
    std::vector<uint32_t> bulk_keys_;
    bool already_consolidated_ = false;
    bool persist_ = true;
    std::string db_filename_ = "tagmatch.db";
    uint32_t partition_size_ = 1000;       // tagmatch.cc:89
    uint32_t partitioning_threads_ = 1;    // tagmatch.cc:90
    uint32_t threads_ = 4, gpus_ = 1;      // tagmatch.cc:170-171
    std::atomic<uint32_t> latency_ms_{0};
    uint32_t batch_limit_ = 65536;

    // consolidated table on the host, in table order
    std::vector<uint32_t> filters_, key_off_{0}, keys_;
    uint64_t table_version_ = 0;

    std::vector<std::unique_ptr<Device>> devs_;
    std::vector<uint64_t> dev_version_;
    std::mutex api_mtx_;  // serialises synchronous calls
    EngineStats stats_;
    bool profile_ = false;
    int base_device_ = 0;
    uint32_t seg_tiles_ = kSegTiles;
    double host_keys_per_query_ = 0;  // output keys per query of match_host's last batch
    double direct_frac_ = -1;         // match_host's adaptive direct share (< 0: not yet set)

    // async path
    std::mutex q_mtx_;
    std::condition_variable q_cv_, done_cv_;
    std::deque<RequestPtr> pending_;
    uint64_t pending_queries_ = 0;
    std::atomic<int> flush_mode_{kFlushFullOrLatency};
    std::atomic<uint64_t> memory_budget_{uint64_t(16) << 30};  // per lane
    std::atomic<uint64_t> bytes_per_query_{64 << 10};         // running estimate
    std::chrono::steady_clock::time_point oldest_;
    uint64_t in_flight_ = 0;
    bool started_ = false, stopping_ = false, flush_now_ = false;
    std::string async_error_;

    Scheduler sched_;
    std::atomic<bool> learned_order_{false};
    std::atomic<uint32_t> latency_target_ms_{25};
    std::atomic<bool> device_results_{false};
    // arrival rate of asynchronous queries (queue lock)
    uint64_t arrived_queries_ = 0, rate_q_ = 0;
    std::chrono::steady_clock::time_point rate_t_{};
    double arrival_qps_ = 0;
};

}  // namespace tmb
