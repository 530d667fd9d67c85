// TagMatch engine implementation.
#include "engine.cuh"
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <immintrin.h>

namespace tmb {

void KeysetChange::apply(std::vector<uint32_t> &keys) const {
    std::vector<uint32_t> out;
    out.reserve(keys.size() + to_add.size());
    std::set<uint32_t> adds = to_add;
    for (uint32_t k : keys) {
        adds.erase(k);
        if (to_remove.count(k)) continue;
        out.push_back(k);
    }
    for (uint32_t k : adds) out.push_back(k);
    keys.swap(out);
}

// Device i of the engine is CUDA device base_device_ + i, base_device_
// being the calling thread's current device when the engine is created
// (one process per GPU: each sets its device first).
Engine::Engine() {
    if (cudaGetDevice(&base_device_) != cudaSuccess) {
        cudaGetLastError();
        base_device_ = 0;
    }
}

Engine::~Engine() {
    try {
        stop();
    } catch (...) {
    }
    for (auto &d : devs_) {
        if (!d) continue;
        cudaSetDevice(d->id);
        if (d->stream) cudaStreamDestroy(d->stream);
        for (auto &ln : d->lanes)
            if (ln.stream) cudaStreamDestroy(ln.stream);
        for (auto &h : d->host) {
            if (h.stream) cudaStreamDestroy(h.stream);
            if (h.staged) cudaEventDestroy(h.staged);
            for (cudaEvent_t ev : h.trace_ev)
                if (ev) cudaEventDestroy(ev);
            for (cudaEvent_t ev : h.copy_ev)
                if (ev) cudaEventDestroy(ev);
        }
    }
}

void Engine::add(const uint32_t *filter, const uint32_t *keys, uint32_t n) {
    std::lock_guard<std::mutex> lk(api_mtx_);
    FilterKey f;
    std::memcpy(f.w.data(), filter, sizeof(f.w));
    KeysetChange &c = updates_[f];
    for (uint32_t i = 0; i < n; ++i) c.to_add.insert(keys[i]);
}

void Engine::remove(const uint32_t *filter, uint32_t key) {
    std::lock_guard<std::mutex> lk(api_mtx_);
    FilterKey f;
    std::memcpy(f.w.data(), filter, sizeof(f.w));
    updates_[f].to_remove.insert(key);
}

namespace {

struct Entry {
    FilterKey f;
    std::vector<uint32_t> keys;
};

// The reference writes each database record as a partition_fib_entry
// (tagmatch.cc:132-142 -> fib.hh:46-49): uint32 partition id, the 24-byte
// filter, uint32 key count, the keys (fib.cc:14-21).  Records are read back
// in that same layout.  (The reference reads them as plain fib_entry,
// tagmatch.cc:101-106, one field short.)
bool read_db(const std::string &fn, std::vector<Entry> &out, std::map<FilterKey, KeysetChange> &updates) {
    std::ifstream in(fn, std::ios::binary);
    if (!in) return false;
    for (;;) {
        uint32_t part, n;
        Entry e;
        if (!in.read(reinterpret_cast<char *>(&part), 4)) break;
        if (!in.read(reinterpret_cast<char *>(e.f.w.data()), 24)) break;
        if (!in.read(reinterpret_cast<char *>(&n), 4)) break;
        e.keys.resize(n);
        if (n && !in.read(reinterpret_cast<char *>(e.keys.data()), std::streamsize(n) * 4)) break;
        auto it = updates.find(e.f);
        if (it != updates.end()) {
            it->second.apply(e.keys);
            updates.erase(it);
        }
        if (!e.keys.empty()) out.push_back(std::move(e));
    }
    return true;
}

// Sorts v with cmp on all hardware threads: sorted chunks, then pairwise
// merges.
template <class T, class Cmp>
void parallel_sort(std::vector<T> &v, Cmp cmp) {
    const size_t n = v.size();
    const unsigned th = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    if (n < (size_t(1) << 16) || th == 1) {
        std::sort(v.begin(), v.end(), cmp);
        return;
    }
    std::vector<size_t> b(th + 1);
    for (unsigned i = 0; i <= th; ++i) b[i] = n * i / th;
    std::vector<std::thread> ts;
    for (unsigned i = 0; i < th; ++i) ts.emplace_back([&, i] { std::sort(v.begin() + b[i], v.begin() + b[i + 1], cmp); });
    for (auto &t : ts) t.join();
    for (unsigned w = 1; w < th; w *= 2) {
        ts.clear();
        for (unsigned i = 0; i + w < th; i += 2 * w) {
            const size_t lo = b[i], mid = b[i + w], hi = b[std::min(i + 2 * w, th)];
            ts.emplace_back([&, lo, mid, hi] { std::inplace_merge(v.begin() + lo, v.begin() + mid, v.begin() + hi, cmp); });
        }
        for (auto &t : ts) t.join();
    }
}

bool write_db(const std::string &fn, const std::vector<Entry> &fib) {
    std::ofstream out(fn, std::ios::binary | std::ios::trunc);
    if (!out) return false;
    const uint32_t part = 0;
    for (const Entry &e : fib) {
        const uint32_t n = uint32_t(e.keys.size());
        out.write(reinterpret_cast<const char *>(&part), 4);
        out.write(reinterpret_cast<const char *>(e.f.w.data()), 24);
        out.write(reinterpret_cast<const char *>(&n), 4);
        if (n) out.write(reinterpret_cast<const char *>(e.keys.data()), std::streamsize(n) * 4);
    }
    return bool(out);
}

}  // namespace

void Engine::consolidate(uint32_t psize, uint32_t threads) {
    std::lock_guard<std::mutex> lk(api_mtx_);
    if (psize == 0) throw Error(TM_ERR_INVALID, "partition size must be at least 1");
    if (started_) throw Error(TM_ERR_STATE, "consolidate() while matching: call stop() first");
    partition_size_ = psize;
    partitioning_threads_ = threads;
    if (!bulk_koff_.empty() && bulk_koff_.size() > 1) {
        if (!already_consolidated_) {
            consolidate_bulk();
            return;
        }
        // incremental update: the bulk adds join the staged updates
        const size_t m = bulk_koff_.size() - 1;
        for (size_t i = 0; i < m; ++i) {
            FilterKey f;
            std::memcpy(f.w.data(), &bulk_words_[i * kWords], 24);
            KeysetChange &c = updates_[f];
            for (uint64_t j = bulk_koff_[i]; j < bulk_koff_[i + 1]; ++j) c.to_add.insert(bulk_keys_[j]);
        }
        clear_bulk();
    }
    std::vector<Entry> fib;
    if (already_consolidated_) {
        if (persist_) {
            if (!read_db(db_filename_, fib, updates_))
                std::cerr << "could not open database file: " << db_filename_ << std::endl;
        } else {
            // in-memory database: the current table
            const uint32_t n = n_filters();
            for (uint32_t i = 0; i < n; ++i) {
                Entry e;
                std::memcpy(e.f.w.data(), &filters_[size_t(i) * kWords], 24);
                e.keys.assign(keys_.begin() + key_off_[i], keys_.begin() + key_off_[i + 1]);
                auto it = updates_.find(e.f);
                if (it != updates_.end()) {
                    it->second.apply(e.keys);
                    updates_.erase(it);
                }
                if (!e.keys.empty()) fib.push_back(std::move(e));
            }
        }
    }
    for (auto &u : updates_) {
        Entry e;
        e.f = u.first;
        u.second.apply(e.keys);
        if (!e.keys.empty()) fib.push_back(std::move(e));
    }
    updates_.clear();
    if (persist_ && !write_db(db_filename_, fib))
        std::cerr << "could not open database file: " << db_filename_ << std::endl;

    uint64_t nk = 0;
    for (const Entry &e : fib) nk += e.keys.size();
    if (nk >= 0xFFFFFFFFull || fib.size() >= 0xFFFFFFFFull) throw Error(TM_ERR_INVALID, "table too large (2^32 keys or filters)");
    filters_.resize(fib.size() * kWords);
    key_off_.assign(fib.size() + 1, 0);
    keys_.clear();
    keys_.reserve(nk);
    for (size_t i = 0; i < fib.size(); ++i) {
        std::memcpy(&filters_[i * kWords], fib[i].f.w.data(), 24);
        keys_.insert(keys_.end(), fib[i].keys.begin(), fib[i].keys.end());
        key_off_[i + 1] = uint32_t(keys_.size());
    }
    ++table_version_;
    // the partitioner runs at consolidation time, on the first device
    build_device_table(device(0));
    already_consolidated_ = true;
}

void Engine::add_many(const uint32_t *filters, uint64_t n, const uint32_t *key_off, const uint32_t *keys) {
    std::lock_guard<std::mutex> lk(api_mtx_);
    if (bulk_koff_.empty()) bulk_koff_.push_back(0);
    bulk_words_.insert(bulk_words_.end(), filters, filters + n * kWords);
    for (uint64_t i = 0; i < n; ++i) {
        bulk_keys_.insert(bulk_keys_.end(), keys + key_off[i], keys + key_off[i + 1]);
        bulk_koff_.push_back(bulk_keys_.size());
    }
}

void Engine::clear_bulk() {
    std::vector<uint32_t>().swap(bulk_words_);
    std::vector<uint64_t>().swap(bulk_koff_);
    std::vector<uint32_t>().swap(bulk_keys_);
}

// First consolidation with bulk adds (tm_add_many): the same table as
// staging every add in the update map and consolidating it -- filters in
// bitvector order (bitvector.hh:389-397), each with the ascending union of
// its keys, empty ones dropped (tagmatch.cc:121-128) -- built by a parallel
// sort of the bulk entries merged with the map's entries instead of one map
// insertion per filter.
void Engine::consolidate_bulk() {
    struct SortEntry {
        uint32_t w[kWords];
        uint32_t idx;
    };
    const size_t m = bulk_koff_.size() - 1;
    std::vector<SortEntry> v(m);
    for (size_t i = 0; i < m; ++i) {
        std::memcpy(v[i].w, &bulk_words_[i * kWords], 24);
        v[i].idx = uint32_t(i);
    }
    auto less_words = [](const uint32_t *a, const uint32_t *b) {
        for (int blk = 0; blk < 3; ++blk) {
            const uint64_t x = uint64_t(a[2 * blk]) | (uint64_t(a[2 * blk + 1]) << 32);
            const uint64_t y = uint64_t(b[2 * blk]) | (uint64_t(b[2 * blk + 1]) << 32);
            if (x != y) return ((y >> __builtin_ctzll(x ^ y)) & 1) != 0;
        }
        return false;
    };
    // stable in effect: equal filters keep their add order (idx breaks ties)
    parallel_sort(v, [&](const SortEntry &a, const SortEntry &b) {
        if (less_words(a.w, b.w)) return true;
        if (less_words(b.w, a.w)) return false;
        return a.idx < b.idx;
    });
    filters_.clear();
    key_off_.assign(1, 0);
    keys_.clear();
    filters_.reserve(m * kWords);
    key_off_.reserve(m + 1);
    keys_.reserve(bulk_keys_.size());
    std::vector<uint32_t> ks;
    auto emit = [&](const uint32_t *w, std::vector<uint32_t> &kv) {
        if (kv.empty()) return;
        filters_.insert(filters_.end(), w, w + kWords);
        keys_.insert(keys_.end(), kv.begin(), kv.end());
        if (keys_.size() >= 0xFFFFFFFFull) throw Error(TM_ERR_INVALID, "table too large (2^32 keys)");
        key_off_.push_back(uint32_t(keys_.size()));
    };
    auto it = updates_.begin();
    size_t i = 0;
    while (i < m || it != updates_.end()) {
        const bool take_map = i == m || (it != updates_.end() && less_words(it->first.w.data(), v[i].w));
        if (take_map) {
            ks.clear();
            it->second.apply(ks);
            emit(it->first.w.data(), ks);
            ++it;
            continue;
        }
        // one group of equal filters from the bulk adds
        size_t j = i;
        ks.clear();
        while (j < m && std::memcmp(v[j].w, v[i].w, 24) == 0) {
            const uint32_t e = v[j].idx;
            ks.insert(ks.end(), bulk_keys_.begin() + bulk_koff_[e], bulk_keys_.begin() + bulk_koff_[e + 1]);
            ++j;
        }
        if (it != updates_.end() && std::memcmp(it->first.w.data(), v[i].w, 24) == 0) {
            KeysetChange c = it->second;
            c.to_add.insert(ks.begin(), ks.end());
            ks.clear();
            c.apply(ks);
            ++it;
        } else {
            std::sort(ks.begin(), ks.end());
            ks.erase(std::unique(ks.begin(), ks.end()), ks.end());
        }
        emit(v[i].w, ks);
        i = j;
    }
    updates_.clear();
    clear_bulk();
    if (persist_) {
        std::ofstream out(db_filename_, std::ios::binary | std::ios::trunc);
        const uint32_t part = 0;
        for (size_t e = 0; out && e + 1 < key_off_.size(); ++e) {
            const uint32_t n = key_off_[e + 1] - key_off_[e];
            out.write(reinterpret_cast<const char *>(&part), 4);
            out.write(reinterpret_cast<const char *>(&filters_[e * kWords]), 24);
            out.write(reinterpret_cast<const char *>(&n), 4);
            out.write(reinterpret_cast<const char *>(&keys_[key_off_[e]]), std::streamsize(n) * 4);
        }
        if (!out) std::cerr << "could not open database file: " << db_filename_ << std::endl;
    }
    ++table_version_;
    build_device_table(device(0));
    already_consolidated_ = true;
}

Engine::Device &Engine::device(int i) {
    while ((int)devs_.size() <= i) {
        auto d = std::make_unique<Device>();
        d->index = int(devs_.size());
        d->id = base_device_ + d->index;
        TM_CUDA(cudaSetDevice(d->id));
        TM_CUDA(cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking));
        devs_.push_back(std::move(d));
        dev_version_.push_back(~0ull);
    }
    return *devs_[i];
}

void Engine::build_device_table(Device &d) {
    TM_CUDA(cudaSetDevice(d.id));
    const uint32_t n = n_filters();
    DevBuf<uint32_t> f, ko, k;
    f.reserve(size_t(n) * kWords);
    ko.reserve(size_t(n) + 1);
    k.reserve(std::max<size_t>(keys_.size(), 1));
    if (n) {
        TM_CUDA(cudaMemcpyAsync(f.p, filters_.data(), filters_.size() * 4, cudaMemcpyHostToDevice, d.stream));
        TM_CUDA(cudaMemcpyAsync(ko.p, key_off_.data(), key_off_.size() * 4, cudaMemcpyHostToDevice, d.stream));
        if (!keys_.empty()) TM_CUDA(cudaMemcpyAsync(k.p, keys_.data(), keys_.size() * 4, cudaMemcpyHostToDevice, d.stream));
    }
    PartitionResult pr;
    gpu_partition(f.p, n, partition_size_, true, pr, d.stream);
    d.table = DevTable();
    build_table(pr, ko.p, k.p, keys_.size(), d.table, d.stream);
    TM_CUDA(cudaStreamSynchronize(d.stream));
    d.table_ready = true;
    dev_version_[d.index] = table_version_;
}

uint32_t Engine::n_partitions() const { return devs_.empty() ? 0 : devs_[0]->table.n_parts; }
uint32_t Engine::n_tiles() const { return devs_.empty() ? 0 : devs_[0]->table.n_tiles; }
size_t Engine::device_bytes() const { return devs_.empty() ? 0 : devs_[0]->table.device_bytes(); }
const DevTable *Engine::table(int dev) const {
    return dev < (int)devs_.size() && devs_[dev]->table_ready ? &devs_[dev]->table : nullptr;
}

void Engine::start(uint32_t threads, uint32_t gpus) {
    std::lock_guard<std::mutex> lk(api_mtx_);
    if (gpus == 0) gpus = 1;
    int count = 0;
    TM_CUDA(cudaGetDeviceCount(&count));
    if (base_device_ + (int)gpus > count)
        throw Error(TM_ERR_INVALID, "start(): " + std::to_string(gpus) + " GPUs requested from device " +
                                        std::to_string(base_device_) + ", " + std::to_string(count) + " present");
    threads_ = threads;
    if (started_) return;  // re-entrant, like front_end::start (front_end.cc:671-691)
    gpus_ = gpus;
    for (uint32_t g = 0; g < gpus_; ++g) {
        Device &d = device(int(g));
        if (dev_version_[g] != table_version_) build_device_table(d);  // replicas (back_end.cc:444-447)
    }
    {
        std::lock_guard<std::mutex> ql(q_mtx_);
        started_ = true;
        stopping_ = false;
        flush_now_ = false;
        if (!pending_.empty()) oldest_ = std::chrono::steady_clock::now();
    }
    for (uint32_t g = 0; g < gpus_; ++g) {
        Device &d = *devs_[g];
        TM_CUDA(cudaSetDevice(d.id));
        for (int l = 0; l < kLanes; ++l) {
            if (!d.lanes[l].stream) TM_CUDA(cudaStreamCreateWithFlags(&d.lanes[l].stream, cudaStreamNonBlocking));
            d.lanes[l].th = std::thread(&Engine::worker_loop, this, int(g), l);
        }
    }
}

void Engine::stop() {
    {
        std::lock_guard<std::mutex> ql(q_mtx_);
        if (!started_ || stopping_) return;
        stopping_ = true;
    }
    q_cv_.notify_all();
    for (auto &d : devs_)
        for (auto &ln : d->lanes)
            if (ln.th.joinable()) ln.th.join();
    std::lock_guard<std::mutex> ql(q_mtx_);
    started_ = false;
    stopping_ = false;
    flush_now_ = false;
}

void Engine::clear() {
    stop();
    std::lock_guard<std::mutex> lk(api_mtx_);
    already_consolidated_ = false;
    updates_.clear();
    clear_bulk();
    filters_.clear();
    key_off_.assign(1, 0);
    keys_.clear();
    ++table_version_;
    for (auto &d : devs_) {
        TM_CUDA(cudaSetDevice(d->id));
        d->table = DevTable();
        d->scratch = MatchScratch();
        for (auto &h : d->host) h.scratch = MatchScratch();
        for (auto &ln : d->lanes) ln.scratch = MatchScratch();
        d->table_ready = false;
    }
}

void Engine::enqueue(RequestPtr r) {
    {
        std::lock_guard<std::mutex> ql(q_mtx_);
        r->arrived = std::chrono::steady_clock::now();
        if (pending_.empty()) oldest_ = r->arrived;
        pending_queries_ += r->n;
        // arrival rate (queries/s), smoothed over windows of >= 10 ms
        arrived_queries_ += r->n;
        const double dt = std::chrono::duration<double>(r->arrived - rate_t_).count();
        if (dt >= 0.01) {
            const double sample = double(arrived_queries_ - rate_q_) / dt;
            arrival_qps_ = dt > 1.0 ? sample : 0.5 * arrival_qps_ + 0.5 * sample;
            rate_t_ = r->arrived;
            rate_q_ = arrived_queries_;
        }
        pending_.push_back(std::move(r));
    }
    q_cv_.notify_all();
}

void Engine::submit(const AsyncRequest &a) {
    auto r = std::make_shared<Request>();
    r->words.assign(a.words, a.words + kWords);
    r->n = 1;
    r->unique = a.unique;
    r->tag = a.tag;
    r->qcb = a.cb;
    r->user = a.user;
    enqueue(std::move(r));
}

void Engine::submit_request(const uint32_t *queries, uint32_t n, bool unique, uint64_t tag, BatchCallback bcb, void *user) {
    auto r = std::make_shared<Request>();
    r->words.assign(queries, queries + size_t(n) * kWords);
    r->n = n;
    r->unique = unique;
    r->tag = tag;
    r->bcb = bcb;
    r->user = user;
    if (n == 0) {  // nothing to match: complete at once
        const uint64_t zero = 0;
        if (bcb) bcb(user, tag, &zero, nullptr, 0, TM_OK);
        return;
    }
    enqueue(std::move(r));
}

// One lane of the asynchronous matcher.  It takes pending requests (or
// pieces of them, up to the batch limit and to the queries that fit the
// device-memory budget), matches them as one device batch on its own
// stream, and completes them.  Two lanes per device keep one batch on the
// GPU while the other is staged or delivered.
void Engine::worker_loop(int dev, int lane) {
    Device &d = *devs_[dev];
    Lane &ln = d.lanes[lane];
    cudaSetDevice(d.id);
    std::vector<Piece> pieces;
    for (;;) {
        pieces.clear();
        bool unique = false;
        uint32_t total = 0;
        {
            std::unique_lock<std::mutex> lk(q_mtx_);
            for (;;) {
                const int mode = flush_mode_.load();
                if (mode == kFlushSingle && lane != 0 && !stopping_) {
                    q_cv_.wait(lk);  // the plain path uses one lane
                    continue;
                }
                if (!pending_.empty()) {
                    if (mode == kFlushLearned && !stopping_ && !flush_now_ && pending_queries_ < batch_limit_ &&
                        sched_.trained()) {
                        // learned flush point: go when the pending queries make a
                        // batch large enough to keep up with the arrival rate
                        // (predicted queries per ms of batch time), or when the
                        // oldest request's wait plus the batch's predicted time
                        // reaches half the latency target; otherwise wait for
                        // more requests.  Below the predicted capacity (a stable
                        // batch under the cap exists) a device with no batch on
                        // it does not wait: waiting would only leave it idle.
                        const uint64_t bq = std::max<uint64_t>(1, memory_budget_.load() / std::max<uint64_t>(1, bytes_per_query_.load()));
                        const uint32_t cap = uint32_t(std::min<uint64_t>(batch_limit_, bq));
                        const uint32_t b0 = uint32_t(std::min<uint64_t>(pending_queries_, cap));
                        const double t0 = sched_.predict_batch_ms(b0);
                        const auto now = std::chrono::steady_clock::now();
                        const double age = std::chrono::duration<double, std::milli>(now - pending_.front()->arrived).count();
                        const double budget = 0.5 * latency_target_ms_.load();
                        const uint32_t need = sched_.stable_batch(arrival_qps_, cap, kLanes);
                        if (b0 >= need || age + t0 >= budget || (d.busy_lanes == 0 && need < cap)) break;
                        double wait_ms = budget - age - t0;
                        if (arrival_qps_ > 0) wait_ms = std::min(wait_ms, 1e3 * double(need - b0) / arrival_qps_);
                        q_cv_.wait_until(lk, now + std::chrono::microseconds(int64_t(1e3 * wait_ms) + 1));
                        continue;
                    }
                    if (stopping_ || flush_now_ || mode != kFlushFullOrLatency || pending_queries_ >= batch_limit_) break;
                    const uint32_t lim = latency_ms_.load();
                    if (lim > 0) {
                        auto due = oldest_ + std::chrono::milliseconds(lim);
                        if (std::chrono::steady_clock::now() >= due) break;
                        q_cv_.wait_until(lk, due);
                        continue;
                    }
                } else if (stopping_) {
                    return;
                }
                q_cv_.wait(lk);
            }
            const int mode = flush_mode_.load();
            const uint64_t budget_q = std::max<uint64_t>(1, memory_budget_.load() / std::max<uint64_t>(1, bytes_per_query_.load()));
            const uint32_t cap = uint32_t(std::min<uint64_t>(batch_limit_, budget_q));
            unique = pending_.front()->unique;
            while (!pending_.empty() && total < cap) {
                RequestPtr &r = pending_.front();
                if (r->unique != unique) break;
                // a request is split over batches only when it alone exceeds
                // the cap; otherwise it waits for the next batch
                if (total > 0 && r->taken == 0 && r->n > cap - total) break;
                const uint32_t take = std::min(r->n - r->taken, cap - total);
                pieces.push_back(Piece{r, r->taken, take});
                r->taken += take;
                total += take;
                if (r->taken == r->n) pending_.pop_front();
                if (mode == kFlushSingle) break;
            }
            pending_queries_ -= total;
            if (!pending_.empty()) oldest_ = std::chrono::steady_clock::now();
            in_flight_ += total;
            ++d.busy_lanes;
        }
        run_pieces(d, ln, pieces, unique);
        {
            std::lock_guard<std::mutex> lk(q_mtx_);
            in_flight_ -= total;
            --d.busy_lanes;
        }
        done_cv_.notify_all();
        q_cv_.notify_all();
    }
}

void Engine::run_pieces(Device &d, Lane &ln, std::vector<Piece> &pieces, bool unique) {
    uint32_t nq = 0;
    for (const Piece &p : pieces) nq += p.n;
    bool ok = true;
    // results left on the device: only for whole requests with a request
    // callback (per-query handlers and split requests get host copies)
    bool dres = device_results_.load();
    for (const Piece &p : pieces)
        if (p.r->qcb || p.q0 != 0 || p.n != p.r->n) dres = false;
    const uint32_t *dkeys_out = nullptr;
    try {
        ln.h_queries.reserve(size_t(nq) * kWords);
        uint32_t at = 0;
        for (const Piece &p : pieces) {
            std::memcpy(ln.h_queries.p + size_t(at) * kWords, p.r->words.data() + size_t(p.q0) * kWords,
                        size_t(p.n) * kWords * sizeof(uint32_t));
            at += p.n;
        }
        ln.scratch.queries.reserve(size_t(nq) * kWords);
        TM_CUDA(cudaMemcpyAsync(ln.scratch.queries.p, ln.h_queries.p, size_t(nq) * 24, cudaMemcpyHostToDevice, ln.stream));
        const uint64_t *doff;
        const uint32_t *dkeys;
        uint64_t nk = 0;
        BatchStats bs;
        prepare(ln.scratch, nq, true);
        const auto tb = std::chrono::steady_clock::now();
        match_batch(d.table, ln.scratch.queries.p, nq, unique, ln.scratch, &doff, &dkeys, &nk, &bs, ln.stream);
        observe(d.table, ln.scratch, nq, std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tb).count(),
                nk);
        ln.h_offsets.reserve(size_t(nq) + 1);
        ln.h_keys.reserve(std::max<uint64_t>(nk, 1));
        TM_CUDA(cudaMemcpyAsync(ln.h_offsets.p, doff, (size_t(nq) + 1) * 8, cudaMemcpyDeviceToHost, ln.stream));
        if (nk && !dres) TM_CUDA(cudaMemcpyAsync(ln.h_keys.p, dkeys, nk * 4, cudaMemcpyDeviceToHost, ln.stream));
        TM_CUDA(cudaStreamSynchronize(ln.stream));
        dkeys_out = dkeys;
        // running estimate of device bytes per query (queues, hit records, keys)
        const uint64_t bytes = bs.routed * (kQueueWords * 4) + bs.records * sizeof(HitRec) + nk * 4 * (unique ? 3 : 1);
        const uint64_t bpq = std::max<uint64_t>(1024, bytes / std::max<uint32_t>(nq, 1));
        bytes_per_query_.store((bytes_per_query_.load() * 3 + bpq) / 4);
    } catch (const Error &e) {
        ok = false;
        std::lock_guard<std::mutex> lk(q_mtx_);
        async_error_ = e.what();
    }
    const uint64_t *off = ln.h_offsets.p;
    const uint32_t *keys = dres ? dkeys_out : ln.h_keys.p;
    uint32_t at = 0;
    std::vector<uint64_t> rebased;
    for (Piece &p : pieces) {
        Request &r = *p.r;
        if (r.qcb) {
            for (uint32_t i = 0; i < p.n; ++i) {
                if (ok) r.qcb(r.user, r.tag + p.q0 + i, keys + off[at + i], off[at + i + 1] - off[at + i]);
                else r.qcb(r.user, r.tag + p.q0 + i, nullptr, 0);
            }
        } else if (r.bcb && p.q0 == 0 && p.n == r.n) {
            // whole request in this batch: offsets rebased to its first key
            rebased.resize(size_t(p.n) + 1);
            const uint64_t b0 = ok ? off[at] : 0;
            for (uint32_t i = 0; i <= p.n; ++i) rebased[i] = ok ? off[at + i] - b0 : 0;
            r.bcb(r.user, r.tag, rebased.data(), ok ? keys + b0 : nullptr, r.n, ok ? TM_OK : TM_ERR_INTERNAL);
        } else if (r.bcb) {
            // a piece of a split request: keep it until every piece is in
            std::lock_guard<std::mutex> rl(r.mtx);
            if (r.counts.empty()) {
                r.counts.assign(r.n, 0);
                r.part.resize(r.n);
            }
            if (ok) {
                for (uint32_t i = 0; i < p.n; ++i) r.counts[p.q0 + i] = uint32_t(off[at + i + 1] - off[at + i]);
                r.part[p.q0].assign(keys + off[at], keys + off[at + p.n]);
            } else {
                r.status = TM_ERR_INTERNAL;
            }
            r.done += p.n;
            if (r.done == r.n) {
                std::vector<uint64_t> o(size_t(r.n) + 1, 0);
                for (uint32_t i = 0; i < r.n; ++i) o[i + 1] = o[i] + r.counts[i];
                std::vector<uint32_t> all;
                all.reserve(o[r.n]);
                for (uint32_t q = 0; q < r.n; ++q)
                    if (!r.part[q].empty()) all.insert(all.end(), r.part[q].begin(), r.part[q].end());
                r.bcb(r.user, r.tag, o.data(), all.data(), r.n, r.status);
            }
        }
        at += p.n;
    }
}

void Engine::match_device(const uint32_t *d_queries, uint32_t nq, bool unique, const uint64_t **d_offsets,
                          const uint32_t **d_keys, uint64_t *n_keys, cudaStream_t st, BatchStats *bs, cudaEvent_t ev0,
                          cudaEvent_t ev1) {
    std::lock_guard<std::mutex> lk(api_mtx_);
    if (!already_consolidated_) throw Error(TM_ERR_STATE, "match before consolidate()");
    Device &d = device(0);
    if (dev_version_[0] != table_version_) build_device_table(d);
    TM_CUDA(cudaSetDevice(d.id));
    BatchStats local;
    d.scratch.profile = profile_;
    prepare(d.scratch, nq, false);
    const auto tb = std::chrono::steady_clock::now();
    match_batch(d.table, d_queries, nq, unique, d.scratch, d_offsets, d_keys, n_keys, &local, st ? st : d.stream, ev0, ev1);
    observe(d.table, d.scratch, nq, std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tb).count(),
            *n_keys);
    stats_.add(local, nq, profile_);
    if (bs) *bs = local;
}

void Engine::match_device_noalloc(const uint32_t *d_queries, uint32_t nq, bool unique, uint64_t *d_offsets,
                                  uint32_t *d_keys, uint64_t capacity, uint64_t *n_keys, cudaStream_t st) {
    std::lock_guard<std::mutex> lk(api_mtx_);
    if (!already_consolidated_ || devs_.empty() || !devs_[0]->table_ready || dev_version_[0] != table_version_)
        throw Error(TM_ERR_STATE, "no device table: call consolidate() first");
    Device &d = *devs_[0];
    TM_CUDA(cudaSetDevice(d.id));
    if (!d.noalloc_scratch) d.noalloc_scratch = noalloc_scratch_address();
    match_batch_noalloc(d.table, d_queries, nq, unique, seg_tiles_, d.noalloc_scratch, d_offsets, d_keys, capacity,
                        n_keys, st ? st : d.stream);
}

void Engine::autotune(const uint32_t *queries, uint32_t n, uint32_t *seg_out, uint32_t *batch_out, double *qps_out) {
    std::lock_guard<std::mutex> lk(api_mtx_);
    if (!already_consolidated_) throw Error(TM_ERR_STATE, "autotune before consolidate()");
    if (n == 0) throw Error(TM_ERR_INVALID, "autotune needs a sample of queries");
    Device &d = device(0);
    if (dev_version_[0] != table_version_) build_device_table(d);
    TM_CUDA(cudaSetDevice(d.id));
    DevBuf<uint32_t> dq;
    dq.reserve(size_t(n) * kWords);
    TM_CUDA(cudaMemcpyAsync(dq.p, queries, size_t(n) * 24, cudaMemcpyHostToDevice, d.stream));
    cudaEvent_t e0, e1;
    TM_CUDA(cudaEventCreate(&e0));
    TM_CUDA(cudaEventCreate(&e1));
    d.scratch.record_items = false;  // the candidates' batches are timed, not recorded
    d.scratch.part_order.clear();
    double best = -1.0;
    uint32_t best_seg = seg_tiles_, best_batch = batch_limit_;
    const uint32_t segs[] = {32, 64, 128, 256, 512, 1024, 2048, 4096, 8192};
    const uint32_t batches[] = {8192, 16384, 32768, 65536, 131072, 262144};
    try {
        for (uint32_t b : batches) {
            if (b > n && b != batches[0]) break;
            const uint32_t bb = std::min(b, n);
            for (uint32_t sg : segs) {
                d.scratch.seg_tiles = sg;
                const uint64_t *doff;
                const uint32_t *dkeys;
                uint64_t nk;
                BatchStats bs;
                // one untimed pass (buffers grow), then the timed pass over the sample
                match_batch(d.table, dq.p, bb, false, d.scratch, &doff, &dkeys, &nk, &bs, d.stream);
                TM_CUDA(cudaEventRecord(e0, d.stream));
                for (uint32_t q0 = 0; q0 + bb <= n; q0 += bb)
                    match_batch(d.table, dq.p + size_t(q0) * kWords, bb, false, d.scratch, &doff, &dkeys, &nk, &bs, d.stream);
                TM_CUDA(cudaEventRecord(e1, d.stream));
                TM_CUDA(cudaEventSynchronize(e1));
                float ms = 0.f;
                TM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                const double qps = double(n / bb * bb) / (ms / 1e3);
                if (qps > best) {
                    best = qps;
                    best_seg = sg;
                    best_batch = bb;
                }
            }
        }
    } catch (...) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        d.scratch.seg_tiles = seg_tiles_;
        throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    batch_limit_ = best_batch;
    apply_seg_tiles(best_seg);
    *seg_out = best_seg;
    *batch_out = best_batch;
    *qps_out = best;
}

void Engine::prepare(MatchScratch &s, uint32_t nq, bool serving) {
    s.record_items = sched_.recording();
    if (learned_order_.load()) s.part_order = sched_.order();
    else s.part_order.clear();
    if (serving) {
        // the learned serving mode also picks each batch's tiles per work
        // item (small batches want more, smaller items); otherwise the
        // engine's (autotuned) value
        const uint32_t best = flush_mode_.load() == kFlushLearned ? sched_.best_seg(nq) : 0u;
        s.seg_tiles = best ? best : seg_tiles_;
    }
}

void Engine::observe(const DevTable &t, const MatchScratch &s, uint32_t nq, double ms, uint64_t keys) {
    if (s.record_items) sched_.absorb(t, s, nq, ms, keys);
    else if (flush_mode_.load() == kFlushLearned) sched_.observe_batch(nq, ms);
}

TrainReport Engine::train_scheduler(uint32_t epochs) {
    std::lock_guard<std::mutex> lk(api_mtx_);
    if (!already_consolidated_) throw Error(TM_ERR_STATE, "train the scheduler after consolidate()");
    Device &d = device(0);
    if (dev_version_[0] != table_version_) build_device_table(d);
    TM_CUDA(cudaSetDevice(d.id));
    int sms = 0, khz = 0;
    TM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d.id));
    TM_CUDA(cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, d.id));
    return sched_.train(d.table, seg_tiles_, sms, double(khz) * 1e3, epochs, d.stream);
}

void Engine::apply_seg_tiles(uint32_t seg) {
    seg_tiles_ = seg;
    for (auto &dv : devs_) {
        dv->scratch.seg_tiles = seg;
        for (auto &h : dv->host) h.scratch.seg_tiles = seg;
        for (auto &ln : dv->lanes) ln.scratch.seg_tiles = seg;
    }
}

void Engine::set_seg_tiles(uint32_t seg) {
    std::lock_guard<std::mutex> lk(api_mtx_);
    if (seg == 0 || seg > (1u << 20)) throw Error(TM_ERR_INVALID, "tiles per work item must be in 1 .. 2^20");
    apply_seg_tiles(seg);
}

void Engine::set_profiling(bool on) {
    std::lock_guard<std::mutex> lk(api_mtx_);
    profile_ = on;
}

namespace {

bool is_pinned(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// memcpy split over a few threads (pinned staging -> pageable caller memory)
void parallel_copy(void *dst, const void *src, size_t bytes) {
    const size_t kMin = size_t(64) << 20;
    const int nt = int(std::min<size_t>(8, std::max<size_t>(1, bytes / kMin)));
    if (nt == 1) {
        std::memcpy(dst, src, bytes);
        return;
    }
    std::vector<std::thread> th;
    const size_t per = (bytes + nt - 1) / nt;
    for (int t = 0; t < nt; ++t) {
        const size_t b = size_t(t) * per, e = std::min(bytes, b + per);
        if (b < e)
            th.emplace_back([=] { std::memcpy(static_cast<char *>(dst) + b, static_cast<const char *>(src) + b, e - b); });
    }
    for (auto &x : th) x.join();
}

// widen 16-bit keys into the caller's 32-bit buffer: AVX2 with streaming
// stores where the CPU has it (no read-for-ownership of the destination),
// split over threads
__attribute__((target("avx2"))) void widen_avx2(uint32_t *d, const uint16_t *s_, uint64_t n) {
    uint64_t i = 0;
    while (i < n && (reinterpret_cast<uintptr_t>(d + i) & 31)) {
        d[i] = s_[i];
        ++i;
    }
    for (; i + 8 <= n; i += 8) {
        const __m128i v = _mm_loadu_si128(reinterpret_cast<const __m128i *>(s_ + i));
        _mm256_stream_si256(reinterpret_cast<__m256i *>(d + i), _mm256_cvtepu16_epi32(v));
    }
    for (; i < n; ++i) d[i] = s_[i];
    _mm_sfence();
}

void widen_scalar(uint32_t *d, const uint16_t *s_, uint64_t n) {
    for (uint64_t i = 0; i < n; ++i) d[i] = s_[i];
}

void parallel_widen(uint32_t *dst, const uint16_t *src, uint64_t n) {
    static const bool avx2 = __builtin_cpu_supports("avx2");
    void (*body)(uint32_t *, const uint16_t *, uint64_t) = avx2 ? widen_avx2 : widen_scalar;
    const uint64_t kMin = uint64_t(8) << 20;
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const int nt = int(std::min<uint64_t>(std::max(1u, hw - 2), std::max<uint64_t>(1, n / kMin)));
    if (nt == 1) {
        body(dst, src, n);
        return;
    }
    std::vector<std::thread> th;
    const uint64_t per = ((n + nt - 1) / nt + 7) & ~uint64_t(7);
    for (int t = 0; t < nt; ++t) {
        const uint64_t b = uint64_t(t) * per, e = std::min(n, b + per);
        if (b < e) th.emplace_back(body, dst + b, src + b, e - b);
    }
    for (auto &x : th) x.join();
}

// Share of a batch's keys that crosses PCIe as 32-bit values straight into
// a pinned caller buffer when the keys could travel narrowed to 16 bits.
// Narrowed keys halve the bytes on the link but cost host memory bandwidth
// (a 2-byte DMA write, a 2-byte read and a 4-byte write per key by the copy
// threads); direct keys cost 4 bytes on the link and one 4-byte DMA write.
// Sending part of each batch direct keeps the link and host memory both
// below the matcher's time per batch.  TM_DIRECT_FRACTION overrides it.
constexpr double kDirectFraction = 0.1;
// smallest batch of match_host's final, halving batches
constexpr uint64_t kTailBatch = 4096;
// output keys per match_host batch (about 2 GB narrowed, 4 GB wide): larger
// batches let a batch's host copies fall behind the matching of the next
// ones, and leave a long copy after the last match.  TM_HOST_BATCH_KEYS
// overrides it (0: no cap).
constexpr double kHostBatchKeys = double(1u << 30);

double host_batch_keys() {
    const char *s = std::getenv("TM_HOST_BATCH_KEYS");
    return s && *s ? std::max(0.0, std::atof(s)) : kHostBatchKeys;
}

// TM_DIRECT_FRACTION fixes the direct share; otherwise (< 0) it adapts.
double direct_fraction_fixed() {
    const char *s = std::getenv("TM_DIRECT_FRACTION");
    if (!s || !*s) return -1.0;
    return std::min(1.0, std::max(0.0, std::atof(s)));
}

// The direct share that balances the two host-side stages of a batch: the
// link carries 2 bytes per narrowed key and 4 per direct key at c bytes/ms,
// host threads widen the narrowed keys at w keys/ms; both take the same
// time when (1 - f) / w = (2 (1 - f) + 4 f) / c, i.e. f = (c - 2w) / (c + 2w).
double balanced_direct_fraction(double c, double w) {
    const double f = (c - 2.0 * w) / (c + 2.0 * w);
    return std::min(0.75, std::max(0.0, f));
}

}  // namespace

// Batches rotate over three lanes (scratch + stream + pinned staging): while
// one batch is matched, the results of the two before it cross PCIe and are
// widened, so the device never waits for the host copies of the batch it
// last finished.  Keys go to the caller's buffer in one of three ways:
// - every key of the table below 65,536: a share of the batch's keys is
//   copied as 32-bit values straight into a pinned caller buffer; the rest
//   crosses as 16-bit values into pinned staging and copy threads widen
//   them into the caller's buffer.  The share adapts from batch to batch:
//   each large batch's measured link rate (CUDA events around its copies)
//   and widening rate give the share that balances the two, and the
//   engine moves halfway to it (TM_DIRECT_FRACTION fixes it instead);
// - otherwise, pinned caller buffer: one 32-bit copy straight into it;
// - otherwise: a 32-bit copy into pinned staging, then copy threads.
void Engine::match_host(const uint32_t *queries, uint64_t nq, bool unique, uint64_t *out_offsets, uint32_t *out_keys,
                        uint64_t capacity, uint64_t *n_keys) {
    std::lock_guard<std::mutex> lk(api_mtx_);
    if (!already_consolidated_) throw Error(TM_ERR_STATE, "match before consolidate()");
    Device &d = device(0);
    if (dev_version_[0] != table_version_) build_device_table(d);
    TM_CUDA(cudaSetDevice(d.id));
    // TM_HOST_TRACE: one stderr line per batch with the host wait, match,
    // copy and widening times (diagnostics)
    const bool trace = std::getenv("TM_HOST_TRACE") != nullptr;
    using TClock = std::chrono::steady_clock;
    const TClock::time_point t_call = TClock::now();
    auto ms_at = [&](TClock::time_point t) { return std::chrono::duration<double, std::milli>(t - t_call).count(); };
    MatchScratch *scr[kHostLanes];
    cudaStream_t str[kHostLanes];
    for (int l = 0; l < kHostLanes; ++l) {
        HostLane &h = d.host[l];
        if (l && !h.stream) TM_CUDA(cudaStreamCreateWithFlags(&h.stream, cudaStreamNonBlocking));
        if (!h.staged) TM_CUDA(cudaEventCreateWithFlags(&h.staged, cudaEventDisableTiming));
        scr[l] = l ? &h.scratch : &d.scratch;
        str[l] = l ? h.stream : d.stream;
        scr[l]->seg_tiles = seg_tiles_;
        if (trace)
            for (cudaEvent_t &ev : h.trace_ev)
                if (!ev) TM_CUDA(cudaEventCreate(&ev));
    }
    const bool narrow = d.table.max_key < 65536u;
    const bool pinned_out = out_keys != nullptr && is_pinned(out_keys);
    const double fixed_frac = direct_fraction_fixed();
    const bool adapt = pinned_out && narrow && fixed_frac < 0;
    if (direct_frac_ < 0) direct_frac_ = kDirectFraction;
    for (int l = 0; l < kHostLanes && adapt; ++l)
        for (cudaEvent_t &ev : d.host[l].copy_ev)
            if (!ev) TM_CUDA(cudaEventCreate(&ev));
    const double batch_keys = host_batch_keys();
    struct Pending {
        bool active = false;
        uint64_t q0 = 0, base = 0, nk = 0, nd = 0;
        uint32_t n = 0;
        std::thread copier;
        uint64_t batch = 0;
        TClock::time_point t_begin, t_matched, t_widen0, t_widen1;
    } pend[kHostLanes];
    uint64_t total = 0;
    bool overflow = false;
    out_offsets[0] = 0;
    auto finish = [&](int l) {
        Pending &p = pend[l];
        if (!p.active) return;
        const TClock::time_point t_wait = TClock::now();
        if (p.copier.joinable()) p.copier.join();
        TM_CUDA(cudaStreamSynchronize(str[l]));
        if (trace) {
            float m16 = 0.f, m32 = 0.f;
            cudaEventElapsedTime(&m16, d.host[l].trace_ev[0], d.host[l].trace_ev[1]);
            cudaEventElapsedTime(&m32, d.host[l].trace_ev[1], d.host[l].trace_ev[2]);
            std::fprintf(stderr,
                         "[tm host] batch %llu lane %d keys %llu direct %llu begin %.1f matched %.1f widen %.1f-%.1f "
                         "narrow_copy_ms %.1f direct_copy_ms %.1f finish_wait_ms %.1f direct_share %.3f\n",
                         (unsigned long long)p.batch, l, (unsigned long long)p.nk, (unsigned long long)p.nd,
                         ms_at(p.t_begin), ms_at(p.t_matched), ms_at(p.t_widen0), ms_at(p.t_widen1), m16, m32,
                         ms_at(TClock::now()) - ms_at(t_wait), direct_frac_);
        }
        if (adapt && p.nk - p.nd >= (uint64_t(1) << 26)) {
            // link and widening rates of this batch -> the balancing share
            float copy_ms = 0.f;
            const double widen_ms = std::chrono::duration<double, std::milli>(p.t_widen1 - p.t_widen0).count();
            if (cudaEventElapsedTime(&copy_ms, d.host[l].copy_ev[0], d.host[l].copy_ev[1]) == cudaSuccess &&
                copy_ms > 0.f && widen_ms > 0.0) {
                const double c = double(2 * (p.nk - p.nd) + 4 * p.nd) / copy_ms;
                const double w = double(p.nk - p.nd) / widen_ms;
                direct_frac_ = 0.5 * direct_frac_ + 0.5 * balanced_direct_fraction(c, w);
            }
        }
        const uint64_t *o = d.host[l].h_offsets.p;
        for (uint32_t i = 1; i <= p.n; ++i) out_offsets[p.q0 + i] = o[i] + p.base;
        p.active = false;
    };
    try {
        uint64_t it = 0;
        for (uint64_t q0 = 0, step = 0; q0 < nq; q0 += step, ++it) {
            // batch size: the device batch limit, lowered so a batch's output
            // stays near kHostBatchKeys keys (keys per query as last seen)
            uint64_t full = batch_limit_;
            if (host_keys_per_query_ > 0 && batch_keys > 0)
                full = std::min<uint64_t>(full, std::max<uint64_t>(kTailBatch, uint64_t(batch_keys / host_keys_per_query_)));
            // full batches, then the last `full` queries in halving batches
            // (down to kTailBatch): what is left to copy and widen after the
            // last match is then a small batch's results
            const uint64_t left = nq - q0;
            step = left > full ? full
                   : left <= 2 * kTailBatch ? left
                                            : std::max<uint64_t>(kTailBatch, left / 2);
            const uint32_t n = uint32_t(step);
            const int l = int(it % kHostLanes);
            finish(l);
            const TClock::time_point t_begin = TClock::now();
            HostLane &h = d.host[l];
            MatchScratch &sc = *scr[l];
            sc.queries.reserve(size_t(n) * kWords);
            TM_CUDA(cudaMemcpyAsync(sc.queries.p, queries + q0 * kWords, size_t(n) * 24, cudaMemcpyHostToDevice, str[l]));
            const uint64_t *doff;
            const uint32_t *dkeys;
            uint64_t nk = 0;
            BatchStats bs;
            sc.profile = profile_;
            prepare(sc, n, false);
            match_batch(d.table, sc.queries.p, n, unique, sc, &doff, &dkeys, &nk, &bs, str[l]);
            observe(d.table, sc, n, std::chrono::duration<double, std::milli>(TClock::now() - t_begin).count(), nk);
            stats_.add(bs, n, profile_);
            stats_.h2d_bytes += uint64_t(n) * 24;
            h.h_offsets.reserve(size_t(n) + 1);
            TM_CUDA(cudaMemcpyAsync(h.h_offsets.p, doff, (size_t(n) + 1) * 8, cudaMemcpyDeviceToHost, str[l]));
            stats_.d2h_bytes += (uint64_t(n) + 1) * 8;
            Pending &p = pend[l];
            p.active = true;
            p.q0 = q0;
            p.n = n;
            p.base = total;
            p.nk = nk;
            p.nd = 0;
            p.batch = it;
            p.t_begin = t_begin;
            p.t_matched = TClock::now();
            p.t_widen0 = p.t_widen1 = p.t_matched;
            if (trace)  // all three recorded; the narrow path records [1] and [2] again after its copies
                for (cudaEvent_t ev : h.trace_ev) TM_CUDA(cudaEventRecord(ev, str[l]));
            if (!overflow && total + nk <= capacity && nk) {
                uint32_t *dst = out_keys + total;
                if (narrow) {
                    // keys [0, nd) direct, [nd, nk) narrowed; nd a multiple
                    // of 4 keeps the narrowing kernel on 16-byte loads
                    const double frac = !pinned_out ? 0.0 : fixed_frac >= 0 ? fixed_frac : direct_frac_;
                    const uint64_t nd = std::min<uint64_t>(nk, uint64_t(double(nk) * frac) & ~uint64_t(3));
                    const uint64_t nn = nk - nd;
                    p.nd = nd;
                    if (nn) {
                        const uint16_t *d16 = narrow_keys(dkeys + nd, nn, sc, str[l]);
                        if (adapt) TM_CUDA(cudaEventRecord(h.copy_ev[0], str[l]));
                        h.h_keys16.reserve(nn);
                        TM_CUDA(cudaMemcpyAsync(h.h_keys16.p, d16, nn * 2, cudaMemcpyDeviceToHost, str[l]));
                        TM_CUDA(cudaEventRecord(h.staged, str[l]));
                        cudaEvent_t ev = h.staged;
                        const uint16_t *src = h.h_keys16.p;
                        uint32_t *wdst = dst + nd;
                        Pending *pp = &p;
                        p.copier = std::thread([=] {
                            if (cudaEventSynchronize(ev) != cudaSuccess) return;
                            pp->t_widen0 = TClock::now();
                            parallel_widen(wdst, src, nn);
                            pp->t_widen1 = TClock::now();
                        });
                    } else if (adapt) {
                        TM_CUDA(cudaEventRecord(h.copy_ev[0], str[l]));
                    }
                    if (trace) TM_CUDA(cudaEventRecord(h.trace_ev[1], str[l]));
                    if (nd) TM_CUDA(cudaMemcpyAsync(dst, dkeys, nd * 4, cudaMemcpyDeviceToHost, str[l]));
                    if (adapt) TM_CUDA(cudaEventRecord(h.copy_ev[1], str[l]));
                    if (trace) TM_CUDA(cudaEventRecord(h.trace_ev[2], str[l]));
                    stats_.d2h_bytes += nn * 2 + nd * 4;
                } else if (pinned_out) {
                    TM_CUDA(cudaMemcpyAsync(dst, dkeys, nk * 4, cudaMemcpyDeviceToHost, str[l]));
                    stats_.d2h_bytes += nk * 4;
                } else {
                    h.h_keys.reserve(nk);
                    TM_CUDA(cudaMemcpyAsync(h.h_keys.p, dkeys, nk * 4, cudaMemcpyDeviceToHost, str[l]));
                    TM_CUDA(cudaEventRecord(h.staged, str[l]));
                    cudaEvent_t ev = h.staged;
                    const uint32_t *src = h.h_keys.p;
                    p.copier = std::thread([=] {
                        if (cudaEventSynchronize(ev) == cudaSuccess) parallel_copy(dst, src, nk * 4);
                    });
                    stats_.d2h_bytes += nk * 4;
                }
            } else if (nk) {
                overflow = true;
            }
            total += nk;
            if (n >= kTailBatch) host_keys_per_query_ = double(nk) / n;
        }
        for (int l = 0; l < kHostLanes; ++l) finish(l);
    } catch (...) {
        for (int l = 0; l < kHostLanes; ++l)
            if (pend[l].copier.joinable()) pend[l].copier.join();
        throw;
    }
    *n_keys = total;
    if (overflow) throw Error(TM_ERR_CAPACITY, "output key buffer too small: " + std::to_string(total) + " keys needed");
}

}  // namespace tmb
