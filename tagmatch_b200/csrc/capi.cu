// C ABI over the engine (declarations and reference citations in
// include/tagmatch_b200.h).
#include "../../include/tagmatch_b200.h"
#include "engine.cuh"
#include <cstring>
#include <new>
#include <string>

struct tm_engine {
    tmb::Engine eng;
    std::string err;
};

namespace {

template <class F>
int guard(tm_engine *e, F &&f) {
    try {
        f();
        if (e) e->err.clear();
        return TM_OK;
    } catch (const tmb::Error &x) {
        if (e) e->err = x.what();
        return x.status;
    } catch (const std::bad_alloc &) {
        if (e) e->err = "host allocation failed";
        return TM_ERR_NOMEM;
    } catch (const std::exception &x) {
        if (e) e->err = x.what();
        return TM_ERR_INTERNAL;
    }
}

}  // namespace

extern "C" {

const char *tm_version(void) { return "tagmatch-b200 0.1 (sm_100a)"; }

int tm_create(tm_engine **out) {
    if (!out) return TM_ERR_INVALID;
    *out = new (std::nothrow) tm_engine();
    return *out ? TM_OK : TM_ERR_NOMEM;
}

void tm_destroy(tm_engine *e) { delete e; }

const char *tm_last_error(const tm_engine *e) { return e ? e->err.c_str() : "null engine"; }

int tm_add(tm_engine *e, const uint32_t filter[TM_FILTER_WORDS], const uint32_t *keys, uint32_t n_keys) {
    if (!e || !filter || (n_keys && !keys)) return TM_ERR_INVALID;
    return guard(e, [&] { e->eng.add(filter, keys, n_keys); });
}

int tm_add_many(tm_engine *e, const uint32_t *filters, uint64_t n, const uint32_t *key_offsets, const uint32_t *keys) {
    if (!e || (n && (!filters || !key_offsets))) return TM_ERR_INVALID;
    return guard(e, [&] { e->eng.add_many(filters, n, key_offsets, keys); });
}

int tm_remove(tm_engine *e, const uint32_t filter[TM_FILTER_WORDS], uint32_t key) {
    if (!e || !filter) return TM_ERR_INVALID;
    return guard(e, [&] { e->eng.remove(filter, key); });
}

int tm_set_database_filename(tm_engine *e, const char *name) {
    if (!e || !name) return TM_ERR_INVALID;
    return guard(e, [&] { e->eng.set_db(name); });
}

const char *tm_get_database_filename(const tm_engine *e) { return e ? e->eng.db().c_str() : nullptr; }

int tm_set_persistence(tm_engine *e, int on) {
    if (!e) return TM_ERR_INVALID;
    return guard(e, [&] { e->eng.set_persist(on != 0); });
}

int tm_consolidate(tm_engine *e, uint32_t partition_size, uint32_t threads) {
    if (!e) return TM_ERR_INVALID;
    return guard(e, [&] { e->eng.consolidate(partition_size, threads); });
}

int tm_consolidate_default(tm_engine *e) {
    if (!e) return TM_ERR_INVALID;
    return guard(e, [&] { e->eng.consolidate(); });
}

int tm_start(tm_engine *e, uint32_t threads, uint32_t gpu_count) {
    if (!e) return TM_ERR_INVALID;
    return guard(e, [&] { e->eng.start(threads, gpu_count); });
}

int tm_stop(tm_engine *e) {
    if (!e) return TM_ERR_INVALID;
    return guard(e, [&] { e->eng.stop(); });
}

int tm_clear(tm_engine *e) {
    if (!e) return TM_ERR_INVALID;
    return guard(e, [&] { e->eng.clear(); });
}

int tm_set_latency_limit_ms(tm_engine *e, uint32_t ms) {
    if (!e) return TM_ERR_INVALID;
    e->eng.set_latency_limit_ms(ms);
    return TM_OK;
}

uint32_t tm_get_latency_limit_ms(const tm_engine *e) { return e ? e->eng.latency_limit_ms() : 0; }

int tm_set_batch_limit(tm_engine *e, uint32_t queries) {
    if (!e || queries == 0) return TM_ERR_INVALID;
    e->eng.set_batch_limit(queries);
    return TM_OK;
}

int tm_match_batch(tm_engine *e, const uint32_t *queries, uint64_t n, int unique, uint64_t *out_offsets,
                   uint32_t *out_keys, uint64_t capacity, uint64_t *n_keys) {
    if (!e || !out_offsets || !n_keys || (n && !queries) || (capacity && !out_keys)) return TM_ERR_INVALID;
    return guard(e, [&] { e->eng.match_host(queries, n, unique != 0, out_offsets, out_keys, capacity, n_keys); });
}

int tm_match_batch_device(tm_engine *e, const uint32_t *d_queries, uint32_t n, int unique, const uint64_t **d_offsets,
                          const uint32_t **d_keys, uint64_t *n_keys, void *stream) {
    if (!e || !d_offsets || !d_keys || !n_keys || (n && !d_queries)) return TM_ERR_INVALID;
    return guard(e, [&] {
        e->eng.match_device(d_queries, n, unique != 0, d_offsets, d_keys, n_keys, static_cast<cudaStream_t>(stream), nullptr,
                            nullptr, nullptr);
    });
}

int tm_match_batch_device_noalloc(tm_engine *e, const uint32_t *d_queries, uint32_t n, int unique,
                                  uint64_t *d_out_offsets, uint32_t *d_out_keys, uint64_t capacity, uint64_t *n_keys,
                                  void *stream) {
    if (!e || !d_out_offsets || !n_keys || (n && !d_queries) || (capacity && !d_out_keys)) return TM_ERR_INVALID;
    return guard(e, [&] {
        e->eng.match_device_noalloc(d_queries, n, unique != 0, d_out_offsets, d_out_keys, capacity, n_keys,
                                    static_cast<cudaStream_t>(stream));
    });
}

int tm_match_async(tm_engine *e, const uint32_t query[TM_FILTER_WORDS], int unique, uint64_t tag, tm_match_callback cb,
                   void *user) {
    if (!e || !query) return TM_ERR_INVALID;
    return guard(e, [&] {
        tmb::AsyncRequest r;
        std::memcpy(r.words, query, sizeof(r.words));
        r.unique = unique != 0;
        r.tag = tag;
        r.cb = cb;
        r.user = user;
        e->eng.submit(r);
    });
}

int tm_submit(tm_engine *e, const uint32_t *queries, uint32_t n, int unique, uint64_t tag, tm_request_callback cb,
              void *user) {
    if (!e || (n && !queries) || !cb) return TM_ERR_INVALID;
    return guard(e, [&] { e->eng.submit_request(queries, n, unique != 0, tag, cb, user); });
}

int tm_set_flush_mode(tm_engine *e, int mode) {
    if (!e || mode < TM_FLUSH_FULL_OR_LATENCY || mode > TM_FLUSH_LEARNED) return TM_ERR_INVALID;
    e->eng.set_flush_mode(mode);
    return TM_OK;
}

int tm_set_serving_results(tm_engine *e, int where) {
    if (!e || (where != TM_RESULTS_HOST && where != TM_RESULTS_DEVICE)) return TM_ERR_INVALID;
    e->eng.set_device_results(where == TM_RESULTS_DEVICE);
    return TM_OK;
}

int tm_set_memory_budget(tm_engine *e, uint64_t bytes) {
    if (!e || bytes == 0) return TM_ERR_INVALID;
    e->eng.set_memory_budget(bytes);
    return TM_OK;
}

int tm_balanced_partitioning(const uint32_t *filters, uint64_t n, uint32_t max_p, uint32_t *partition_of,
                             uint32_t *masks, uint32_t *sizes, uint64_t capacity, uint64_t *n_partitions) {
    if ((n && (!filters || !partition_of)) || !n_partitions || max_p == 0) return TM_ERR_INVALID;
    if (n >= 0xFFFFFFFFull) return TM_ERR_INVALID;
    try {
        cudaStream_t st;
        TM_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        struct StreamGuard {
            cudaStream_t s;
            ~StreamGuard() { cudaStreamDestroy(s); }
        } sg{st};
        tmb::DevBuf<uint32_t> f;
        f.reserve(size_t(n) * TM_FILTER_WORDS);
        if (n) TM_CUDA(cudaMemcpyAsync(f.p, filters, size_t(n) * 24, cudaMemcpyHostToDevice, st));
        tmb::PartitionResult pr;
        tmb::gpu_partition(f.p, uint32_t(n), max_p, false, pr, st);
        const uint64_t np = pr.parts.size();
        *n_partitions = np;
        std::vector<uint32_t> order(n), words(size_t(n) * TM_FILTER_WORDS);
        if (n) {
            TM_CUDA(cudaMemcpy(order.data(), pr.order.p, size_t(n) * 4, cudaMemcpyDeviceToHost));
            TM_CUDA(cudaMemcpy(words.data(), pr.words.p, size_t(n) * 24, cudaMemcpyDeviceToHost));
        }
        for (uint64_t p = 0; p < np; ++p) {
            const tmb::Range r = pr.parts[p];
            uint32_t m[TM_FILTER_WORDS];
            for (int k = 0; k < TM_FILTER_WORDS; ++k) m[k] = 0xFFFFFFFFu;
            for (uint32_t i = r.begin; i < r.end; ++i) {
                partition_of[order[i]] = uint32_t(p);
                for (int k = 0; k < TM_FILTER_WORDS; ++k) m[k] &= words[size_t(i) * TM_FILTER_WORDS + k];
            }
            if (p < capacity) {
                if (masks) std::memcpy(masks + p * TM_FILTER_WORDS, m, sizeof(m));
                if (sizes) sizes[p] = r.end - r.begin;
            }
        }
        return np > capacity ? TM_ERR_CAPACITY : TM_OK;
    } catch (const tmb::Error &x) {
        return x.status;
    } catch (...) {
        return TM_ERR_INTERNAL;
    }
}

int tm_autotune(tm_engine *e, const uint32_t *queries, uint32_t n, uint32_t *seg_tiles, uint32_t *batch_limit,
                double *queries_per_s) {
    if (!e || !queries || n == 0 || !seg_tiles || !batch_limit || !queries_per_s) return TM_ERR_INVALID;
    return guard(e, [&] { e->eng.autotune(queries, n, seg_tiles, batch_limit, queries_per_s); });
}

int tm_sched_record(tm_engine *e, int on) {
    if (!e) return TM_ERR_INVALID;
    return guard(e, [&] { e->eng.scheduler().set_recording(on != 0); });
}

int tm_sched_samples(tm_engine *e, float *features, float *log_cycles, uint64_t capacity, uint64_t *n) {
    if (!e || !n) return TM_ERR_INVALID;
    return guard(e, [&] { e->eng.scheduler().export_samples(features, log_cycles, capacity, n); });
}

int tm_sched_train(tm_engine *e, uint32_t epochs, tm_sched_report *rep) {
    if (!e || epochs == 0) return TM_ERR_INVALID;
    return guard(e, [&] {
        const tmb::TrainReport r = e->eng.train_scheduler(epochs);
        if (rep) {
            rep->samples = r.samples;
            rep->steps = r.steps;
            rep->train_mse = r.train_mse;
            rep->val_mse = r.val_mse;
            rep->val_r2 = r.val_r2;
            rep->mean_mse = r.mean_mse;
            rep->ms = r.ms;
        }
    });
}

int tm_sched_use_order(tm_engine *e, int on) {
    if (!e) return TM_ERR_INVALID;
    return guard(e, [&] {
        if (on && !e->eng.scheduler().trained()) throw tmb::Error(TM_ERR_STATE, "the cost model is not trained");
        e->eng.set_learned_order(on != 0);
    });
}

int tm_sched_predict_batch_ms(tm_engine *e, uint32_t queries, double *ms) {
    if (!e || !ms) return TM_ERR_INVALID;
    return guard(e, [&] { *ms = e->eng.scheduler().predict_batch_ms(queries); });
}

int tm_set_latency_target_ms(tm_engine *e, uint32_t ms) {
    if (!e || ms == 0) return TM_ERR_INVALID;
    return guard(e, [&] { e->eng.set_latency_target_ms(ms); });
}

uint32_t tm_mlp_param_count(void) { return uint32_t(tmb::kMlpParams); }

int tm_mlp_loss_grad(const float *params, const float *features, const float *targets, uint32_t n, float *outputs,
                     float *grad, float *loss) {
    if (!params || !grad || !loss || (n && (!features || !targets || !outputs))) return TM_ERR_INVALID;
    try {
        tmb::CostModel::loss_grad(params, features, targets, n, outputs, grad, loss, nullptr);
        return TM_OK;
    } catch (const tmb::Error &x) {
        return x.status;
    } catch (...) {
        return TM_ERR_INTERNAL;
    }
}

int tm_set_tiles_per_item(tm_engine *e, uint32_t seg_tiles) {
    if (!e) return TM_ERR_INVALID;
    return guard(e, [&] { e->eng.set_seg_tiles(seg_tiles); });
}

uint32_t tm_get_tiles_per_item(const tm_engine *e) { return e ? e->eng.seg_tiles() : 0; }

int tm_get_table_info(tm_engine *e, tm_table_info *info) {
    if (!e || !info) return TM_ERR_INVALID;
    return guard(e, [&] {
        const tmb::DevTable *t = e->eng.table(0);
        info->filters = e->eng.n_filters();
        info->keys = e->eng.keys().size();
        info->partitions = t ? t->n_parts : 0;
        info->tiles = t ? t->n_tiles : 0;
        info->device_bytes = t ? t->device_bytes() : 0;
        info->max_key = t ? t->max_key : 0;
    });
}

int tm_get_match_stats(tm_engine *e, tm_match_stats *st) {
    if (!e || !st) return TM_ERR_INVALID;
    const tmb::EngineStats &s = e->eng.stats();
    st->batches = s.batches;
    st->queries = s.queries;
    st->routed = s.routed;
    st->items = s.items;
    st->pairs = s.pairs;
    st->keys = s.keys;
    st->pair_retries = s.pair_retries;
    st->match_kernel_launches = s.match_launches;
    st->match_kernel_ms = s.match_ms;
    st->dense_tests = s.dense;
    st->kernel_launches = s.launches;
    st->h2d_bytes = s.h2d_bytes;
    st->d2h_bytes = s.d2h_bytes;
    st->records = s.records;
    return TM_OK;
}

int tm_reset_match_stats(tm_engine *e) {
    if (!e) return TM_ERR_INVALID;
    e->eng.reset_stats();
    return TM_OK;
}

int tm_set_profiling(tm_engine *e, int on) {
    if (!e) return TM_ERR_INVALID;
    return guard(e, [&] { e->eng.set_profiling(on != 0); });
}

}  // extern "C"
