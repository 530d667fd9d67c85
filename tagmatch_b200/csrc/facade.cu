// The reference's static tagmatch API (tagmatch.hh:11-37) over one
// process-wide engine.  The API has no status codes (the reference prints
// and exits on CUDA errors, gpu.cu:14-24); here failures are printed and the
// call returns, and match()/match_unique() stay noexcept: a query that
// cannot be queued completes at once with no keys.
#include <cstdio>
#include <iostream>
#include "tagmatch.hh"
#include "engine.cuh"

namespace {

tmb::Engine &engine() {
    static tmb::Engine e;
    return e;
}

template <class F>
void report(const char *what, F &&f) {
    try {
        f();
    } catch (const std::exception &x) {
        std::cerr << "tagmatch::" << what << ": " << x.what() << std::endl;
    }
}

void words_of(const filter_t &f, uint32_t *w) { f.copy_into_uint32_array(w); }

void deliver(void *, uint64_t tag, const uint32_t *keys, uint64_t n) {
    reinterpret_cast<tagmatch_query *>(tag)->deliver(keys, n);
}

void enqueue(tagmatch_query *q, match_handler *h, bool unique) noexcept {
    q->match_unique = unique;
    q->set_match_handler(h);
    try {
        tmb::AsyncRequest r;
        words_of(q->filter, r.words);
        r.unique = unique;
        r.tag = reinterpret_cast<uint64_t>(q);
        r.cb = deliver;
        r.user = nullptr;
        engine().submit(r);
    } catch (const std::exception &x) {
        std::cerr << "tagmatch::match: " << x.what() << std::endl;
        q->deliver(nullptr, 0);
    }
}

}  // namespace

void tagmatch::add(const filter_t &s, const std::vector<tagmatch_key_t> &keys) {
    uint32_t w[6];
    words_of(s, w);
    report("add", [&] { engine().add(w, keys.data(), uint32_t(keys.size())); });
}

void tagmatch::add(const filter_t &s, tagmatch_key_t key) {
    uint32_t w[6];
    words_of(s, w);
    report("add", [&] { engine().add(w, &key, 1); });
}

void tagmatch::remove(const filter_t &s, tagmatch_key_t key) {
    uint32_t w[6];
    words_of(s, w);
    report("remove", [&] { engine().remove(w, key); });
}

void tagmatch::consolidate() { report("consolidate", [&] { engine().consolidate(); }); }

void tagmatch::consolidate(unsigned int psize, unsigned int threads) {
    report("consolidate", [&] { engine().consolidate(psize, threads); });
}

const char *tagmatch::get_database_filename() { return engine().db().c_str(); }
void tagmatch::set_database_filename(const char *name) { engine().set_db(name ? name : "tagmatch.db"); }

void tagmatch::start() { report("start", [&] { engine().start(); }); }
void tagmatch::start(unsigned int threads, unsigned int gpus) { report("start", [&] { engine().start(threads, gpus); }); }
void tagmatch::stop() { report("stop", [&] { engine().stop(); }); }
void tagmatch::clear() { report("clear", [&] { engine().clear(); }); }

unsigned int tagmatch::get_latency_limit_ms() { return engine().latency_limit_ms(); }
void tagmatch::set_latency_limit_ms(unsigned int ms) { engine().set_latency_limit_ms(ms); }

void tagmatch::match(tagmatch_query *q, match_handler *h) noexcept { enqueue(q, h, false); }
void tagmatch::match_unique(tagmatch_query *q, match_handler *h) noexcept { enqueue(q, h, true); }
