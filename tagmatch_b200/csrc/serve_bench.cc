// Serving load generator over the public C ABI (tm_submit).
//
// Requests of 1..4096 queries (log-uniform sizes) arrive as a Poisson
// process at a given rate of queries per second; each request's latency is
// the time from its scheduled arrival to its completion callback.  The
// table and the query pool come from the seeded workload generator.  For
// every (mode, rate) pair one JSON line is printed:
//   {"mode", "offered_qps", "sustained_qps", "requests", "queries",
//    "p50_ms", "p99_ms", "p999_ms", "keys"}
// Modes: "plain" = one request per device batch on one lane
// (TM_FLUSH_SINGLE); "continuous" = all pending requests share the next
// batch on either of two lanes (TM_FLUSH_IMMEDIATE).
//
// usage: tagmatch_serve_bench [filters=N] [pool=Q] [seed=S] [maxp=P]
//          [rates=r1,r2,...] [modes=plain,continuous] [seconds=T] [unique=0|1]
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <random>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "tagmatch_b200.h"

extern "C" int64_t tmw_generate_filters(uint64_t seed, uint64_t n, double zipf_s, uint32_t n_tags, uint32_t *filters,
                                        uint32_t *key_offsets, uint32_t *keys);
extern "C" int tmw_generate_queries(uint64_t seed, uint64_t nq, const uint32_t *filters, uint64_t n, double zipf_s,
                                    uint32_t n_tags, double superset_fraction, uint32_t *queries);

using Clock = std::chrono::steady_clock;

namespace {

struct Rec {
    Clock::time_point arrival, done;
    uint32_t n = 0;
};

std::vector<Rec> g_recs;
std::atomic<uint64_t> g_done_requests{0}, g_keys{0};

void on_done(void *, uint64_t tag, const uint64_t *offsets, const uint32_t *, uint32_t n, int status) {
    g_recs[tag].done = Clock::now();
    if (status == TM_OK) g_keys += offsets[n];
    g_done_requests++;
}

std::vector<std::string> split(const std::string &s) {
    std::vector<std::string> out;
    std::stringstream ss(s);
    std::string t;
    while (std::getline(ss, t, ',')) out.push_back(t);
    return out;
}

double pct(std::vector<double> &v, double p) {
    if (v.empty()) return 0;
    size_t k = std::min(v.size() - 1, size_t(p * (v.size() - 1) + 0.5));
    std::nth_element(v.begin(), v.begin() + k, v.end());
    return v[k];
}

}  // namespace

int main(int argc, char **argv) {
    uint64_t filters = 10000000, pool = 1 << 20, seed = 2;
    uint32_t maxp = 65536;
    std::string rates = "100000,300000,1000000", modes = "plain,continuous";
    double seconds = 5.0;
    int unique = 0;
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        auto v = a.substr(a.find('=') + 1);
        if (a.rfind("filters=", 0) == 0) filters = std::stoull(v);
        else if (a.rfind("pool=", 0) == 0) pool = std::stoull(v);
        else if (a.rfind("seed=", 0) == 0) seed = std::stoull(v);
        else if (a.rfind("maxp=", 0) == 0) maxp = uint32_t(std::stoul(v));
        else if (a.rfind("rates=", 0) == 0) rates = v;
        else if (a.rfind("modes=", 0) == 0) modes = v;
        else if (a.rfind("seconds=", 0) == 0) seconds = std::stod(v);
        else if (a.rfind("unique=", 0) == 0) unique = std::stoi(v);
    }
    std::vector<uint32_t> f(filters * 6), ko(filters + 1), keys(filters * 4), q(pool * 6);
    const int64_t nk = tmw_generate_filters(seed, filters, 1.0, 100000, f.data(), ko.data(), keys.data());
    if (nk < 0 || tmw_generate_queries(seed, pool, f.data(), filters, 1.0, 100000, 0.5, q.data()) != 0) {
        std::fprintf(stderr, "workload generation failed\n");
        return 2;
    }
    tm_engine *e = nullptr;
    if (tm_create(&e) != TM_OK) return 2;
    tm_set_persistence(e, 0);
    if (tm_add_many(e, f.data(), filters, ko.data(), keys.data()) != TM_OK ||
        tm_consolidate(e, maxp, 1) != TM_OK) {
        std::fprintf(stderr, "build failed: %s\n", tm_last_error(e));
        return 2;
    }
    tm_set_batch_limit(e, 16384);  // bounds one batch's latency
    std::mt19937_64 rng(seed * 7 + 1);
    const double mean_size = (4096.0 - 1.0) / std::log(4096.0);  // log-uniform on [1, 4096]
    for (const std::string &mode : split(modes)) {
        for (const std::string &rs : split(rates)) {
            const double rate = std::stod(rs);
            tm_set_flush_mode(e, mode == "plain" ? TM_FLUSH_SINGLE : TM_FLUSH_IMMEDIATE);
            if (tm_start(e, 4, 1) != TM_OK) {
                std::fprintf(stderr, "start failed: %s\n", tm_last_error(e));
                return 2;
            }
            // warm-up: grow the lanes' buffers to the largest batch before timing
            {
                g_recs.assign(16, Rec());
                for (uint64_t i = 0; i < 16; ++i)
                    tm_submit(e, q.data() + (i * 4096 % (pool - 4096)) * 6, 4096, unique, i, on_done, nullptr);
                tm_stop(e);
                tm_start(e, 4, 1);
            }
            // arrival schedule
            std::exponential_distribution<double> gap(rate / mean_size);
            std::uniform_real_distribution<double> u(0.0, std::log(4097.0));
            std::uniform_int_distribution<uint64_t> off(0, pool - 4096);
            std::vector<double> t_arr;
            std::vector<uint32_t> sizes;
            std::vector<uint64_t> starts;
            for (double t = 0; t < seconds; t += gap(rng)) {
                t_arr.push_back(t);
                sizes.push_back(std::min<uint32_t>(4096, std::max<uint32_t>(1, uint32_t(std::exp(u(rng))))));
                starts.push_back(off(rng));
            }
            g_recs.assign(t_arr.size(), Rec());
            g_done_requests = 0;
            g_keys = 0;
            const Clock::time_point t0 = Clock::now() + std::chrono::milliseconds(20);
            uint64_t queries = 0;
            for (size_t i = 0; i < t_arr.size(); ++i) {
                const auto at = t0 + std::chrono::nanoseconds(int64_t(t_arr[i] * 1e9));
                std::this_thread::sleep_until(at);
                g_recs[i].arrival = at;
                g_recs[i].n = sizes[i];
                queries += sizes[i];
                if (tm_submit(e, q.data() + starts[i] * 6, sizes[i], unique, i, on_done, nullptr) != TM_OK) {
                    std::fprintf(stderr, "submit failed: %s\n", tm_last_error(e));
                    return 2;
                }
            }
            tm_stop(e);  // drains: every callback has fired on return
            std::vector<double> lat;
            Clock::time_point last = t0;
            for (const Rec &r : g_recs) {
                lat.push_back(std::chrono::duration<double, std::milli>(r.done - r.arrival).count());
                last = std::max(last, r.done);
            }
            const double span = std::chrono::duration<double>(last - t0).count();
            std::printf(
                "{\"mode\": \"%s\", \"offered_qps\": %.0f, \"sustained_qps\": %.0f, \"requests\": %zu, \"queries\": %llu, "
                "\"p50_ms\": %.3f, \"p99_ms\": %.3f, \"p999_ms\": %.3f, \"keys\": %llu, \"unique\": %d}\n",
                mode.c_str(), rate, queries / std::max(span, 1e-9), t_arr.size(), (unsigned long long)queries,
                pct(lat, 0.50), pct(lat, 0.99), pct(lat, 0.999), (unsigned long long)g_keys.load(), unique);
            std::fflush(stdout);
        }
    }
    tm_destroy(e);
    return 0;
}
