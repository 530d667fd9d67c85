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
// batch on either of two lanes (TM_FLUSH_IMMEDIATE); "learned" = continuous
// batching with the learned scheduler's flush points and per-batch tiles
// per work item (TM_FLUSH_LEARNED).  Before the first "learned" run the
// engine records timing samples while it serves a calibration load in
// continuous mode (the first and the last rate, calib=T seconds split over
// five tiles per item values), trains its cost model on the GPU and prints the
// training report as a line with "mode": "learned-training".
//
// usage: tagmatch_serve_bench [filters=N] [pool=Q] [seed=S] [maxp=P]
//          [rates=r1,r2,...] [modes=plain,continuous,learned] [seconds=T]
//          [unique=0|1] [target_ms=M] [calib=T] [epochs=E] [plain_rates=...]
//          [results=host,device]
// (plain_rates: the rates of the plain mode, which saturates far below the
// others; default: rates.  results: where the keys go, each in turn --
// host memory, or left in device memory (TM_RESULTS_DEVICE); every line
// says which.)
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
    std::string rates = "100000,300000,1000000", modes = "plain,continuous", plain_rates, results = "host";
    std::string residency = "host";
    double seconds = 5.0, calib = 3.0;
    int unique = 0;
    uint32_t target_ms = 25, epochs = 30;
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        auto v = a.substr(a.find('=') + 1);
        if (a.rfind("filters=", 0) == 0) filters = std::stoull(v);
        else if (a.rfind("pool=", 0) == 0) pool = std::stoull(v);
        else if (a.rfind("seed=", 0) == 0) seed = std::stoull(v);
        else if (a.rfind("maxp=", 0) == 0) maxp = uint32_t(std::stoul(v));
        else if (a.rfind("rates=", 0) == 0) rates = v;
        else if (a.rfind("plain_rates=", 0) == 0) plain_rates = v;
        else if (a.rfind("results=", 0) == 0) results = v;
        else if (a.rfind("modes=", 0) == 0) modes = v;
        else if (a.rfind("seconds=", 0) == 0) seconds = std::stod(v);
        else if (a.rfind("unique=", 0) == 0) unique = std::stoi(v);
        else if (a.rfind("target_ms=", 0) == 0) target_ms = uint32_t(std::stoul(v));
        else if (a.rfind("calib=", 0) == 0) calib = std::stod(v);
        else if (a.rfind("epochs=", 0) == 0) epochs = uint32_t(std::stoul(v));
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
    tm_set_latency_target_ms(e, target_ms);
    // one Poisson load at `rate` for `secs` seconds in flush mode `fm`;
    // returns false on an API failure
    auto run = [&](int fm, double rate, double secs, const char *label, bool print) -> bool {
        tm_set_flush_mode(e, fm);
        if (tm_start(e, 4, 1) != TM_OK) {
            std::fprintf(stderr, "start failed: %s\n", tm_last_error(e));
            return false;
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
        for (double t = 0; t < secs; t += gap(rng)) {
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
                return false;
            }
        }
        tm_stop(e);  // drains: every callback has fired on return
        if (!print) return true;
        std::vector<double> lat;
        Clock::time_point last = t0;
        for (const Rec &r : g_recs) {
            lat.push_back(std::chrono::duration<double, std::milli>(r.done - r.arrival).count());
            last = std::max(last, r.done);
        }
        const double span = std::chrono::duration<double>(last - t0).count();
        std::printf(
            "{\"mode\": \"%s\", \"results\": \"%s\", \"offered_qps\": %.0f, \"sustained_qps\": %.0f, \"requests\": %zu, "
            "\"queries\": %llu, \"p50_ms\": %.3f, \"p99_ms\": %.3f, \"p999_ms\": %.3f, \"keys\": %llu, \"unique\": %d}\n",
            label, residency.c_str(), rate, queries / std::max(span, 1e-9), t_arr.size(), (unsigned long long)queries,
            pct(lat, 0.50), pct(lat, 0.99), pct(lat, 0.999), (unsigned long long)g_keys.load(), unique);
        std::fflush(stdout);
        return true;
    };
    for (const std::string &res : split(results)) {
        residency = res;
        tm_set_serving_results(e, res == "device" ? TM_RESULTS_DEVICE : TM_RESULTS_HOST);
        bool trained = false;
        for (const std::string &mode : split(modes)) {
            int fm = mode == "plain" ? TM_FLUSH_SINGLE : mode == "learned" ? TM_FLUSH_LEARNED : TM_FLUSH_IMMEDIATE;
            if (mode == "learned" && !trained) {
                // calibration: timing samples from continuous serving at several
                // tiles per work item (the model chooses among them), then training
                tm_sched_record(e, 1);
                const uint32_t seg0 = tm_get_tiles_per_item(e);
                const double r_lo = std::stod(split(rates).front()), r_hi = std::stod(split(rates).back());
                for (uint32_t sg : {32u, 128u, 512u, 2048u, 8192u}) {
                    tm_set_tiles_per_item(e, sg);
                    // small batches at the lowest rate, large ones at the highest
                    if (!run(TM_FLUSH_IMMEDIATE, r_lo, calib / 10, "calibration", false) ||
                        !run(TM_FLUSH_IMMEDIATE, r_hi, calib / 10, "calibration", false))
                        return 2;
                }
                tm_set_tiles_per_item(e, seg0);
                tm_sched_record(e, 0);
                tm_sched_report rep{};
                if (tm_sched_train(e, epochs, &rep) != TM_OK) {
                    std::fprintf(stderr, "training failed: %s\n", tm_last_error(e));
                    return 2;
                }
                double p1k = 0, p16k = 0;
                tm_sched_predict_batch_ms(e, 1024, &p1k);
                tm_sched_predict_batch_ms(e, 16384, &p16k);
                std::printf("{\"mode\": \"learned-training\", \"results\": \"%s\", \"samples\": %llu, \"steps\": %llu, "
                            "\"train_mse\": %.4f, \"val_mse\": %.4f, \"val_r2\": %.4f, \"mean_mse\": %.4f, "
                            "\"train_ms\": %.1f, \"pred_ms_1024\": %.3f, \"pred_ms_16384\": %.3f, \"target_ms\": %u}\n",
                            residency.c_str(), (unsigned long long)rep.samples, (unsigned long long)rep.steps,
                            rep.train_mse, rep.val_mse, rep.val_r2, rep.mean_mse, rep.ms, p1k, p16k, target_ms);
                std::fflush(stdout);
                trained = true;
            }
            for (const std::string &rs : split(mode == "plain" && !plain_rates.empty() ? plain_rates : rates))
                if (!run(fm, std::stod(rs), seconds, mode.c_str(), true)) return 2;
        }
    }
    tm_destroy(e);
    return 0;
}
