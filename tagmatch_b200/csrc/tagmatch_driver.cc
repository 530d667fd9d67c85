// Streaming driver over the tagmatch.hh-compatible API, following the flow
// of the reference's tagmatch_main.cc (:122-225): load filters in chunks,
// consolidate, start, match every query of a query file asynchronously,
// stop (drain), clear; per chunk it prints the consolidate, enqueue and
// drain times, the number of completed queries and keys, and the
// end-to-end rate including the drain.  It can also write the partitioning
// client's files (test_partitioning_client.cc:84-221): partition_prefix
// records and partition_fib_entry records (fib.hh:41-77).
//
// usage: tagmatch_driver in=<filters> [Q=<queries>] [-b|-p] [m=<max partition>]
//          [t=<threads>] [u=<partitioner threads>] [gg=<gpus>] [chunk=<filters>]
//          [unique=0|1] [latency=<ms>] [part_out=<prefix>] [db=<file>]
//   in=   binary fib_entry records (24-byte filter, u32 n, n keys) with -b
//         (default), or partition_fib_entry records (u32 partition first)
//         with -p
//   Q=    binary 24-byte query records
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "tagmatch.hh"
#include "tagmatch_b200.h"

using Clock = std::chrono::steady_clock;

namespace {

class match_counter : public match_handler {
public:
    std::atomic<uint64_t> queries{0}, keys{0};
    void process_results(query *q) override {
        queries++;
        keys += q->output_keys.size();
    }
};

struct Record {
    filter_t filter;
    std::vector<tagmatch_key_t> keys;
};

// Reads up to `limit` records; false at end of input.
bool read_records(std::istream &in, bool with_partition, size_t limit, std::vector<Record> &out) {
    out.clear();
    while (out.size() < limit) {
        uint32_t part = 0, n = 0;
        if (with_partition && !in.read(reinterpret_cast<char *>(&part), 4)) return false;
        Record r;
        if (!r.filter.read_binary(in)) return false;
        if (!in.read(reinterpret_cast<char *>(&n), 4)) return false;
        r.keys.resize(n);
        if (n && !in.read(reinterpret_cast<char *>(r.keys.data()), std::streamsize(n) * 4)) return false;
        out.push_back(std::move(r));
    }
    return true;
}

double ms_since(Clock::time_point t) { return std::chrono::duration<double, std::milli>(Clock::now() - t).count(); }

int write_partitions(const std::vector<Record> &fib, unsigned maxp, const std::string &prefix) {
    std::vector<uint32_t> words(fib.size() * 6), part(fib.size());
    for (size_t i = 0; i < fib.size(); ++i) fib[i].filter.copy_into_uint32_array(&words[i * 6]);
    uint64_t np = 0, cap = fib.size() / 8 + 1024;
    std::vector<uint32_t> masks, sizes;
    int st;
    do {
        masks.assign(cap * 6, 0);
        sizes.assign(cap, 0);
        st = tm_balanced_partitioning(words.data(), fib.size(), maxp, part.data(), masks.data(), sizes.data(), cap, &np);
        if (st == TM_ERR_CAPACITY) cap = np;
    } while (st == TM_ERR_CAPACITY);
    if (st != TM_OK) {
        std::cerr << "partitioning failed: " << st << std::endl;
        return 1;
    }
    std::ofstream pf(prefix + ".partitions", std::ios::binary), ff(prefix + ".filters", std::ios::binary);
    for (uint64_t p = 0; p < np; ++p) {
        filter_t m;
        m.assign_uint32_array(&masks[p * 6]);
        const uint8_t length = 192;
        const uint32_t pid = uint32_t(p), size = sizes[p];
        m.write_binary(pf);  // partition_prefix::write_binary (fib.hh:63-69)
        pf.write(reinterpret_cast<const char *>(&length), 1);
        pf.write(reinterpret_cast<const char *>(&pid), 4);
        pf.write(reinterpret_cast<const char *>(&size), 4);
    }
    for (size_t i = 0; i < fib.size(); ++i) {  // partition_fib_entry::write_binary (fib.hh:46-49)
        const uint32_t n = uint32_t(fib[i].keys.size());
        ff.write(reinterpret_cast<const char *>(&part[i]), 4);
        fib[i].filter.write_binary(ff);
        ff.write(reinterpret_cast<const char *>(&n), 4);
        ff.write(reinterpret_cast<const char *>(fib[i].keys.data()), std::streamsize(n) * 4);
    }
    std::printf("partitions=%llu written to %s.partitions / %s.filters\n", (unsigned long long)np, prefix.c_str(),
                prefix.c_str());
    return 0;
}

}  // namespace

int main(int argc, char **argv) {
    std::string in_f, q_f, part_out, db = "tagmatch_driver.db";
    unsigned maxp = 65536, threads = 4, pthreads = 1, gpus = 1, latency = 0;
    size_t chunk = size_t(1) << 62;
    bool with_partition = false, unique = false;
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        auto val = [&](const char *k) { return a.substr(std::strlen(k)); };
        if (a.rfind("in=", 0) == 0) in_f = val("in=");
        else if (a.rfind("Q=", 0) == 0) q_f = val("Q=");
        else if (a == "-b") with_partition = false;
        else if (a == "-p") with_partition = true;
        else if (a.rfind("m=", 0) == 0) maxp = unsigned(std::stoul(val("m=")));
        else if (a.rfind("t=", 0) == 0) threads = unsigned(std::stoul(val("t=")));
        else if (a.rfind("u=", 0) == 0) pthreads = unsigned(std::stoul(val("u=")));
        else if (a.rfind("gg=", 0) == 0) gpus = unsigned(std::stoul(val("gg=")));
        else if (a.rfind("chunk=", 0) == 0) chunk = std::stoull(val("chunk="));
        else if (a.rfind("unique=", 0) == 0) unique = std::stoi(val("unique=")) != 0;
        else if (a.rfind("latency=", 0) == 0) latency = unsigned(std::stoul(val("latency=")));
        else if (a.rfind("part_out=", 0) == 0) part_out = val("part_out=");
        else if (a.rfind("db=", 0) == 0) db = val("db=");
        else {
            std::cerr << "unknown argument " << a << std::endl;
            return 1;
        }
    }
    if (in_f.empty()) {
        std::cerr << "usage: " << argv[0] << " in=<filters> [Q=<queries>] ..." << std::endl;
        return 1;
    }
    std::ifstream input(in_f, std::ios::binary);
    if (!input) {
        std::cerr << "could not open input file " << in_f << std::endl;
        return 1;
    }
    std::vector<filter_t> qs;
    if (!q_f.empty()) {
        std::ifstream qin(q_f, std::ios::binary);
        basic_query bq;
        while (bq.read_binary(qin)) qs.push_back(bq.filter);
    }
    tagmatch::set_database_filename(db.c_str());
    std::vector<Record> fib;
    bool more = true;
    for (int round = 0; more; ++round) {
        more = read_records(input, with_partition, chunk, fib);
        if (fib.empty()) break;
        for (const Record &r : fib) tagmatch::add(r.filter, r.keys);
        auto t0 = Clock::now();
        tagmatch::consolidate(maxp, pthreads);
        const double t_cons = ms_since(t0);
        if (!part_out.empty() && write_partitions(fib, maxp, part_out + (round ? "." + std::to_string(round) : "")))
            return 1;
        std::vector<tagmatch_query> queries;
        queries.reserve(qs.size());
        for (const filter_t &f : qs) queries.emplace_back(f);
        tagmatch::set_latency_limit_ms(latency);
        tagmatch::start(threads, gpus);
        match_counter counter;
        t0 = Clock::now();
        for (tagmatch_query &q : queries) {
            if (unique) tagmatch::match_unique(&q, &counter);
            else tagmatch::match(&q, &counter);
        }
        const double t_enq = ms_since(t0);
        const auto t1 = Clock::now();
        tagmatch::stop();  // drains every pending query
        const double t_drain = ms_since(t1);
        const double t_total = ms_since(t0);
        std::printf(
            "round=%d filters=%zu consolidate_ms=%.1f queries=%zu enqueue_ms=%.1f drain_ms=%.1f completed=%llu keys=%llu "
            "qps=%.1f\n",
            round, fib.size(), t_cons, queries.size(), t_enq, t_drain, (unsigned long long)counter.queries.load(),
            (unsigned long long)counter.keys.load(), t_total > 0 ? 1e3 * queries.size() / t_total : 0.0);
        std::fflush(stdout);
        tagmatch::clear();
    }
    return 0;
}
