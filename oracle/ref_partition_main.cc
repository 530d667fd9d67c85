// Harness around the reference's own CPU partitioner (partitioning.cc, built
// from the reference sources by oracle/Makefile without GPU partitioning).
// TEST INFRASTRUCTURE ONLY.
//
// usage: ref_partition <max_p> <threads> < filters.bin > partitions.txt
//   filters.bin: n records of 24 bytes (the bitvector binary image,
//   bitvector.hh write_binary).
//   Output: one line per input filter "f <index> <partition id>", then one
//   line per partition "p <id> <size> <6 mask words in hex>".
#include <cstdio>
#include <cstdint>
#include <cstdlib>
#include <vector>
#include <iostream>

#include "partitioning.hh"
#include "fib.hh"

int main(int argc, char **argv) {
    if (argc < 3) { std::fprintf(stderr, "usage: %s max_p threads\n", argv[0]); return 2; }
    unsigned maxp = std::strtoul(argv[1], nullptr, 10);
    unsigned threads = std::strtoul(argv[2], nullptr, 10);
    std::vector<partition_fib_entry *> fib;
    std::vector<partition_fib_entry *> by_input;
    uint32_t w[6];
    while (std::fread(w, sizeof(uint32_t), 6, stdin) == 6) {
        fib_entry fe;
        uint64_t b[3] = {w[0] | (uint64_t(w[1]) << 32), w[2] | (uint64_t(w[3]) << 32), w[4] | (uint64_t(w[5]) << 32)};
        fe.filter = filter_t(b);
        fe.keys.push_back(uint32_t(by_input.size()));
        partition_fib_entry *p = new partition_fib_entry(fe);
        fib.push_back(p);
        by_input.push_back(p);
    }
    std::vector<partition_prefix> masks;
    partitioning::set_maxp(maxp);
    partitioning::set_cpu_threads(threads);
    partitioning::balanced_partitioning(fib, masks);
    for (size_t i = 0; i < by_input.size(); ++i)
        std::printf("f %zu %u\n", i, by_input[i]->partition);
    for (const partition_prefix &pp : masks) {
        std::printf("p %u %u", pp.partition, pp.size);
        for (unsigned k = 0; k < 6; ++k) std::printf(" %08x", pp.filter.uint32_value(k));
        std::printf("\n");
    }
    for (partition_fib_entry *p : by_input) delete p;
    return 0;
}
