// tagmatch: the reference's static API (tagmatch.hh:11-37), backed by the
// B200 engine (include/tagmatch_b200.h).  Same methods, same meaning:
// add/remove stage changes, consolidate() merges them into the table
// (database file + GPU partitioner), start()/stop() run the matcher,
// match()/match_unique() are asynchronous and complete through the query's
// match_handler on an engine thread.
#ifndef TAGMATCH_TAGMATCH_HH_INCLUDED
#define TAGMATCH_TAGMATCH_HH_INCLUDED
#include <vector>
#include "filter.hh"
#include "key.hh"
#include "query.hh"
#include "tagmatch_query.hh"

class tagmatch {
public:
    static void add(const filter_t &set, const std::vector<tagmatch_key_t> &keys);
    static void add(const filter_t &set, tagmatch_key_t key);
    static void remove(const filter_t &set, tagmatch_key_t key);

    static void consolidate();
    static void consolidate(unsigned int partition_size, unsigned int threads);

    static const char *get_database_filename();
    static void set_database_filename(const char *);

    static void start();
    static void start(unsigned int threads, unsigned int gpu_count);
    static void stop();
    static void clear();

    static unsigned int get_latency_limit_ms();
    static void set_latency_limit_ms(unsigned int latency_limit);

    static void match(tagmatch_query *q, match_handler *h) noexcept;
    static void match_unique(tagmatch_query *q, match_handler *h) noexcept;
};
#endif
