// tagmatch_query (tagmatch_query.hh of the reference): a query with its
// completion handler.  The engine fills output_keys (sorted and unique for
// match_unique, tagmatch_query.hh:99-119) and then calls the handler's
// match_done() exactly once.
#ifndef TAGMATCH_TAGMATCH_QUERY_HH_INCLUDED
#define TAGMATCH_TAGMATCH_QUERY_HH_INCLUDED
#include <cstdint>
#include "match_handler.hh"
#include "query.hh"

class tagmatch_query : public query {
    match_handler *handler = nullptr;

public:
    tagmatch_query() : query() {}
    tagmatch_query(const filter_t &f) : query(f) {}
    tagmatch_query(const std::string &f) : query(f) {}
    tagmatch_query(const tagmatch_query &x) : query(x), handler(x.handler) {}
    tagmatch_query(tagmatch_query &&x) : query(std::move(x)), handler(x.handler) { x.handler = nullptr; }

    void set_match_handler(match_handler *h) { handler = h; }
    match_handler *get_match_handler() const { return handler; }

    // called by the engine with the query's keys
    void deliver(const uint32_t *keys, uint64_t n) {
        output_keys.assign(keys, keys + n);
        if (handler) handler->match_done(this);
    }
};
#endif
