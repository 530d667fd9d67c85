// match_handler (match_handler.hh:15-22 of the reference): asynchronous
// completion callback.  match_done() runs on an engine thread, once per
// query, after output_keys is filled; by default it calls process_results().
#ifndef TAGMATCH_MATCH_HANDLER_HH_INCLUDED
#define TAGMATCH_MATCH_HANDLER_HH_INCLUDED
#include "query.hh"

class match_handler {
public:
    virtual void match_done(query *q) { process_results(q); }
    virtual void process_results(query *q) = 0;
    virtual ~match_handler() {}
};
#endif
