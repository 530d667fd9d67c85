// synchronous_match_handler (synchronous_match_handler.hh of the
// reference): lets one caller thread wait for a query's completion and then
// process its results on that thread.
#ifndef TAGMATCH_SYNCHRONOUS_MATCH_HANDLER_HH_INCLUDED
#define TAGMATCH_SYNCHRONOUS_MATCH_HANDLER_HH_INCLUDED
#include <condition_variable>
#include <mutex>
#include "match_handler.hh"

class synchronous_match_handler : public match_handler {
    std::mutex mtx;
    std::condition_variable cv;
    query *ready = nullptr;

public:
    virtual void process_results(query *q) = 0;
    virtual void match_done(query *q) {
        std::lock_guard<std::mutex> lk(mtx);
        ready = q;
        cv.notify_all();
    }
    virtual void synchronize_and_process() {
        query *q;
        {
            std::unique_lock<std::mutex> lk(mtx);
            cv.wait(lk, [this] { return ready != nullptr; });
            q = ready;
            ready = nullptr;
        }
        process_results(q);
    }
};
#endif
