// Known-answer tests of the tagmatch.hh-compatible C++ API, case for case
// after the reference's test/test_tagmatch.cc (Boost.Test there; a minimal
// harness here).  The fixture filters (F, Q) and the reference
// test_matcher's expected sets are read from the golden fixture file.
//
// usage: tagmatch_facade_test <tagmatch_fixtures.txt> <database path> [case]
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <functional>
#include <iostream>
#include <map>
#include <set>
#include <sstream>
#include <string>
#include <vector>

#include "synchronous_match_handler.hh"
#include "tagmatch.hh"

using std::set;
using std::vector;

static int g_checks = 0, g_failures = 0;
#define CHECK(c)                                                                         \
    do {                                                                                 \
        ++g_checks;                                                                      \
        if (!(c)) {                                                                      \
            ++g_failures;                                                                \
            std::fprintf(stderr, "%s:%d: check failed: %s\n", __FILE__, __LINE__, #c);  \
        }                                                                                \
    } while (0)

static vector<filter_t> F, Q;
static vector<set<tagmatch_key_t>> EXPECTED;  // reference test_matcher on F x Q
static const filter_t ALL_ONES(std::string(192, '1'));
static const filter_t ALL_ZEROS(std::string(192, '0'));

static void init_test() {
    tagmatch::set_latency_limit_ms(200);
    tagmatch::clear();
}

class general_matcher : public synchronous_match_handler {
public:
    void process_results(query *q) override {
        for (tagmatch_key_t k : q->output_keys) keys.insert(k);
    }
    set<tagmatch_key_t> keys;
};

class finder_matcher : public synchronous_match_handler {
public:
    explicit finder_matcher(tagmatch_key_t t) : target(t) {}
    void process_results(query *q) override {
        for (tagmatch_key_t k : q->output_keys)
            if (k == target) found = true;
    }
    tagmatch_key_t target;
    bool found = false;
};

class deferred_matching_checks {
    struct check {
        tagmatch_query *q;
        general_matcher *h;
        set<tagmatch_key_t> expected;
    };
    vector<check> checks;

public:
    void run_query(const filter_t &f, const set<tagmatch_key_t> &s) {
        check c{new tagmatch_query(f), new general_matcher(), s};
        checks.push_back(c);
        tagmatch::match_unique(c.q, c.h);
    }
    void check_results() {
        for (size_t i = 0; i < checks.size(); ++i) {
            checks[i].h->synchronize_and_process();
            if (checks[i].h->keys != checks[i].expected)
                std::fprintf(stderr, "  query %zu: unexpected results\n", i);
            CHECK(checks[i].h->keys == checks[i].expected);
        }
    }
    ~deferred_matching_checks() {
        for (check &c : checks) {
            delete c.q;
            delete c.h;
        }
    }
};

// ---- basics ----
static void consolidate_empty() {
    tagmatch::set_latency_limit_ms(200);
    tagmatch::consolidate();
    tagmatch::clear();
}

static void start_and_stop() {
    tagmatch::consolidate();
    tagmatch::start();
    tagmatch::stop();
    tagmatch::start(4, 1);
    tagmatch::stop();
    tagmatch::clear();
    tagmatch::consolidate();
    tagmatch::start(4, 1);
    tagmatch::stop();
    tagmatch::start();
    tagmatch::stop();
    tagmatch::clear();
}

static void consolidate_no_match_action() {
    for (int round = 0; round < 2; ++round) {
        for (int i = 0; i < 5; ++i) tagmatch::add(F[i], tagmatch_key_t(i));
        tagmatch::consolidate();
        tagmatch::start();
        tagmatch::stop();
        tagmatch::start(4, 1);
        tagmatch::stop();
        tagmatch::clear();
    }
}

static void repeated_stop() {
    tagmatch::start();
    tagmatch::stop();
    tagmatch::stop();
    tagmatch::clear();
    tagmatch::start();
    for (int i = 0; i < 4; ++i) tagmatch::stop();
    tagmatch::clear();
    tagmatch::clear();
    tagmatch::start();
    for (int i = 0; i < 8; ++i) tagmatch::stop();
    tagmatch::clear();
}

static void find_one_filter() {
    tagmatch::clear();
    tagmatch::add(F[1], 1);
    tagmatch::consolidate();
    tagmatch::start();
    finder_matcher f1(1), f2(1), f3(1), f4(1);
    tagmatch_query q1(F[1]), q2(F[2]), q3(ALL_ZEROS), q4(ALL_ONES);
    tagmatch::match_unique(&q1, &f1);
    tagmatch::match_unique(&q2, &f2);
    tagmatch::match_unique(&q3, &f3);
    tagmatch::match_unique(&q4, &f4);
    tagmatch::stop();
    f1.synchronize_and_process();
    f2.synchronize_and_process();
    f3.synchronize_and_process();
    f4.synchronize_and_process();
    CHECK(f1.found);
    CHECK(!f2.found);
    CHECK(!f3.found);
    CHECK(f4.found);
    tagmatch::clear();
}

static void clear_case() {
    tagmatch::clear();
    tagmatch::add(F[1], 1);
    tagmatch::consolidate();
    tagmatch::start();
    finder_matcher f1(1);
    tagmatch_query q1(F[1]);
    tagmatch::match_unique(&q1, &f1);
    tagmatch::stop();
    f1.synchronize_and_process();
    CHECK(f1.found);
    tagmatch::clear();
    tagmatch::consolidate();
    tagmatch::start();
    finder_matcher f2(1);
    tagmatch_query q2(F[1]);
    tagmatch::match_unique(&q2, &f2);
    tagmatch::stop();
    f2.synchronize_and_process();
    CHECK(!f2.found);
}

// ---- same_filter ----
static void add_same_filter() {
    tagmatch::clear();
    tagmatch::add(F[1], 2);
    tagmatch::add(F[1], 3);
    tagmatch::add(F[1], 4);
    tagmatch::consolidate();
    tagmatch::start();
    general_matcher m1, m2;
    tagmatch_query q1(F[1]), q2(F[2]);
    tagmatch::match_unique(&q1, &m1);
    tagmatch::match_unique(&q2, &m2);
    tagmatch::stop();
    m1.synchronize_and_process();
    m2.synchronize_and_process();
    CHECK((m1.keys == set<tagmatch_key_t>{2, 3, 4}));
    CHECK(m2.keys.empty());
    tagmatch::clear();
}

// ---- finding_filters ----
static void add_and_find_multi() {
    tagmatch::set_latency_limit_ms(400);
    tagmatch::clear();
    tagmatch::add(F[1], 1);
    tagmatch::add(F[1], 2);
    tagmatch::add(F[2], 3);
    tagmatch::add(F[3], 4);
    tagmatch::consolidate();
    deferred_matching_checks C;
    C.run_query(F[1], {1, 2});
    C.run_query(F[2], {3});
    C.run_query(F[3], {4});
    tagmatch::start();  // queries issued before start() wait for it
    tagmatch::stop();
    C.check_results();
    tagmatch::clear();
}

static void add_and_find_multi2() {
    init_test();
    tagmatch::add(F[1], 1);
    tagmatch::add(F[1], 2);
    tagmatch::add(F[2], 3);
    tagmatch::add(F[3], 4);
    tagmatch::consolidate();
    tagmatch::start();
    deferred_matching_checks C;
    C.run_query(F[1], {1, 2});
    C.run_query(F[2], {3});
    C.run_query(F[3], {4});
    tagmatch::stop();
    C.check_results();
    tagmatch::clear();
}

static void add_and_clear() {
    deferred_matching_checks C;
    init_test();
    tagmatch::consolidate();
    tagmatch::start(4, 1);
    C.run_query(F[1], {});
    tagmatch::stop();
    tagmatch::add(F[1], 3);
    tagmatch::consolidate();
    tagmatch::start(4, 1);
    C.run_query(F[1], {3});
    tagmatch::stop();
    tagmatch::clear();
    tagmatch::consolidate();
    tagmatch::start(4, 1);
    C.run_query(F[1], {});
    tagmatch::stop();
    C.check_results();
    tagmatch::clear();
}

static void add_many_and_find() {
    init_test();
    deferred_matching_checks C;
    for (int i = 1; i <= 10; ++i) tagmatch::add(F[i], tagmatch_key_t(i));
    tagmatch::consolidate();
    tagmatch::start(4, 1);
    for (int i = 1; i <= 10; ++i) C.run_query(F[i], {tagmatch_key_t(i)});
    tagmatch::stop();
    C.check_results();
    tagmatch::clear();
}

// ---- subset_search ----
static void misc_subsets() {
    init_test();
    deferred_matching_checks C;
    for (size_t i = 0; i < F.size(); ++i) tagmatch::add(F[i], tagmatch_key_t(i));
    tagmatch::consolidate();
    tagmatch::start(4, 1);
    for (size_t i = 0; i < Q.size(); ++i) {
        set<tagmatch_key_t> expected;
        for (size_t j = 0; j < F.size(); ++j)
            if (F[j].subset_of(Q[i])) expected.insert(tagmatch_key_t(j));
        CHECK(expected == EXPECTED[i]);  // this build's subset_of agrees with the reference matcher
        C.run_query(Q[i], expected);
    }
    tagmatch::stop();
    C.check_results();
    tagmatch::clear();
}

static void misc_subsets_Q1() {
    init_test();
    for (size_t i = 0; i < F.size(); ++i) tagmatch::add(F[i], tagmatch_key_t(i));
    tagmatch::consolidate();
    tagmatch::start(4, 1);
    deferred_matching_checks C;
    C.run_query(Q[1], {2});
    tagmatch::stop();
    C.check_results();
    tagmatch::clear();
}

static void corner_case_filters() {
    init_test();
    filter_t f_first, f_last;
    f_first.set_bit(0);
    f_last.set_bit(filter_t::WIDTH - 1);
    tagmatch::add(f_first, 1);
    tagmatch::add(f_last, 2);
    filter_t has_first, has_last, has_none, has_both;
    for (unsigned b : {0u, 10u, 100u, filter_t::WIDTH - 2}) has_first.set_bit(b);
    for (unsigned b : {1u, 10u, 100u, filter_t::WIDTH - 1}) has_last.set_bit(b);
    for (unsigned b : {1u, 10u, 100u, filter_t::WIDTH - 2}) has_none.set_bit(b);
    for (unsigned b : {0u, 10u, 100u, filter_t::WIDTH - 1}) has_both.set_bit(b);
    tagmatch::consolidate();
    tagmatch::start(4, 1);
    deferred_matching_checks C;
    C.run_query(has_none, {});
    C.run_query(has_first, {1});
    C.run_query(has_last, {2});
    C.run_query(has_both, {1, 2});
    tagmatch::stop();
    C.check_results();
    tagmatch::clear();
}

static void single_bit_filters() {
    init_test();
    deferred_matching_checks C;
    set<tagmatch_key_t> all;
    for (unsigned i = 0; i < filter_t::WIDTH; ++i) {
        filter_t f;
        f.set_bit(i);
        tagmatch::add(f, i);
        all.insert(i);
    }
    tagmatch::consolidate();
    tagmatch::start(4, 1);
    C.run_query(ALL_ONES, all);
    tagmatch::stop();
    C.check_results();
    tagmatch::clear();
}

static void deepest_trie() {
    init_test();
    deferred_matching_checks C;
    filter_t f;
    set<tagmatch_key_t> all;
    for (unsigned i = 0; i < filter_t::WIDTH; ++i) {
        f.set_bit(i);
        tagmatch::add(f, i);
        all.insert(i);
    }
    tagmatch::consolidate();
    tagmatch::start(4, 1);
    C.run_query(ALL_ONES, all);
    tagmatch::stop();
    C.check_results();
    tagmatch::clear();
}

// match (not unique) returns every key of every matching filter
static void match_multiset() {
    init_test();
    tagmatch::add(F[1], std::vector<tagmatch_key_t>{7, 8});
    tagmatch::add(F[2], std::vector<tagmatch_key_t>{7});
    tagmatch::consolidate();
    tagmatch::start(2, 1);
    general_matcher m;
    struct counting : synchronous_match_handler {
        std::multiset<tagmatch_key_t> keys;
        void process_results(query *q) override { keys.insert(q->output_keys.begin(), q->output_keys.end()); }
    } h;
    filter_t u = F[1];
    u |= F[2];
    tagmatch_query q(u);
    tagmatch::match(&q, &h);
    tagmatch::stop();
    h.synchronize_and_process();
    CHECK((h.keys == std::multiset<tagmatch_key_t>{7, 7, 8}));
    tagmatch::clear();
}

int main(int argc, char **argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s fixtures.txt database [case]\n", argv[0]);
        return 2;
    }
    std::ifstream in(argv[1]);
    if (!in) {
        std::fprintf(stderr, "cannot read %s\n", argv[1]);
        return 2;
    }
    std::map<int, std::string> fs, qs;
    std::map<int, set<tagmatch_key_t>> es;
    std::string line;
    while (std::getline(in, line)) {
        std::istringstream ls(line);
        std::string tag;
        int idx;
        if (!(ls >> tag >> idx)) continue;
        if (tag == "F" || tag == "Q") {
            std::string s;
            ls >> s;
            (tag == "F" ? fs : qs)[idx] = s;
        } else if (tag == "E") {
            set<tagmatch_key_t> e;
            tagmatch_key_t k;
            while (ls >> k) e.insert(k);
            es[idx] = e;
        }
    }
    for (auto &kv : fs) F.push_back(filter_t(kv.second));
    for (auto &kv : qs) Q.push_back(filter_t(kv.second));
    for (auto &kv : es) EXPECTED.push_back(kv.second);
    if (F.size() != 11 || Q.size() != 13 || EXPECTED.size() != Q.size()) {
        std::fprintf(stderr, "fixture file incomplete\n");
        return 2;
    }
    tagmatch::set_database_filename(argv[2]);

    const std::vector<std::pair<const char *, std::function<void()>>> cases = {
        {"consolidate_empty", consolidate_empty},
        {"start_and_stop", start_and_stop},
        {"consolidate_no_match_action", consolidate_no_match_action},
        {"repeated_stop", repeated_stop},
        {"find_one_filter", find_one_filter},
        {"clear", clear_case},
        {"add_same_filter", add_same_filter},
        {"add_and_find_multi", add_and_find_multi},
        {"add_and_find_multi2", add_and_find_multi2},
        {"add_and_clear", add_and_clear},
        {"add_many_and_find", add_many_and_find},
        {"misc_subsets", misc_subsets},
        {"misc_subsets_Q1", misc_subsets_Q1},
        {"corner_case_filters", corner_case_filters},
        {"single_bit_filters", single_bit_filters},
        {"deepest_trie", deepest_trie},
        {"match_multiset", match_multiset},
    };
    for (auto &c : cases) {
        if (argc > 3 && std::string(argv[3]) != c.first) continue;
        const int before = g_failures;
        c.second();
        std::printf("%-30s %s\n", c.first, g_failures == before ? "ok" : "FAILED");
    }
    std::printf("%d checks, %d failures\n", g_checks, g_failures);
    return g_failures ? 1 : 0;
}
