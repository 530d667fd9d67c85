// basic_query / query (query.hh of the reference): a query filter plus its
// output keys.
#ifndef TAGMATCH_QUERY_HH_INCLUDED
#define TAGMATCH_QUERY_HH_INCLUDED
#include <iostream>
#include <sstream>
#include <string>
#include <vector>
#include "filter.hh"
#include "key.hh"

class basic_query {
public:
    filter_t filter;
    bool match_unique;

    basic_query() : filter(), match_unique(false) {}
    basic_query(const filter_t &f) : filter(f), match_unique(false) {}
    basic_query(const std::string &f) : filter(f), match_unique(false) {}
    basic_query(const basic_query &q) : filter(q.filter), match_unique(q.match_unique) {}

    // binary record: the 24-byte filter (query.cc:11-19)
    std::ostream &write_binary(std::ostream &out) const { return filter.write_binary(out); }
    std::istream &read_binary(std::istream &in) { return filter.read_binary(in); }
    // ASCII record: "! <filter>" (query.cc:21-40)
    std::ostream &write_ascii(std::ostream &out) const {
        out << "! ";
        filter.write_ascii(out);
        return out << '\n';
    }
    std::istream &read_ascii(std::istream &in) {
        std::string line;
        if (std::getline(in, line)) {
            std::istringstream ls(line);
            std::string cmd;
            ls >> cmd;
            if (cmd == "!") filter.read_ascii(ls);
        }
        return in;
    }
};

class query : public basic_query {
public:
    std::vector<tagmatch_key_t> output_keys;

    query() : basic_query() {}
    query(const filter_t &f) : basic_query(f) {}
    query(const std::string &f) : basic_query(f) {}
    query(const query &q) : basic_query(q), output_keys(q.output_keys) {}
    query(query &&q) : basic_query(q), output_keys(std::move(q.output_keys)) {}
};
#endif
