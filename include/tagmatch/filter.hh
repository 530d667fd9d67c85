// filter_t (filter.hh:7 of the reference): a 192-bit Bloom filter.
#ifndef TAGMATCH_FILTER_HH_INCLUDED
#define TAGMATCH_FILTER_HH_INCLUDED
#include <cstdint>
#include "bitvector.hh"
typedef bitvector<192> filter_t;
typedef uint8_t filter_pos_t;
#endif
