// tagmatch_key_t (key.hh:6 of the reference).
#ifndef TAGMATCH_KEY_HH_INCLUDED
#define TAGMATCH_KEY_HH_INCLUDED
#include <cstdint>
typedef uint32_t tagmatch_key_t;
#endif
