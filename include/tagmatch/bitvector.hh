// Fixed-width bit vector with the interface of the reference's
// bitvector<Size> (bitvector.hh:98-581), written for this library.
//
// Layout (same as the reference, so binary records are interchangeable):
// bit p lives in 64-bit block p / 64 at bit p % 64; the string "0101..."
// sets bit i for the i-th character; the binary image is the blocks in
// little-endian order (test_io.cc:50-68).  Order (operator<): in the first
// differing block, the lowest differing bit decides and the vector holding a
// 1 there is the greater one (bitvector.hh:389-397).
#ifndef TAGMATCH_BITVECTOR_HH_INCLUDED
#define TAGMATCH_BITVECTOR_HH_INCLUDED

#include <cctype>
#include <cstdint>
#include <cstring>
#include <iostream>
#include <string>

typedef uint64_t block_t;

template <unsigned int Size>
class bitvector {
    static_assert(Size % 64 == 0, "bitvector width must be a multiple of 64");
    static const int N = Size / 64;
    block_t b[N];

    static int low_bit(block_t x) noexcept { return __builtin_ctzll(x); }
    // mask of the low `n` bits of a block (n in [0, 64])
    static block_t low_mask(unsigned n) noexcept { return n >= 64 ? ~block_t(0) : ((block_t(1) << n) - 1); }

public:
    static const unsigned int WIDTH = Size;

    bitvector() noexcept { clear(); }
    bitvector(const std::string &s) noexcept {
        clear();
        const size_t n = s.size() < Size ? s.size() : Size;
        for (size_t i = 0; i < n; ++i)
            if (s[i] == '1') set_bit(unsigned(i));
    }
    bitvector(const block_t *p) noexcept { assign(p); }
    bitvector(const bitvector &o) noexcept { assign(o.b); }

    const block_t *begin() const noexcept { return b; }
    const block_t *end() const noexcept { return b + N; }
    const uint64_t *begin64() const noexcept { return b; }
    const uint64_t *end64() const noexcept { return b + N; }

    uint32_t uint32_value(unsigned i) const noexcept {
        return uint32_t(i & 1 ? b[i / 2] >> 32 : b[i / 2]);
    }
    void copy_into_uint32_array(uint32_t *x) const noexcept {
        for (unsigned i = 0; i < Size / 32; ++i) x[i] = uint32_value(i);
    }
    void assign_uint32_array(const uint32_t *x) noexcept {
        for (int i = 0; i < N; ++i) b[i] = block_t(x[2 * i]) | (block_t(x[2 * i + 1]) << 32);
    }

    void assign(const block_t *p) noexcept { std::memcpy(b, p, sizeof(b)); }
    bitvector &operator=(const bitvector &o) noexcept { assign(o.b); return *this; }
    void clear() noexcept { std::memset(b, 0, sizeof(b)); }
    void fill() noexcept { std::memset(b, 0xFF, sizeof(b)); }
    bool is_empty() const noexcept {
        block_t acc = 0;
        for (int i = 0; i < N; ++i) acc |= b[i];
        return acc == 0;
    }

    void set_bit(unsigned pos) noexcept { b[pos / 64] |= block_t(1) << (pos % 64); }
    bool operator[](unsigned pos) const noexcept { return (b[pos / 64] >> (pos % 64)) & 1; }

    bitvector &operator|=(const bitvector &x) noexcept { for (int i = 0; i < N; ++i) b[i] |= x.b[i]; return *this; }
    bitvector &operator&=(const bitvector &x) noexcept { for (int i = 0; i < N; ++i) b[i] &= x.b[i]; return *this; }
    bitvector &operator^=(const bitvector &x) noexcept { for (int i = 0; i < N; ++i) b[i] ^= x.b[i]; return *this; }
    bool operator==(const bitvector &x) const noexcept { return std::memcmp(b, x.b, sizeof(b)) == 0; }
    bool operator!=(const bitvector &x) const noexcept { return !(*this == x); }

    // this is a subset of p: no bit set here is clear in p
    bool subset_of(const block_t *p) const noexcept {
        block_t acc = 0;
        for (int i = 0; i < N; ++i) acc |= b[i] & ~p[i];
        return acc == 0;
    }
    bool subset_of(const bitvector &x) const noexcept { return subset_of(x.b); }

    // subset test restricted to bit positions [left, right)
    bool range_subset_of(const bitvector &x, unsigned left, unsigned right) const noexcept {
        for (unsigned i = left / 64; i * 64 < right && i < unsigned(N); ++i) {
            const unsigned lo = i * 64;
            block_t m = ~block_t(0);
            if (left > lo) m &= ~low_mask(left - lo);
            if (right < lo + 64) m &= low_mask(right - lo);
            if (b[i] & ~x.b[i] & m) return false;
        }
        return true;
    }
    bool prefix_subset_of(const bitvector &x, unsigned right) const noexcept {
        return right == 0 ? true : range_subset_of(x, 0, right);
    }
    bool suffix_subset_of(const bitvector &x, unsigned left) const noexcept { return range_subset_of(x, left, Size); }
    bool prefix_equal(const bitvector &x, unsigned right) const noexcept {
        for (unsigned i = 0; i * 64 < right; ++i) {
            const block_t m = right >= (i + 1) * 64 ? ~block_t(0) : low_mask(right - i * 64);
            if ((b[i] ^ x.b[i]) & m) return false;
        }
        return true;
    }

    bool operator<(const bitvector &x) const noexcept {
        for (int i = 0; i < N; ++i)
            if (b[i] != x.b[i]) return (x.b[i] >> low_bit(b[i] ^ x.b[i])) & 1;
        return false;
    }
    bool operator>(const bitvector &x) const noexcept { return x < *this; }

    // position of the first differing bit, or WIDTH when equal
    unsigned leftmost_diff(const bitvector &x) const noexcept {
        for (int i = 0; i < N; ++i)
            if (b[i] != x.b[i]) return unsigned(i * 64 + low_bit(b[i] ^ x.b[i]));
        return Size;
    }
    static unsigned leftmost_diff(const bitvector &x, const bitvector &y) noexcept { return x.leftmost_diff(y); }

    // first set bit at or after pos, or WIDTH
    unsigned next_bit(unsigned pos) const noexcept {
        for (unsigned i = pos / 64; i < unsigned(N); ++i) {
            block_t v = b[i];
            if (i == pos / 64) v &= ~low_mask(pos % 64);
            if (v) return i * 64 + unsigned(low_bit(v));
        }
        return Size;
    }

    unsigned popcount() const noexcept {
        unsigned c = 0;
        for (int i = 0; i < N; ++i) c += unsigned(__builtin_popcountll(b[i]));
        return c;
    }
    unsigned prefix_popcount(unsigned right) const noexcept {
        unsigned c = 0;
        for (unsigned i = 0; i * 64 < right; ++i)
            c += unsigned(__builtin_popcountll(b[i] & (right >= (i + 1) * 64 ? ~block_t(0) : low_mask(right - i * 64))));
        return c;
    }
    unsigned suffix_popcount(unsigned left) const noexcept { return left >= Size ? 0 : popcount() - prefix_popcount(left); }

    std::ostream &write_binary(std::ostream &out) const {
        unsigned char buf[sizeof(b)];
        for (int i = 0; i < N; ++i)
            for (int k = 0; k < 8; ++k) buf[i * 8 + k] = (unsigned char)(b[i] >> (8 * k));
        return out.write(reinterpret_cast<const char *>(buf), sizeof(buf));
    }
    std::istream &read_binary(std::istream &in) {
        unsigned char buf[sizeof(b)];
        if (in.read(reinterpret_cast<char *>(buf), sizeof(buf))) {
            for (int i = 0; i < N; ++i) {
                b[i] = 0;
                for (int k = 0; k < 8; ++k) b[i] |= block_t(buf[i * 8 + k]) << (8 * k);
            }
        }
        return in;
    }
    std::ostream &write_ascii(std::ostream &out) const {
        for (unsigned p = 0; p < Size; ++p) out << ((*this)[p] ? '1' : '0');
        return out;
    }
    std::ostream &write_ascii(std::ostream &out, uint8_t prefix_len) const {
        for (unsigned p = 0; p < Size && p < prefix_len; ++p) out << ((*this)[p] ? '1' : '0');
        return out;
    }
    // reads up to WIDTH '0'/'1' characters after leading blanks; stops at
    // the first other character, leaving the remaining bits clear
    std::istream &read_ascii(std::istream &in) {
        while (std::isspace(in.peek())) in.get();
        clear();
        for (unsigned p = 0; p < Size; ++p) {
            const int c = in.peek();
            if (c != '0' && c != '1') { if (c != EOF) in.get(); break; }
            in.get();
            if (c == '1') set_bit(p);
        }
        return in;
    }
};

#endif
