// Exact decimal -> double conversion for MPS number tokens.
//
// parse_decimal(p, n, &out) returns true and sets `out` to the correctly
// rounded (to nearest, ties to even) double of the token when the token is
// a plain decimal -- [+-] digits [. digits] [(e|E|d|D) [+-] digits] -- with
// at most 19 significant digits whose value is a normal double well inside
// the exponent range.  In every other case, and in every case where the
// fast computation cannot prove its rounding, it returns false and the
// caller converts with strtod; so the result is always strtod's.
//
// Method: the multiply-by-a-truncated-128-bit-power-of-five scheme of
// Eisel and Lemire (D. Lemire, "Number Parsing at a Gigabyte per Second",
// Software: Practice and Experience 51(8), 2021), with a simpler
// acceptance test than the paper's:
//   w  = the decimal significand (< 10^19), normalised so bit 63 is set;
//   T  = floor(5^q * 2^s), the 128-bit scaled power of five, exact bignum
//        arithmetic at first use (so |T - 5^q 2^s| < 1);
//   R  = floor(w*T / 2^64), computed exactly from two 64x64 products.
// The true w * 5^q * 2^s / 2^64 lies in (R - 1, R + 2).  With M the top 54
// bits of R (mantissa and round bit) and r the bits below them (F values),
// rounding is decided unless the truth can sit on a halfway point:
// M odd with r <= 1, or M even with r >= F - 2.  Those cases (which include
// every exact tie) go to strtod.
#pragma once

#include <cstdint>
#include <cstring>
#include <mutex>
#include <vector>

namespace nir {
namespace decimal {

constexpr int kQMin = -342;
constexpr int kQMax = 308;

struct Pow5 {
    uint64_t hi, lo;  // T = hi * 2^64 + lo, bit 127 set
    int32_t s;        // T = floor(5^q * 2^s)
};

// Little-endian base-2^64 unsigned bignum, just enough for the table.
struct Big {
    std::vector<uint64_t> d;
    int bits() const {
        for (int i = int(d.size()) - 1; i >= 0; --i)
            if (d[i]) return i * 64 + 64 - __builtin_clzll(d[i]);
        return 0;
    }
    bool bit(int k) const {
        const size_t w = size_t(k) / 64;
        return w < d.size() && ((d[w] >> (k % 64)) & 1);
    }
    void mul_small(uint64_t m) {
        unsigned __int128 c = 0;
        for (auto& x : d) {
            c += (unsigned __int128)x * m;
            x = uint64_t(c);
            c >>= 64;
        }
        if (c) d.push_back(uint64_t(c));
    }
    void shl1() {
        uint64_t c = 0;
        for (auto& x : d) {
            const uint64_t nc = x >> 63;
            x = (x << 1) | c;
            c = nc;
        }
        if (c) d.push_back(c);
    }
    bool ge(const Big& o) const {
        const size_t n = std::max(d.size(), o.d.size());
        for (size_t i = n; i-- > 0;) {
            const uint64_t a = i < d.size() ? d[i] : 0, b = i < o.d.size() ? o.d[i] : 0;
            if (a != b) return a > b;
        }
        return true;
    }
    void sub(const Big& o) {  // requires *this >= o
        uint64_t br = 0;
        for (size_t i = 0; i < d.size(); ++i) {
            const uint64_t b = i < o.d.size() ? o.d[i] : 0;
            const unsigned __int128 t = (unsigned __int128)d[i] - b - br;
            d[i] = uint64_t(t);
            br = (t >> 64) ? 1 : 0;
        }
    }
};

inline const Pow5* table() {
    static std::vector<Pow5> tab;
    static std::once_flag once;
    std::call_once(once, [] {
        tab.resize(size_t(kQMax - kQMin + 1));
        // q >= 0: the top 128 bits of 5^q
        Big p{{1}};
        for (int q = 0; q <= kQMax; ++q) {
            if (q) p.mul_small(5);
            const int L = p.bits();
            unsigned __int128 t = 0;
            for (int k = 0; k < 128; ++k) {
                const int src = L - 1 - k;
                t = (t << 1) | (src >= 0 && p.bit(src) ? 1u : 0u);
            }
            tab[size_t(q - kQMin)] = {uint64_t(t >> 64), uint64_t(t), 128 - L};
        }
        // q < 0: floor(2^k / 5^|q|) with k = bits(5^|q|) + 127, by binary
        // long division (the quotient has 128 bits)
        Big d{{1}};
        for (int a = 1; a <= -kQMin; ++a) {
            d.mul_small(5);
            const int L = d.bits();
            const int k = L + 127;
            Big rem{{0}};
            unsigned __int128 quo = 0;
            for (int i = k; i >= 0; --i) {
                rem.shl1();
                if (i == k) rem.d[0] |= 1;
                const bool take = rem.ge(d);
                if (take) rem.sub(d);
                if (i < 128) quo = (quo << 1) | (take ? 1u : 0u);
                else if (take) quo = ~(unsigned __int128)0;  // not reached: the quotient is < 2^128
            }
            tab[size_t(-a - kQMin)] = {uint64_t(quo >> 64), uint64_t(quo), k};
        }
    });
    return tab.data();
}

// Eight ASCII bytes (little-endian in v) that are all digits?
inline bool eight_digits(uint64_t v) {
    return ((v & 0xF0F0F0F0F0F0F0F0ULL) | (((v + 0x0606060606060606ULL) & 0xF0F0F0F0F0F0F0F0ULL) >> 4)) ==
           0x3333333333333333ULL;
}
// Their value, first byte most significant: pairwise combination of
// neighbouring digits, then pairs, then quads (multiply-shift per lane).
inline uint64_t eight_value(uint64_t v) {
    v -= 0x3030303030303030ULL;
    v = (v * 10 + (v >> 8)) & 0x00FF00FF00FF00FFULL;
    v = (v * 100 + (v >> 16)) & 0x0000FFFF0000FFFFULL;
    return (v * 10000 + (v >> 32)) & 0xFFFFFFFFULL;
}

// Accumulates the digits at p into w (digits counted in `digits`); returns
// the end of the digit run, or nullptr when a 20th significant digit shows.
inline const char* take_digits(const char* p, const char* e, uint64_t& w, int& digits) {
    while (digits <= 11 && e - p >= 8) {
        uint64_t v;
        std::memcpy(&v, p, 8);
        if (!eight_digits(v)) break;
        w = w * 100000000ULL + eight_value(v);
        digits += 8;
        p += 8;
    }
    while (p < e && *p >= '0' && *p <= '9') {
        if (digits == 19) return nullptr;
        w = w * 10 + uint64_t(*p - '0');
        ++digits;
        ++p;
    }
    return p;
}

// Fast path only; false means "use strtod".
inline bool parse_decimal(const char* p, size_t n, double& out) {
    const char* e = p + n;
    bool neg = false;
    if (p < e && (*p == '+' || *p == '-')) {
        neg = *p == '-';
        ++p;
    }
    uint64_t w = 0;
    int digits = 0;   // significant digits taken into w
    int64_t q = 0;    // decimal exponent of w
    bool any = false;
    // integer part: leading zeros are not significant
    while (p < e && *p == '0') {
        any = true;
        ++p;
    }
    {
        const char* s = p;
        p = take_digits(p, e, w, digits);
        if (!p) return false;
        any |= p != s;
    }
    if (p < e && *p == '.') {
        ++p;
        const char* s = p;
        if (w == 0)
            while (p < e && *p == '0') ++p;  // zeros right after the point scale only
        const char* d = p;
        p = take_digits(p, e, w, digits);
        if (!p) return false;
        q -= int64_t(p - s);
        any |= p != s;
        (void)d;
    }
    if (!any) return false;
    if (p < e && (*p == 'e' || *p == 'E' || *p == 'd' || *p == 'D')) {
        ++p;
        bool eneg = false;
        if (p < e && (*p == '+' || *p == '-')) {
            eneg = *p == '-';
            ++p;
        }
        if (p == e || *p < '0' || *p > '9') return false;
        int64_t x = 0;
        while (p < e && *p >= '0' && *p <= '9') {
            if (x > 100000) return false;
            x = x * 10 + (*p - '0');
            ++p;
        }
        q += eneg ? -x : x;
    }
    if (p != e) return false;
    if (w == 0) {
        out = neg ? -0.0 : 0.0;
        return true;
    }
    if (q < kQMin || q > kQMax) return false;
    const Pow5& T = table()[q - kQMin];
    const int l = __builtin_clzll(w);
    const uint64_t wn = w << l;
    // R = floor(wn * T / 2^64) = wn*hi + high64(wn*lo)
    const unsigned __int128 a = (unsigned __int128)wn * T.hi;
    const unsigned __int128 b = (unsigned __int128)wn * T.lo;
    const unsigned __int128 R = a + (b >> 64);
    const uint64_t Rh = uint64_t(R >> 64), Rl = uint64_t(R);
    const int h = Rh >> 63 ? 127 : 126;  // leading bit of R (R >= 2^126)
    // M = top 54 bits, r = the h - 53 bits below them
    const int rb = h - 53;  // 73 or 74
    const uint64_t M = uint64_t(R >> rb);
    const unsigned __int128 r = R & ((((unsigned __int128)1) << rb) - 1);
    const unsigned __int128 F = ((unsigned __int128)1) << rb;
    if ((M & 1) ? (r <= 1) : (r >= F - 2)) return false;
    (void)Rl;
    uint64_t m = (M >> 1) + (M & 1);  // round half up is exact here: no ties reach this point
    // v = R * 2^(64 + q - l - s); R's leading bit h, mantissa exponent:
    int64_t E = int64_t(h) - 52 + 64 + q - l - T.s;
    if (m == (uint64_t(1) << 53)) {
        m >>= 1;
        ++E;
    }
    const int64_t eb = E + 52 + 1023;
    if (eb <= 1 || eb >= 2046) return false;  // near subnormal or overflow: strtod decides
    const uint64_t bits = (uint64_t(neg) << 63) | (uint64_t(eb) << 52) | (m & ((uint64_t(1) << 52) - 1));
    std::memcpy(&out, &bits, 8);
    return true;
}

}  // namespace decimal
}  // namespace nir
