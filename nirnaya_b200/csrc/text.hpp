// Text scanning shared by the MPS and SOL readers: white space as the C
// locale's isspace (what istream's >> splits on), 16-byte SSE2 token
// scanning, name hashing and an open-addressing name table, and a simple
// fork/join over threads.
#pragma once

#include <emmintrin.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <memory>
#include <thread>
#include <utility>
#include <vector>

namespace nir {
namespace text {

// An allocator whose resize leaves new elements uninitialised (default-
// initialised), for large buffers that are about to be written anyway: the
// pages are then first touched by the threads that fill them.
template <class T>
struct NoInit : std::allocator<T> {
    template <class U>
    struct rebind {
        using other = NoInit<U>;
    };
    NoInit() = default;
    template <class U>
    NoInit(const NoInit<U>&) noexcept {}
    template <class U>
    void construct(U* p) noexcept {
        ::new (static_cast<void*>(p)) U;
    }
    template <class U, class... A>
    void construct(U* p, A&&... a) {
        ::new (static_cast<void*>(p)) U(std::forward<A>(a)...);
    }
};
template <class T>
using uvector = std::vector<T, NoInit<T>>;

// isspace in the C locale, which is what istream's >> splits on
inline bool is_space(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r'; }

struct Tok {
    const char* p;
    uint32_t n;
};

// Bit i set when p[i] is white space (' ' or 0x09-0x0D), 16 bytes at once.
// Reads p[0..15]: the file buffer is padded so that this stays inside it.
inline uint32_t space_mask16(const char* p) {
    const __m128i v = _mm_loadu_si128(reinterpret_cast<const __m128i*>(p));
    const __m128i sp = _mm_cmpeq_epi8(v, _mm_set1_epi8(' '));
    const __m128i t = _mm_sub_epi8(v, _mm_set1_epi8(0x09));
    const __m128i ctl = _mm_cmpeq_epi8(_mm_min_epu8(t, _mm_set1_epi8(4)), t);  // 0x09 <= c <= 0x0D
    return uint32_t(_mm_movemask_epi8(_mm_or_si128(sp, ctl)));
}

// The tokens of [b, e), split on white space as istream >> splits them.
inline void tokenize(const char* b, const char* e, std::vector<Tok>& out) {
    out.clear();
    const char* tok = nullptr;  // start of a token still open
    for (const char* p = b; p < e; p += 16) {
        uint32_t sp = space_mask16(p);
        const size_t lim = size_t(e - p);
        if (lim < 16) sp |= (0xFFFFu << lim) & 0xFFFFu;  // bytes past the end count as space
        uint32_t pos = 0;
        for (;;) {
            if (!tok) {
                const uint32_t ns = ~sp & (0xFFFFu << pos) & 0xFFFFu;
                if (!ns) break;
                pos = uint32_t(__builtin_ctz(ns));
                tok = p + pos;
            }
            const uint32_t s = sp & (0xFFFFu << pos);
            if (!s) break;  // the token goes on in the next block
            pos = uint32_t(__builtin_ctz(s));
            out.push_back({tok, uint32_t(p + pos - tok)});
            tok = nullptr;
        }
    }
    if (tok) out.push_back({tok, uint32_t(e - tok)});
}

// 64-bit hash of a name: 8-byte words folded by multiply-xorshift, then the
// murmur3 finaliser so that every input bit reaches the low (index) bits.
inline uint64_t hash_name(const char* p, size_t n) {
    uint64_t h = 0x9E3779B97F4A7C15ULL ^ (uint64_t(n) * 0xC2B2AE3D27D4EB4FULL);
    size_t i = 0;
    for (; i + 8 <= n; i += 8) {
        uint64_t w;
        std::memcpy(&w, p + i, 8);
        h = (h ^ w) * 0x9FB21C651E98DF25ULL;
        h ^= h >> 32;
    }
    uint64_t w = 0;
    std::memcpy(&w, p + i, n - i);
    h ^= w;
    h ^= h >> 33;
    h *= 0xFF51AFD7ED558CCDULL;
    h ^= h >> 33;
    h *= 0xC4CEB9FE1A85EC53ULL;
    h ^= h >> 33;
    return h;
}

// Open-addressing table of names -> index.  Names of up to 16 bytes are
// kept in the slot, so most probes touch one cache line; longer names are
// compared through a pointer into the file buffer.
struct NameMap {
    struct Slot {
        uint32_t tag = 0;
        uint32_t n = 0;
        int32_t v = -1;
        uint32_t pad = 0;
        char key[16];
        const char* p = nullptr;
    };
    std::vector<Slot> slots;
    size_t count = 0;

    NameMap() { slots.resize(1024); }

    static bool same(const Slot& s, uint32_t tag, const char* p, size_t n) {
        if (s.tag != tag || s.n != n) return false;
        return n <= 16 ? std::memcmp(s.key, p, n) == 0 : std::memcmp(s.p, p, n) == 0;
    }
    const Slot* slot_for(uint64_t h) const { return &slots[h & (slots.size() - 1)]; }
    int32_t find_h(uint64_t h, const char* p, size_t n) const {
        const size_t mask = slots.size() - 1;
        const uint32_t tag = uint32_t(h >> 32);
        for (size_t i = h & mask;; i = (i + 1) & mask) {
            const Slot& s = slots[i];
            if (s.v < 0) return -1;
            if (same(s, tag, p, n)) return s.v;
        }
    }
    int32_t find(const char* p, size_t n) const { return find_h(hash_name(p, n), p, n); }
    // returns the existing value, or inserts v and returns -1
    int32_t insert(const char* p, size_t n, int32_t v) { return insert_h(hash_name(p, n), p, p, n, v); }
    // inserts, or sets the value of a name already there
    void assign(const char* p, size_t n, int32_t v) {
        if (2 * (count + 1) > slots.size()) grow();
        const uint64_t h = hash_name(p, n);
        const size_t mask = slots.size() - 1;
        const uint32_t tag = uint32_t(h >> 32);
        for (size_t i = h & mask;; i = (i + 1) & mask) {
            Slot& s = slots[i];
            if (s.v < 0) {
                s.tag = tag;
                s.n = uint32_t(n);
                s.v = v;
                s.p = p;
                std::memcpy(s.key, p, std::min<size_t>(n, 16));
                ++count;
                return;
            }
            if (same(s, tag, p, n)) {
                s.v = v;
                return;
            }
        }
    }
    // with the hash given; `cmp` holds the name's bytes (a copy of the first
    // 16 when n <= 16 is enough), `p` is what the slot keeps
    int32_t insert_h(uint64_t h, const char* cmp, const char* p, size_t n, int32_t v) {
        if (2 * (count + 1) > slots.size()) grow();
        const size_t mask = slots.size() - 1;
        const uint32_t tag = uint32_t(h >> 32);
        for (size_t i = h & mask;; i = (i + 1) & mask) {
            Slot& s = slots[i];
            if (s.v < 0) {
                s.tag = tag;
                s.n = uint32_t(n);
                s.v = v;
                s.p = p;
                std::memcpy(s.key, cmp, std::min<size_t>(n, 16));
                ++count;
                return -1;
            }
            if (same(s, tag, cmp, n)) return s.v;
        }
    }
    // room for n names without growing
    void reserve(size_t n) {
        size_t want = slots.size();
        while (want < 2 * n + 2) want *= 2;
        if (want > slots.size()) rehash(want);
    }
    void grow() { rehash(slots.size() * 2); }
    void rehash(size_t size) {
        std::vector<Slot> old(size);
        old.swap(slots);
        const size_t mask = slots.size() - 1;
        for (const Slot& s : old) {
            if (s.v < 0) continue;
            size_t i = hash_name(s.n <= 16 ? s.key : s.p, s.n) & mask;
            while (slots[i].v >= 0) i = (i + 1) & mask;
            slots[i] = s;
        }
    }
};

template <class F>
void run_threads(int nt, F&& f) {
    if (nt <= 1) {
        f(0);
        return;
    }
    std::vector<std::thread> th;
    th.reserve(size_t(nt - 1));
    for (int k = 1; k < nt; ++k) th.emplace_back([&f, k] { f(k); });
    f(0);
    for (auto& x : th) x.join();
}

}  // namespace text
}  // namespace nir
