// Warp row-block layout of a CSR orientation (host only).
//
// A descriptor list blk[0..nblk] holds (first row, first nonzero) of every
// warp row block plus an end entry (rows, nnz).  A block either packs at
// most kRowsPerWarpBlock consecutive rows whose nonzeros total at most
// `cap` (<= kWarpCapMax), or holds one row of any length.  The iteration
// kernels stage a packed block's products in a kWarpCapMax-entry shared
// slice per warp, so these invariants are what keeps them in bounds:
// check_row_blocks verifies them before any list is uploaded.
#pragma once

#include <vector_types.h>

#include <algorithm>
#include <stdexcept>
#include <vector>

namespace nir {

#ifndef NIR_WARP_U
#define NIR_WARP_U 8
#endif
constexpr int kWarpU = NIR_WARP_U;           // nonzeros per lane per round
constexpr int kWarpCapMax = 32 * kWarpU;     // largest warp row block (256 for 8 per lane)
constexpr int kRowsPerWarpBlock = 32;        // rows in one warp row block

// Greedy packing of consecutive rows; rp[0] may be any offset.
inline std::vector<int2> build_row_blocks(const std::vector<int>& rp, int cap) {
    const int rows = int(rp.size()) - 1;
    std::vector<int2> blk;
    if (rows <= 0) {
        const int p = rp.empty() ? 0 : rp[0];
        blk.push_back(int2{0, p});
        blk.push_back(int2{0, p});
        return blk;
    }
    blk.push_back(int2{0, rp[0]});
    int s = 0;
    while (s < rows) {
        int r = s + 1;
        if (rp[s + 1] - rp[s] <= cap) {
            while (r < rows && rp[r + 1] - rp[s] <= cap && r - s < kRowsPerWarpBlock) ++r;
        }
        blk.push_back(int2{r, rp[r]});
        s = r;
    }
    return blk;
}

inline void check_row_blocks(const std::vector<int2>& b, const std::vector<int>& rp, int cap) {
    const int rows = int(rp.size()) - 1;
    if (cap < 1 || cap > kWarpCapMax) throw std::runtime_error("internal: row block capacity out of range");
    if (b.size() < 2 || b.front().x != 0 || b.back().x != std::max(rows, 0))
        throw std::runtime_error("internal: row blocks do not cover the rows");
    for (size_t k = 0; k + 1 < b.size(); ++k) {
        const int r0 = b[k].x, r1 = b[k + 1].x, p0 = b[k].y, p1 = b[k + 1].y;
        if (rows <= 0) {
            if (r0 != 0 || r1 != 0 || p0 != p1) throw std::runtime_error("internal: malformed empty row block");
            continue;
        }
        if (!(r0 < r1 && r1 <= rows) || p0 != rp[r0] || p1 != rp[r1])
            throw std::runtime_error("internal: malformed row block descriptor");
        if (!(r1 - r0 == 1 || (p1 - p0 <= cap && r1 - r0 <= kRowsPerWarpBlock)))
            throw std::runtime_error("internal: row block exceeds its capacity");
    }
}

// ---------------------------------------------------------------- CTA blocks

constexpr int kCtaRowsMax = 256;  // rows of one packed CTA block: one epilogue thread each

// CTA blocks (k_cta.cuh): consecutive rows packed while their nonzeros
// total at most cap and they are at most kCtaRowsMax; a row with more than
// cap nonzeros gets a block of its own.  Descriptor b is (first row, first
// nonzero in the CSR, first entry in the padded stream, 0); the end entry
// is (rows, nnz, padded length, 0).  Block b's nonzeros occupy padded
// positions [q0, q0 + p1 - p0), q0 a multiple of 4, and zeros fill the
// gap up to the next block, so every 16-byte load of a block's run of
// indices or values is aligned and never reads another block's entries.
// rp[0] may be any offset; row numbers are relative to rp.
inline std::vector<int4> build_cta_blocks(const std::vector<int>& rp, int cap, long long q_base = 0) {
    const int rows = int(rp.size()) - 1;
    std::vector<int4> blk;
    long long q = q_base;
    auto pad4 = [](long long v) { return (v + 3) & ~3LL; };
    auto push = [&](int r, int p) {
        if (q > (1LL << 31) - 64) throw std::runtime_error("padded matrix stream exceeds 2^31 entries");
        blk.push_back(int4{r, p, int(q), 0});
    };
    if (rows <= 0) {
        const int p = rp.empty() ? 0 : rp[0];
        push(0, p);
        push(0, p);
        return blk;
    }
    int s = 0;
    while (s < rows) {
        push(s, rp[s]);
        int r = s + 1;
        if (rp[s + 1] - rp[s] <= cap) {
            while (r < rows && rp[r + 1] - rp[s] <= cap && r - s < kCtaRowsMax) ++r;
        }
        q = pad4(q + (rp[r] - rp[s]));
        s = r;
    }
    push(rows, rp[rows]);
    return blk;
}

// The invariants k_cta.cuh relies on to stay in bounds: rows covered in
// order, p = rp of each first row, q multiples of 4 with room for each
// block's nonzeros, packed blocks within cap and kCtaRowsMax rows.
inline void check_cta_blocks(const std::vector<int4>& b, const std::vector<int>& rp, int cap) {
    const int rows = int(rp.size()) - 1;
    if (cap < 1) throw std::runtime_error("internal: CTA block capacity out of range");
    if (b.size() < 2 || b.front().x != 0 || b.back().x != std::max(rows, 0))
        throw std::runtime_error("internal: CTA blocks do not cover the rows");
    for (size_t k = 0; k + 1 < b.size(); ++k) {
        const int r0 = b[k].x, r1 = b[k + 1].x, p0 = b[k].y, p1 = b[k + 1].y, q0 = b[k].z, q1 = b[k + 1].z;
        if ((q0 & 3) || (q1 & 3) || q1 - q0 < p1 - p0 || q0 < 0)
            throw std::runtime_error("internal: malformed padded stream offsets");
        if (rows <= 0) {
            if (r0 != 0 || r1 != 0 || p0 != p1) throw std::runtime_error("internal: malformed empty CTA block");
            continue;
        }
        if (!(r0 < r1 && r1 <= rows) || p0 != rp[r0] || p1 != rp[r1])
            throw std::runtime_error("internal: malformed CTA block descriptor");
        if (!(r1 - r0 == 1 || (p1 - p0 <= cap && r1 - r0 <= kCtaRowsMax)))
            throw std::runtime_error("internal: CTA block exceeds its capacity");
    }
}

// CTA blocks of a block-diagonal batch: instance i owns rows
// [off[i], off[i+1]) of rp, and no block crosses an instance.  The 4th
// component of each descriptor is the block's instance; lo[i] is instance
// i's first block (lo[count] = number of blocks).  The padded stream of the
// instances follows their order.
inline std::vector<int4> build_batch_cta_blocks(const std::vector<int>& rp, const std::vector<int>& off, int cap,
                                                std::vector<int>* lo) {
    const int count = int(off.size()) - 1;
    std::vector<int4> all;
    lo->clear();
    long long q = 0;
    for (int i = 0; i < count; ++i) {
        lo->push_back(int(all.size()));
        if (off[i + 1] == off[i]) continue;  // no rows of this orientation
        std::vector<int> seg(rp.begin() + off[i], rp.begin() + off[i + 1] + 1);
        const std::vector<int4> b = build_cta_blocks(seg, cap, q);  // rows relative to the instance
        for (size_t k = 0; k + 1 < b.size(); ++k) all.push_back(int4{b[k].x + off[i], b[k].y, b[k].z, i});
        q = b.back().z;
    }
    lo->push_back(int(all.size()));
    const int rows = int(rp.size()) - 1;
    if (all.empty()) all.push_back(int4{0, rp.empty() ? 0 : rp[0], 0, 0});  // one empty block, as for a single LP
    all.push_back(int4{std::max(rows, 0), rows >= 0 ? rp[rows] : 0, int(q), 0});
    check_cta_blocks(all, rp, cap);
    return all;
}

// Row blocks of a block-diagonal batch: instance i owns rows
// [off[i], off[i+1]) of rp, and no block crosses an instance.  Also returns
// the instance of every block (owner) and each instance's first block
// (lo[i], with lo[count] = number of blocks).
inline std::vector<int2> build_batch_row_blocks(const std::vector<int>& rp, const std::vector<int>& off, int cap,
                                                std::vector<int>* owner, std::vector<int>* lo) {
    const int count = int(off.size()) - 1;
    std::vector<int2> all;
    owner->clear();
    lo->clear();
    for (int i = 0; i < count; ++i) {
        lo->push_back(int(all.size()));
        if (off[i + 1] == off[i]) continue;  // no rows of this orientation
        std::vector<int> seg(rp.begin() + off[i], rp.begin() + off[i + 1] + 1);
        const std::vector<int2> b = build_row_blocks(seg, cap);  // rows relative to the instance
        for (size_t k = 0; k + 1 < b.size(); ++k) {
            all.push_back(int2{b[k].x + off[i], b[k].y});
            owner->push_back(i);
        }
    }
    lo->push_back(int(all.size()));
    const int rows = int(rp.size()) - 1;
    if (all.empty()) all.push_back(int2{0, rp.empty() ? 0 : rp[0]});  // one empty block, as for a single LP
    all.push_back(int2{std::max(rows, 0), rows >= 0 ? rp[rows] : 0});
    check_row_blocks(all, rp, cap);
    return all;
}

}  // namespace nir
