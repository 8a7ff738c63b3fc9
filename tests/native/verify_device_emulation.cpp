// Host emulation of the device solution check (nirnaya_b200/csrc/k_verify.cuh),
// for tests/test_zz_verify_device.py.
//
// Compiled with g++ (-ffp-contract=off) from the same header the kernels
// use, so the per-element arithmetic is the kernels' own.  What the kernels
// add around it is restated here step for step:
//   - the batch's layout (engine_batch.cuh: block-diagonal CSC, bounds
//     sanitised to +-inf, a stable sort of the entries by row);
//   - each kernel's partition of columns and rows over threads;
//   - the warp shuffle-down trees of block_best / block_min, with a lane
//     whose source is out of range keeping its own value.
// The test compares its reports with nir_verify_solution's, bit for bit.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#include "k_verify.cuh"
#include "nir_lp.h"

using nir::vfy::Rec;

namespace {

constexpr int kBlock = 256;  // kVfyBlock

Rec warp_best(const Rec* in) {  // lane 0's value after the shuffle-down tree
    Rec r[32];
    for (int l = 0; l < 32; ++l) r[l] = in[l];
    for (int o = 16; o > 0; o >>= 1) {
        Rec old[32];
        for (int l = 0; l < 32; ++l) old[l] = r[l];
        for (int l = 0; l < 32; ++l) r[l] = nir::vfy::best(old[l], l + o < 32 ? old[l + o] : old[l]);
    }
    return r[0];
}

Rec block_best(const std::vector<Rec>& t) {  // t: kBlock thread values
    Rec part[kBlock / 32];
    for (int w = 0; w < kBlock / 32; ++w) part[w] = warp_best(&t[size_t(w) * 32]);
    Rec lane[32];
    for (int l = 0; l < 32; ++l) lane[l] = l < kBlock / 32 ? part[l] : nir::vfy::rec0();
    return warp_best(lane);
}

long long block_min(const std::vector<long long>& t) {
    auto warp_min = [](long long* r) {
        for (int o = 16; o > 0; o >>= 1) {
            long long old[32];
            std::memcpy(old, r, sizeof(old));
            for (int l = 0; l < 32; ++l) r[l] = std::min(old[l], l + o < 32 ? old[l + o] : old[l]);
        }
        return r[0];
    };
    long long part[kBlock / 32], warp0[32];
    for (int w = 0; w < kBlock / 32; ++w) {
        long long r[32];
        for (int l = 0; l < 32; ++l) r[l] = t[size_t(w) * 32 + size_t(l)];
        part[w] = warp_min(r);
        if (w == 0) std::memcpy(warp0, r, sizeof(r));  // warp 0's lanes after its own tree
    }
    long long r[32];
    for (int l = 0; l < 32; ++l) r[l] = l < kBlock / 32 ? part[l] : warp0[l];
    return warp_min(r);
}

double sanitize(double b, bool lower) {
    const bool f = std::isfinite(b) && std::fabs(b) < 1e20;
    return f ? b : (lower ? -INFINITY : INFINITY);
}

}  // namespace

extern "C" int emu_batch_verify(const nir_lp_view* lps, int count, const double* x, const int8_t* vartype,
                                const double* claimed, double tol, nir_verify_report* out) {
    // the batch's layout
    std::vector<int> row_off(1, 0), col_off(1, 0);
    std::vector<double> offsets;
    for (int k = 0; k < count; ++k) {
        row_off.push_back(row_off.back() + lps[k].nrow);
        col_off.push_back(col_off.back() + lps[k].ncol);
        offsets.push_back(lps[k].obj_offset);
    }
    const long long m = row_off.back(), n = col_off.back();
    std::vector<double> c(static_cast<size_t>(n)), lo(static_cast<size_t>(n)), up(static_cast<size_t>(n)), rl(static_cast<size_t>(m)), ru(static_cast<size_t>(m));
    std::vector<int> row_inst(static_cast<size_t>(m));
    // (row, column, value) in CSC order, then a stable sort by row
    std::vector<int> cnt(size_t(m) + 1, 0);
    struct E {
        int row, col;
        double v;
    };
    std::vector<E> csc;
    for (int k = 0; k < count; ++k) {
        const nir_lp_view& v = lps[k];
        for (int j = 0; j < v.ncol; ++j) {
            const int g = col_off[size_t(k)] + j;
            c[size_t(g)] = v.cost[j];
            lo[size_t(g)] = sanitize(v.collo[j], true);
            up[size_t(g)] = sanitize(v.colup[j], false);
            for (int64_t q = v.col_start[j]; q < v.col_start[j + 1]; ++q)
                csc.push_back({v.row_index[q] + row_off[size_t(k)], g, v.value[q]});
        }
        for (int i = 0; i < v.nrow; ++i) {
            const int r = row_off[size_t(k)] + i;
            rl[size_t(r)] = sanitize(v.rowlo[i], true);
            ru[size_t(r)] = sanitize(v.rowup[i], false);
            row_inst[size_t(r)] = k;
        }
    }
    for (const E& e : csc) ++cnt[size_t(e.row) + 1];
    std::vector<int> rp(size_t(m) + 1, 0);
    for (long long i = 0; i < m; ++i) rp[size_t(i) + 1] = rp[size_t(i)] + cnt[size_t(i) + 1];
    std::vector<int> ci(csc.size()), fill(rp.begin(), rp.end() - 1);
    std::vector<double> val(csc.size());
    for (const E& e : csc) {
        const int p = fill[size_t(e.row)]++;
        ci[size_t(p)] = e.col;
        val[size_t(p)] = e.v;
    }

    // k_vfy_cols: one block per instance, column j on thread j % kBlock
    std::vector<long long> fb(static_cast<size_t>(count));
    std::vector<Rec> B(static_cast<size_t>(count)), G(static_cast<size_t>(count));
    for (int k = 0; k < count; ++k) {
        const long long c0 = col_off[size_t(k)], nk = col_off[size_t(k) + 1] - c0;
        std::vector<long long> tf(kBlock, nk);
        for (int t = 0; t < kBlock; ++t)
            for (long long j = t; j < nk; j += kBlock)
                if (!std::isfinite(x[c0 + j])) {
                    tf[size_t(t)] = j;
                    break;
                }
        const long long f = block_min(tf);
        std::vector<Rec> tb(kBlock, nir::vfy::rec0()), tg(kBlock, nir::vfy::rec0());
        for (int t = 0; t < kBlock; ++t)
            for (long long j = t; j < f; j += kBlock)
                nir::vfy::col_check(x[c0 + j], lo[size_t(c0 + j)], up[size_t(c0 + j)],
                                    vartype ? vartype[c0 + j] : int8_t(0), j, tb[size_t(t)], tg[size_t(t)]);
        fb[size_t(k)] = f;
        B[size_t(k)] = block_best(tb);
        G[size_t(k)] = block_best(tg);
    }

    // k_vfy_rows: the objectives, then one thread per row
    std::vector<double> obj(static_cast<size_t>(count)), rv(static_cast<size_t>(m));
    std::vector<int8_t> rs(static_cast<size_t>(m));
    for (int k = 0; k < count; ++k) {
        const long long c0 = col_off[size_t(k)], c1 = col_off[size_t(k) + 1];
        obj[size_t(k)] = fb[size_t(k)] < c1 - c0 ? 0.0 : nir::vfy::objective(offsets[size_t(k)], c0, c1, c.data(), x);
    }
    for (long long r = 0; r < m; ++r) {
        const int k = row_inst[size_t(r)];
        if (fb[size_t(k)] < (long long)(col_off[size_t(k) + 1] - col_off[size_t(k)])) {
            rv[size_t(r)] = 0.0;
            rs[size_t(r)] = 0;
            continue;
        }
        const Rec R = nir::vfy::row_check(r - row_off[size_t(k)], rp[size_t(r)], rp[size_t(r) + 1], ci.data(),
                                          val.data(), x, rl[size_t(r)], ru[size_t(r)]);
        rv[size_t(r)] = R.v;
        rs[size_t(r)] = R.pos >= 0 ? int8_t(R.pos & 1) : int8_t(0);
    }

    // k_vfy_report: one block per instance, row i on thread i % kBlock
    for (int k = 0; k < count; ++k) {
        const long long r0 = row_off[size_t(k)], mk = row_off[size_t(k) + 1] - r0;
        std::vector<Rec> tr(kBlock, nir::vfy::rec0());
        for (int t = 0; t < kBlock; ++t)
            for (long long i = t; i < mk; i += kBlock)
                nir::vfy::see(tr[size_t(t)], rv[size_t(r0 + i)], 2 * i + rs[size_t(r0 + i)]);
        const Rec R = block_best(tr);
        const double cl = claimed ? claimed[k] : std::numeric_limits<double>::quiet_NaN();
        out[k] = nir::vfy::assemble(fb[size_t(k)], col_off[size_t(k) + 1] - col_off[size_t(k)], B[size_t(k)],
                                    G[size_t(k)], R, obj[size_t(k)], cl, tol);
    }
    return 0;
}
