// Seeded synthetic LP instances (see include/nir_lpgen.h for the kinds).
//
// Host-only C++17; compiled into libnir_lpgen.so so that CPU tests, the
// benchmark and the CUDA engine's tests all see bit-identical instances.
// The random stream is xoshiro256** (Blackman & Vigna) seeded by splitmix64,
// the same generator family the reference ships (src/core/rng.hpp:8-77).

#include "nir_lpgen.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

thread_local std::string g_err;

struct Rng {
    uint64_t s[4];
    explicit Rng(uint64_t seed) {
        uint64_t x = seed;
        for (auto& w : s) w = mix(x);
    }
    static uint64_t mix(uint64_t& x) {
        uint64_t z = (x += 0x9e3779b97f4a7c15ULL);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
        return z ^ (z >> 31);
    }
    static uint64_t rotl(uint64_t v, int k) { return (v << k) | (v >> (64 - k)); }
    uint64_t next() {
        const uint64_t r = rotl(s[1] * 5, 7) * 9;
        const uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
    double uniform() { return static_cast<double>(next() >> 11) * 0x1.0p-53; }        // [0,1)
    double uniform(double a, double b) { return a + (b - a) * uniform(); }
    // Box-Muller, one variate per call.
    double normal() {
        double u1 = 1.0 - uniform();  // (0,1]
        double u2 = uniform();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
    // Uniform integer in [0, n).
    int64_t below(int64_t n) { return static_cast<int64_t>(uniform() * static_cast<double>(n)); }
};

// k distinct integers from [0, n), returned ascending.
void sample_distinct(Rng& r, int64_t k, int64_t n, std::vector<int32_t>& out) {
    out.clear();
    if (k >= n) {
        for (int64_t i = 0; i < n; ++i) out.push_back(static_cast<int32_t>(i));
        return;
    }
    while (static_cast<int64_t>(out.size()) < k) {
        int64_t need = k - static_cast<int64_t>(out.size());
        for (int64_t t = 0; t < need; ++t) out.push_back(static_cast<int32_t>(r.below(n)));
        std::sort(out.begin(), out.end());
        out.erase(std::unique(out.begin(), out.end()), out.end());
    }
}

constexpr double kInf = std::numeric_limits<double>::infinity();

struct Lp {
    int32_t m = 0, n = 0;
    std::vector<int64_t> start;
    std::vector<int32_t> index;
    std::vector<double> value;
    std::vector<double> cost, collo, colup, rowlo, rowup, x0;
    std::vector<double> demand_factor, cost_factor;
    int32_t n_demand = 0;
};

// Column-major assembly from per-row entry lists (rows visited in order, so
// every column's rows come out ascending and distinct).
struct RowBuilder {
    int32_t m, n;
    std::vector<std::vector<std::pair<int32_t, double>>> rows;  // per row: (col, val)
    RowBuilder(int32_t m_, int32_t n_) : m(m_), n(n_), rows(m_) {}
    void to_csc(Lp& lp) {
        lp.m = m;
        lp.n = n;
        std::vector<int64_t> cnt(n + 1, 0);
        for (auto& r : rows)
            for (auto& e : r) cnt[e.first + 1]++;
        for (int32_t j = 0; j < n; ++j) cnt[j + 1] += cnt[j];
        lp.start = cnt;
        lp.index.assign(cnt[n], 0);
        lp.value.assign(cnt[n], 0.0);
        std::vector<int64_t> pos(cnt.begin(), cnt.end() - 1);
        for (int32_t i = 0; i < m; ++i)
            for (auto& e : rows[i]) {
                int64_t p = pos[e.first]++;
                lp.index[p] = i;
                lp.value[p] = e.second;
            }
        rows.clear();
        rows.shrink_to_fit();
    }
};

std::vector<double> mul_A(const Lp& lp, const std::vector<double>& x) {
    std::vector<double> y(lp.m, 0.0);
    for (int32_t j = 0; j < lp.n; ++j)
        for (int64_t k = lp.start[j]; k < lp.start[j + 1]; ++k) y[lp.index[k]] += lp.value[k] * x[j];
    return y;
}

std::vector<double> mul_At(const Lp& lp, const std::vector<double>& y) {
    std::vector<double> c(lp.n, 0.0);
    for (int32_t j = 0; j < lp.n; ++j) {
        double s = 0.0;
        for (int64_t k = lp.start[j]; k < lp.start[j + 1]; ++k) s += lp.value[k] * y[lp.index[k]];
        c[j] = s;
    }
    return c;
}

// c = A^T y0 + s, s ~ U[0,1]
void finish_cost(Lp& lp, Rng& r, const std::vector<double>& y0) {
    lp.cost = mul_At(lp, y0);
    for (auto& cj : lp.cost) cj += r.uniform();
}

void gen_random_eq(Lp& lp, uint64_t seed, const nir_lpgen_opts& o) {
    const int32_t m = o.m ? o.m : 2000, n = o.n ? o.n : 5000, k = o.per_col ? o.per_col : 8;
    Rng r(seed);
    lp.m = m;
    lp.n = n;
    lp.start.assign(n + 1, 0);
    std::vector<int32_t> rows;
    for (int32_t j = 0; j < n; ++j) {
        sample_distinct(r, std::min<int64_t>(k, m), m, rows);
        for (int32_t i : rows) {
            lp.index.push_back(i);
            lp.value.push_back(r.normal());
        }
        lp.start[j + 1] = static_cast<int64_t>(lp.index.size());
    }
    lp.collo.assign(n, 0.0);
    lp.colup.assign(n, 10.0);
    lp.x0.resize(n);
    for (auto& v : lp.x0) v = r.uniform(0.0, 10.0);
    lp.rowlo = mul_A(lp, lp.x0);
    lp.rowup = lp.rowlo;
    std::vector<double> y0(m);
    for (auto& v : y0) v = r.normal();
    finish_cost(lp, r, y0);
}

void gen_zipf(Lp& lp, uint64_t seed, const nir_lpgen_opts& o) {
    const int32_t m = o.m ? o.m : 200000, n = o.n ? o.n : 500000;
    const int32_t cap = o.zipf_cap ? o.zipf_cap : 2000;
    const int64_t target = o.target_nnz ? o.target_nnz : 5000000;
    Rng r(seed);
    // Truncated Zipf(1.5) on 1..cap by inverse CDF.
    std::vector<double> cdf(cap);
    double acc = 0.0;
    for (int32_t L = 1; L <= cap; ++L) {
        acc += std::pow(static_cast<double>(L), -1.5);
        cdf[L - 1] = acc;
    }
    for (auto& v : cdf) v /= acc;
    std::vector<int64_t> len(m);
    int64_t total = 0;
    for (int32_t i = 0; i < m; ++i) {
        double u = r.uniform();
        int64_t L = static_cast<int64_t>(std::lower_bound(cdf.begin(), cdf.end(), u) - cdf.begin()) + 1;
        len[i] = std::min<int64_t>(L, cap);
        total += len[i];
    }
    // Realisation rule: rescale all lengths by target/total (when the draw
    // overshoots), round, keep >= 1 and <= min(cap, n).
    if (total > target) {
        const double f = static_cast<double>(target) / static_cast<double>(total);
        for (auto& L : len) L = std::max<int64_t>(1, std::llround(static_cast<double>(L) * f));
    }
    for (auto& L : len) L = std::min<int64_t>(L, std::min<int64_t>(cap, n));
    RowBuilder rb(m, n);
    std::vector<int32_t> cols;
    for (int32_t i = 0; i < m; ++i) {
        sample_distinct(r, len[i], n, cols);
        auto& row = rb.rows[i];
        row.reserve(cols.size());
        for (int32_t j : cols) {
            double mag = std::pow(10.0, r.uniform(-2.0, 2.0));
            double sgn = (r.next() >> 63) ? -1.0 : 1.0;
            row.push_back({j, sgn * mag});
        }
    }
    rb.to_csc(lp);
    lp.collo.assign(n, 0.0);
    lp.colup.resize(n);
    lp.x0.resize(n);
    for (int32_t j = 0; j < n; ++j) {
        lp.colup[j] = r.uniform(1.0, 100.0);
        lp.x0[j] = r.uniform(0.0, lp.colup[j]);
    }
    lp.rowlo = mul_A(lp, lp.x0);
    lp.rowup = lp.rowlo;
    std::vector<double> y0(m);
    for (auto& v : y0) v = r.normal();
    finish_cost(lp, r, y0);
}

void gen_multiperiod(Lp& lp, uint64_t seed, const nir_lpgen_opts& o) {
    const int32_t m = o.m ? o.m : 5000;
    const int32_t n = o.n ? o.n : static_cast<int32_t>(std::llround(2.5 * m));
    const int32_t P = 12;
    if (m < 10 * P) throw std::invalid_argument("multiperiod needs m >= 120");
    Rng r(seed);
    auto rblk = [&](int32_t p) { return std::make_pair(int64_t(m) * p / P, int64_t(m) * (p + 1) / P); };
    auto cblk = [&](int32_t p) { return std::make_pair(int64_t(n) * p / P, int64_t(n) * (p + 1) / P); };
    // Column-wise entries inside the column's period block.
    std::vector<std::vector<std::pair<int32_t, double>>> col(n);
    std::vector<int32_t> rows;
    for (int32_t p = 0; p < P; ++p) {
        auto rb = rblk(p);
        auto cb = cblk(p);
        for (int64_t j = cb.first; j < cb.second; ++j) {
            sample_distinct(r, std::min<int64_t>(10, rb.second - rb.first), rb.second - rb.first, rows);
            for (int32_t i : rows) col[j].push_back({static_cast<int32_t>(rb.first + i), r.uniform(0.5, 2.0)});
        }
    }
    // Inventory links: the first tenth of the rows of period p>0 take +1 from
    // a column of period p-1 and -1 from a column of period p.
    auto has_row = [&](int64_t j, int32_t i) {
        for (auto& e : col[j])
            if (e.first == i) return true;
        return false;
    };
    for (int32_t p = 1; p < P; ++p) {
        auto rb = rblk(p);
        auto cprev = cblk(p - 1);
        auto ccur = cblk(p);
        int64_t nlink = std::max<int64_t>(1, (rb.second - rb.first) / 10);
        for (int64_t t = 0; t < nlink; ++t) {
            int32_t i = static_cast<int32_t>(rb.first + t);
            int64_t jin = cprev.first + r.below(cprev.second - cprev.first);
            col[jin].push_back({i, 1.0});
            int64_t jout;
            do {
                jout = ccur.first + r.below(ccur.second - ccur.first);
            } while (has_row(jout, i));
            col[jout].push_back({i, -1.0});
        }
    }
    lp.m = m;
    lp.n = n;
    lp.start.assign(n + 1, 0);
    for (int32_t j = 0; j < n; ++j) {
        std::sort(col[j].begin(), col[j].end());
        for (auto& e : col[j]) {
            lp.index.push_back(e.first);
            lp.value.push_back(e.second);
        }
        lp.start[j + 1] = static_cast<int64_t>(lp.index.size());
    }
    lp.collo.assign(n, 0.0);
    lp.colup.assign(n, 10.0);
    lp.x0.resize(n);
    for (auto& v : lp.x0) v = r.uniform(0.0, 10.0);
    std::vector<double> ax = mul_A(lp, lp.x0);
    lp.rowlo.resize(m);
    lp.rowup.resize(m);
    std::vector<double> y0(m);
    for (int32_t i = 0; i < m; ++i) {
        if (i % 2 == 0) {  // equality
            lp.rowlo[i] = lp.rowup[i] = ax[i];
            y0[i] = r.normal();
        } else {  // <= with slack
            lp.rowlo[i] = -kInf;
            lp.rowup[i] = ax[i] + r.uniform();
            y0[i] = -std::fabs(r.normal());
        }
    }
    finish_cost(lp, r, y0);
}

void gen_blend_family(Lp& lp, uint64_t seed, const nir_lpgen_opts& o) {
    const int32_t m = o.m ? o.m : 20000, n = o.n ? o.n : 50000;
    const int64_t nnz_target = o.target_nnz ? o.target_nnz : 400000;
    const int32_t per_col = static_cast<int32_t>(std::max<int64_t>(3, nnz_target / n));
    const int32_t nd = std::max(1, m / 10);          // demand rows (>=)
    const int32_t nq = (m - nd) / 2;                 // quality rows (<=)
    const int32_t nc = m - nd - nq;                  // capacity rows (<=)
    const int32_t kd = std::max(1, per_col / 4);     // demand entries per column
    const int32_t kq = std::max(1, (per_col - kd) / 2);
    const int32_t kc = std::max(1, per_col - kd - kq);
    Rng fr(o.family_seed);  // the fixed matrix
    lp.m = m;
    lp.n = n;
    lp.start.assign(n + 1, 0);
    std::vector<int32_t> a, b, c;
    for (int32_t j = 0; j < n; ++j) {
        sample_distinct(fr, kd, nd, a);
        sample_distinct(fr, kq, nq, b);
        sample_distinct(fr, kc, nc, c);
        for (int32_t i : a) {
            lp.index.push_back(i);
            lp.value.push_back(fr.uniform(0.5, 2.0));
        }
        for (int32_t i : b) {
            lp.index.push_back(nd + i);
            lp.value.push_back(fr.normal());
        }
        for (int32_t i : c) {
            lp.index.push_back(nd + nq + i);
            lp.value.push_back(fr.uniform(0.5, 2.0));
        }
        lp.start[j + 1] = static_cast<int64_t>(lp.index.size());
    }
    lp.collo.assign(n, 0.0);
    lp.colup.resize(n);
    lp.x0.resize(n);
    for (int32_t j = 0; j < n; ++j) {
        lp.colup[j] = fr.uniform(1.0, 10.0);
        lp.x0[j] = fr.uniform(0.0, lp.colup[j]);
    }
    std::vector<double> ax = mul_A(lp, lp.x0);
    lp.rowlo.resize(m);
    lp.rowup.resize(m);
    std::vector<double> y0(m);
    for (int32_t i = 0; i < m; ++i) {
        if (i < nd) {
            lp.rowlo[i] = 0.5 * ax[i];
            lp.rowup[i] = kInf;
            y0[i] = std::fabs(fr.normal());
        } else {
            lp.rowlo[i] = -kInf;
            lp.rowup[i] = ax[i] + fr.uniform();
            y0[i] = -std::fabs(fr.normal());
        }
    }
    finish_cost(lp, fr, y0);
    // Instance perturbation (seed): demand b by (1+0.2N), c by (1+0.1N),
    // clamped so that x0 stays feasible and every cost keeps its sign.
    Rng r(seed);
    lp.n_demand = nd;
    lp.demand_factor.resize(nd);
    for (int32_t i = 0; i < nd; ++i) {
        double f = std::min(1.9, std::max(0.1, 1.0 + 0.2 * r.normal()));
        lp.demand_factor[i] = f;
        lp.rowlo[i] *= f;
    }
    lp.cost_factor.resize(n);
    for (int32_t j = 0; j < n; ++j) {
        double f = std::min(1.5, std::max(0.5, 1.0 + 0.1 * r.normal()));
        lp.cost_factor[j] = f;
        lp.cost[j] *= f;
    }
}

void gen_badly_scaled(Lp& lp, uint64_t seed, const nir_lpgen_opts& o) {
    const int32_t m = o.m ? o.m : 50000, n = o.n ? o.n : 120000;
    const int64_t nnz_target = o.target_nnz ? o.target_nnz : 1000000;
    const double d = o.scale_decades > 0 ? o.scale_decades : 4.0;
    const int32_t nb = n / 2;                 // base columns; the rest duplicate them
    const int64_t base_nnz = nnz_target / 2;
    Rng r(seed);
    std::vector<double> R(m), C(nb);
    for (auto& v : R) v = std::pow(10.0, r.uniform(-d, d));
    for (auto& v : C) v = std::pow(10.0, r.uniform(-d, d));
    lp.m = m;
    lp.n = 2 * nb + (n - 2 * nb);
    lp.start.assign(lp.n + 1, 0);
    std::vector<std::vector<std::pair<int32_t, double>>> base(nb);
    std::vector<int32_t> rows;
    for (int32_t j = 0; j < nb; ++j) {
        int64_t k = base_nnz / nb + ((j < base_nnz % nb) ? 1 : 0);
        sample_distinct(r, std::max<int64_t>(1, std::min<int64_t>(k, m)), m, rows);
        for (int32_t i : rows) base[j].push_back({i, R[i] * r.normal() * C[j]});
    }
    int32_t col = 0;
    auto emit = [&](const std::vector<std::pair<int32_t, double>>& e) {
        for (auto& p : e) {
            lp.index.push_back(p.first);
            lp.value.push_back(p.second);
        }
        lp.start[++col] = static_cast<int64_t>(lp.index.size());
    };
    for (int32_t j = 0; j < nb; ++j) emit(base[j]);
    for (int32_t j = 0; j < nb; ++j) {
        auto dup = base[j];
        for (auto& p : dup) p.second *= 1.0 + 1e-9 * r.normal();
        emit(dup);
    }
    while (col < lp.n) emit({});  // odd n: one empty column
    lp.collo.assign(lp.n, 0.0);
    lp.colup.assign(lp.n, 10.0);
    lp.x0.resize(lp.n);
    for (auto& v : lp.x0) v = r.uniform(0.0, 10.0);
    lp.rowlo = mul_A(lp, lp.x0);
    lp.rowup = lp.rowlo;
    std::vector<double> y0(m);
    for (int32_t i = 0; i < m; ++i) y0[i] = r.normal() / R[i];
    finish_cost(lp, r, y0);
}

}  // namespace

struct nir_lpgen {
    Lp lp;
};

extern "C" {

int nir_lpgen_create(int kind, uint64_t seed, const nir_lpgen_opts* opts, nir_lpgen** out) {
    if (!out) {
        g_err = "null output pointer";
        return 1;
    }
    *out = nullptr;
    nir_lpgen_opts o;
    std::memset(&o, 0, sizeof(o));
    if (opts) o = *opts;
    if (o.m < 0 || o.n < 0 || o.target_nnz < 0 || o.per_col < 0) {
        g_err = "negative size";
        return 1;
    }
    try {
        auto g = std::make_unique<nir_lpgen>();
        switch (kind) {
            case NIR_GEN_RANDOM_EQ: gen_random_eq(g->lp, seed, o); break;
            case NIR_GEN_ZIPF: gen_zipf(g->lp, seed, o); break;
            case NIR_GEN_MULTIPERIOD: gen_multiperiod(g->lp, seed, o); break;
            case NIR_GEN_BLEND_FAMILY: gen_blend_family(g->lp, seed, o); break;
            case NIR_GEN_BADLY_SCALED: gen_badly_scaled(g->lp, seed, o); break;
            default: g_err = "unknown instance kind"; return 1;
        }
        *out = g.release();
        return 0;
    } catch (const std::bad_alloc&) {
        g_err = "out of host memory";
    } catch (const std::exception& e) {
        g_err = e.what();
    }
    return 1;
}

int nir_lpgen_view(const nir_lpgen* g, nir_lp_view* v) {
    if (!g || !v) return 1;
    const Lp& lp = g->lp;
    v->nrow = lp.m;
    v->ncol = lp.n;
    v->nnz = lp.start.empty() ? 0 : lp.start.back();
    v->col_start = lp.start.data();
    v->row_index = lp.index.data();
    v->value = lp.value.data();
    v->cost = lp.cost.data();
    v->collo = lp.collo.data();
    v->colup = lp.colup.data();
    v->rowlo = lp.rowlo.data();
    v->rowup = lp.rowup.data();
    v->obj_offset = 0.0;
    return 0;
}

const double* nir_lpgen_x0(const nir_lpgen* g) { return g ? g->lp.x0.data() : nullptr; }

const double* nir_lpgen_demand_factors(const nir_lpgen* g, int32_t* n_demand) {
    if (n_demand) *n_demand = g ? g->lp.n_demand : 0;
    return (g && !g->lp.demand_factor.empty()) ? g->lp.demand_factor.data() : nullptr;
}

const double* nir_lpgen_cost_factors(const nir_lpgen* g) {
    return (g && !g->lp.cost_factor.empty()) ? g->lp.cost_factor.data() : nullptr;
}

void nir_lpgen_free(nir_lpgen* g) { delete g; }

const char* nir_lpgen_last_error(void) { return g_err.c_str(); }

}  // extern "C"
