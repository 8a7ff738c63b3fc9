// Presolve and scaling ahead of the PDHG path (C ABI: include/nir_facade.h).
//
// nir_presolve follows sov::Presolver::presolve (src/presolve/presolve.hpp:
// 32-345) rule for rule; nir_scale follows sov::scale_model
// (src/model/scaling.hpp:56-154).  The reference runs both on one thread;
// here every pass that reads the model without changing it runs over rows
// or columns in parallel, and every change is applied on one thread in the
// reference's order with the reference's expressions, so that the results
// are bit-identical:
//   R4  fixed columns: found in parallel; the right-hand-side updates they
//       cause are applied per row, in parallel over rows, in the order of
//       the columns (which is the reference's order for each row);
//   R1/R3 empty and singleton rows: active entries counted in parallel;
//       the rows with at most one are handled in row order;
//   R5/R6/R14/R7 activity rules: every row's activity bounds computed in
//       parallel; the rows are then walked in order, and a row whose columns
//       an earlier row of the same pass changed (a forcing row fixing them,
//       an integer bound tightened) has its activity recomputed first;
//   R2  empty columns: found in parallel, fixed in column order.
// Compile without FMA contraction (-ffp-contract=off), as the reference's
// x86-64 build has none.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "nir_facade.h"
#include "text.hpp"

namespace {

using nir::text::uvector;  // buffers that are written in full right after they are sized

thread_local std::string g_err;

constexpr double kInf = std::numeric_limits<double>::infinity();
constexpr double kInfInput = 1e20;  // src/core/types.hpp:16

// is_finite_bound (src/core/types.hpp:49-51)
inline bool fin(double b) { return std::isfinite(b) && std::abs(b) < kInfInput; }

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

// f(begin, end) over [0, n) in nt contiguous ranges
template <class F>
void parallel_ranges(int64_t n, int threads, int64_t grain, F&& f) {
    const int nt = int(std::max<int64_t>(1, std::min<int64_t>(threads, n / std::max<int64_t>(grain, 1) + 1)));
    run_threads(nt, [&](int k) { f(n * k / nt, n * (k + 1) / nt); });
}

int hw_threads(int t) { return t > 0 ? t : int(std::max(1u, std::thread::hardware_concurrency())); }

// CSR of a CSC in CsrMatrix::from_csc's entry order (src/core/csc_matrix.hpp:
// 160-182): columns ascending, CSC order within a column.  Built in
// parallel over column ranges; each range writes after the ranges before it.
struct Csr {
    std::vector<int64_t> start;
    uvector<int32_t> index;
    uvector<double> value;
};

Csr csr_of(int32_t m, int32_t n, const int64_t* cs, const int32_t* ci, const double* cv, int threads) {
    Csr r;
    const int64_t nnz = cs[n];
    const int nt = int(std::max<int64_t>(1, std::min<int64_t>(threads, nnz / 65536 + 1)));
    std::vector<int32_t> jb(size_t(nt) + 1, n);
    jb[0] = 0;
    for (int k = 1; k < nt; ++k) {
        jb[size_t(k)] = int32_t(std::lower_bound(cs, cs + n + 1, nnz * k / nt) - cs);
        jb[size_t(k)] = std::max(jb[size_t(k) - 1], std::min(jb[size_t(k)], n));
    }
    std::vector<std::vector<int64_t>> pos(static_cast<size_t>(nt));
    run_threads(nt, [&](int k) {
        auto& c = pos[size_t(k)];
        c.assign(size_t(m), 0);
        for (int64_t q = cs[jb[size_t(k)]]; q < cs[jb[size_t(k) + 1]]; ++q) ++c[size_t(ci[q])];
    });
    r.start.assign(size_t(m) + 1, 0);
    for (int32_t i = 0; i < m; ++i) {
        int64_t s = r.start[size_t(i)];
        for (int k = 0; k < nt; ++k) {
            const int64_t c = pos[size_t(k)][size_t(i)];
            pos[size_t(k)][size_t(i)] = s;
            s += c;
        }
        r.start[size_t(i) + 1] = s;
    }
    r.index.resize(size_t(nnz));
    r.value.resize(size_t(nnz));
    run_threads(nt, [&](int k) {
        auto& w = pos[size_t(k)];
        for (int32_t j = jb[size_t(k)]; j < jb[size_t(k) + 1]; ++j)
            for (int64_t q = cs[j]; q < cs[j + 1]; ++q) {
                const int64_t p = w[size_t(ci[q])]++;
                r.index[size_t(p)] = j;
                r.value[size_t(p)] = cv[q];
            }
    });
    return r;
}

bool check_view(const nir_lp_view* v) {
    if (!v || v->nrow < 0 || v->ncol < 0 || !v->col_start) return false;
    if (v->ncol > 0 && (!v->cost || !v->collo || !v->colup)) return false;
    if (v->nrow > 0 && (!v->rowlo || !v->rowup)) return false;
    if (v->col_start[0] != 0 || v->col_start[v->ncol] != v->nnz) return false;
    if (v->nnz > 0 && (!v->row_index || !v->value)) return false;
    for (int32_t j = 0; j < v->ncol; ++j)
        if (v->col_start[j] > v->col_start[j + 1]) return false;
    for (int64_t k = 0; k < v->nnz; ++k)
        if (v->row_index[k] < 0 || v->row_index[k] >= v->nrow) return false;
    return true;
}

}  // namespace

struct nir_presolved {
    int32_t status = 0, solved = 0;
    int32_t rows_removed = 0, cols_removed = 0, tightenings = 0;
    int32_t nrow = 0, ncol = 0;
    double obj_offset = 0.0;
    std::vector<int64_t> start{0};
    nir::text::uvector<int32_t> index;
    nir::text::uvector<double> value;
    std::vector<double> cost, collo, colup, rowlo, rowup;
    std::vector<int8_t> vartype;
    std::vector<int32_t> col_map, row_map;
    std::vector<double> fixed_x;
    std::vector<uint8_t> is_fixed;
};

namespace {

enum : int32_t { kOptimal = 0, kInfeasible = 1, kUnbounded = 2 };

struct Presolve {
    const nir_lp_view& A;
    const int32_t m, n;
    const int64_t* cs;
    const int32_t* ci;
    const double* cv;
    const double* cost;
    int threads;
    nir_presolved& res;

    std::vector<double> collo, colup, rowlo, rowup;
    std::vector<int8_t> vt;
    double obj_offset;
    Csr csr;
    std::vector<uint8_t> row_del, col_del;
    std::vector<uint8_t> row_int;  // the row has an integer column (R7 can act on it)
    // activity bounds kept from one pass to the next: a row's stay valid
    // until one of its columns is deleted or has a bound changed (such a
    // column is marked in col_touched)
    std::vector<uint8_t> col_touched, row_valid;

    Presolve(const nir_lp_view& a, const int8_t* vtype, int th, nir_presolved& r)
        : A(a), m(a.nrow), n(a.ncol), cs(a.col_start), ci(a.row_index), cv(a.value), cost(a.cost), threads(th),
          res(r) {
        collo.assign(a.collo, a.collo + n);
        colup.assign(a.colup, a.colup + n);
        rowlo.assign(a.rowlo, a.rowlo + m);
        rowup.assign(a.rowup, a.rowup + m);
        vt.assign(size_t(n), 0);
        if (vtype) vt.assign(vtype, vtype + n);
        obj_offset = a.obj_offset;
    }

    // fix_col (src/presolve/presolve.hpp:53-67)
    void fix_col(int32_t j, double val) {
        if (col_del[size_t(j)]) return;
        col_del[size_t(j)] = 1;
        col_touched[size_t(j)] = 1;
        res.is_fixed[size_t(j)] = 1;
        res.fixed_x[size_t(j)] = val;
        obj_offset += cost[j] * val;
        for (int64_t k = cs[j]; k < cs[j + 1]; ++k) {
            const int32_t i = ci[k];
            if (row_del[size_t(i)]) continue;
            const double aij = cv[k];
            if (fin(rowlo[size_t(i)])) rowlo[size_t(i)] -= aij * val;
            if (fin(rowup[size_t(i)])) rowup[size_t(i)] -= aij * val;
        }
        ++res.cols_removed;
    }

    void stop(int32_t status) {
        res.status = status;
        res.solved = 1;
    }

    struct Act {
        double min_act, max_act;
        int32_t min_inf, max_inf;
    };
    std::vector<Act> act;

    // the activity bounds of row i (src/presolve/presolve.hpp:142-161)
    Act activity(int32_t i) const {
        Act a{0.0, 0.0, 0, 0};
        for (int64_t k = csr.start[size_t(i)]; k < csr.start[size_t(i) + 1]; ++k) {
            const int32_t j = csr.index[size_t(k)];
            if (col_del[size_t(j)]) continue;
            const double v = csr.value[size_t(k)];
            if (v > 0.0) {
                if (fin(collo[size_t(j)])) a.min_act += v * collo[size_t(j)];
                else ++a.min_inf;
                if (fin(colup[size_t(j)])) a.max_act += v * colup[size_t(j)];
                else ++a.max_inf;
            } else if (v < 0.0) {
                if (fin(colup[size_t(j)])) a.min_act += v * colup[size_t(j)];
                else ++a.min_inf;
                if (fin(collo[size_t(j)])) a.max_act += v * collo[size_t(j)];
                else ++a.max_inf;
            }
        }
        return a;
    }

    // returns false when presolve stops (infeasible / unbounded)
    bool round(bool& changed) {
        // R4: fixed columns
        {
            std::vector<uint8_t> fx(size_t(n), 0);
            parallel_ranges(n, threads, 1 << 14, [&](int64_t a, int64_t b) {
                for (int64_t j = a; j < b; ++j)
                    fx[size_t(j)] = !col_del[size_t(j)] && fin(collo[size_t(j)]) && fin(colup[size_t(j)]) &&
                                    std::abs(colup[size_t(j)] - collo[size_t(j)]) <= 1e-11;
            });
            bool any = false;
            for (int32_t j = 0; j < n; ++j) {
                if (!fx[size_t(j)]) continue;
                any = true;
                const double val = collo[size_t(j)];
                col_del[size_t(j)] = 1;
                col_touched[size_t(j)] = 1;
                res.is_fixed[size_t(j)] = 1;
                res.fixed_x[size_t(j)] = val;
                obj_offset += cost[j] * val;
                ++res.cols_removed;
            }
            if (any) {
                changed = true;
                // each row gets its updates in column order, as fix_col
                // called for j = 0, 1, ... gives them
                parallel_ranges(m, threads, 1 << 13, [&](int64_t a, int64_t b) {
                    for (int64_t i = a; i < b; ++i) {
                        if (row_del[size_t(i)]) continue;
                        for (int64_t k = csr.start[size_t(i)]; k < csr.start[size_t(i) + 1]; ++k) {
                            const int32_t j = csr.index[size_t(k)];
                            if (!fx[size_t(j)]) continue;
                            const double aij = csr.value[size_t(k)], val = res.fixed_x[size_t(j)];
                            if (fin(rowlo[size_t(i)])) rowlo[size_t(i)] -= aij * val;
                            if (fin(rowup[size_t(i)])) rowup[size_t(i)] -= aij * val;
                        }
                    }
                });
            }
        }

        // R1 & R3: empty rows and row singletons
        {
            std::vector<uint8_t> cnt(size_t(m), 2);
            std::vector<int32_t> sj(size_t(m), -1);
            std::vector<double> sa(size_t(m), 0.0);
            parallel_ranges(m, threads, 1 << 13, [&](int64_t a, int64_t b) {
                for (int64_t i = a; i < b; ++i) {
                    if (row_del[size_t(i)]) continue;
                    int c = 0;
                    for (int64_t k = csr.start[size_t(i)]; k < csr.start[size_t(i) + 1]; ++k) {
                        const int32_t j = csr.index[size_t(k)];
                        if (!col_del[size_t(j)] && std::abs(csr.value[size_t(k)]) > 1e-13) {
                            if (++c > 1) break;
                            sj[size_t(i)] = j;
                            sa[size_t(i)] = csr.value[size_t(k)];
                        }
                    }
                    cnt[size_t(i)] = uint8_t(std::min(c, 2));
                }
            });
            for (int32_t i = 0; i < m; ++i) {
                if (row_del[size_t(i)] || cnt[size_t(i)] > 1) continue;
                if (cnt[size_t(i)] == 0) {
                    if ((fin(rowlo[size_t(i)]) && rowlo[size_t(i)] > 1e-7) ||
                        (fin(rowup[size_t(i)]) && rowup[size_t(i)] < -1e-7)) {
                        stop(kInfeasible);
                        return false;
                    }
                    row_del[size_t(i)] = 1;
                    ++res.rows_removed;
                    changed = true;
                    continue;
                }
                const int32_t j = sj[size_t(i)];
                const double a = sa[size_t(i)];
                col_touched[size_t(j)] = 1;  // its bounds may change below
                double lo_b = -kInf, up_b = kInf;
                if (a > 0.0) {
                    if (fin(rowlo[size_t(i)])) lo_b = rowlo[size_t(i)] / a;
                    if (fin(rowup[size_t(i)])) up_b = rowup[size_t(i)] / a;
                } else {
                    if (fin(rowup[size_t(i)])) lo_b = rowup[size_t(i)] / a;
                    if (fin(rowlo[size_t(i)])) up_b = rowlo[size_t(i)] / a;
                }
                if (vt[size_t(j)] != 0) {
                    if (fin(lo_b)) lo_b = std::ceil(lo_b - 1e-7);
                    if (fin(up_b)) up_b = std::floor(up_b + 1e-7);
                }
                if (lo_b > collo[size_t(j)] + 1e-9) {
                    collo[size_t(j)] = lo_b;
                    ++res.tightenings;
                }
                if (up_b < colup[size_t(j)] - 1e-9) {
                    colup[size_t(j)] = up_b;
                    ++res.tightenings;
                }
                if (collo[size_t(j)] > colup[size_t(j)] + 1e-7) {
                    stop(kInfeasible);
                    return false;
                }
                if (collo[size_t(j)] > colup[size_t(j)]) collo[size_t(j)] = colup[size_t(j)];
                row_del[size_t(i)] = 1;
                ++res.rows_removed;
                changed = true;
            }
        }

        // R5, R6, R7, R14: activity bounds, redundancy, forcing rows,
        // integer bound tightening
        {
            for (int32_t j = 0; j < n; ++j) {
                if (!col_touched[size_t(j)]) continue;
                col_touched[size_t(j)] = 0;
                for (int64_t k = cs[j]; k < cs[j + 1]; ++k) row_valid[size_t(ci[k])] = 0;
            }
            parallel_ranges(m, threads, 1 << 13, [&](int64_t a, int64_t b) {
                for (int64_t i = a; i < b; ++i)
                    if (!row_del[size_t(i)] && !row_valid[size_t(i)]) {
                        act[size_t(i)] = activity(int32_t(i));
                        row_valid[size_t(i)] = 1;
                    }
            });
            // changes made by rows of this pass reach later rows, which are
            // recomputed when the walk gets to them
            std::vector<uint8_t> dirty(static_cast<size_t>(m), 0);
            auto touch = [&](int32_t j) {
                col_touched[size_t(j)] = 1;
                for (int64_t k = cs[j]; k < cs[j + 1]; ++k) dirty[size_t(ci[k])] = 1;
            };
            for (int32_t i = 0; i < m; ++i) {
                if (row_del[size_t(i)]) continue;
                const Act a = dirty[size_t(i)] ? activity(i) : act[size_t(i)];
                const double lo = rowlo[size_t(i)], up = rowup[size_t(i)];
                // R6
                if ((a.min_inf == 0 && fin(up) && a.min_act > up + 1e-7) ||
                    (a.max_inf == 0 && fin(lo) && a.max_act < lo - 1e-7)) {
                    stop(kInfeasible);
                    return false;
                }
                // R5
                const bool lo_red = !fin(lo) || (a.min_inf == 0 && a.min_act >= lo - 1e-9);
                const bool up_red = !fin(up) || (a.max_inf == 0 && a.max_act <= up + 1e-9);
                if (lo_red && up_red) {
                    row_del[size_t(i)] = 1;
                    ++res.rows_removed;
                    changed = true;
                    continue;
                }
                // R14
                if (a.min_inf == 0 && fin(rowup[size_t(i)]) && std::abs(a.min_act - rowup[size_t(i)]) <= 1e-9) {
                    force(i, true, touch);
                    changed = true;
                    continue;
                }
                if (a.max_inf == 0 && fin(rowlo[size_t(i)]) && std::abs(a.max_act - rowlo[size_t(i)]) <= 1e-9) {
                    force(i, false, touch);
                    changed = true;
                    continue;
                }
                // R7 (its loops skip continuous columns: rows without an
                // integer column are passed over whole)
                if (!row_int[size_t(i)]) continue;
                if (a.min_inf == 0 && fin(rowup[size_t(i)])) {
                    const double slack = rowup[size_t(i)] - a.min_act;
                    for (int64_t k = csr.start[size_t(i)]; k < csr.start[size_t(i) + 1]; ++k) {
                        const int32_t j = csr.index[size_t(k)];
                        if (col_del[size_t(j)] || vt[size_t(j)] == 0) continue;
                        const double v = csr.value[size_t(k)];
                        if (v > 1e-9 && fin(collo[size_t(j)])) {
                            const double new_u = std::floor(collo[size_t(j)] + (slack / v) + 1e-6);
                            if (new_u < colup[size_t(j)] - 0.5) {
                                colup[size_t(j)] = new_u;
                                ++res.tightenings;
                                changed = true;
                                touch(j);
                            }
                        } else if (v < -1e-9 && fin(colup[size_t(j)])) {
                            const double new_l = std::ceil(colup[size_t(j)] + (slack / v) - 1e-6);
                            if (new_l > collo[size_t(j)] + 0.5) {
                                collo[size_t(j)] = new_l;
                                ++res.tightenings;
                                changed = true;
                                touch(j);
                            }
                        }
                    }
                }
                if (a.max_inf == 0 && fin(rowlo[size_t(i)])) {
                    const double slack = a.max_act - rowlo[size_t(i)];
                    for (int64_t k = csr.start[size_t(i)]; k < csr.start[size_t(i) + 1]; ++k) {
                        const int32_t j = csr.index[size_t(k)];
                        if (col_del[size_t(j)] || vt[size_t(j)] == 0) continue;
                        const double v = csr.value[size_t(k)];
                        if (v > 1e-9 && fin(colup[size_t(j)])) {
                            const double new_l = std::ceil(colup[size_t(j)] - (slack / v) - 1e-6);
                            if (new_l > collo[size_t(j)] + 0.5) {
                                collo[size_t(j)] = new_l;
                                ++res.tightenings;
                                changed = true;
                                touch(j);
                            }
                        } else if (v < -1e-9 && fin(collo[size_t(j)])) {
                            const double new_u = std::floor(collo[size_t(j)] - (slack / v) + 1e-6);
                            if (new_u < colup[size_t(j)] - 0.5) {
                                colup[size_t(j)] = new_u;
                                ++res.tightenings;
                                changed = true;
                                touch(j);
                            }
                        }
                    }
                }
            }
        }

        // R2: empty columns
        {
            std::vector<uint8_t> empty(size_t(n), 0);
            parallel_ranges(n, threads, 1 << 14, [&](int64_t a, int64_t b) {
                for (int64_t j = a; j < b; ++j) {
                    if (col_del[size_t(j)]) continue;
                    bool active = false;
                    for (int64_t k = cs[j]; k < cs[j + 1] && !active; ++k) active = !row_del[size_t(ci[k])];
                    empty[size_t(j)] = !active;
                }
            });
            for (int32_t j = 0; j < n; ++j) {
                if (!empty[size_t(j)] || col_del[size_t(j)]) continue;
                const double cj = cost[j];
                if (cj > 1e-12) {
                    if (!fin(collo[size_t(j)])) {
                        stop(kUnbounded);
                        return false;
                    }
                    fix_col(j, collo[size_t(j)]);
                } else if (cj < -1e-12) {
                    if (!fin(colup[size_t(j)])) {
                        stop(kUnbounded);
                        return false;
                    }
                    fix_col(j, colup[size_t(j)]);
                } else {
                    double v = 0.0;
                    if (fin(collo[size_t(j)]) && v < collo[size_t(j)]) v = collo[size_t(j)];
                    if (fin(colup[size_t(j)]) && v > colup[size_t(j)]) v = colup[size_t(j)];
                    fix_col(j, v);
                }
                changed = true;
            }
        }
        return true;
    }

    // a forcing row: every active column to the bound that attains the
    // activity bound (src/presolve/presolve.hpp:182-203)
    template <class Touch>
    void force(int32_t i, bool at_min, Touch& touch) {
        for (int64_t k = csr.start[size_t(i)]; k < csr.start[size_t(i) + 1]; ++k) {
            const int32_t j = csr.index[size_t(k)];
            if (col_del[size_t(j)]) continue;
            const bool pos = csr.value[size_t(k)] > 0.0;
            fix_col(j, at_min ? (pos ? collo[size_t(j)] : colup[size_t(j)]) : (pos ? colup[size_t(j)] : collo[size_t(j)]));
            touch(j);
        }
        row_del[size_t(i)] = 1;
        ++res.rows_removed;
    }

    void finalize() {
        std::vector<int32_t> new_col(size_t(n), -1), new_row(size_t(m), -1);
        for (int32_t j = 0; j < n; ++j)
            if (!col_del[size_t(j)]) {
                new_col[size_t(j)] = res.ncol++;
                res.col_map.push_back(j);
            }
        for (int32_t i = 0; i < m; ++i)
            if (!row_del[size_t(i)]) {
                new_row[size_t(i)] = res.nrow++;
                res.row_map.push_back(i);
            }
        res.obj_offset = obj_offset;
        const int32_t N = res.ncol, M = res.nrow;
        res.cost.resize(size_t(N));
        res.collo.resize(size_t(N));
        res.colup.resize(size_t(N));
        res.vartype.resize(size_t(N));
        for (int32_t c = 0; c < N; ++c) {
            const int32_t j = res.col_map[size_t(c)];
            res.cost[size_t(c)] = cost[j];
            res.collo[size_t(c)] = collo[size_t(j)];
            res.colup[size_t(c)] = colup[size_t(j)];
            res.vartype[size_t(c)] = vt[size_t(j)];
        }
        res.rowlo.resize(size_t(M));
        res.rowup.resize(size_t(M));
        for (int32_t r = 0; r < M; ++r) {
            res.rowlo[size_t(r)] = rowlo[size_t(res.row_map[size_t(r)])];
            res.rowup[size_t(r)] = rowup[size_t(res.row_map[size_t(r)])];
        }
        // CscMatrix::from_triplets of the kept entries, column by column in
        // parallel: zeros dropped, rows sorted (stably), duplicates summed,
        // zero sums dropped
        std::vector<int64_t> cnt(size_t(N) + 1, 0);
        parallel_ranges(N, threads, 1 << 12, [&](int64_t a, int64_t b) {
            for (int64_t c = a; c < b; ++c) {
                const int32_t j = res.col_map[size_t(c)];
                int64_t q = 0;
                for (int64_t k = cs[j]; k < cs[j + 1]; ++k) q += !row_del[size_t(ci[k])] && cv[k] != 0.0;
                cnt[size_t(c) + 1] = q;
            }
        });
        for (int32_t c = 0; c < N; ++c) cnt[size_t(c) + 1] += cnt[size_t(c)];
        uvector<int32_t> ri(size_t(cnt[size_t(N)]));
        uvector<double> rv(size_t(cnt[size_t(N)]));
        std::vector<int64_t> kept(size_t(N), 0);
        parallel_ranges(N, threads, 1 << 12, [&](int64_t a, int64_t b) {
            std::vector<std::pair<int32_t, double>> buf;
            for (int64_t c = a; c < b; ++c) {
                const int32_t j = res.col_map[size_t(c)];
                int64_t w = cnt[size_t(c)];
                bool sorted = true;
                for (int64_t k = cs[j]; k < cs[j + 1]; ++k) {
                    if (row_del[size_t(ci[k])] || cv[k] == 0.0) continue;
                    const int32_t r = new_row[size_t(ci[k])];
                    if (w > cnt[size_t(c)] && ri[size_t(w - 1)] >= r) sorted = false;
                    ri[size_t(w)] = r;
                    rv[size_t(w)] = cv[k];
                    ++w;
                }
                const int64_t s = cnt[size_t(c)], e = w;
                if (sorted || s == e) {
                    kept[size_t(c)] = e - s;
                    continue;
                }
                buf.clear();
                for (int64_t k = s; k < e; ++k) buf.push_back({ri[size_t(k)], rv[size_t(k)]});
                std::stable_sort(buf.begin(), buf.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
                int64_t o = s;
                int32_t cur_r = buf[0].first;
                double cur_v = buf[0].second;
                for (size_t k = 1; k < buf.size(); ++k) {
                    if (buf[k].first == cur_r) {
                        cur_v += buf[k].second;
                    } else {
                        if (cur_v != 0.0) {
                            ri[size_t(o)] = cur_r;
                            rv[size_t(o)] = cur_v;
                            ++o;
                        }
                        cur_r = buf[k].first;
                        cur_v = buf[k].second;
                    }
                }
                if (cur_v != 0.0) {
                    ri[size_t(o)] = cur_r;
                    rv[size_t(o)] = cur_v;
                    ++o;
                }
                kept[size_t(c)] = o - s;
            }
        });
        bool merged = false;
        for (int32_t c = 0; c < N && !merged; ++c) merged = kept[size_t(c)] != cnt[size_t(c) + 1] - cnt[size_t(c)];
        if (!merged) {
            res.start.swap(cnt);
            res.index.swap(ri);
            res.value.swap(rv);
        } else {
            res.start.assign(size_t(N) + 1, 0);
            for (int32_t c = 0; c < N; ++c) res.start[size_t(c) + 1] = res.start[size_t(c)] + kept[size_t(c)];
            res.index.resize(size_t(res.start[size_t(N)]));
            res.value.resize(size_t(res.start[size_t(N)]));
            for (int32_t c = 0; c < N; ++c) {
                std::memcpy(res.index.data() + res.start[size_t(c)], ri.data() + cnt[size_t(c)],
                            size_t(kept[size_t(c)]) * sizeof(int32_t));
                std::memcpy(res.value.data() + res.start[size_t(c)], rv.data() + cnt[size_t(c)],
                            size_t(kept[size_t(c)]) * sizeof(double));
            }
        }
        if (res.ncol == 0 && res.nrow == 0) {
            res.solved = 1;
            res.status = kOptimal;
        }
    }

    void run(int max_rounds) {
        res.fixed_x.assign(size_t(n), 0.0);
        res.is_fixed.assign(size_t(n), 0);
        csr = csr_of(m, n, cs, ci, cv, threads);
        row_int.assign(size_t(m), 0);
        parallel_ranges(m, threads, 1 << 13, [&](int64_t a, int64_t b) {
            for (int64_t i = a; i < b; ++i)
                for (int64_t k = csr.start[size_t(i)]; k < csr.start[size_t(i) + 1] && !row_int[size_t(i)]; ++k)
                    row_int[size_t(i)] = vt[size_t(csr.index[size_t(k)])] != 0;
        });
        row_del.assign(size_t(m), 0);
        col_del.assign(size_t(n), 0);
        col_touched.assign(size_t(n), 0);
        row_valid.assign(size_t(m), 0);
        act.resize(size_t(m));
        for (int r = 0; r < max_rounds; ++r) {
            bool changed = false;
            if (!round(changed)) return;  // the reduced model stays empty
            if (!changed) break;
        }
        finalize();
    }
};

}  // namespace

extern "C" {

int nir_presolve(const nir_lp_view* lp, const int8_t* vartype, int32_t max_rounds, int32_t threads,
                 nir_presolved** out) {
    if (!out || !check_view(lp)) {
        g_err = "null or inconsistent argument";
        return 12;
    }
    *out = nullptr;
    try {
        auto r = std::make_unique<nir_presolved>();
        Presolve p(*lp, vartype, hw_threads(threads), *r);
        p.run(max_rounds);
        *out = r.release();
    } catch (const std::exception& e) {
        g_err = e.what();
        return 14;
    }
    return 0;
}

int nir_presolved_status(const nir_presolved* r, int32_t* status, int32_t* solved, int32_t* counters3) {
    if (!r) return 12;
    if (status) *status = r->status;
    if (solved) *solved = r->solved;
    if (counters3) {
        counters3[0] = r->rows_removed;
        counters3[1] = r->cols_removed;
        counters3[2] = r->tightenings;
    }
    return 0;
}

int nir_presolved_reduced(const nir_presolved* r, nir_lp_view* v, const int8_t** vartype) {
    if (!r || !v) return 12;
    v->nrow = r->nrow;
    v->ncol = r->ncol;
    v->nnz = r->start.back();
    v->col_start = r->start.data();
    v->row_index = r->index.data();
    v->value = r->value.data();
    v->cost = r->cost.data();
    v->collo = r->collo.data();
    v->colup = r->colup.data();
    v->rowlo = r->rowlo.data();
    v->rowup = r->rowup.data();
    v->obj_offset = r->obj_offset;
    if (vartype) *vartype = r->vartype.data();
    return 0;
}

int nir_presolved_maps(const nir_presolved* r, const int32_t** col_map, const int32_t** row_map,
                       const double** fixed_x, const uint8_t** is_col_fixed) {
    if (!r) return 12;
    if (col_map) *col_map = r->col_map.data();
    if (row_map) *row_map = r->row_map.data();
    if (fixed_x) *fixed_x = r->fixed_x.data();
    if (is_col_fixed) *is_col_fixed = r->is_fixed.data();
    return 0;
}

void nir_presolved_free(nir_presolved* r) { delete r; }

// ScalingInfo::round_pow2 (src/model/scaling.hpp:14-19)
static double round_pow2(double v) {
    if (v <= 0.0 || !std::isfinite(v)) return 1.0;
    int e = static_cast<int>(std::round(std::log2(v)));
    e = std::max(-30, std::min(30, e));
    return std::ldexp(1.0, e);
}

int nir_scale(const nir_lp_view* lp, const int8_t* vartype, int32_t enable, int64_t qnnz, const int64_t* q_start,
              const int32_t* q_index, const double* q_value, int32_t threads_in, double* R, double* C,
              int32_t* active, double* cost, double* collo, double* colup, double* value, double* rowlo,
              double* rowup, double* q_value_out) {
    if (!check_view(lp) || !R || !C || !active || !cost || (lp->ncol > 0 && (!collo || !colup)) ||
        (lp->nrow > 0 && (!rowlo || !rowup)) || (lp->nnz > 0 && !value) ||
        (qnnz > 0 && (!q_start || !q_index || !q_value || !q_value_out))) {
        g_err = "null or inconsistent argument";
        return 12;
    }
    const int T = hw_threads(threads_in);
    const int32_t m = lp->nrow, n = lp->ncol;
    const int64_t nnz = lp->nnz;
    const int64_t* cs = lp->col_start;
    const int32_t* ci = lp->row_index;
    const double* cv = lp->value;
    auto is_cont = [&](int32_t j) { return !vartype || vartype[j] == 0; };
    auto copy_out = [&] {
        std::copy(lp->cost, lp->cost + n, cost);
        std::copy(lp->collo, lp->collo + n, collo);
        std::copy(lp->colup, lp->colup + n, colup);
        std::copy(cv, cv + nnz, value);
        std::copy(lp->rowlo, lp->rowlo + m, rowlo);
        std::copy(lp->rowup, lp->rowup + m, rowup);
        if (qnnz > 0) std::copy(q_value, q_value + qnnz, q_value_out);
    };
    std::fill(R, R + m, 1.0);
    std::fill(C, C + n, 1.0);
    *active = 0;
    if (!enable || nnz == 0) {
        copy_out();
        return 0;
    }
    try {
        // the coefficient range (min/max: the order does not matter)
        double max_a = 0.0, min_a = kInf;
        {
            const int nt = int(std::max<int64_t>(1, std::min<int64_t>(T, nnz / 65536 + 1)));
            std::vector<double> mx(size_t(nt), 0.0), mn(size_t(nt), kInf);
            run_threads(nt, [&](int k) {
                double hi = 0.0, lo = kInf;  // in registers: the slots below share a cache line
                for (int64_t q = nnz * k / nt; q < nnz * (k + 1) / nt; ++q) {
                    const double av = std::abs(cv[q]);
                    if (av > 0.0) {
                        hi = std::max(hi, av);
                        lo = std::min(lo, av);
                    }
                }
                mx[size_t(k)] = hi;
                mn[size_t(k)] = lo;
            });
            for (int k = 0; k < nt; ++k) {
                max_a = std::max(max_a, mx[size_t(k)]);
                min_a = std::min(min_a, mn[size_t(k)]);
            }
        }
        if (min_a >= kInf || (max_a / min_a) <= 10.0) {
            copy_out();
            return 0;
        }
        *active = 1;
        const int passes = ((max_a / min_a) < 1e3) ? 2 : 6;
        std::vector<double> Rw(size_t(m), 1.0), Cw(size_t(n), 1.0);
        const Csr csr = csr_of(m, n, cs, ci, cv, T);
        for (int pass = 0; pass < passes; ++pass) {
            // rows: |a_ij| R_i C_j over each row's entries
            const int nr = int(std::max<int64_t>(1, std::min<int64_t>(T, m / 4096 + 1)));
            std::vector<double> change(size_t(std::max(nr, T)), 1.0);
            run_threads(nr, [&](int k) {
                double mc = 1.0;
                for (int64_t i = int64_t(m) * k / nr; i < int64_t(m) * (k + 1) / nr; ++i) {
                    double rmin = kInf, rmax = 0.0;
                    for (int64_t q = csr.start[size_t(i)]; q < csr.start[size_t(i) + 1]; ++q) {
                        const double v = std::abs(csr.value[size_t(q)]) * Rw[size_t(i)] * Cw[size_t(csr.index[size_t(q)])];
                        if (v > 0.0) {
                            rmin = std::min(rmin, v);
                            rmax = std::max(rmax, v);
                        }
                    }
                    if (rmax > 0.0 && rmin < kInf) {
                        const double f = 1.0 / std::sqrt(rmin * rmax);
                        mc = std::max(mc, std::max(f, 1.0 / f));
                        Rw[size_t(i)] *= f;
                    }
                }
                change[size_t(k)] = mc;
            });
            double max_change = 1.0;
            for (int k = 0; k < nr; ++k) max_change = std::max(max_change, change[size_t(k)]);
            // columns (continuous only): with the new row scales
            const int nc = int(std::max<int64_t>(1, std::min<int64_t>(T, n / 4096 + 1)));
            std::fill(change.begin(), change.end(), 1.0);
            run_threads(nc, [&](int k) {
                double mc = 1.0;
                for (int64_t j = int64_t(n) * k / nc; j < int64_t(n) * (k + 1) / nc; ++j) {
                    if (!is_cont(int32_t(j))) continue;
                    double cmin = kInf, cmax = 0.0;
                    for (int64_t q = cs[j]; q < cs[j + 1]; ++q) {
                        const double v = std::abs(cv[q]) * Rw[size_t(ci[q])] * Cw[size_t(j)];
                        if (v > 0.0) {
                            cmin = std::min(cmin, v);
                            cmax = std::max(cmax, v);
                        }
                    }
                    if (cmax > 0.0 && cmin < kInf) {
                        const double f = 1.0 / std::sqrt(cmin * cmax);
                        mc = std::max(mc, std::max(f, 1.0 / f));
                        Cw[size_t(j)] *= f;
                    }
                }
                change[size_t(k)] = mc;
            });
            for (int k = 0; k < nc; ++k) max_change = std::max(max_change, change[size_t(k)]);
            if (max_change < 1.05) break;
        }
        for (int32_t i = 0; i < m; ++i) R[i] = round_pow2(Rw[size_t(i)]);
        for (int32_t j = 0; j < n; ++j) C[j] = is_cont(j) ? round_pow2(Cw[size_t(j)]) : 1.0;
        parallel_ranges(n, T, 1 << 12, [&](int64_t a, int64_t b) {
            for (int64_t j = a; j < b; ++j) {
                const double cj = C[j];
                cost[j] = lp->cost[j] * cj;
                collo[j] = fin(lp->collo[j]) ? lp->collo[j] / cj : lp->collo[j];
                colup[j] = fin(lp->colup[j]) ? lp->colup[j] / cj : lp->colup[j];
                for (int64_t q = cs[j]; q < cs[j + 1]; ++q) value[q] = cv[q] * R[ci[q]] * cj;
            }
        });
        for (int32_t i = 0; i < m; ++i) {
            const double ri = R[i];
            rowlo[i] = fin(lp->rowlo[i]) ? lp->rowlo[i] * ri : lp->rowlo[i];
            rowup[i] = fin(lp->rowup[i]) ? lp->rowup[i] * ri : lp->rowup[i];
        }
        if (qnnz > 0)
            for (int32_t j = 0; j < n; ++j)
                for (int64_t q = q_start[j]; q < q_start[j + 1]; ++q)
                    q_value_out[q] = q_value[q] * C[q_index[q]] * C[j];
    } catch (const std::exception& e) {
        g_err = e.what();
        return 14;
    }
    return 0;
}

const char* nir_facade_last_error(void) { return g_err.c_str(); }

}  // extern "C"
