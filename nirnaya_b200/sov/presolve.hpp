// Drop-in replacement for the reference's src/presolve/presolve.hpp.
//
// Same names and signatures as the file it replaces
// (src/presolve/presolve.hpp:9-32): `sov::PresolveResult` (with postsolve)
// and `sov::Presolver::presolve(const Model&, int level, int max_rounds)`,
// which Solver::solve calls before dispatching to PDHG
// (include/sov/solver.hpp:159).  Level <= 0 and models with a quadratic
// block are copied through unchanged, as the reference does.  Otherwise the
// rounds run in libnir_facade.so (include/nir_facade.h), on all host
// threads, or NIR_FACADE_THREADS.  The reduced model, the maps, the fixed
// values, the counters and the status are the reference's, bit for bit.
// Names come from the original model through the maps; the reduced model is
// called name + "_pre".
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>

#include "../model/model.hpp"
#include "nir_facade.h"

namespace sov {

struct PresolveResult {
    Status status = Status::Optimal;  // Optimal: continue with the reduced model, or solved in presolve
    bool solved_in_presolve = false;
    Model reduced;
    std::vector<Idx> orig_col_map;  // reduced col j -> original col idx
    std::vector<Idx> orig_row_map;  // reduced row i -> original row idx
    std::vector<double> fixed_x;    // size orig.ncol
    std::vector<bool> is_col_fixed;
    Idx rows_removed = 0;
    Idx cols_removed = 0;
    Idx bound_tightenings = 0;

    void postsolve(const std::vector<double>& x_red, std::vector<double>& x_orig) const {
        x_orig = fixed_x;
        for (size_t j = 0; j < orig_col_map.size() && j < x_red.size(); ++j) x_orig[size_t(orig_col_map[j])] = x_red[j];
    }
};

class Presolver {
public:
    static PresolveResult presolve(const Model& orig, int level, int max_rounds = 20) {
        PresolveResult res;
        res.fixed_x.assign(size_t(orig.ncol), 0.0);
        res.is_col_fixed.assign(size_t(orig.ncol), false);
        if (level <= 0 || orig.is_qp()) {
            res.reduced = orig;
            res.orig_col_map.resize(size_t(orig.ncol));
            for (Idx j = 0; j < orig.ncol; ++j) res.orig_col_map[size_t(j)] = j;
            res.orig_row_map.resize(size_t(orig.nrow));
            for (Idx i = 0; i < orig.nrow; ++i) res.orig_row_map[size_t(i)] = i;
            return res;
        }
        nir_lp_view v;
        v.nrow = orig.nrow;
        v.ncol = orig.ncol;
        v.nnz = orig.A.nnz();
        v.col_start = orig.A.start.data();
        v.row_index = orig.A.index.data();
        v.value = orig.A.value.data();
        v.cost = orig.cost.data();
        v.collo = orig.collo.data();
        v.colup = orig.colup.data();
        v.rowlo = orig.rowlo.data();
        v.rowup = orig.rowup.data();
        v.obj_offset = orig.obj_offset;
        std::vector<int8_t> vt(size_t(orig.ncol));
        for (Idx j = 0; j < orig.ncol; ++j) vt[size_t(j)] = static_cast<int8_t>(orig.vartype[size_t(j)]);
        const char* env = std::getenv("NIR_FACADE_THREADS");
        nir_presolved* h = nullptr;
        if (nir_presolve(&v, vt.data(), max_rounds, env ? std::atoi(env) : 0, &h) != 0)
            throw std::runtime_error(std::string("presolve: ") + nir_facade_last_error());
        int32_t st = 0, solved = 0, cnt[3] = {0, 0, 0};
        nir_presolved_status(h, &st, &solved, cnt);
        res.status = static_cast<Status>(st);
        res.solved_in_presolve = solved != 0;
        res.rows_removed = cnt[0];
        res.cols_removed = cnt[1];
        res.bound_tightenings = cnt[2];
        const int32_t* cm = nullptr;
        const int32_t* rm = nullptr;
        const double* fx = nullptr;
        const uint8_t* isf = nullptr;
        nir_presolved_maps(h, &cm, &rm, &fx, &isf);
        res.fixed_x.assign(fx, fx + orig.ncol);
        for (Idx j = 0; j < orig.ncol; ++j) res.is_col_fixed[size_t(j)] = isf[j] != 0;
        const bool stopped = res.solved_in_presolve && res.status != Status::Optimal;
        if (!stopped) {  // an infeasible or unbounded stop leaves the reduced model empty
            nir_lp_view r;
            const int8_t* rvt = nullptr;
            nir_presolved_reduced(h, &r, &rvt);
            Model red;
            red.name = orig.name + "_pre";
            red.sense = orig.sense;
            red.obj_offset = r.obj_offset;
            red.ncol = r.ncol;
            red.nrow = r.nrow;
            res.orig_col_map.assign(cm, cm + r.ncol);
            res.orig_row_map.assign(rm, rm + r.nrow);
            red.cost.assign(r.cost, r.cost + r.ncol);
            red.collo.assign(r.collo, r.collo + r.ncol);
            red.colup.assign(r.colup, r.colup + r.ncol);
            red.vartype.resize(size_t(r.ncol));
            red.col_names.resize(size_t(r.ncol));
            for (Idx j = 0; j < r.ncol; ++j) {
                red.vartype[size_t(j)] = static_cast<VarType>(rvt[j]);
                if (size_t(cm[j]) < orig.col_names.size()) red.col_names[size_t(j)] = orig.col_names[size_t(cm[j])];
            }
            red.rowlo.assign(r.rowlo, r.rowlo + r.nrow);
            red.rowup.assign(r.rowup, r.rowup + r.nrow);
            red.row_names.resize(size_t(r.nrow));
            for (Idx i = 0; i < r.nrow; ++i)
                if (size_t(rm[i]) < orig.row_names.size()) red.row_names[size_t(i)] = orig.row_names[size_t(rm[i])];
            red.A = CscMatrix(r.nrow, r.ncol);
            red.A.start.assign(r.col_start, r.col_start + r.ncol + 1);
            red.A.index.assign(r.row_index, r.row_index + r.nnz);
            red.A.value.assign(r.value, r.value + r.nnz);
            red.Q = CscMatrix(r.ncol, r.ncol);
            res.reduced = std::move(red);
        }
        nir_presolved_free(h);
        return res;
    }
};

}  // namespace sov
