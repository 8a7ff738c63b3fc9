// Drop-in replacement for the reference's src/io/sol_io.hpp.
//
// Same names and signatures as the file it replaces
// (src/io/sol_io.hpp:14-25, :108-134): `sov::VerificationReport`,
// `sov::verify_solution(model, x, claimed_obj, tol)` and
// `sov::SolIo::write_sol / read_sol`, which the Solver (after the PDHG path
// and in its MIP/MIQP searches), the MIP solver and tools/checker.cpp call.
// The work runs in libnir_mps.so (include/nir_sol.h):
//   * verify_solution: the same report, bit for bit (double-double row
//     activities in the reference's order, in parallel over rows);
//   * write_sol: the same bytes, formatted in parallel;
//   * read_sol: the same x and objective; values are extracted as
//     `istream >> double` extracts them, and the objective goes through
//     std::stod here, so a bad objective token throws what the reference
//     throws.  The one difference: when it throws, x already holds every
//     line's value (the reference has assigned the lines before it).
// NIR_SOL_THREADS sets the thread count (default: all hardware threads).
#pragma once
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "../core/dd_real.hpp"
#include "../model/model.hpp"
#include "nir_sol.h"

namespace sov {

struct VerificationReport {
    bool passed = true;
    double max_bound_viol = 0.0;
    double max_row_viol = 0.0;
    double max_int_viol = 0.0;
    double computed_obj = 0.0;
    double obj_rel_err = 0.0;
    std::string worst_item;
};

namespace sol_detail {

inline int32_t threads() {
    const char* e = std::getenv("NIR_SOL_THREADS");
    return e ? static_cast<int32_t>(std::atoi(e)) : 0;
}

inline std::string name_of(const std::vector<std::string>& names, int64_t i) {
    return i >= 0 && static_cast<size_t>(i) < names.size() ? names[static_cast<size_t>(i)] : std::string();
}

inline nir_lp_view view_of(const Model& m) {
    nir_lp_view v;
    v.nrow = m.nrow;
    v.ncol = m.ncol;
    v.nnz = m.A.nnz();
    v.col_start = m.A.start.data();
    v.row_index = m.A.index.data();
    v.value = m.A.value.data();
    v.cost = m.cost.data();
    v.collo = m.collo.data();
    v.colup = m.colup.data();
    v.rowlo = m.rowlo.data();
    v.rowup = m.rowup.data();
    v.obj_offset = m.obj_offset;
    return v;
}

}  // namespace sol_detail

inline VerificationReport verify_solution(const Model& model, const std::vector<double>& x, double claimed_obj,
                                          double tol = 1e-6) {
    const nir_lp_view v = sol_detail::view_of(model);
    std::vector<int8_t> vt(model.vartype.size());
    for (size_t j = 0; j < vt.size(); ++j) vt[j] = static_cast<int8_t>(model.vartype[j]);
    const int64_t qnnz = model.Q.nnz();
    nir_verify_report r;
    nir_verify_solution(&v, vt.empty() ? nullptr : vt.data(), qnnz, qnnz > 0 ? model.Q.start.data() : nullptr,
                        qnnz > 0 ? model.Q.index.data() : nullptr, qnnz > 0 ? model.Q.value.data() : nullptr,
                        x.data(), static_cast<int64_t>(x.size()), claimed_obj, tol, sol_detail::threads(), &r);
    VerificationReport rep;
    rep.passed = r.passed != 0;
    rep.max_bound_viol = r.max_bound_viol;
    rep.max_row_viol = r.max_row_viol;
    rep.max_int_viol = r.max_int_viol;
    rep.computed_obj = r.computed_obj;
    rep.obj_rel_err = r.obj_rel_err;
    switch (r.worst_kind) {
        case 1: rep.worst_item = "Solution size mismatch"; break;
        case 2: rep.worst_item = "NaN/Inf in variable " + sol_detail::name_of(model.col_names, r.worst_index); break;
        case 3: rep.worst_item = "Lower bound on " + sol_detail::name_of(model.col_names, r.worst_index); break;
        case 4: rep.worst_item = "Upper bound on " + sol_detail::name_of(model.col_names, r.worst_index); break;
        case 5: rep.worst_item = "Integrality on " + sol_detail::name_of(model.col_names, r.worst_index); break;
        case 6: rep.worst_item = "Row lower bound on " + sol_detail::name_of(model.row_names, r.worst_index); break;
        case 7: rep.worst_item = "Row upper bound on " + sol_detail::name_of(model.row_names, r.worst_index); break;
        default: break;
    }
    return rep;
}

class SolIo {
public:
    static bool write_sol(const std::string& path, const Model& model, Status status, double obj, double gap,
                          const std::vector<double>& x) {
        std::vector<const char*> names(model.col_names.size());
        for (size_t j = 0; j < names.size(); ++j) names[j] = model.col_names[j].c_str();
        return nir_sol_write(path.c_str(), status_to_string(status), obj, gap, model.ncol, x.data(),
                             static_cast<int64_t>(x.size()), names.empty() ? nullptr : names.data(),
                             static_cast<int64_t>(names.size()), sol_detail::threads()) == 0;
    }

    static bool read_sol(const std::string& path, const Model& model, Status& out_status, double& out_obj,
                         std::vector<double>& out_x) {
        std::vector<const char*> names(static_cast<size_t>(model.ncol), "");
        for (Idx j = 0; j < model.ncol && static_cast<size_t>(j) < model.col_names.size(); ++j)
            names[static_cast<size_t>(j)] = model.col_names[static_cast<size_t>(j)].c_str();
        std::vector<double> x(static_cast<size_t>(model.ncol), 0.0);
        double obj = 0.0;
        int32_t nobj = 0;
        const int st = nir_sol_read(path.c_str(), model.ncol, names.empty() ? nullptr : names.data(),
                                    sol_detail::threads(), x.data(), &obj, &nobj);
        if (st == 14) return false;
        out_x = std::move(x);
        out_status = Status::Optimal;
        out_obj = 0.0;
        for (int32_t k = 0; k < nobj; ++k) out_obj = std::stod(nir_sol_objective_token(k));
        return true;
    }
};

}  // namespace sov
