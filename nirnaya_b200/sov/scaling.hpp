// Drop-in replacement for the reference's src/model/scaling.hpp.
//
// Same names and signatures as the file it replaces
// (src/model/scaling.hpp:9-56): `sov::ScalingInfo` (round_pow2 and the
// three unscale helpers, unchanged) and `sov::scale_model(const Model&,
// bool, ScalingInfo&)`, which Solver::solve calls on the presolved model
// before PDHG (include/sov/solver.hpp:180-181).  The equilibration runs in
// libnir_facade.so (nir_scale, include/nir_facade.h) on all host threads
// or NIR_FACADE_THREADS.  Its scales and scaled arrays are the reference's,
// bit for bit.  The scales are also recorded (include/nir_sov_glue.hpp) for
// the drop-in PdhgSolver, which undoes them before the GPU engine runs.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>

#include "model.hpp"
#include "nir_facade.h"
#include "nir_sov_glue.hpp"

namespace sov {

struct ScalingInfo {
    bool active = false;
    std::vector<double> R;  // Row scales (m)
    std::vector<double> C;  // Col scales (n)

    static double round_pow2(double v) {
        if (v <= 0.0 || !std::isfinite(v)) return 1.0;
        int exp = static_cast<int>(std::round(std::log2(v)));
        exp = std::max(-30, std::min(30, exp));
        return std::ldexp(1.0, exp);
    }

    void unscale_primal(const std::vector<double>& x_scaled, std::vector<double>& x_orig) const {
        x_orig.resize(x_scaled.size());
        if (!active) {
            x_orig = x_scaled;
            return;
        }
        for (size_t j = 0; j < x_scaled.size(); ++j) x_orig[j] = x_scaled[j] * C[j];
    }

    void unscale_row_duals(const std::vector<double>& y_scaled, std::vector<double>& y_orig) const {
        y_orig.resize(y_scaled.size());
        if (!active) {
            y_orig = y_scaled;
            return;
        }
        for (size_t i = 0; i < y_scaled.size(); ++i) y_orig[i] = y_scaled[i] * R[i];
    }

    void unscale_reduced_costs(const std::vector<double>& d_scaled, std::vector<double>& d_orig) const {
        d_orig.resize(d_scaled.size());
        if (!active) {
            d_orig = d_scaled;
            return;
        }
        for (size_t j = 0; j < d_scaled.size(); ++j) d_orig[j] = d_scaled[j] / C[j];
    }
};

inline Model scale_model(const Model& orig, bool enable_scaling, ScalingInfo& info) {
    info.R.assign(size_t(orig.nrow), 1.0);
    info.C.assign(size_t(orig.ncol), 1.0);
    info.active = false;
    nir::sov_glue::LastScaling& last = nir::sov_glue::last_scaling();  // read by the drop-in PdhgSolver
    last.active = false;
    if (!enable_scaling || orig.A.nnz() == 0) return orig;
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
    Model scaled = orig;
    const int64_t qnnz = orig.Q.nnz();
    const char* env = std::getenv("NIR_FACADE_THREADS");
    int32_t active = 0;
    const int st = nir_scale(&v, vt.data(), 1, qnnz, qnnz > 0 ? orig.Q.start.data() : nullptr,
                             qnnz > 0 ? orig.Q.index.data() : nullptr, qnnz > 0 ? orig.Q.value.data() : nullptr,
                             env ? std::atoi(env) : 0, info.R.data(), info.C.data(), &active, scaled.cost.data(),
                             scaled.collo.data(), scaled.colup.data(), scaled.A.value.data(), scaled.rowlo.data(),
                             scaled.rowup.data(), qnnz > 0 ? scaled.Q.value.data() : nullptr);
    if (st != 0) throw std::runtime_error(std::string("scale_model: ") + nir_facade_last_error());
    info.active = active != 0;
    last.active = info.active;
    last.R = info.R;
    last.C = info.C;
    return scaled;
}

}  // namespace sov
