// Drop-in replacement for the reference's src/gpu/pdhg_solver.hpp.
//
// Same names and signature as the file it replaces
// (src/gpu/pdhg_solver.hpp:14-25): `sov::PdhgResult` and
// `sov::PdhgSolver::solve(const Model&, const Options&, const Deadline&)`,
// so Solver::solve (include/sov/solver.hpp:235-244), the CLI's
// `--method pdhg` and the C API's `method=pdhg` reach the B200 engine
// unchanged.  The body hands the model's CSC matrix and vectors as they are
// to libnir_pdhg.so through its C ABI (include/nir_pdhg.h) and maps the
// result back:
//   * the iteration cap follows the reference's rule
//     max(5000, simplex_iter_limit / 10) (src/gpu/pdhg_solver.hpp:60),
//     scaled by 10 for the restarted method, whose iterations it replaces;
//   * the Deadline (stop flag, wall clock) is polled between launch chunks,
//     as src/gpu/pdhg_solver.hpp:63 polls it every 256 iterations;
//   * the objective is the model's own dd_real eval_objective
//     (src/model/model.hpp:73-98), as at src/gpu/pdhg_solver.hpp:105;
//   * statuses are honest: IterationLimit and NumericalTrouble are reported
//     as such (the reference reports Optimal at its cap).  The one exception
//     is a point that meets 1e-6 relative KKT at the cap but not yet the row
//     margin below: it is Optimal, and Solver's dd check has the last word;
//   * the solve stops at 1e-6 relative KKT and, so that Solver's dd_real
//     verification passes, at a per-row relative violation of at most
//     0.1 * tol.checker_tol.
//   * the scales of scale_model (which Solver applies just before) are
//     undone exactly before the engine runs and the solution is mapped
//     back: the engine preconditions by itself, and power-of-two
//     equilibration ahead of it slows the restarted PDHG's duality gap;
//   * when only that row margin is missing at the cap, the solve goes on
//     once in FP64 on the GPU from the point it reached (the retry that
//     Solver's presolve-less fallback would otherwise make from scratch);
//   * optionally, a crossover turns the engine's point into a vertex: a
//     basis is read off the point and the program's own simplex
//     (sov::LpSolver) is warm-started from it (nir::dropin::crossover
//     below).
// Environment knobs (no Options field is added, so options.hpp stays as
// it is): NIR_PDHG_ALGO = pdlp | pdhg | reference, NIR_PDHG_PRECISION =
// mixed | fp64 | fp32, NIR_PDHG_TOL, NIR_PDHG_MAX_ITERS, NIR_PDHG_DEVICE,
// NIR_PDHG_KEEP_SCALING=1 (solve the scaled model as given), NIR_PDHG_RETRY=0
// (no FP64 retry on the GPU when only the row margin is missing at the cap),
// NIR_PDHG_CROSSOVER = 1 (after every solve) | auto (when the engine stops
// short of Optimal), NIR_PDHG_CROSSOVER_TOL (relative distance at which a
// value sits at its bound, default 1e-6), NIR_PDHG_CROSSOVER_METHOD =
// primal (default) | dual (the simplex that finishes the crossover).
// There is no CPU fallback: an engine error is thrown as
// std::runtime_error, which the C API turns into its -1 + last_error.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../core/options.hpp"
#include "../core/status.hpp"
#include "../core/timer.hpp"
#include "../core/types.hpp"
#include "../lp/lp_solver.hpp"
#include "../model/model.hpp"
#include "nir_pdhg.h"
#include "nir_sov_glue.hpp"

namespace nir {
namespace dropin {

// The result of a crossover from an approximate LP optimum to a vertex.
struct CrossoverResult {
    sov::Status status = sov::Status::NumericalTrouble;
    std::vector<double> x;           // the vertex (model columns)
    std::vector<double> y;           // row duals, as LpSolver gives them to Solver
    sov::Idx simplex_iterations = 0;
    sov::Idx crash_structurals = 0;  // structural columns in the crash basis
};

// Crossover: from (x, y), an approximate optimum of `model`, to an optimal
// vertex.
//   1. The crash basis, by complementarity.  For every column and every row
//      logical (whose value is the row activity), two measures:
//      - p, its relative distance to the nearer bound (0 within tol, inf
//        when free);
//      - q, its reduced cost over a common dual scale: c_j - (A'y)_j for a
//        column, y_i for a row.
//      A basic variable has p large and q near zero; a nonbasic one the
//      reverse.  Ranked by p / (p + q), ties by q ascending, the first nrow
//      are basic.  The others sit at their nearer bound.
//   2. The program's own simplex (sov::LpSolver, src/lp/lp_solver.hpp) is
//      warm-started from that basis (set_basis, :896-907) and solves to
//      optimality, by default with its primal simplex (:576).  Its
//      factorisation swaps logicals in for dependent columns (:183-212).
// Near an optimum most of the basis is already right, so few pivots are
// left to make.
inline CrossoverResult crossover(const sov::Model& model, const std::vector<double>& x, const std::vector<double>& y,
                                 const sov::Options& opt, const sov::Deadline& deadline, double tol,
                                 const char* method = "primal") {
    using sov::Idx;
    using sov::VarStatus;
    const Idx n = model.ncol, m = model.nrow;
    std::vector<double> act(size_t(m), 0.0), d(model.cost.begin(), model.cost.end());
    for (Idx j = 0; j < n; ++j)
        for (sov::Off k = model.A.start[size_t(j)]; k < model.A.start[size_t(j) + 1]; ++k) {
            const size_t i = size_t(model.A.index[size_t(k)]);
            act[i] += model.A.value[size_t(k)] * x[size_t(j)];
            d[size_t(j)] -= model.A.value[size_t(k)] * y[i];
        }
    double dscale = 0.0;
    for (double c : model.cost) dscale = std::max(dscale, std::abs(c));
    for (double v : y) dscale = std::max(dscale, std::abs(v));
    dscale += 1.0;
    struct Key {
        double r, q;
        Idx v;
    };
    std::vector<Key> keys;
    keys.reserve(size_t(n + m));
    std::vector<VarStatus> st(size_t(n + m));
    for (Idx v = 0; v < n + m; ++v) {
        const bool col = v < n;
        const size_t i = size_t(col ? v : v - n);
        const double val = col ? x[i] : act[i];
        const double lo = col ? model.collo[i] : model.rowlo[i], up = col ? model.colup[i] : model.rowup[i];
        const bool fl = sov::is_finite_bound(lo), fu = sov::is_finite_bound(up);
        const double dl = fl ? (val - lo) / (1.0 + std::abs(lo)) : sov::kInf;
        const double du = fu ? (up - val) / (1.0 + std::abs(up)) : sov::kInf;
        // the place of a nonbasic variable: the nearer finite bound
        if (fl && fu && lo == up) st[size_t(v)] = VarStatus::Fixed;
        else if (!fl && !fu) st[size_t(v)] = VarStatus::FreeZero;
        else st[size_t(v)] = (fl && dl <= du) ? VarStatus::AtLower : VarStatus::AtUpper;
        double p = std::min(dl, du);
        if (p <= tol) p = 0.0;
        const double q = std::abs(col ? d[i] : y[i]) / dscale;
        double r;
        if (st[size_t(v)] == VarStatus::Fixed) r = -1.0;
        else if (!std::isfinite(p)) r = 1.0;
        else r = p > 0.0 ? p / (p + q) : 0.0;
        keys.push_back({r, q, v});
    }
    std::stable_sort(keys.begin(), keys.end(), [](const Key& a, const Key& b) {
        return a.r > b.r || (a.r == b.r && a.q < b.q);
    });
    sov::BasisSnapshot snap;
    CrossoverResult r;
    for (size_t k = 0; k < size_t(m); ++k) {
        st[size_t(keys[k].v)] = VarStatus::Basic;
        snap.basic_index.push_back(keys[k].v);
        if (keys[k].v < n) ++r.crash_structurals;
    }
    snap.status = st;
    sov::Options lp_opt = opt;
    // "primal" (the default): LpSolver's primal simplex, which starts from
    // the crash basis's nearly feasible point.  Otherwise its dual path,
    // whose artificial-bounds phase 1 can wander off a basis with small
    // dual infeasibilities.
    if (method && *method) lp_opt.method = method;
    sov::LpSolver lp(lp_opt);
    lp.load(model);
    lp.set_basis(snap);
    r.status = lp.solve(deadline);
    r.simplex_iterations = lp.stats.iterations;
    r.x.assign(lp.value.begin(), lp.value.begin() + n);
    r.y = lp.row_duals;
    return r;
}

}  // namespace dropin
}  // namespace nir

namespace sov {

struct PdhgResult {
    Status status = Status::Optimal;
    double objective = 0.0;
    std::vector<double> x;
    std::vector<double> y;
    Idx iterations = 0;
};

class PdhgSolver {
public:
    static PdhgResult solve(const Model& model, const Options& opt, const Deadline& deadline) {
        PdhgResult res;
        nir_lp_view lp;
        std::memset(&lp, 0, sizeof(lp));
        lp.nrow = model.nrow;
        lp.ncol = model.ncol;
        lp.nnz = model.A.nnz();
        lp.col_start = model.A.start.data();
        lp.row_index = model.A.index.data();
        lp.value = model.A.value.data();
        lp.cost = model.cost.data();
        lp.collo = model.collo.data();
        lp.colup = model.colup.data();
        lp.rowlo = model.rowlo.data();
        lp.rowup = model.rowup.data();
        lp.obj_offset = model.obj_offset;

        // Undo the scales of the scale_model call that produced this model
        // (Solver scales, then calls here), exactly: they are powers of two.
        // The engine preconditions by itself, and the relative KKT, the row
        // margin and Solver's check then all refer to the same space.
        // NIR_PDHG_KEEP_SCALING=1 solves the model as given.
        const nir::sov_glue::LastScaling& sc = nir::sov_glue::last_scaling();
        const bool undo = sc.active && sc.R.size() == size_t(model.nrow) && sc.C.size() == size_t(model.ncol) &&
                          env_int("NIR_PDHG_KEEP_SCALING", 0) == 0;
        std::vector<double> uc, ulo, uup, uval, url, uru;
        if (undo) {
            uc.resize(size_t(model.ncol));
            ulo.resize(size_t(model.ncol));
            uup.resize(size_t(model.ncol));
            uval.resize(size_t(lp.nnz));
            for (Idx j = 0; j < model.ncol; ++j) {
                const double cj = sc.C[size_t(j)];
                uc[size_t(j)] = model.cost[size_t(j)] / cj;
                ulo[size_t(j)] = is_finite_bound(model.collo[size_t(j)]) ? model.collo[size_t(j)] * cj : model.collo[size_t(j)];
                uup[size_t(j)] = is_finite_bound(model.colup[size_t(j)]) ? model.colup[size_t(j)] * cj : model.colup[size_t(j)];
                for (Off k = model.A.start[size_t(j)]; k < model.A.start[size_t(j) + 1]; ++k)
                    uval[size_t(k)] = model.A.value[size_t(k)] / sc.R[size_t(model.A.index[size_t(k)])] / cj;
            }
            url.resize(size_t(model.nrow));
            uru.resize(size_t(model.nrow));
            for (Idx i = 0; i < model.nrow; ++i) {
                const double ri = sc.R[size_t(i)];
                url[size_t(i)] = is_finite_bound(model.rowlo[size_t(i)]) ? model.rowlo[size_t(i)] / ri : model.rowlo[size_t(i)];
                uru[size_t(i)] = is_finite_bound(model.rowup[size_t(i)]) ? model.rowup[size_t(i)] / ri : model.rowup[size_t(i)];
            }
            lp.cost = uc.data();
            lp.collo = ulo.data();
            lp.colup = uup.data();
            lp.value = uval.data();
            lp.rowlo = url.data();
            lp.rowup = uru.data();
        }

        nir_pdhg_params p;
        nir_pdhg_default_params(&p);
        const long long ref_cap = std::max<long long>(5000, static_cast<long long>(opt.simplex_iter_limit) / 10);
        p.max_iters = 10 * ref_cap;
        p.feas_tol = 0.1 * opt.tol.checker_tol;
        apply_env(p, ref_cap);

        res.x.assign(model.ncol, 0.0);
        res.y.assign(model.nrow, 0.0);
        nir_pdhg_info info;
        const int device = env_int("NIR_PDHG_DEVICE", 0);
        int st = nir_pdhg_solve_lp(&lp, device, &p, &poll_deadline, const_cast<Deadline*>(&deadline), res.x.data(),
                                   res.y.data(), &info);
        if (st == NIR_STATUS_INPUT_ERROR || st == NIR_STATUS_INTERNAL_ERROR)
            throw std::runtime_error(std::string("B200 PDHG engine: ") + nir_pdhg_last_error());
        // The FP64 retry on the GPU.  When the solve met the relative KKT but
        // not the row margin at its cap (the case in which Solver's dd check
        // can fail and its fallback re-runs everything presolve-less,
        // include/sov/solver.hpp:283-296), it goes on once in FP64 from the
        // point it reached, with its primal weight and a second cap.  The
        // retry's point replaces the first only if it meets the KKT
        // tolerance.  NIR_PDHG_RETRY=0 turns it off.
        if (st == NIR_STATUS_ITERATION_LIMIT && p.feas_tol > 0.0 && info.rel_kkt <= p.tol &&
            p.algorithm != NIR_ALGO_REFERENCE && env_int("NIR_PDHG_RETRY", 1) != 0 && !deadline.expired()) {
            nir_pdhg_params q = p;
            q.precision = NIR_PREC_FP64;
            const std::vector<double> x0 = res.x, y0 = res.y;
            q.x_init = x0.data();
            q.y_init = y0.data();
            q.omega_init = info.primal_weight;
            nir_pdhg_info info2;
            const int st2 = nir_pdhg_solve_lp(&lp, device, &q, &poll_deadline, const_cast<Deadline*>(&deadline),
                                              res.x.data(), res.y.data(), &info2);
            if (st2 == NIR_STATUS_INPUT_ERROR || st2 == NIR_STATUS_INTERNAL_ERROR)
                throw std::runtime_error(std::string("B200 PDHG engine: ") + nir_pdhg_last_error());
            if (st2 == NIR_STATUS_OPTIMAL || info2.rel_kkt <= p.tol) {
                info2.iterations += info.iterations;
                info = info2;
                st = st2;
            } else {
                res.x = x0;
                res.y = y0;
                info.iterations += info2.iterations;
            }
        }
        res.status = static_cast<Status>(st);
        // The engine iterates until the relative KKT is below tol and, as a
        // margin for Solver's double-double check, every row's relative
        // violation is below feas_tol.  When only that margin is missing at
        // the cap, the point meets the PDHG criterion: it is reported Optimal
        // and Solver's verification (include/sov/solver.hpp:283) judges the
        // rows, as it does for the reference's own PDHG.
        if (st == NIR_STATUS_ITERATION_LIMIT && p.feas_tol > 0.0 && info.rel_kkt <= p.tol)
            res.status = Status::Optimal;
        res.iterations = static_cast<Idx>(std::min<int64_t>(info.iterations, 2147483647));
        if (undo) {  // back to the variables of the model given: x / C, y / R
            for (Idx j = 0; j < model.ncol; ++j) res.x[size_t(j)] /= sc.C[size_t(j)];
            for (Idx i = 0; i < model.nrow; ++i) res.y[size_t(i)] /= sc.R[size_t(i)];
        }
        // Crossover to a vertex of the model given, when asked for.  Its
        // result replaces the engine's only when the simplex proves it
        // optimal; its pivots count as iterations.
        const char* xo = std::getenv("NIR_PDHG_CROSSOVER");
        const std::string mode = xo ? xo : "";
        bool finite = true;
        for (double v : res.x) finite = finite && std::isfinite(v);
        for (double v : res.y) finite = finite && std::isfinite(v);
        if ((mode == "1" || (mode == "auto" && res.status != Status::Optimal)) && model.nrow > 0 && finite &&
            res.status != Status::TimeLimit && !deadline.expired()) {
            const char* t = std::getenv("NIR_PDHG_CROSSOVER_TOL");
            const char* how = std::getenv("NIR_PDHG_CROSSOVER_METHOD");
            const nir::dropin::CrossoverResult c = nir::dropin::crossover(
                model, res.x, res.y, opt, deadline, t && *t ? std::atof(t) : 1e-6, how && *how ? how : "primal");
            if (c.status == Status::Optimal) {
                res.x = c.x;
                res.y = c.y;
                res.status = Status::Optimal;
            }
            res.iterations += c.simplex_iterations;
        }
        res.objective = model.eval_objective(res.x);
        return res;
    }

private:
    static int poll_deadline(void* ctx) { return static_cast<const Deadline*>(ctx)->expired() ? 1 : 0; }

    static int env_int(const char* k, int dflt) {
        const char* v = std::getenv(k);
        return (v && *v) ? std::atoi(v) : dflt;
    }

    static void apply_env(nir_pdhg_params& p, long long ref_cap) {
        if (const char* a = std::getenv("NIR_PDHG_ALGO")) {
            const std::string s(a);
            if (s == "reference") {
                p.algorithm = NIR_ALGO_REFERENCE;
                p.max_iters = ref_cap;
            } else if (s == "pdhg") {
                p.algorithm = NIR_ALGO_PDHG;
            } else if (s == "pdlp") {
                p.algorithm = NIR_ALGO_PDLP;
            }
        }
        if (const char* a = std::getenv("NIR_PDHG_PRECISION")) {
            const std::string s(a);
            if (s == "fp64") p.precision = NIR_PREC_FP64;
            else if (s == "fp32") p.precision = NIR_PREC_FP32;
            else if (s == "mixed") p.precision = NIR_PREC_MIXED;
        }
        if (const char* a = std::getenv("NIR_PDHG_TOL")) p.tol = std::atof(a);
        if (const char* a = std::getenv("NIR_PDHG_MAX_ITERS")) p.max_iters = std::atoll(a);
    }
};

}  // namespace sov
