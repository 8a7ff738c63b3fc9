// Checks the drop-in PdhgSolver's crossover (nir::dropin::crossover in
// nirnaya_b200/sov/pdhg_solver.hpp) without a GPU.  The engine entry point is
// replaced by a stand-in for PDLP.  It solves the LP it is given with the
// program's own simplex and returns that optimum perturbed by about 1e-8
// relative, clipped into the bounds: an approximate optimum of the kind the
// engine stops at.  Built against a tree of the reference's headers with the
// drop-in headers linked in (tests/test_dropin.py).
//
// The checks, on the reference's own known-answer LPs
// (tests/unit_tests.cpp:115-142 and :316-331, tools/bench_runner.cpp:24-39)
// and on seeded random LPs:
//   1. crossover from the perturbed point reaches the simplex's optimal
//      objective, with a passing dd_real verification at 1e-9;
//   2. it takes fewer simplex iterations than the simplex from its slack
//      basis;
//   3. through Solver::solve with method=pdhg and NIR_PDHG_CROSSOVER=1, with
//      presolve and scaling on and off, the result passes Solver's own
//      check.  On the worked example it gives x = (3, 1) and the simplex's
//      duals (1.5, 0.5);
//   4. NIR_PDHG_CROSSOVER=auto runs only when the engine stopped short of
//      Optimal, and then turns its IterationLimit into Optimal;
//   5. from real PDHG iterates (the reference loop run to 1e-6 relative KKT
//      by the oracle), crossover reaches the simplex's optimum.
// Prints one line per model, then "ok" and exits 0.  Otherwise it names the
// first failed check and exits 1.
//
// With the argument "c1" (or "measure <kind> <seed> [m]") it measures
// instead, on the C1 model (random_eq_2000x5000, seed 1) or the generator
// model named.  It runs the reference loop (oracle) for its own cap and for
// six times that, crosses over from each point (240 s limit), and times the
// simplex from its slack basis (300 s limit).
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "include/sov/solver.hpp"
#include "nir_lpgen.h"   // the seeded generator of the benchmark models
#include "nir_oracle.h"  // the reference PDHG loop restated in C, for a real PDHG iterate

namespace {

int g_status = NIR_STATUS_OPTIMAL;  // what the stand-in engine reports

sov::Model model_from(const nir_lp_view* lp) {
    sov::Model m;
    m.ncol = lp->ncol;
    m.nrow = lp->nrow;
    m.obj_offset = lp->obj_offset;
    m.cost.assign(lp->cost, lp->cost + lp->ncol);
    m.collo.assign(lp->collo, lp->collo + lp->ncol);
    m.colup.assign(lp->colup, lp->colup + lp->ncol);
    m.rowlo.assign(lp->rowlo, lp->rowlo + lp->nrow);
    m.rowup.assign(lp->rowup, lp->rowup + lp->nrow);
    m.vartype.assign(size_t(lp->ncol), sov::VarType::Continuous);
    m.A = sov::CscMatrix(lp->nrow, lp->ncol);
    m.A.start.assign(lp->col_start, lp->col_start + lp->ncol + 1);
    m.A.index.assign(lp->row_index, lp->row_index + lp->nnz);
    m.A.value.assign(lp->value, lp->value + lp->nnz);
    return m;
}

// The simplex optimum of `m`, perturbed by ~eps relative and clipped into
// the bounds.  Returns the simplex's iteration count.
long long approximate_optimum(const sov::Model& m, std::vector<double>& x, std::vector<double>& y,
                              double eps = 1e-8) {
    sov::Options o;
    o.log_level = 0;
    sov::LpSolver lp(o);
    lp.load(m);
    sov::Deadline dl;
    if (lp.solve(dl) != sov::Status::Optimal) return -1;
    x.assign(lp.value.begin(), lp.value.begin() + m.ncol);
    y = lp.row_duals;
    for (sov::Idx j = 0; j < m.ncol; ++j) {
        double v = x[size_t(j)] + eps * (1.0 + std::abs(x[size_t(j)])) * std::sin(1.0 + 7.0 * j);
        if (sov::is_finite_bound(m.collo[size_t(j)])) v = std::max(v, m.collo[size_t(j)]);
        if (sov::is_finite_bound(m.colup[size_t(j)])) v = std::min(v, m.colup[size_t(j)]);
        x[size_t(j)] = v;
    }
    for (size_t i = 0; i < y.size(); ++i) y[i] *= 1.0 + eps * std::cos(3.0 + i);
    return lp.stats.iterations;
}

}  // namespace

extern "C" int nir_pdhg_default_params(nir_pdhg_params* p) {
    std::memset(p, 0, sizeof(*p));
    p->tol = 1e-6;
    return 0;
}

extern "C" int nir_pdhg_solve_lp(const nir_lp_view* lp, int, const nir_pdhg_params*, int (*)(void*), void*,
                                 double* x, double* y, nir_pdhg_info* info) {
    std::vector<double> xa, ya;
    if (approximate_optimum(model_from(lp), xa, ya) < 0) return NIR_STATUS_NUMERICAL_TROUBLE;
    std::memcpy(x, xa.data(), xa.size() * sizeof(double));
    std::memcpy(y, ya.data(), ya.size() * sizeof(double));
    std::memset(info, 0, sizeof(*info));
    info->iterations = 7;
    info->rel_kkt = 1e-3;  // far from tolerance: the drop-in must not call this Optimal by itself
    return g_status;
}

extern "C" const char* nir_pdhg_last_error(void) { return ""; }

static int fail(const char* model, const char* what) {
    std::printf("failed: %s: %s\n", model, what);
    return 1;
}

static sov::Model appendix_a5() {  // tests/unit_tests.cpp:115-142
    sov::ModelBuilder mb("Appendix_A5");
    const sov::Idx x1 = mb.add_col(2.0, 0.0, sov::kInf), x2 = mb.add_col(3.0, 0.0, sov::kInf);
    mb.add_row(4.0, sov::kInf, {x1, x2}, {1.0, 1.0});
    mb.add_row(6.0, sov::kInf, {x1, x2}, {1.0, 3.0});
    return mb.finalize();
}

static sov::Model pdhg_lp() {  // tests/unit_tests.cpp:316-331
    sov::ModelBuilder mb("PDHG_LP");
    const sov::Idx x1 = mb.add_col(2.0, 0.0, 20.0), x2 = mb.add_col(3.0, 0.0, 20.0);
    mb.add_row(4.0, 20.0, {x1, x2}, {1.0, 1.0});
    mb.add_row(6.0, 30.0, {x1, x2}, {1.0, 3.0});
    return mb.finalize();
}

static sov::Model transport() {  // tools/bench_runner.cpp:24-39, optimum 13
    sov::ModelBuilder mb("Degenerate_Transport_LP");
    const int N = 5;
    std::vector<std::vector<sov::Idx>> f(N, std::vector<sov::Idx>(N));
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) f[size_t(i)][size_t(j)] = mb.add_col(double((i + 1) * (j + 2) % 7 + 1), 0.0, 1.0);
    for (int i = 0; i < N; ++i) {
        mb.add_row(1.0, 1.0, f[size_t(i)], std::vector<double>(N, 1.0));
        std::vector<sov::Idx> c;
        for (int r = 0; r < N; ++r) c.push_back(f[size_t(r)][size_t(i)]);
        mb.add_row(1.0, 1.0, c, std::vector<double>(N, 1.0));
    }
    return mb.finalize();
}

// A feasible, bounded LP: rows around A x0 (equalities, ranges and one-sided
// rows), costs A'y0 + s with s >= 0 on columns bounded below.
struct Lcg {  // a small deterministic generator for the test models
    unsigned long long s;
    double uniform() {
        s = s * 6364136223846793005ULL + 1442695040888963407ULL;
        return double(s >> 11) * (1.0 / 9007199254740992.0);
    }
};

// zero_cost: every feasible point is optimal; *x0_out receives the strictly
// feasible point the rows are built around.
static sov::Model random_lp(unsigned seed, int m, int n, bool zero_cost = false,
                            std::vector<double>* x0_out = nullptr) {
    Lcg rng{0x9E3779B97F4A7C15ULL ^ seed};
    sov::ModelBuilder mb("random");
    std::vector<double> x0(static_cast<size_t>(n));
    std::vector<std::vector<std::pair<int, double>>> cols(static_cast<size_t>(n));
    std::vector<double> y0(static_cast<size_t>(m));
    for (int i = 0; i < m; ++i) y0[size_t(i)] = rng.uniform() * 2.0 - 1.0;
    std::vector<double> ax(size_t(m), 0.0);
    for (int j = 0; j < n; ++j) {
        x0[size_t(j)] = rng.uniform() * 10.0;
        for (int k = 0; k < 3; ++k) {
            const int i = int(rng.uniform() * m) % m;
            const double v = rng.uniform() * 4.0 - 2.0;
            cols[size_t(j)].push_back({i, v});
            ax[size_t(i)] += v * x0[size_t(j)];
        }
    }
    std::vector<sov::Idx> id(static_cast<size_t>(n));
    for (int j = 0; j < n; ++j) {
        double c = rng.uniform();
        for (auto& e : cols[size_t(j)]) c += e.second * y0[size_t(e.first)];
        const double up = (j % 4 == 0) ? sov::kInf : 10.0 + 5.0 * rng.uniform();
        id[size_t(j)] = mb.add_col(zero_cost ? 0.0 : c, 0.0, up);
    }
    std::vector<std::vector<sov::Idx>> ri(static_cast<size_t>(m));
    std::vector<std::vector<double>> rv(static_cast<size_t>(m));
    for (int j = 0; j < n; ++j)
        for (auto& e : cols[size_t(j)]) {
            ri[size_t(e.first)].push_back(id[size_t(j)]);
            rv[size_t(e.first)].push_back(e.second);
        }
    for (int i = 0; i < m; ++i) {
        const double a = ax[size_t(i)];
        switch (i % 3) {
            case 0: mb.add_row(a, a, ri[size_t(i)], rv[size_t(i)]); break;
            case 1: mb.add_row(a - 1.0, a + 2.0, ri[size_t(i)], rv[size_t(i)]); break;
            default: mb.add_row(-sov::kInf, a + 0.5, ri[size_t(i)], rv[size_t(i)]); break;
        }
    }
    if (x0_out) *x0_out = x0;
    return mb.finalize();
}

static double seconds_since(const std::chrono::steady_clock::time_point& t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

static sov::Model model_of(const nir_lp_view& v) { return model_from(&v); }

// kind, seed, m: a generator model (include/nir_lpgen.h); m = 0 is the
// kind's default.
static int measure(int kind, unsigned long long seed, int m) {
    std::setvbuf(stdout, nullptr, _IOLBF, 0);  // each line out as it is made
    nir_lpgen* g = nullptr;
    nir_lpgen_opts o;
    std::memset(&o, 0, sizeof(o));
    o.m = m;
    if (nir_lpgen_create(kind, seed, &o, &g) != 0) return fail("measure", "generator");
    nir_lp_view v;
    nir_lpgen_view(g, &v);
    const sov::Model f = model_of(v);
    sov::Options opt;
    opt.log_level = 0;
    std::printf("kind %d seed %llu: m=%d n=%d nnz=%lld\n", kind, seed, int(f.nrow), int(f.ncol),
                (long long)f.A.nnz());
    bool ok = true;
    // the reference loop run for its own cap, max(5000, simplex_iter_limit / 10),
    // and for six times as many iterations; then crossover from each point
    const long long cap = std::max<long long>(5000, static_cast<long long>(opt.simplex_iter_limit) / 10);
    for (long long iters : {cap, 6 * cap}) {
        std::vector<double> xp(size_t(f.ncol)), yp(size_t(f.nrow));
        or_pdhg_out po;
        auto t0 = std::chrono::steady_clock::now();
        or_ref_pdhg(&v, iters, 0, 0.0, 0, xp.data(), yp.data(), &po);
        const double t_pdhg = seconds_since(t0);
        or_kkt kk;
        or_rel_kkt(&v, xp.data(), yp.data(), &kk);
        std::printf("reference PDHG loop (oracle, 1 thread): %lld iterations, %.2f s, rel KKT %.2e, max rel row "
                    "violation %.2e\n",
                    (long long)po.iterations, t_pdhg, kk.rel_kkt, kk.max_rel_row_viol);
        for (const char* method : {"dual", "primal"}) {
            sov::Deadline dl;
            dl.wall_limit_sec = 240.0;
            t0 = std::chrono::steady_clock::now();
            const nir::dropin::CrossoverResult r = nir::dropin::crossover(f, xp, yp, opt, dl, 1e-6, method);
            const double t_x = seconds_since(t0);
            const double obj = f.eval_objective(r.x);
            const bool pass = r.status == sov::Status::Optimal && sov::verify_solution(f, r.x, obj, 1e-9).passed;
            std::printf("  crossover (%s): status %d, %lld pivots, %.2f s, crash basic columns %lld, objective "
                        "%.12g, dd check at 1e-9 %s\n",
                        method, int(r.status), (long long)r.simplex_iterations, t_x, (long long)r.crash_structurals,
                        obj, pass ? "PASS" : "FAIL");
            ok = ok && pass;
        }
    }
    sov::Deadline limit;
    limit.wall_limit_sec = 300.0;
    sov::LpSolver lp(opt);
    lp.load(f);
    auto t0 = std::chrono::steady_clock::now();
    const sov::Status st = lp.solve(limit);
    std::printf("simplex from slacks: status %d, %lld iterations, %.2f s%s\n", int(st), (long long)lp.stats.iterations,
                seconds_since(t0), st == sov::Status::Optimal ? "" : " (stopped)");
    nir_lpgen_free(g);
    return ok ? 0 : 1;
}

// "mps <file>...": each model's LP (integrality dropped; models with a
// quadratic objective are skipped), crossover from its simplex optimum
// perturbed by 1e-6, against the simplex from slacks.
static int check_files(int argc, char** argv) {
    sov::Options opt;
    opt.log_level = 0;
    for (int a = 2; a < argc; ++a) {
        sov::Model f;
        std::string err;
        if (sov::MpsReader::read(argv[a], f, err) != sov::Status::Optimal) return fail(argv[a], err.c_str());
        if (f.is_qp()) continue;
        if (f.sense == sov::Sense::Maximize) {  // the LP as the solver minimises it
            for (double& c : f.cost) c = -c;
            f.obj_offset = -f.obj_offset;
            f.sense = sov::Sense::Minimize;
        }
        f.vartype.assign(size_t(f.ncol), sov::VarType::Continuous);
        std::vector<double> xa, ya;
        const long long scratch = approximate_optimum(f, xa, ya, 1e-6);
        if (scratch < 0) return fail(argv[a], "the simplex does not solve its LP");
        sov::LpSolver ref(opt);
        ref.load(f);
        sov::Deadline dl;
        ref.solve(dl);
        const double obj_ref = f.eval_objective(std::vector<double>(ref.value.begin(), ref.value.begin() + f.ncol));
        const nir::dropin::CrossoverResult r = nir::dropin::crossover(f, xa, ya, opt, dl, 1e-6);
        const double obj = f.eval_objective(r.x);
        if (r.status != sov::Status::Optimal || std::abs(obj - obj_ref) > 1e-9 * (1.0 + std::abs(obj_ref)) ||
            !sov::verify_solution(f, r.x, obj, 1e-9).passed)
            return fail(argv[a], "crossover on the model's LP");
        std::printf("%s: m=%d n=%d objective %.12g, simplex from slacks %lld iterations, crossover %lld\n",
                    f.name.c_str(), int(f.nrow), int(f.ncol), obj, scratch, (long long)r.simplex_iterations);
    }
    std::printf("ok\n");
    return 0;
}

int main(int argc, char** argv) {
    if (argc > 1 && std::strcmp(argv[1], "mps") == 0) return check_files(argc, argv);
    if (argc > 1 && std::strcmp(argv[1], "c1") == 0) return measure(NIR_GEN_RANDOM_EQ, 1, 0);
    if (argc > 3 && std::strcmp(argv[1], "measure") == 0)
        return measure(std::atoi(argv[2]), std::strtoull(argv[3], nullptr, 10), argc > 4 ? std::atoi(argv[4]) : 0);
    struct Case {
        const char* name;
        sov::Model m;
    };
    std::vector<Case> cases;
    cases.push_back({"appendix_a5", appendix_a5()});
    cases.push_back({"pdhg_lp", pdhg_lp()});
    cases.push_back({"transport", transport()});
    const char* rnames[] = {"random_0", "random_1", "random_2", "random_3"};
    for (unsigned s = 0; s < 4; ++s) cases.push_back({rnames[s], random_lp(11 + s, 40 + 20 * int(s), 100 + 40 * int(s))});

    sov::Options opt;
    opt.log_level = 0;
    sov::Deadline dl;
    for (const Case& c : cases) {
        // 1-2: crossover from the perturbed optimum
        std::vector<double> xa, ya;
        const long long scratch = approximate_optimum(c.m, xa, ya);
        if (scratch < 0) return fail(c.name, "the simplex does not solve it");
        sov::LpSolver ref(opt);
        ref.load(c.m);
        ref.solve(dl);
        const std::vector<double> xs(ref.value.begin(), ref.value.begin() + c.m.ncol);
        const double obj_ref = c.m.eval_objective(xs);
        const nir::dropin::CrossoverResult r = nir::dropin::crossover(c.m, xa, ya, opt, dl, 1e-6);
        if (r.status != sov::Status::Optimal) return fail(c.name, "crossover not optimal");
        const double obj = c.m.eval_objective(r.x);
        if (std::abs(obj - obj_ref) > 1e-9 * (1.0 + std::abs(obj_ref))) return fail(c.name, "crossover objective");
        if (!sov::verify_solution(c.m, r.x, obj, 1e-9).passed) return fail(c.name, "crossover point fails dd check");
        if (r.simplex_iterations > scratch) return fail(c.name, "crossover took more pivots than the simplex alone");
        // a point as far off as PDLP's tolerance: the same optimum, whatever the pivots
        std::vector<double> xb, yb;
        approximate_optimum(c.m, xb, yb, 1e-6);
        const nir::dropin::CrossoverResult r6 = nir::dropin::crossover(c.m, xb, yb, opt, dl, 1e-6);
        if (r6.status != sov::Status::Optimal ||
            std::abs(c.m.eval_objective(r6.x) - obj_ref) > 1e-9 * (1.0 + std::abs(obj_ref)))
            return fail(c.name, "crossover from a point 1e-6 off");
        std::printf("%s: m=%d n=%d objective %.12g, simplex from slacks %lld iterations, crossover %lld from 1e-8 "
                    "off (crash: %lld basic columns), %lld from 1e-6 off\n",
                    c.name, int(c.m.nrow), int(c.m.ncol), obj, scratch, (long long)r.simplex_iterations,
                    (long long)r.crash_structurals, (long long)r6.simplex_iterations);

        // 3: through Solver, method=pdhg, crossover after the engine
        setenv("NIR_PDHG_CROSSOVER", "1", 1);
        for (int variant = 0; variant < 2; ++variant) {
            sov::Options so = opt;
            so.method = "pdhg";
            so.presolve = variant ? 2 : 0;
            so.scale = variant != 0;
            g_status = NIR_STATUS_OPTIMAL;
            const sov::SolveResult res = sov::Solver(so).solve(c.m);
            if (res.status != sov::Status::Optimal || !res.verification.passed)
                return fail(c.name, variant ? "Solver with presolve and scaling" : "Solver without presolve");
            if (std::abs(res.objective - obj_ref) > 1e-9 * (1.0 + std::abs(obj_ref)))
                return fail(c.name, "Solver objective");
            if (std::strcmp(c.name, "appendix_a5") == 0 && variant == 0 &&
                (std::abs(res.x[0] - 3.0) > 1e-12 || std::abs(res.x[1] - 1.0) > 1e-12 ||
                 std::abs(res.row_duals[0] - 1.5) > 1e-12 || std::abs(res.row_duals[1] - 0.5) > 1e-12))
                return fail(c.name, "vertex or duals of the worked example");
        }

        // 3b: the dual finish, selected through the environment, reaches the same optimum
        setenv("NIR_PDHG_CROSSOVER_METHOD", "dual", 1);
        {
            sov::Options so = opt;
            so.method = "pdhg";
            g_status = NIR_STATUS_OPTIMAL;
            const sov::SolveResult res = sov::Solver(so).solve(c.m);
            if (res.status != sov::Status::Optimal || !res.verification.passed ||
                std::abs(res.objective - obj_ref) > 1e-9 * (1.0 + std::abs(obj_ref)))
                return fail(c.name, "Solver with NIR_PDHG_CROSSOVER_METHOD=dual");
        }
        unsetenv("NIR_PDHG_CROSSOVER_METHOD");

        // 4: auto runs only when the engine stopped short
        setenv("NIR_PDHG_CROSSOVER", "auto", 1);
        sov::Options so = opt;
        so.method = "pdhg";
        so.presolve = 0;
        so.scale = false;
        g_status = NIR_STATUS_OPTIMAL;
        sov::SolveResult res = sov::Solver(so).solve(c.m);
        if (res.iterations != 7) return fail(c.name, "auto ran a crossover after an optimal engine result");
        g_status = NIR_STATUS_ITERATION_LIMIT;
        res = sov::Solver(so).solve(c.m);
        if (res.status != sov::Status::Optimal || !res.verification.passed || res.iterations < 7)
            return fail(c.name, "auto did not finish an engine result stopped at its cap");
        unsetenv("NIR_PDHG_CROSSOVER");
    }
    // an interior point of the optimal face: with zero costs every feasible
    // point is optimal, and x0 lies strictly inside its column bounds, so
    // there are more basic candidates than rows
    {
        std::vector<double> x0;
        const sov::Model z = random_lp(99, 60, 150, true, &x0);
        const nir::dropin::CrossoverResult r =
            nir::dropin::crossover(z, x0, std::vector<double>(size_t(z.nrow), 0.0), opt, dl, 1e-6);
        if (r.status != sov::Status::Optimal || !sov::verify_solution(z, r.x, 0.0, 1e-9).passed)
            return fail("zero_cost", "crossover from an interior feasible point");
        int inside = 0;
        for (sov::Idx j = 0; j < z.ncol; ++j)
            if (r.x[size_t(j)] > z.collo[size_t(j)] + 1e-9 &&
                (!sov::is_finite_bound(z.colup[size_t(j)]) || r.x[size_t(j)] < z.colup[size_t(j)] - 1e-9))
                ++inside;
        if (inside > z.nrow) return fail("zero_cost", "more columns inside their bounds than rows: not a vertex");
        std::printf("zero_cost: m=%d n=%d crash basic columns %lld, %lld pivots, %d columns inside their bounds\n",
                    int(z.nrow), int(z.ncol), (long long)r.crash_structurals, (long long)r.simplex_iterations, inside);
    }
    // a point 1e-3 off, as an early stop of the engine leaves it
    {
        const sov::Model f = random_lp(21, 80, 200);
        std::vector<double> xa, ya;
        approximate_optimum(f, xa, ya, 1e-3);
        sov::LpSolver ref(opt);
        ref.load(f);
        ref.solve(dl);
        const double obj_ref = f.eval_objective(std::vector<double>(ref.value.begin(), ref.value.begin() + f.ncol));
        const nir::dropin::CrossoverResult r = nir::dropin::crossover(f, xa, ya, opt, dl, 1e-6);
        if (r.status != sov::Status::Optimal ||
            std::abs(f.eval_objective(r.x) - obj_ref) > 1e-9 * (1.0 + std::abs(obj_ref)))
            return fail("far", "crossover from a point 1e-3 off");
        std::printf("far: m=%d n=%d from 1e-3 off: %lld pivots (simplex from slacks %lld)\n", int(f.nrow),
                    int(f.ncol), (long long)r.simplex_iterations, (long long)ref.stats.iterations);
    }
    // real PDHG iterates: the reference loop (oracle) to 1e-6 relative KKT
    for (unsigned seed = 0; seed < 3; ++seed) {
        const sov::Model f = random_lp(31 + seed, 30 + 10 * int(seed), 80 + 20 * int(seed));
        nir_lp_view v;
        std::memset(&v, 0, sizeof(v));
        v.nrow = f.nrow;
        v.ncol = f.ncol;
        v.nnz = f.A.nnz();
        v.col_start = f.A.start.data();
        v.row_index = f.A.index.data();
        v.value = f.A.value.data();
        v.cost = f.cost.data();
        v.collo = f.collo.data();
        v.colup = f.colup.data();
        v.rowlo = f.rowlo.data();
        v.rowup = f.rowup.data();
        std::vector<double> xp(size_t(f.ncol)), yp(size_t(f.nrow));
        or_pdhg_out po;
        or_ref_pdhg(&v, 3000000, 64, 1e-6, 1, xp.data(), yp.data(), &po);
        sov::LpSolver ref(opt);
        ref.load(f);
        ref.solve(dl);
        const double obj_ref = f.eval_objective(std::vector<double>(ref.value.begin(), ref.value.begin() + f.ncol));
        const nir::dropin::CrossoverResult r = nir::dropin::crossover(f, xp, yp, opt, dl, 1e-6);
        if (r.status != sov::Status::Optimal ||
            std::abs(f.eval_objective(r.x) - obj_ref) > 1e-9 * (1.0 + std::abs(obj_ref)))
            return fail("pdhg_iterate", "crossover from a PDHG iterate");
        std::printf("pdhg_iterate_%u: m=%d n=%d PDHG %lld iterations (rel KKT %.1e), crossover %lld pivots "
                    "(simplex from slacks %lld)\n",
                    seed, int(f.nrow), int(f.ncol), (long long)po.iterations, po.last_kkt,
                    (long long)r.simplex_iterations, (long long)ref.stats.iterations);
    }
    std::printf("ok\n");
    return 0;
}
