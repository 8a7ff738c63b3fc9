// Checks the drop-in PdhgSolver's FP64 retry on the GPU without a GPU: the
// engine entry point is replaced by a stand-in that plays back scripted
// results and records the parameters of every call.  Built against a tree of
// the reference's headers with the drop-in headers linked in
// (tests/test_dropin.py).
//
// The checks (the model is not scaled, so the engine's space is the model's):
//   1. a solve that meets the relative KKT but not the row margin at its cap
//      goes on once in FP64, from the point it reached, with its primal
//      weight; the retry's Optimal point is returned, iterations summed;
//   2. a retry that does not meet the KKT tolerance leaves the first point,
//      reported Optimal as before (Solver's dd check judges the rows);
//   3. an Optimal first solve, a first solve above the KKT tolerance, and
//      NIR_PDHG_RETRY=0 make no retry.
// Prints "ok" and exits 0, or names the first failed check and exits 1.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "include/sov/solver.hpp"

namespace {
struct Reply {
    int status;
    double rel_kkt;
    double omega;
    long long iterations;
    double xval;  // every x entry of the returned point
};
struct Call {
    int precision;
    bool warm;
    double x_init0;
    double omega_init;
};
std::vector<Reply> g_script;
std::vector<Call> g_calls;
int g_n = 0, g_m = 0;
}  // namespace

extern "C" int nir_pdhg_default_params(nir_pdhg_params* p) {
    std::memset(p, 0, sizeof(*p));
    p->algorithm = NIR_ALGO_PDLP;
    p->precision = NIR_PREC_MIXED;
    p->tol = 1e-6;
    p->max_iters = 1000;
    return 0;
}

extern "C" int nir_pdhg_solve_lp(const nir_lp_view*, int, const nir_pdhg_params* p, int (*)(void*), void*,
                                 double* x, double* y, nir_pdhg_info* info) {
    g_calls.push_back(Call{p->precision, p->x_init != nullptr && p->y_init != nullptr,
                           p->x_init ? p->x_init[0] : 0.0, p->omega_init});
    const Reply r = g_script.at(g_calls.size() - 1);
    for (int j = 0; j < g_n; ++j) x[j] = r.xval;
    for (int i = 0; i < g_m; ++i) y[i] = -r.xval;
    std::memset(info, 0, sizeof(*info));
    info->status = r.status;
    info->rel_kkt = r.rel_kkt;
    info->primal_weight = r.omega;
    info->iterations = r.iterations;
    return r.status;
}

extern "C" const char* nir_pdhg_last_error(void) { return ""; }

static int fail(const char* what) {
    std::printf("failed: %s\n", what);
    return 1;
}

int main() {
    sov::ModelBuilder mb("retry_check");
    g_n = 6;
    g_m = 3;
    std::vector<sov::Idx> cols;
    for (int j = 0; j < g_n; ++j) cols.push_back(mb.add_col(1.0 + j, 0.0, 10.0));
    for (int i = 0; i < g_m; ++i) mb.add_row(1.0, 1.0, {cols[size_t(i)], cols[size_t(i + 3)]}, {1.0, 2.0});
    const sov::Model model = mb.finalize();
    sov::Options opt;
    sov::Deadline dl;
    unsetenv("NIR_PDHG_RETRY");

    // 1. margin missing at the cap, the retry meets everything
    g_calls.clear();
    g_script = {{NIR_STATUS_ITERATION_LIMIT, 5e-7, 0.25, 100, 1.5}, {NIR_STATUS_OPTIMAL, 4e-7, 0.3, 40, 2.5}};
    sov::PdhgResult r = sov::PdhgSolver::solve(model, opt, dl);
    if (g_calls.size() != 2) return fail("no retry after a missing row margin");
    if (g_calls[1].precision != NIR_PREC_FP64) return fail("the retry is not FP64");
    if (!g_calls[1].warm || g_calls[1].x_init0 != 1.5) return fail("the retry does not start from the point reached");
    if (g_calls[1].omega_init != 0.25) return fail("the retry does not keep the primal weight");
    if (r.status != sov::Status::Optimal || r.x[0] != 2.5 || r.iterations != 140)
        return fail("the retry's optimal point is not returned");

    // 2. the retry stays above the KKT tolerance: the first point stands
    g_calls.clear();
    g_script = {{NIR_STATUS_ITERATION_LIMIT, 5e-7, 0.25, 100, 1.5}, {NIR_STATUS_ITERATION_LIMIT, 3e-6, 0.3, 40, 2.5}};
    r = sov::PdhgSolver::solve(model, opt, dl);
    if (g_calls.size() != 2) return fail("no retry in case 2");
    if (r.status != sov::Status::Optimal || r.x[0] != 1.5 || r.iterations != 140)
        return fail("a worse retry replaced the first point");

    // 3. no retry: Optimal at once, KKT not met, or turned off
    g_calls.clear();
    g_script = {{NIR_STATUS_OPTIMAL, 5e-7, 0.25, 100, 1.5}};
    r = sov::PdhgSolver::solve(model, opt, dl);
    if (g_calls.size() != 1 || r.status != sov::Status::Optimal) return fail("retry after an optimal solve");
    g_calls.clear();
    g_script = {{NIR_STATUS_ITERATION_LIMIT, 5e-6, 0.25, 100, 1.5}};
    r = sov::PdhgSolver::solve(model, opt, dl);
    if (g_calls.size() != 1 || r.status != sov::Status::IterationLimit) return fail("retry above the KKT tolerance");
    g_calls.clear();
    setenv("NIR_PDHG_RETRY", "0", 1);
    g_script = {{NIR_STATUS_ITERATION_LIMIT, 5e-7, 0.25, 100, 1.5}};
    r = sov::PdhgSolver::solve(model, opt, dl);
    if (g_calls.size() != 1 || r.status != sov::Status::Optimal) return fail("NIR_PDHG_RETRY=0 did not turn it off");
    std::printf("ok\n");
    return 0;
}
