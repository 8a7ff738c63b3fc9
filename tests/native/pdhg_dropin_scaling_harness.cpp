// Checks the drop-in PdhgSolver's handling of scale_model's scales without a
// GPU: the engine entry point is replaced by a stand-in that records the LP it
// is given and returns a known point.  Built against a tree of the
// reference's headers with the drop-in headers linked in (tests/test_dropin.py).
//
// The checks:
//   1. with scaling active, the engine receives the unscaled model bit for bit;
//   2. the point it returns comes back divided by C (x) and R (y), so that
//      Solver's unscale_primal / unscale_row_duals give it back exactly;
//   3. with scaling off, or NIR_PDHG_KEEP_SCALING=1, the engine receives the
//      model as given.
// Prints "ok" and exits 0, or names the first failed check and exits 1.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "include/sov/solver.hpp"

namespace {
std::vector<double> g_cost, g_lo, g_up, g_val, g_rl, g_ru;
std::vector<double> g_x0, g_y0;

bool same(const std::vector<double>& a, const double* b) {
    return std::memcmp(a.data(), b, a.size() * sizeof(double)) == 0;
}
}  // namespace

extern "C" int nir_pdhg_default_params(nir_pdhg_params* p) {
    std::memset(p, 0, sizeof(*p));
    p->tol = 1e-6;
    return 0;
}

extern "C" int nir_pdhg_solve_lp(const nir_lp_view* lp, int, const nir_pdhg_params*, int (*)(void*), void*,
                                 double* x, double* y, nir_pdhg_info* info) {
    g_cost.assign(lp->cost, lp->cost + lp->ncol);
    g_lo.assign(lp->collo, lp->collo + lp->ncol);
    g_up.assign(lp->colup, lp->colup + lp->ncol);
    g_val.assign(lp->value, lp->value + lp->nnz);
    g_rl.assign(lp->rowlo, lp->rowlo + lp->nrow);
    g_ru.assign(lp->rowup, lp->rowup + lp->nrow);
    std::memcpy(x, g_x0.data(), g_x0.size() * sizeof(double));
    std::memcpy(y, g_y0.data(), g_y0.size() * sizeof(double));
    std::memset(info, 0, sizeof(*info));
    info->iterations = 7;
    return NIR_STATUS_OPTIMAL;
}

extern "C" const char* nir_pdhg_last_error(void) { return ""; }

static int fail(const char* what) {
    std::printf("failed: %s\n", what);
    return 1;
}

int main() {
    // a model whose coefficients span six decades, so that scale_model is active
    sov::ModelBuilder mb("scaling_check");
    const int n = 40, m = 25;
    std::vector<sov::Idx> cols;
    for (int j = 0; j < n; ++j)
        cols.push_back(mb.add_col(1.0 + 0.25 * j, j % 5 == 0 ? -sov::kInf : -1.0 * j, j % 7 == 0 ? sov::kInf : 3.0 + j));
    for (int i = 0; i < m; ++i) {
        std::vector<sov::Idx> idx;
        std::vector<double> val;
        for (int k = 0; k < 4; ++k) {
            idx.push_back(cols[size_t((i * 3 + k * 7) % n)]);
            val.push_back(std::pow(10.0, double((i + k) % 7) - 3.0) * (k % 2 ? -1.5 : 1.25));
        }
        mb.add_row(i % 3 == 0 ? -sov::kInf : -5.0 - i, i % 4 == 0 ? sov::kInf : 7.0 + i, idx, val);
    }
    const sov::Model orig = mb.finalize();
    sov::Options opt;
    sov::Deadline dl;
    g_x0.resize(size_t(n));
    g_y0.resize(size_t(m));
    for (int j = 0; j < n; ++j) g_x0[size_t(j)] = 0.1 * j - 1.0;
    for (int i = 0; i < m; ++i) g_y0[size_t(i)] = 0.3 * i - 2.0;

    sov::ScalingInfo si;
    const sov::Model sc = sov::scale_model(orig, true, si);
    if (!si.active) return fail("scale_model inactive on the test model");
    sov::PdhgResult r = sov::PdhgSolver::solve(sc, opt, dl);
    if (!same(g_cost, orig.cost.data()) || !same(g_lo, orig.collo.data()) || !same(g_up, orig.colup.data()) ||
        !same(g_val, orig.A.value.data()) || !same(g_rl, orig.rowlo.data()) || !same(g_ru, orig.rowup.data()))
        return fail("the engine did not receive the unscaled model");
    std::vector<double> xo, yo;
    si.unscale_primal(r.x, xo);
    si.unscale_row_duals(r.y, yo);
    if (!same(xo, g_x0.data()) || !same(yo, g_y0.data())) return fail("the point did not map back exactly");

    sov::ScalingInfo off;
    const sov::Model same_model = sov::scale_model(orig, false, off);
    r = sov::PdhgSolver::solve(same_model, opt, dl);
    if (!same(g_val, orig.A.value.data()) || !same(r.x, g_x0.data())) return fail("scaling off: model changed");

    sov::ScalingInfo again;
    const sov::Model sc2 = sov::scale_model(orig, true, again);
    setenv("NIR_PDHG_KEEP_SCALING", "1", 1);
    r = sov::PdhgSolver::solve(sc2, opt, dl);
    if (!same(g_val, sc2.A.value.data()) || !same(r.x, g_x0.data())) return fail("keep-scaling: model changed");
    std::printf("ok\n");
    return 0;
}
