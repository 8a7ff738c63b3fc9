// Near-parallel columns, re-expressed so that PDHG does not stall on them.
// Host side, included by engine.cu.
//
// When column j' of A is (nearly) a multiple of column j, A_j' = lambda A_j
// + eps with eps tiny, the primal iterates of PDHG cannot tell the two
// apart: moving mass from x_j' to x_j leaves A x (almost) unchanged, and
// the only force along that direction is the cost difference, which the
// diagonal preconditioning makes vanishingly small when the columns are
// large.  The two columns then stay split evenly between their bounds,
// the duals cannot price both, and the duality gap stops shrinking (a
// badly scaled LP whose columns are duplicated with a 1e-9 perturbation
// plateaus at a relative gap of ~5e-4).
//
// The handle therefore solves an equivalent LP.  For a group of columns
// j (the representative) and j'_1..j'_K parallel to it (lambda_k):
//   v   = x_j + sum_k lambda_k x_j'_k    takes column j:   A_j,  cost c_j
//   w_k = x_j'_k                         takes column j'_k: A_j'_k - lambda_k A_j
//                                                          (= eps_k), cost c_j'_k - lambda_k c_j
//   one new row  v - sum_k lambda_k w_k = x_j  with the bounds of x_j,
//   v bounded by the sums of its parts' bounds, w_k by x_j'_k's.
// A_j v + sum_k eps_k w_k = A_j x_j + sum_k A_j'_k x_j'_k, so the LP is the
// same one, exactly (up to the rounding of eps); the split of the group now
// sits in variables that the matrix does not couple, and PDHG resolves it.
// The solution maps back as x_j = v - sum_k lambda_k w_k, x_j'_k = w_k, and
// y = the duals of the original rows.  The relative KKT error and objective
// the solve reports are evaluated on the original LP.
//
// No counterpart in the reference, whose PDHG (src/gpu/pdhg_solver.hpp) works
// on the model as given; its presolve (src/presolve/presolve.hpp) has no
// parallel-column rule.
#pragma once

namespace {

// Columns whose |eps| stays within this share of the column's largest entry
// are treated as parallel.
constexpr double kParallelRtol = 1e-6;

// Finds groups of parallel columns: columns with the same row pattern (by
// hash, then compared exactly) whose values are proportional within
// kParallelRtol.  The first column of a group in index order is its
// representative.  Columns with a single nonzero are never grouped: each is
// parallel to every other single-entry column of its row, a coincidence
// that is common (slack-like columns; a handful among the 500,000 columns of
// the power-law LP) and that PDHG resolves on its own -- re-expressing those
// pairs there made the PDLP solve stall at a relative gap of 2e-4 where it
// otherwise converges in 155,000 iterations.
ParallelGroups find_parallel(const nir_lp_view* lp) {
    const int n = lp->ncol;
    ParallelGroups g;
    g.rep_of.assign(size_t(n), -1);
    g.lam.assign(size_t(n), 0.0);
    g.row_of.assign(size_t(n), -1);
    std::vector<std::pair<unsigned long long, int>> key;
    key.reserve(size_t(n));
    for (int j = 0; j < n; ++j) {
        const long long s = lp->col_start[j], e = lp->col_start[j + 1];
        if (e - s < 2) continue;
        unsigned long long h = 1469598103934665603ULL ^ (unsigned long long)(e - s);
        for (long long k = s; k < e; ++k) {
            h ^= (unsigned long long)(unsigned)lp->row_index[k];
            h *= 1099511628211ULL;
        }
        key.emplace_back(h, j);
    }
    std::sort(key.begin(), key.end());
    std::vector<int> reps;
    for (size_t a = 0; a < key.size();) {
        size_t b = a + 1;
        while (b < key.size() && key[b].first == key[a].first) ++b;
        if (b - a >= 2) {
            reps.clear();
            for (size_t t = a; t < b; ++t) {
                const int j = key[t].second;
                const long long s = lp->col_start[j], len = lp->col_start[j + 1] - s;
                bool matched = false;
                for (int r : reps) {
                    const long long sr = lp->col_start[r];
                    if (lp->col_start[r + 1] - sr != len) continue;
                    if (!std::equal(lp->row_index + s, lp->row_index + s + len, lp->row_index + sr)) continue;
                    long long kmax = 0;
                    double amax = 0.0, bmax = 0.0;
                    for (long long k = 0; k < len; ++k) {
                        if (std::fabs(lp->value[sr + k]) > amax) {
                            amax = std::fabs(lp->value[sr + k]);
                            kmax = k;
                        }
                        bmax = std::max(bmax, std::fabs(lp->value[s + k]));
                    }
                    if (!(amax > 0.0)) continue;
                    const double lam = lp->value[s + kmax] / lp->value[sr + kmax];
                    if (!(lam != 0.0) || !std::isfinite(lam)) continue;
                    double emax = 0.0;
                    for (long long k = 0; k < len; ++k)
                        emax = std::max(emax, std::fabs(lp->value[s + k] - lam * lp->value[sr + k]));
                    if (emax <= kParallelRtol * bmax) {
                        g.rep_of[size_t(j)] = r;
                        g.lam[size_t(j)] = lam;
                        matched = true;
                        break;
                    }
                }
                if (!matched) reps.push_back(j);
            }
        }
        a = b;
    }
    for (int j = 0; j < n; ++j) {
        const int r = g.rep_of[size_t(j)];
        if (r >= 0 && g.row_of[size_t(r)] < 0) g.row_of[size_t(r)] = lp->nrow + g.groups++;
    }
    return g;
}

// lam * [lo, hi] as an interval.
inline void scaled_interval(double lam, double lo, double hi, double& a, double& b) {
    if (lam > 0.0) {
        a = lam * lo;
        b = lam * hi;
    } else {
        a = lam * hi;
        b = lam * lo;
    }
}

// The equivalent LP's cost, column bounds and row bounds from the
// original vectors (host copies, bounds already sanitised to +-inf).
void parallel_vectors(const nir_pdhg* h, std::vector<double>& c, std::vector<double>& l, std::vector<double>& u,
                      std::vector<double>& rl, std::vector<double>& ru) {
    const ParallelGroups& g = *h->par;
    const int n = h->n, m = h->m;
    c = h->h_c;
    l = h->h_l;
    u = h->h_u;
    rl = h->h_rl;
    ru = h->h_ru;
    rl.resize(size_t(m + g.groups));
    ru.resize(size_t(m + g.groups));
    for (int j = 0; j < n; ++j) {
        const int r = g.row_of[size_t(j)];
        if (r >= 0) {
            rl[size_t(r)] = h->h_l[size_t(j)];
            ru[size_t(r)] = h->h_u[size_t(j)];
        }
    }
    for (int j = 0; j < n; ++j) {
        const int rep = g.rep_of[size_t(j)];
        if (rep < 0) continue;
        const double lam = g.lam[size_t(j)];
        c[size_t(j)] = h->h_c[size_t(j)] - lam * h->h_c[size_t(rep)];
        double a, b;
        scaled_interval(lam, h->h_l[size_t(j)], h->h_u[size_t(j)], a, b);
        l[size_t(rep)] += a;  // an infinite part makes the sum infinite
        u[size_t(rep)] += b;
    }
}

// Builds the equivalent LP on the device (h->inner) when the LP has
// parallel columns.
void build_parallel(nir_pdhg* h, const nir_lp_view* lp, int device) {
    const char* env = std::getenv("NIR_PDHG_PARALLEL_COLUMNS");
    if (env && std::string(env) == "0") return;
    auto g = std::make_unique<ParallelGroups>(find_parallel(lp));
    if (g->groups == 0) return;
    const int n = lp->ncol, m = lp->nrow, m2 = m + g->groups;
    std::vector<int64_t> start(static_cast<size_t>(n) + 1, 0);
    std::vector<int> index;
    std::vector<double> value;
    index.reserve(size_t(lp->nnz) + size_t(2 * g->groups));
    value.reserve(size_t(lp->nnz) + size_t(2 * g->groups));
    for (int j = 0; j < n; ++j) {
        const long long s = lp->col_start[j], e = lp->col_start[j + 1];
        const int rep = g->rep_of[size_t(j)];
        if (rep < 0) {
            for (long long k = s; k < e; ++k) {
                index.push_back(lp->row_index[k]);
                value.push_back(lp->value[k]);
            }
            if (g->row_of[size_t(j)] >= 0) {
                index.push_back(g->row_of[size_t(j)]);
                value.push_back(1.0);
            }
        } else {
            const double lam = g->lam[size_t(j)];
            const long long sr = lp->col_start[rep];
            for (long long k = s; k < e; ++k) {
                const double eps = lp->value[k] - lam * lp->value[sr + (k - s)];
                if (eps != 0.0) {
                    index.push_back(lp->row_index[k]);
                    value.push_back(eps);
                }
            }
            index.push_back(g->row_of[size_t(rep)]);
            value.push_back(-lam);
        }
        start[size_t(j) + 1] = int64_t(index.size());
    }
    h->par = std::move(g);
    std::vector<double> c, l, u, rl, ru;
    parallel_vectors(h, c, l, u, rl, ru);
    nir_lp_view v{};
    v.nrow = m2;
    v.ncol = n;
    v.nnz = (long long)index.size();
    v.col_start = start.data();
    v.row_index = index.data();
    v.value = value.data();
    v.cost = c.data();
    v.collo = l.data();
    v.colup = u.data();
    v.rowlo = rl.data();
    v.rowup = ru.data();
    v.obj_offset = lp->obj_offset;
    validate_lp(&v);
    h->inner = std::make_unique<nir_pdhg>();
    h->inner->device = -1;
    create_impl(h->inner.get(), &v, device);
}

void parallel_update_vectors(nir_pdhg* h) {
    std::vector<double> c, l, u, rl, ru;
    parallel_vectors(h, c, l, u, rl, ru);
    upload_vectors(h->inner.get(), c.data(), l.data(), u.data(), rl.data(), ru.data());
}

// Original point -> the equivalent LP's point.
void parallel_map_in(const nir_pdhg* h, const double* x, std::vector<double>& xv) {
    const ParallelGroups& g = *h->par;
    xv.assign(x, x + h->n);
    for (int j = 0; j < h->n; ++j) {
        const int rep = g.rep_of[size_t(j)];
        if (rep >= 0) xv[size_t(rep)] += g.lam[size_t(j)] * x[j];
    }
}

// The equivalent LP's point -> original point (partners in index order).
void parallel_map_out(const nir_pdhg* h, const std::vector<double>& xv, std::vector<double>& x) {
    const ParallelGroups& g = *h->par;
    x = xv;
    for (int j = 0; j < h->n; ++j) {
        const int rep = g.rep_of[size_t(j)];
        if (rep >= 0) x[size_t(rep)] -= g.lam[size_t(j)] * xv[size_t(j)];
    }
}

// Relative KKT error of (x, y) on the handle's own (original) LP, evaluated
// on the device in FP64 with the KKT kernels of the solve on unit scales.
struct KktReport {
    double kkt, kp, kd, kg, max_rel_row;
};

KktReport kkt_of_point(nir_pdhg* h, const nir_pdhg_params& p, const std::vector<double>& x,
                       const std::vector<double>& y) {
    cudaStream_t s = h->stream;
    const int n = h->n, m = h->m;
    if (h->A.lay < 0 || h->At.lay < 0) use_layouts(h, default_layouts(h));
    precondition(h, p, false);  // unit scales: the scaled copies equal the original LP
    pad_scaled(h);
    ensure_partials(h);
    const PartLayout L = part_layout(h);
    NIR_CUDA(cudaMemcpyAsync(h->xp64, x.data(), size_t(n) * sizeof(double), cudaMemcpyHostToDevice, s));
    NIR_CUDA(cudaMemcpyAsync(h->yp64, y.data(), size_t(m) * sizeof(double), cudaMemcpyHostToDevice, s));
    nir::DevState st0{};
    st0.probe_hit = -1;
    NIR_CUDA(cudaMemcpyAsync(h->st, &st0, sizeof(st0), cudaMemcpyHostToDevice, s));
    int gkr = 0, gkc = 0;
    launch_kkt<double>(h, 0, L.KR, L.KC, h->xp64, h->yp64, &gkr, &gkc);
    nir::k_ref_probe<<<1, nir::kBlock, 0, s>>>(L.KR, gkr, L.KC, gkc, rhs_norm(h), norm2(h->h_c), h->offset, -1.0,
                                               h->st);
    NIR_LAUNCHED();
    h->launches += 1;
    nir::DevState st;
    d2h(h, &st, h->st, sizeof(st));
    return KktReport{st.kkt, st.kp, st.kd, st.kg, st.max_rel_row};
}

// PDHG / PDLP on the equivalent LP, reported on the original one.  The two
// LPs share the primal objective and the original rows, but not the dual
// objective: the equivalent LP relaxes the box of each representative x_j
// into a row, so at the same point its dual bound is the lower one, and a
// primal iterate that is slightly infeasible (hence below the optimum) can
// meet the tolerance there while the original's gap does not.  When the
// equivalent LP met the tolerance and the original did not, the solve
// therefore goes on from where it stopped with a ten times tighter
// tolerance, up to kParallelTightenings times; it reports Optimal only when
// the original LP's relative KKT error meets the tolerance, and otherwise
// the status of the last inner solve, with Optimal turned into
// NIR_STATUS_NUMERICAL_TROUBLE.
constexpr int kParallelTightenings = 4;

int solve_parallel(nir_pdhg* h, const nir_pdhg_params& p, int (*poll)(void*), void* ctx, double* x_out,
                   double* y_out, nir_pdhg_info* info) {
    nir_pdhg* in = h->inner.get();
    const int n = h->n, m = h->m, m2 = in->m;
    const double t0 = now_sec();
    nir_pdhg_params q = p;
    std::vector<double> xi, yi;
    if (p.x_init) {
        parallel_map_in(h, p.x_init, xi);
        q.x_init = xi.data();
    }
    if (p.y_init) {
        yi.assign(p.y_init, p.y_init + m);
        yi.resize(size_t(m2), 0.0);
        q.y_init = yi.data();
    }
    in->profiling = h->profiling;
    std::vector<double> xv(static_cast<size_t>(n)), yv(static_cast<size_t>(m2)), x, y;
    int status = solve_fast(in, q, poll, ctx, xv.data(), yv.data(), info);
    parallel_map_out(h, xv, x);
    y.assign(yv.begin(), yv.begin() + m);
    KktReport k = kkt_of_point(h, p, x, y);
    auto met = [&p](const KktReport& r) {
        return r.kkt <= p.tol && (p.feas_tol <= 0.0 || r.max_rel_row <= p.feas_tol);
    };
    for (int t = 0; t < kParallelTightenings && status == NIR_STATUS_OPTIMAL && p.tol > 0.0 && !met(k) &&
                    info->iterations < p.max_iters;
         ++t) {
        nir_pdhg_info more{};
        q.tol *= 0.1;
        q.feas_tol *= 0.1;
        q.x_init = xv.data();
        q.y_init = yv.data();
        q.omega_init = info->primal_weight;
        q.max_iters = p.max_iters - info->iterations;
        if (p.time_limit > 0.0) q.time_limit = std::max(1e-3, p.time_limit - (now_sec() - t0));
        std::vector<double> xv2(static_cast<size_t>(n)), yv2(static_cast<size_t>(m2));
        status = solve_fast(in, q, poll, ctx, xv2.data(), yv2.data(), &more);
        more.iterations += info->iterations;
        more.iterations_fp64 += info->iterations_fp64;
        more.restarts += info->restarts;
        more.setup_seconds += info->setup_seconds;
        *info = more;
        xv.swap(xv2);
        yv.swap(yv2);
        parallel_map_out(h, xv, x);
        y.assign(yv.begin(), yv.begin() + m);
        k = kkt_of_point(h, p, x, y);
    }
    if (status == NIR_STATUS_OPTIMAL && p.tol > 0.0 && !met(k)) status = NIR_STATUS_NUMERICAL_TROUBLE;
    NIR_CUDA(cudaMemcpyAsync(h->out_x, x.data(), size_t(n) * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    NIR_CUDA(cudaMemcpyAsync(h->out_y, y.data(), size_t(m) * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    NIR_CUDA(cudaStreamSynchronize(h->stream));
    h->last_x = h->out_x;
    if (x_out) std::memcpy(x_out, x.data(), size_t(n) * sizeof(double));
    if (y_out) std::memcpy(y_out, y.data(), size_t(m) * sizeof(double));
    info->objective = host_objective(h, x);
    info->rel_kkt = k.kkt;
    info->rel_primal = k.kp;
    info->rel_dual = k.kd;
    info->rel_gap = k.kg;
    info->max_rel_row_viol = k.max_rel_row;
    info->parallel_groups = h->par->groups;
    h->ktime = in->ktime;
    h->launches += in->launches;
    in->launches = 0;
    info->status = status;
    return status;
}

}  // namespace
