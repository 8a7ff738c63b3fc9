/*
 * nir_oracle.c -- CPU oracle for the NIRNAYA PDHG path (test infrastructure
 * only; see nir_oracle.h for who may use it and what each function restates).
 *
 * Build with -O2 -fno-fast-math -ffp-contract=off so that no multiply-add is
 * fused: the reference is compiled as ISO C++17 without FMA contraction, and
 * bit-identical iterates depend on the same rounding of every product.
 */
#include "nir_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---------------- double-double (src/core/dd_real.hpp:8-82) ---------------- */

typedef struct { double hi, lo; } dd;

static void two_sum(double a, double b, double* s, double* e) {
    double ss = a + b;
    double bb = ss - a;
    *e = (a - (ss - bb)) + (b - bb);
    *s = ss;
}

static void quick_two_sum(double a, double b, double* s, double* e) {
    double ss = a + b;
    *e = b - (ss - a);
    *s = ss;
}

static dd dd_add_d(dd a, double b) {  /* dd_real::operator+=(double), :38-44 */
    double s1, s2;
    two_sum(a.hi, b, &s1, &s2);
    s2 += a.lo;
    dd r;
    quick_two_sum(s1, s2, &r.hi, &r.lo);
    return r;
}

static dd dd_add(dd a, dd b) {  /* dd_real::operator+=(const dd_real&), :46-55 */
    double s1, s2, t1, t2;
    two_sum(a.hi, b.hi, &s1, &s2);
    two_sum(a.lo, b.lo, &t1, &t2);
    s2 += t1;
    quick_two_sum(s1, s2, &s1, &s2);
    s2 += t2;
    dd r;
    quick_two_sum(s1, s2, &r.hi, &r.lo);
    return r;
}

static dd dd_add_prod(dd a, double x, double y) {  /* dd_real::add_prod, :77-81 */
    dd p;
    p.hi = x * y;
    p.lo = fma(x, y, -p.hi);
    return dd_add(a, p);
}

static double dd_val(dd a) { return a.hi + a.lo; }

double or_dd_cancellation_probe(double a, double b, double c) {
    dd acc = {0.0, 0.0};
    acc = dd_add_d(acc, a);
    acc = dd_add_d(acc, b);
    acc = dd_add_d(acc, c);
    return dd_val(acc);
}

/* NeumaierSum, src/core/dd_real.hpp:89-104 */
double or_neumaier_probe(double a, double b, double c) {
    double s = 0.0, comp = 0.0, v[3] = {a, b, c};
    for (int k = 0; k < 3; ++k) {
        double t = s + v[k];
        if (fabs(s) >= fabs(v[k])) comp += (s - t) + v[k];
        else comp += (v[k] - t) + s;
        s = t;
    }
    return s + comp;
}

/* ---------------- helpers with the reference's exact semantics ---------------- */

/* is_finite_bound, src/core/types.hpp:49-51 */
static int fin(double b) { return isfinite(b) && fabs(b) < 1e20; }
/* std::max(a, b) and std::min(a, b) exactly (ties and signed zeros included) */
static double smax(double a, double b) { return (a < b) ? b : a; }
static double smin(double a, double b) { return (b < a) ? b : a; }

/* ---------------- SpMV pair (src/core/csc_matrix.hpp:99-120) ---------------- */

void or_spmv(const nir_lp_view* lp, const double* x, double* y) {
    for (int32_t i = 0; i < lp->nrow; ++i) y[i] = 0.0;
    for (int32_t j = 0; j < lp->ncol; ++j) {
        double xj = x[j];
        if (xj == 0.0) continue;
        for (int64_t k = lp->col_start[j]; k < lp->col_start[j + 1]; ++k)
            y[lp->row_index[k]] += lp->value[k] * xj;
    }
}

void or_spmv_t(const nir_lp_view* lp, const double* x, double* y) {
    for (int32_t j = 0; j < lp->ncol; ++j) {
        double s = 0.0;
        for (int64_t k = lp->col_start[j]; k < lp->col_start[j + 1]; ++k)
            s += lp->value[k] * x[lp->row_index[k]];
        y[j] = s;
    }
}

/* ---------------- CSC from triplets (src/core/csc_matrix.hpp:30-96) ---------------- */

typedef struct { int32_t row; int32_t ord; double val; } trip_rv;

static int cmp_row(const void* a, const void* b) {
    const trip_rv* p = (const trip_rv*)a;
    const trip_rv* q = (const trip_rv*)b;
    if (p->row != q->row) return p->row < q->row ? -1 : 1;
    return p->ord < q->ord ? -1 : (p->ord > q->ord);
}

int64_t or_csc_from_triplets(int32_t nrow, int32_t ncol, int64_t ntrip, const int32_t* trow,
                             const int32_t* tcol, const double* tval, int64_t* start_out,
                             int32_t* index_out, double* value_out) {
    int64_t* cnt = (int64_t*)calloc((size_t)ncol + 1, sizeof(int64_t));
    for (int64_t t = 0; t < ntrip; ++t)
        if (trow[t] >= 0 && trow[t] < nrow && tcol[t] >= 0 && tcol[t] < ncol && tval[t] != 0.0)
            cnt[tcol[t] + 1]++;
    for (int32_t j = 0; j < ncol; ++j) cnt[j + 1] += cnt[j];
    int64_t total = cnt[ncol];
    trip_rv* buf = (trip_rv*)malloc(sizeof(trip_rv) * (size_t)(total ? total : 1));
    int64_t* pos = (int64_t*)malloc(sizeof(int64_t) * ((size_t)ncol + 1));
    memcpy(pos, cnt, sizeof(int64_t) * ((size_t)ncol + 1));
    for (int64_t t = 0; t < ntrip; ++t)
        if (trow[t] >= 0 && trow[t] < nrow && tcol[t] >= 0 && tcol[t] < ncol && tval[t] != 0.0) {
            int64_t p = pos[tcol[t]]++;
            buf[p].row = trow[t];
            buf[p].ord = (int32_t)(p - cnt[tcol[t]]);
            buf[p].val = tval[t];
        }
    int64_t w = 0;
    start_out[0] = 0;
    for (int32_t j = 0; j < ncol; ++j) {
        int64_t s = cnt[j], e = cnt[j + 1];
        if (e > s) {
            /* insertion order breaks ties, i.e. a stable sort by row */
            qsort(buf + s, (size_t)(e - s), sizeof(trip_rv), cmp_row);
            int32_t cur_r = buf[s].row;
            double cur_v = buf[s].val;
            for (int64_t k = s + 1; k < e; ++k) {
                if (buf[k].row == cur_r) {
                    cur_v += buf[k].val;
                } else {
                    if (cur_v != 0.0) { index_out[w] = cur_r; value_out[w] = cur_v; ++w; }
                    cur_r = buf[k].row;
                    cur_v = buf[k].val;
                }
            }
            if (cur_v != 0.0) { index_out[w] = cur_r; value_out[w] = cur_v; ++w; }
        }
        start_out[j + 1] = w;
    }
    free(cnt);
    free(buf);
    free(pos);
    return w;
}

/* ---------------- objective and checker ---------------- */

double or_eval_objective(const nir_lp_view* lp, const double* x) {
    dd sum = {lp->obj_offset, 0.0};
    for (int32_t j = 0; j < lp->ncol; ++j)
        if (lp->cost[j] != 0.0 && x[j] != 0.0) sum = dd_add_prod(sum, lp->cost[j], x[j]);
    return dd_val(sum);
}

void or_verify(const nir_lp_view* lp, const double* x, double claimed_obj, double tol,
               or_verify_report* rep) {
    memset(rep, 0, sizeof(*rep));
    rep->passed = 1;
    for (int32_t j = 0; j < lp->ncol; ++j) {
        double v = x[j];
        if (!isfinite(v)) { rep->passed = 0; return; }
        if (fin(lp->collo[j])) {
            double viol = smax(0.0, lp->collo[j] - v) / (1.0 + fabs(lp->collo[j]));
            if (viol > rep->max_bound_viol) rep->max_bound_viol = viol;
        }
        if (fin(lp->colup[j])) {
            double viol = smax(0.0, v - lp->colup[j]) / (1.0 + fabs(lp->colup[j]));
            if (viol > rep->max_bound_viol) rep->max_bound_viol = viol;
        }
    }
    dd* act = (dd*)calloc((size_t)lp->nrow + 1, sizeof(dd));
    for (int32_t j = 0; j < lp->ncol; ++j) {
        double xj = x[j];
        if (xj == 0.0) continue;
        for (int64_t k = lp->col_start[j]; k < lp->col_start[j + 1]; ++k)
            act[lp->row_index[k]] = dd_add_prod(act[lp->row_index[k]], lp->value[k], xj);
    }
    for (int32_t i = 0; i < lp->nrow; ++i) {
        double r = dd_val(act[i]);
        if (fin(lp->rowlo[i])) {
            double viol = smax(0.0, lp->rowlo[i] - r) / (1.0 + fabs(lp->rowlo[i]));
            if (viol > rep->max_row_viol) rep->max_row_viol = viol;
        }
        if (fin(lp->rowup[i])) {
            double viol = smax(0.0, r - lp->rowup[i]) / (1.0 + fabs(lp->rowup[i]));
            if (viol > rep->max_row_viol) rep->max_row_viol = viol;
        }
    }
    free(act);
    rep->computed_obj = or_eval_objective(lp, x);
    if (isfinite(claimed_obj))
        rep->obj_rel_err = fabs(rep->computed_obj - claimed_obj) / (1.0 + fabs(rep->computed_obj));
    if (rep->max_bound_viol > tol || rep->max_row_viol > tol || rep->obj_rel_err > 1e-5) rep->passed = 0;
}

/* ---------------- relative KKT error ---------------- */

void or_rel_kkt(const nir_lp_view* lp, const double* x, const double* y, or_kkt* out) {
    const int32_t m = lp->nrow, n = lp->ncol;
    dd* ax = (dd*)calloc((size_t)m + 1, sizeof(dd));
    for (int32_t j = 0; j < n; ++j)
        for (int64_t k = lp->col_start[j]; k < lp->col_start[j + 1]; ++k)
            ax[lp->row_index[k]] = dd_add_prod(ax[lp->row_index[k]], lp->value[k], x[j]);
    dd pres2 = {0, 0}, rhs2 = {0, 0}, dres2 = {0, 0}, c2 = {0, 0};
    dd pobj = {lp->obj_offset, 0.0}, dobj = {lp->obj_offset, 0.0};
    double max_rel_row = 0.0;
    for (int32_t i = 0; i < m; ++i) {
        double a = dd_val(ax[i]);
        double lo = lp->rowlo[i], up = lp->rowup[i];
        double r = 0.0, b = 0.0;
        if (fin(lo) && a < lo) r = a - lo;
        if (fin(up) && a > up) r = a - up;
        if (fin(lo)) b = fabs(lo);
        if (fin(up) && fabs(up) > b) b = fabs(up);
        pres2 = dd_add_prod(pres2, r, r);
        rhs2 = dd_add_prod(rhs2, b, b);
        if (r != 0.0) {
            double bb = (r < 0.0) ? fabs(lo) : fabs(up);
            double rel = fabs(r) / (1.0 + bb);
            if (rel > max_rel_row) max_rel_row = rel;
        }
        /* dual objective and wrong-sign multipliers */
        double yi = y[i];
        if (yi > 0.0) {
            if (fin(lo)) dobj = dd_add_prod(dobj, lo, yi);
            else dres2 = dd_add_prod(dres2, yi, yi);
        } else if (yi < 0.0) {
            if (fin(up)) dobj = dd_add_prod(dobj, up, yi);
            else dres2 = dd_add_prod(dres2, yi, yi);
        }
    }
    for (int32_t j = 0; j < n; ++j) {
        dd s = {0, 0};
        for (int64_t k = lp->col_start[j]; k < lp->col_start[j + 1]; ++k)
            s = dd_add_prod(s, lp->value[k], y[lp->row_index[k]]);
        double rc = dd_val(dd_add(dd_add_d((dd){0, 0}, lp->cost[j]), (dd){-s.hi, -s.lo}));
        double l = lp->collo[j], u = lp->colup[j];
        double lam = 0.0;
        if (rc > 0.0 && fin(l)) lam = rc;
        if (rc < 0.0 && fin(u)) lam = rc;
        double d = rc - lam;
        dres2 = dd_add_prod(dres2, d, d);
        if (lam > 0.0) dobj = dd_add_prod(dobj, l, lam);
        else if (lam < 0.0) dobj = dd_add_prod(dobj, u, lam);
        c2 = dd_add_prod(c2, lp->cost[j], lp->cost[j]);
        pobj = dd_add_prod(pobj, lp->cost[j], x[j]);
        double xb = 0.0;
        if (fin(l) && x[j] < l) xb = x[j] - l;
        if (fin(u) && x[j] > u) xb = x[j] - u;
        pres2 = dd_add_prod(pres2, xb, xb);
    }
    free(ax);
    out->pobj = dd_val(pobj);
    out->dobj = dd_val(dobj);
    out->rel_primal = sqrt(dd_val(pres2)) / (1.0 + sqrt(dd_val(rhs2)));
    out->rel_dual = sqrt(dd_val(dres2)) / (1.0 + sqrt(dd_val(c2)));
    out->rel_gap = fabs(out->pobj - out->dobj) / (1.0 + fabs(out->pobj) + fabs(out->dobj));
    double k = out->rel_primal;
    if (out->rel_dual > k) k = out->rel_dual;
    if (out->rel_gap > k) k = out->rel_gap;
    out->rel_kkt = k;
    out->max_rel_row_viol = max_rel_row;
}

/* ---------------- the reference PDHG loop (src/gpu/pdhg_solver.hpp:25-107) ---------------- */

void or_ref_pdhg(const nir_lp_view* lp, int64_t max_iters, int64_t probe_every, double probe_tol,
                 int stop_at_probe, double* x, double* y, or_pdhg_out* out) {
    const int32_t n = lp->ncol, m = lp->nrow;
    double* u = (double*)malloc(sizeof(double) * ((size_t)n + 1));
    double* v = (double*)malloc(sizeof(double) * ((size_t)m + 1));
    double* xbar = (double*)calloc((size_t)n + 1, sizeof(double));
    double* aty = (double*)calloc((size_t)n + 1, sizeof(double));
    double* axb = (double*)calloc((size_t)m + 1, sizeof(double));
    memset(out, 0, sizeof(*out));
    out->first_hit = -1;
    out->last_kkt = NAN;

    /* power iteration for ||A||_2, :33-45 */
    for (int32_t j = 0; j < n; ++j) u[j] = 1.0;
    double norm_est = 1.0;
    for (int p = 0; p < 12; ++p) {
        or_spmv(lp, u, v);
        or_spmv_t(lp, v, u);
        double n2 = 0.0;
        for (int32_t j = 0; j < n; ++j) n2 += u[j] * u[j];
        norm_est = sqrt(smax(1e-12, n2));
        for (int32_t j = 0; j < n; ++j) u[j] /= norm_est;
    }
    double sigma_max = sqrt(norm_est);
    double tau = 0.85 / smax(1e-6, sigma_max);
    double sigma = 0.85 / smax(1e-6, sigma_max);
    out->tau = tau;
    out->sigma = sigma;

    /* box-midpoint start, :47-57 */
    for (int32_t j = 0; j < n; ++j) {
        double lo = lp->collo[j], up = lp->colup[j];
        x[j] = 0.0;
        if (fin(lo) && fin(up)) x[j] = 0.5 * (lo + up);
        else if (fin(lo)) x[j] = smax(0.0, lo);
        else if (fin(up)) x[j] = smin(0.0, up);
    }
    for (int32_t i = 0; i < m; ++i) y[i] = 0.0;

    int64_t iters = 0;
    for (int64_t iter = 0; iter < max_iters; ++iter) {
        iters = iter + 1;
        /* primal step, :69-78 */
        or_spmv_t(lp, y, aty);
        for (int32_t j = 0; j < n; ++j) {
            double cand = x[j] - tau * (lp->cost[j] - aty[j]);
            if (fin(lp->collo[j])) cand = smax(lp->collo[j], cand);
            if (fin(lp->colup[j])) cand = smin(lp->colup[j], cand);
            xbar[j] = 2.0 * cand - x[j];
            x[j] = cand;
        }
        /* dual step and row violation, :80-95 */
        or_spmv(lp, xbar, axb);
        double max_p_viol = 0.0;
        for (int32_t i = 0; i < m; ++i) {
            double target = axb[i] - y[i] / sigma;
            double r = target;
            if (fin(lp->rowlo[i])) r = smax(lp->rowlo[i], r);
            if (fin(lp->rowup[i])) r = smin(lp->rowup[i], r);
            y[i] += sigma * (r - axb[i]);
            double viol = 0.0;
            if (fin(lp->rowlo[i])) viol = smax(viol, lp->rowlo[i] - axb[i]);
            if (fin(lp->rowup[i])) viol = smax(viol, axb[i] - lp->rowup[i]);
            max_p_viol = smax(max_p_viol, viol);
        }
        if (probe_every > 0 && ((iter + 1) % probe_every) == 0) {
            or_kkt k;
            or_rel_kkt(lp, x, y, &k);
            out->last_kkt = k.rel_kkt;
            if (k.rel_kkt <= probe_tol && out->first_hit < 0) {
                out->first_hit = iter + 1;
                if (stop_at_probe) break;
            }
        }
        /* stop test, :97-100 */
        if (iter > 20 && (iter & 31) == 0 && max_p_viol <= 1e-6) {
            out->stopped = 1;
            break;
        }
    }
    out->iterations = iters;
    out->objective = or_eval_objective(lp, x);
    free(u);
    free(v);
    free(xbar);
    free(aty);
    free(axb);
}
