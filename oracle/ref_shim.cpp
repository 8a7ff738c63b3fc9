// ref_shim.cpp -- C ABI over the reference's own code, compiled from the
// reference's sources in place (oracle/Makefile, output oracle/_ref/).
//
// TEST INFRASTRUCTURE ONLY: the tests use it to pin the oracle and the CUDA
// engine against the reference itself, and the benchmark's CPU-baseline leg
// times sov::PdhgSolver::solve through it.  It holds no algorithm of its
// own; every entry point forwards to a reference function:
//   ref_pdhg_solve      sov::PdhgSolver::solve        src/gpu/pdhg_solver.hpp:25-107
//   ref_solver_solve    sov::Solver::solve            include/sov/solver.hpp:128-326
//   ref_verify          sov::verify_solution          src/io/sol_io.hpp:25-106
//   ref_eval_objective  sov::Model::eval_objective    src/model/model.hpp:73-98
//   ref_spmv(_t)        sov::CscMatrix::spmv(_transpose) src/core/csc_matrix.hpp:99-120
//   ref_from_triplets   sov::CscMatrix::from_triplets src/core/csc_matrix.hpp:30-96
//   ref_read_mps        sov::MpsReader::read          src/io/mps_reader.hpp:15-304
//   ref_write_mps       sov::MpsReader::write         src/io/mps_reader.hpp:306-412
//   ref_mps_roundtrip   MpsReader::read then ::write  (names and all kept)
//   ref_presolve        sov::Presolver::presolve      src/presolve/presolve.hpp:32-345
//   ref_write_sol       sov::SolIo::write_sol         src/io/sol_io.hpp:110-132
//   ref_verify_full     sov::verify_solution          src/io/sol_io.hpp:25-106 (every field)
//   ref_scale           sov::scale_model              src/model/scaling.hpp:56-154
//   ref_dd_probe        sov::dd_real / NeumaierSum    src/core/dd_real.hpp:27-104

#include "include/sov/solver.hpp"

#include <cstdio>
#include <cstring>
#include <memory>
#include <string>

#include "../include/nir_lp.h"

namespace {

thread_local std::string g_err;
thread_local int g_status = 0;

sov::Model to_model(const nir_lp_view* v) {
    sov::Model m;
    m.name = "shim";
    m.sense = sov::Sense::Minimize;
    m.obj_offset = v->obj_offset;
    m.ncol = v->ncol;
    m.nrow = v->nrow;
    m.cost.assign(v->cost, v->cost + v->ncol);
    m.collo.assign(v->collo, v->collo + v->ncol);
    m.colup.assign(v->colup, v->colup + v->ncol);
    m.vartype.assign(v->ncol, sov::VarType::Continuous);
    m.rowlo.assign(v->rowlo, v->rowlo + v->nrow);
    m.rowup.assign(v->rowup, v->rowup + v->nrow);
    m.A = sov::CscMatrix(v->nrow, v->ncol);
    m.A.start.assign(v->col_start, v->col_start + v->ncol + 1);
    m.A.index.assign(v->row_index, v->row_index + v->nnz);
    m.A.value.assign(v->value, v->value + v->nnz);
    m.Q = sov::CscMatrix(v->ncol, v->ncol);
    for (sov::Idx j = 0; j < v->ncol; ++j) m.col_names.push_back("C" + std::to_string(j));
    for (sov::Idx i = 0; i < v->nrow; ++i) m.row_names.push_back("R" + std::to_string(i));
    return m;
}

}  // namespace

struct ref_model {
    sov::Model m;
    int sense = 1;
};

extern "C" {

const char* ref_last_error(void) { return g_err.c_str(); }

// PdhgSolver::solve on an already-internal (minimisation) LP.
int ref_pdhg_solve(const nir_lp_view* v, int threads, int simplex_iter_limit, double time_limit,
                   double* x_out, double* y_out, int* status, double* objective, int* iterations) {
    try {
        sov::Model m = to_model(v);
        sov::Options opt;
        opt.threads = threads;
        opt.simplex_iter_limit = simplex_iter_limit;
        opt.log_level = 0;
        sov::Deadline dl;
        dl.wall_limit_sec = time_limit;
        sov::PdhgResult r = sov::PdhgSolver::solve(m, opt, dl);
        if (x_out) std::memcpy(x_out, r.x.data(), sizeof(double) * r.x.size());
        if (y_out) std::memcpy(y_out, r.y.data(), sizeof(double) * r.y.size());
        *status = static_cast<int>(r.status);
        *objective = r.objective;
        *iterations = r.iterations;
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

// Solver::solve with a method ("auto" = dual simplex, "ipm", "pdhg") on a
// model with the given sense; x_out gets the user-space solution.
int ref_solver_solve(const nir_lp_view* v, int sense, const char* method, int presolve, int scale,
                     double* x_out, int* status, double* objective, int* verified) {
    try {
        sov::Model m = to_model(v);
        m.sense = sense < 0 ? sov::Sense::Maximize : sov::Sense::Minimize;
        sov::Options opt;
        opt.log_level = 0;
        opt.method = method ? method : "auto";
        opt.presolve = presolve;
        opt.scale = scale != 0;
        sov::Solver s(opt);
        sov::SolveResult r = s.solve(m);
        *status = static_cast<int>(r.status);
        *objective = r.objective;
        *verified = r.verification.passed ? 1 : 0;
        if (x_out && r.x.size() == static_cast<size_t>(v->ncol))
            std::memcpy(x_out, r.x.data(), sizeof(double) * r.x.size());
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

int ref_verify(const nir_lp_view* v, const double* x, double claimed, double tol, int* passed,
               double* max_bound_viol, double* max_row_viol, double* computed_obj, double* obj_rel_err) {
    sov::Model m = to_model(v);
    std::vector<double> xv(x, x + v->ncol);
    sov::VerificationReport r = sov::verify_solution(m, xv, claimed, tol);
    *passed = r.passed ? 1 : 0;
    *max_bound_viol = r.max_bound_viol;
    *max_row_viol = r.max_row_viol;
    *computed_obj = r.computed_obj;
    *obj_rel_err = r.obj_rel_err;
    return 0;
}

double ref_eval_objective(const nir_lp_view* v, const double* x) {
    sov::Model m = to_model(v);
    return m.eval_objective(std::vector<double>(x, x + v->ncol));
}

void ref_spmv(const nir_lp_view* v, const double* x, double* y) {
    sov::Model m = to_model(v);
    std::vector<double> yy;
    m.A.spmv(std::vector<double>(x, x + v->ncol), yy);
    std::memcpy(y, yy.data(), sizeof(double) * yy.size());
}

void ref_spmv_t(const nir_lp_view* v, const double* x, double* y) {
    sov::Model m = to_model(v);
    std::vector<double> yy;
    m.A.spmv_transpose(std::vector<double>(x, x + v->nrow), yy);
    std::memcpy(y, yy.data(), sizeof(double) * yy.size());
}

int64_t ref_from_triplets(int32_t nrow, int32_t ncol, int64_t ntrip, const int32_t* r, const int32_t* c,
                          const double* val, int64_t* start, int32_t* index, double* value) {
    std::vector<sov::Triplet> t(ntrip);
    for (int64_t k = 0; k < ntrip; ++k) t[k] = {r[k], c[k], val[k]};
    sov::CscMatrix A = sov::CscMatrix::from_triplets(nrow, ncol, t);
    std::memcpy(start, A.start.data(), sizeof(int64_t) * A.start.size());
    std::memcpy(index, A.index.data(), sizeof(int32_t) * A.index.size());
    std::memcpy(value, A.value.data(), sizeof(double) * A.value.size());
    return A.nnz();
}

void ref_dd_probe(double a, double b, double c, double* dd_out, double* neumaier_out) {
    sov::dd_real acc(0.0);
    acc += a;
    acc += b;
    acc += c;
    *dd_out = acc.to_double();
    sov::NeumaierSum s;
    s.add(a);
    s.add(b);
    s.add(c);
    *neumaier_out = s.result();
}

// MPS reader: returns a handle whose internal-minimisation LP is exposed
// through ref_model_view (sense is +1 min / -1 max of the file).
ref_model* ref_read_mps(const char* path) {
    auto h = std::make_unique<ref_model>();
    std::string err;
    sov::Status st;
    try {
        st = sov::MpsReader::read(path, h->m, err);
    } catch (const std::exception& e) {
        // the reader lets std::stod's exceptions escape
        g_err = std::string("exception: ") + e.what();
        g_status = -1;
        return nullptr;
    }
    if (st != sov::Status::Optimal) {
        g_err = err;
        g_status = static_cast<int>(st);
        return nullptr;
    }
    g_status = 0;
    h->sense = (h->m.sense == sov::Sense::Maximize) ? -1 : 1;
    h->m = h->m.to_internal_min();
    return h.release();
}

int ref_last_status(void) { return g_status; }

// Reads `in` with the reference reader and writes the model back with the
// reference writer; 0 on success, else the read status (-1: exception).
int ref_mps_roundtrip(const char* in, const char* out) {
    sov::Model m;
    std::string err;
    try {
        const sov::Status st = sov::MpsReader::read(in, m, err);
        if (st != sov::Status::Optimal) {
            g_err = err;
            return static_cast<int>(st);
        }
    } catch (const std::exception& e) {
        g_err = std::string("exception: ") + e.what();
        return -1;
    }
    return sov::MpsReader::write(out, m) ? 0 : 14;
}

int ref_model_vartypes(const ref_model* h, int8_t* out) {
    if (!h) return 1;
    for (sov::Idx j = 0; j < h->m.ncol; ++j) out[j] = static_cast<int8_t>(h->m.vartype[j]);
    return 0;
}

int64_t ref_model_qnnz(const ref_model* h) { return h ? h->m.Q.nnz() : 0; }

int ref_model_q(const ref_model* h, int64_t* start, int32_t* index, double* value) {
    if (!h) return 1;
    const sov::CscMatrix& Q = h->m.Q;
    for (sov::Idx j = 0; j <= h->m.ncol; ++j) start[j] = Q.start.empty() ? 0 : Q.start[j];
    for (sov::Off k = 0; k < Q.nnz(); ++k) {
        index[k] = Q.index[k];
        value[k] = Q.value[k];
    }
    return 0;
}

// MPS writer over an LP view with variable types and a sense (+1 / -1).
int ref_write_mps(const nir_lp_view* v, const int8_t* vartype, int sense, const char* path) {
    sov::Model m = to_model(v);
    m.name = "written";
    m.sense = sense < 0 ? sov::Sense::Maximize : sov::Sense::Minimize;
    if (vartype)
        for (sov::Idx j = 0; j < v->ncol; ++j) m.vartype[j] = static_cast<sov::VarType>(vartype[j]);
    return sov::MpsReader::write(path, m) ? 0 : 1;
}

int ref_model_view(const ref_model* h, nir_lp_view* v, int* sense) {
    if (!h) return 1;
    const sov::Model& m = h->m;
    v->nrow = m.nrow;
    v->ncol = m.ncol;
    v->nnz = m.A.nnz();
    v->col_start = m.A.start.data();
    v->row_index = m.A.index.data();
    v->value = m.A.value.data();
    v->cost = m.cost.data();
    v->collo = m.collo.data();
    v->colup = m.colup.data();
    v->rowlo = m.rowlo.data();
    v->rowup = m.rowup.data();
    v->obj_offset = m.obj_offset;
    *sense = h->sense;
    return 0;
}

void ref_model_free(ref_model* h) { delete h; }

struct ref_presolved {
    sov::PresolveResult r;
};

ref_presolved* ref_presolve(const nir_lp_view* v, const int8_t* vartype, int level, int rounds) {
    sov::Model m = to_model(v);
    if (vartype)
        for (sov::Idx j = 0; j < v->ncol; ++j) m.vartype[size_t(j)] = static_cast<sov::VarType>(vartype[j]);
    auto h = std::make_unique<ref_presolved>();
    h->r = sov::Presolver::presolve(m, level, rounds);
    return h.release();
}

int ref_presolved_status(const ref_presolved* h, int* status, int* solved, int* counters3) {
    *status = static_cast<int>(h->r.status);
    *solved = h->r.solved_in_presolve ? 1 : 0;
    counters3[0] = h->r.rows_removed;
    counters3[1] = h->r.cols_removed;
    counters3[2] = h->r.bound_tightenings;
    return 0;
}

int ref_presolved_reduced(const ref_presolved* h, nir_lp_view* v, int8_t* vartype) {
    const sov::Model& m = h->r.reduced;
    v->nrow = m.nrow;
    v->ncol = m.ncol;
    v->nnz = m.A.nnz();
    v->col_start = m.A.start.data();
    v->row_index = m.A.index.data();
    v->value = m.A.value.data();
    v->cost = m.cost.data();
    v->collo = m.collo.data();
    v->colup = m.colup.data();
    v->rowlo = m.rowlo.data();
    v->rowup = m.rowup.data();
    v->obj_offset = m.obj_offset;
    if (vartype)
        for (sov::Idx j = 0; j < m.ncol; ++j) vartype[j] = static_cast<int8_t>(m.vartype[size_t(j)]);
    return 0;
}

// sizes: col_map / row_map as the reduced model, fixed_x / is_fixed as the original
int ref_presolved_maps(const ref_presolved* h, int32_t* col_map, int32_t* row_map, double* fixed_x, uint8_t* is_fixed) {
    for (size_t j = 0; j < h->r.orig_col_map.size(); ++j) col_map[j] = h->r.orig_col_map[j];
    for (size_t i = 0; i < h->r.orig_row_map.size(); ++i) row_map[i] = h->r.orig_row_map[i];
    for (size_t j = 0; j < h->r.fixed_x.size(); ++j) fixed_x[j] = h->r.fixed_x[j];
    for (size_t j = 0; j < h->r.is_col_fixed.size(); ++j) is_fixed[j] = h->r.is_col_fixed[j] ? 1 : 0;
    return 0;
}

int64_t ref_presolved_map_sizes(const ref_presolved* h, int64_t* ncols) {
    *ncols = int64_t(h->r.orig_col_map.size());
    return int64_t(h->r.orig_row_map.size());
}

void ref_presolved_free(ref_presolved* h) { delete h; }

namespace {
sov::Model named_model(const nir_lp_view* v, const int8_t* vartype, const char* const* names) {
    sov::Model m = to_model(v);
    if (vartype)
        for (sov::Idx j = 0; j < v->ncol; ++j) m.vartype[size_t(j)] = static_cast<sov::VarType>(vartype[j]);
    if (names)
        for (sov::Idx j = 0; j < v->ncol; ++j) m.col_names[size_t(j)] = names[j];
    return m;
}
}  // namespace

int ref_write_sol(const nir_lp_view* v, const char* const* names, int status, double obj, double gap,
                  const double* x, int64_t nx, const char* path) {
    sov::Model m = named_model(v, nullptr, names);
    std::vector<double> xv(x, x + nx);
    return sov::SolIo::write_sol(path, m, static_cast<sov::Status>(status), obj, gap, xv) ? 0 : 14;
}

int ref_verify_full(const nir_lp_view* v, const int8_t* vartype, const char* const* names, const double* x,
                    int64_t nx, double claimed, double tol, int* passed, double* out5, char* worst, int worst_cap) {
    sov::Model m = named_model(v, vartype, names);
    std::vector<double> xv(x, x + nx);
    sov::VerificationReport r = sov::verify_solution(m, xv, claimed, tol);
    *passed = r.passed ? 1 : 0;
    out5[0] = r.max_bound_viol;
    out5[1] = r.max_row_viol;
    out5[2] = r.max_int_viol;
    out5[3] = r.computed_obj;
    out5[4] = r.obj_rel_err;
    std::snprintf(worst, size_t(worst_cap), "%s", r.worst_item.c_str());
    return 0;
}

// scale_model: scales and the scaled arrays (Q scaled when qnnz > 0)
int ref_scale(const nir_lp_view* v, const int8_t* vartype, int enable, int64_t qnnz, const int64_t* q_start,
              const int32_t* q_index, const double* q_value, double* R, double* C, int* active, double* cost,
              double* collo, double* colup, double* value, double* rowlo, double* rowup, double* q_out) {
    sov::Model m = to_model(v);
    if (vartype)
        for (sov::Idx j = 0; j < v->ncol; ++j) m.vartype[size_t(j)] = static_cast<sov::VarType>(vartype[j]);
    if (qnnz > 0) {
        m.Q.start.assign(q_start, q_start + v->ncol + 1);
        m.Q.index.assign(q_index, q_index + qnnz);
        m.Q.value.assign(q_value, q_value + qnnz);
    }
    sov::ScalingInfo info;
    sov::Model s = sov::scale_model(m, enable != 0, info);
    *active = info.active ? 1 : 0;
    std::copy(info.R.begin(), info.R.end(), R);
    std::copy(info.C.begin(), info.C.end(), C);
    std::copy(s.cost.begin(), s.cost.end(), cost);
    std::copy(s.collo.begin(), s.collo.end(), collo);
    std::copy(s.colup.begin(), s.colup.end(), colup);
    std::copy(s.A.value.begin(), s.A.value.end(), value);
    std::copy(s.rowlo.begin(), s.rowlo.end(), rowlo);
    std::copy(s.rowup.begin(), s.rowup.end(), rowup);
    if (qnnz > 0) std::copy(s.Q.value.begin(), s.Q.value.end(), q_out);
    return 0;
}

}  // extern "C"
