// Drop-in replacement for the reference's src/io/mps_reader.hpp.
//
// Same class and signatures as the file it replaces
// (src/io/mps_reader.hpp:13-15, :306): `sov::MpsReader::read(path, Model&,
// std::string&)` and `sov::MpsReader::write(path, const Model&)`, so the
// CLI (src/driver/cli_main.cpp:89), the C API's sov_read_mps /
// sov_write_mps (src/driver/c_api.cpp:101-120), Solver and the checker
// (tools/checker.cpp:17) read and write through libnir_mps.so
// (include/nir_mps.h):
//   * read: the multi-threaded reader returns the model MpsReader::read
//     builds -- name, sense, offset, matrix, bounds, variable types, names,
//     the quadratic block -- already through Model::validate, whose status
//     (0, 1 infeasible bounds, 12 input error) and message it returns.  A
//     token that is not a number gives InputError with its line, where the
//     reference lets std::stod's exception escape;
//   * write: the parallel writer emits MpsReader::write's bytes.
// NIR_MPS_THREADS sets the thread count (default: all hardware threads).
#pragma once
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "../model/model.hpp"
#include "nir_mps.h"

namespace sov {

class MpsReader {
public:
    static Status read(const std::string& path, Model& out_model, std::string& error_msg) {
        nir_mps* h = nullptr;
        const int st = nir_mps_read(path.c_str(), threads(), &h);
        if (st != 0) {
            error_msg = nir_mps_last_error();
            return static_cast<Status>(st);
        }
        nir_lp_view v;
        int32_t sense = 1;
        nir_mps_view(h, &v, &sense);
        Model m;
        m.name = nir_mps_model_name(h);
        m.sense = sense < 0 ? Sense::Maximize : Sense::Minimize;
        m.obj_offset = v.obj_offset;
        m.ncol = v.ncol;
        m.nrow = v.nrow;
        m.cost.assign(v.cost, v.cost + v.ncol);
        m.collo.assign(v.collo, v.collo + v.ncol);
        m.colup.assign(v.colup, v.colup + v.ncol);
        const int8_t* vt = nir_mps_vartypes(h);
        m.vartype.resize(size_t(v.ncol));
        for (Idx j = 0; j < v.ncol; ++j) m.vartype[size_t(j)] = static_cast<VarType>(vt[j]);
        m.A = CscMatrix(v.nrow, v.ncol);
        m.A.start.assign(v.col_start, v.col_start + v.ncol + 1);
        m.A.index.assign(v.row_index, v.row_index + v.nnz);
        m.A.value.assign(v.value, v.value + v.nnz);
        m.rowlo.assign(v.rowlo, v.rowlo + v.nrow);
        m.rowup.assign(v.rowup, v.rowup + v.nrow);
        names(h, 0, v.ncol, m.col_names);
        names(h, 1, v.nrow, m.row_names);
        int64_t qnnz = 0;
        const int64_t* qs = nullptr;
        const int32_t* qi = nullptr;
        const double* qv = nullptr;
        nir_mps_quadratic(h, &qnnz, &qs, &qi, &qv);
        m.Q = CscMatrix(v.ncol, v.ncol);
        m.Q.start.assign(qs, qs + v.ncol + 1);
        m.Q.index.assign(qi, qi + qnnz);
        m.Q.value.assign(qv, qv + qnnz);
        nir_mps_free(h);
        out_model = std::move(m);
        return Status::Optimal;
    }

    static bool write(const std::string& path, const Model& m) {
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
        std::vector<int8_t> vt(size_t(m.ncol));
        for (Idx j = 0; j < m.ncol; ++j) vt[size_t(j)] = static_cast<int8_t>(m.vartype[size_t(j)]);
        // the reference's per-index fallback to generated names
        std::vector<std::string> gen;
        gen.reserve(size_t(m.ncol) + size_t(m.nrow));
        std::vector<const char*> cn(size_t(m.ncol)), rn(size_t(m.nrow));
        for (Idx j = 0; j < m.ncol; ++j) {
            if (j < static_cast<Idx>(m.col_names.size())) {
                cn[size_t(j)] = m.col_names[size_t(j)].c_str();
            } else {
                gen.push_back("C" + std::to_string(j));
                cn[size_t(j)] = gen.back().c_str();
            }
        }
        for (Idx i = 0; i < m.nrow; ++i) {
            if (i < static_cast<Idx>(m.row_names.size())) {
                rn[size_t(i)] = m.row_names[size_t(i)].c_str();
            } else {
                gen.push_back("R" + std::to_string(i));
                rn[size_t(i)] = gen.back().c_str();
            }
        }
        const int64_t qnnz = m.Q.nnz();
        return nir_mps_write(&v, vt.data(), m.sense == Sense::Maximize ? -1 : 1, m.name.c_str(), cn.data(), rn.data(),
                             qnnz, qnnz > 0 ? m.Q.start.data() : nullptr, qnnz > 0 ? m.Q.index.data() : nullptr,
                             qnnz > 0 ? m.Q.value.data() : nullptr, threads(), path.c_str()) == 0;
    }

private:
    static int32_t threads() {
        const char* e = std::getenv("NIR_MPS_THREADS");
        return e ? static_cast<int32_t>(std::atoi(e)) : 0;
    }
    static void names(const nir_mps* h, int32_t rows, Idx n, std::vector<std::string>& out) {
        const char* chars = nullptr;
        const int64_t* off = nullptr;
        nir_mps_names(h, rows, &chars, &off);
        out.clear();
        out.reserve(size_t(n));
        for (Idx i = 0; i < n; ++i) out.emplace_back(chars + off[i], size_t(off[i + 1] - off[i]));
    }
};

}  // namespace sov
