// Multi-threaded MPS writer (C ABI: include/nir_mps.h, nir_mps_write).
//
// The bytes are those of sov::MpsReader::write (src/io/mps_reader.hpp:
// 306-412): the same sections and line formats (printf "%-10s" name fields,
// "%.17g" numbers, 256-byte line buffers), the same row-type and bound-type
// choices, markers around runs of integer columns, generated C<j> / R<i>
// names where none are given.  Every section is cut into one range of rows
// or columns per thread, formatted into memory in parallel and written with
// one pwrite per range at its offset.
#include <fcntl.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "nir_mps.h"

namespace {

constexpr double kInfInput = 1e20;  // src/core/types.hpp:16

inline bool finite_bound(double b) { return std::isfinite(b) && std::abs(b) < kInfInput; }

struct Names {
    const char* const* given;
    char prefix;
    // the name of item i: the given one, or prefix + decimal index
    const char* get(int64_t i, char* tmp) const {
        if (given) return given[i];
        std::snprintf(tmp, 32, "%c%lld", prefix, (long long)i);
        return tmp;
    }
};

// snprintf into a 256-byte buffer and append what it holds, as the
// reference does with `snprintf(buf, sizeof(buf), ...); out << buf;`
template <class... A>
inline void line(std::string& out, const char* fmt, A... a) {
    char buf[256];
    const int r = std::snprintf(buf, sizeof(buf), fmt, a...);
    if (r > 0) out.append(buf, size_t(std::min(r, int(sizeof(buf)) - 1)));
}

template <class F>
void run_threads(int nt, F&& f) {
    if (nt <= 1) {
        f(0);
        return;
    }
    std::vector<std::thread> th;
    for (int k = 1; k < nt; ++k) th.emplace_back([&f, k] { f(k); });
    f(0);
    for (auto& x : th) x.join();
}

}  // namespace

namespace nir {
void set_mps_error(const std::string& msg);  // mps.cpp: what nir_mps_last_error returns
}

extern "C" int nir_mps_write(const nir_lp_view* lp, const int8_t* vartype, int32_t sense, const char* model_name,
                             const char* const* col_names, const char* const* row_names, int64_t qnnz,
                             const int64_t* q_start, const int32_t* q_index, const double* q_value, int32_t threads,
                             const char* path) {
    if (!lp || !path || (qnnz > 0 && (!q_start || !q_index || !q_value))) {
        nir::set_mps_error("null argument");
        return 12;
    }
    const int32_t nrow = lp->nrow, ncol = lp->ncol;
    const int T = threads > 0 ? threads : int(std::max(1u, std::thread::hardware_concurrency()));
    const Names cn{col_names, 'C'}, rn{row_names, 'R'};
    auto is_int = [&](int32_t j) { return vartype && (vartype[j] == 1 || vartype[j] == 2); };

    // chunks in file order; each section's ranges are filled in parallel
    std::vector<std::string> chunks;
    auto section = [&](int64_t n, const std::string& head, auto&& body, const std::string& tail = std::string()) {
        chunks.push_back(head);
        const int nt = int(std::max<int64_t>(1, std::min<int64_t>(T, n / 4096 + 1)));
        const size_t c0 = chunks.size();
        chunks.resize(c0 + size_t(nt));
        run_threads(nt, [&](int k) {
            std::string& out = chunks[c0 + size_t(k)];
            const int64_t a = n * k / nt, b = n * (k + 1) / nt;
            out.reserve(size_t(b - a) * 48);
            for (int64_t i = a; i < b; ++i) body(out, i);
        });
        if (!tail.empty()) chunks.push_back(tail);
    };

    std::string head = std::string("NAME          ") + (model_name ? model_name : "") + "\n";
    head += std::string("OBJSENSE\n  ") + (sense < 0 ? "MAX" : "MIN") + "\n";
    head += "ROWS\n N  OBJ\n";
    section(nrow, head, [&](std::string& out, int64_t i) {
        const double lo = lp->rowlo[i], up = lp->rowup[i];
        char rt = 'E';
        if (!finite_bound(lo) && finite_bound(up)) rt = 'L';
        else if (finite_bound(lo) && !finite_bound(up)) rt = 'G';
        else if (lo < up) rt = 'G';  // ranged: the RANGES line follows
        char tmp[32];
        out += ' ';
        out += rt;
        out += "  ";
        out += rn.get(i, tmp);
        out += '\n';
    });
    section(ncol, "COLUMNS\n", [&](std::string& out, int64_t j) {
        const bool now_int = is_int(int32_t(j)), before = j > 0 && is_int(int32_t(j - 1));
        if (now_int && !before) out += "    MARK0000  'MARKER'                 'INTORG'\n";
        else if (!now_int && before) out += "    MARK0001  'MARKER'                 'INTEND'\n";
        char tmp[32], tmp2[32];
        const char* c = cn.get(j, tmp);
        if (lp->cost[j] != 0.0) line(out, "    %-10s %-10s %.17g\n", c, "OBJ", lp->cost[j]);
        for (int64_t k = lp->col_start[j]; k < lp->col_start[j + 1]; ++k)
            line(out, "    %-10s %-10s %.17g\n", c, rn.get(lp->row_index[k], tmp2), lp->value[k]);
    }, ncol > 0 && is_int(ncol - 1) ? std::string("    MARK0001  'MARKER'                 'INTEND'\n") : "");
    std::string rhs_head = "RHS\n";
    if (lp->obj_offset != 0.0) line(rhs_head, "    RHS1       %-10s %.17g\n", "OBJ", -lp->obj_offset);
    section(nrow, rhs_head, [&](std::string& out, int64_t i) {
        const double v = finite_bound(lp->rowlo[i]) ? lp->rowlo[i] : lp->rowup[i];
        char tmp[32];
        if (v != 0.0 && finite_bound(v)) line(out, "    RHS1       %-10s %.17g\n", rn.get(i, tmp), v);
    });
    section(nrow, "RANGES\n", [&](std::string& out, int64_t i) {
        const double lo = lp->rowlo[i], up = lp->rowup[i];
        char tmp[32];
        if (finite_bound(lo) && finite_bound(up) && lo < up)
            line(out, "    RNG1       %-10s %.17g\n", rn.get(i, tmp), up - lo);
    });
    section(ncol, "BOUNDS\n", [&](std::string& out, int64_t j) {
        const double lo = lp->collo[j], up = lp->colup[j];
        char tmp[32];
        const char* c = cn.get(j, tmp);
        if (vartype && vartype[j] == 2 && lo == 0.0 && up == 1.0) {
            line(out, " BV BND1       %s\n", c);
            return;
        }
        if (!finite_bound(lo) && !finite_bound(up)) {
            line(out, " FR BND1       %s\n", c);
            return;
        }
        if (finite_bound(lo) && finite_bound(up) && lo == up) {
            line(out, " FX BND1       %-10s %.17g\n", c, lo);
            return;
        }
        if (!finite_bound(lo)) line(out, " MI BND1       %s\n", c);
        else if (lo != 0.0) line(out, " LO BND1       %-10s %.17g\n", c, lo);
        if (finite_bound(up)) line(out, " UP BND1       %-10s %.17g\n", c, up);
    });
    if (qnnz > 0) {
        section(ncol, "QUADOBJ\n", [&](std::string& out, int64_t j) {
            char tmp[32], tmp2[32];
            const char* c2 = cn.get(j, tmp2);
            for (int64_t k = q_start[j]; k < q_start[j + 1]; ++k)
                line(out, "    %-10s %-10s %.17g\n", cn.get(q_index[k], tmp), c2, q_value[k]);
        });
    }
    chunks.push_back("ENDATA\n");

    const int fd = ::open(path, O_WRONLY | O_CREAT | O_TRUNC, 0666);
    if (fd < 0) {
        nir::set_mps_error(std::string("Cannot open ") + path + " for writing");
        return 14;
    }
    std::vector<size_t> off(chunks.size() + 1, 0);
    for (size_t c = 0; c < chunks.size(); ++c) off[c + 1] = off[c] + chunks[c].size();
    const int nt = int(std::max<size_t>(1, std::min<size_t>(size_t(T), chunks.size())));
    std::vector<int> fail(size_t(nt), 0);
    run_threads(nt, [&](int k) {
        for (size_t c = size_t(k); c < chunks.size(); c += size_t(nt)) {
            size_t done = 0;
            while (done < chunks[c].size()) {
                const ssize_t w = ::pwrite(fd, chunks[c].data() + done, chunks[c].size() - done, off_t(off[c] + done));
                if (w < 0 && errno == EINTR) continue;
                if (w <= 0) {
                    fail[size_t(k)] = 1;
                    return;
                }
                done += size_t(w);
            }
        }
    });
    const bool closed = ::close(fd) == 0;
    for (int f : fail)
        if (f || !closed) {
            nir::set_mps_error(std::string("Cannot write ") + path);
            return 14;
        }
    return 0;
}
