// SOL file I/O and the double-double solution check (C ABI: include/nir_sol.h).
//
// The reference's SolIo::write_sol / read_sol and verify_solution
// (src/io/sol_io.hpp:25-170) work on one thread.  Here:
//   write   each thread formats a range of columns with the reference's
//           snprintf formats into memory; the ranges are written with one
//           pwrite each at their offsets, so the bytes are the same;
//   read    each thread takes a range of lines: tokens split as istream's
//           >> splits them, the value taken as num_get takes a double in
//           the C locale (below), the name looked up in a table of the
//           model's names; the assignments are then applied in file order;
//   verify  bounds and integrality in parallel over columns, double-double
//           row activities in parallel over rows (each row's terms added in
//           ascending column order, the order of the reference's column
//           scatter), reductions that keep the first index of each maximum
//           so the reference's choice of worst item is reproduced.
// Compiled without FMA contraction: the double-double steps rely on exact
// roundings of each operation, as in the reference's build.
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <limits>
#include <string>

#include "decimal.hpp"
#include "nir_sol.h"
#include "text.hpp"

namespace {

using namespace nir::text;

constexpr double kInfInput = 1e20;  // src/core/types.hpp:16
inline bool fin(double b) { return std::isfinite(b) && std::abs(b) < kInfInput; }

thread_local std::vector<std::string> g_obj_tokens;

int hw(int t) { return t > 0 ? t : int(std::max(1u, std::thread::hardware_concurrency())); }

// ---- double-double arithmetic (Knuth two-sum, Dekker's product via fma):
// the reference's dd_real steps (src/core/dd_real.hpp:7-83) in the same
// order, so that every rounding is the same
struct DD {
    double hi = 0.0, lo = 0.0;
};

inline void two_sum(double a, double b, double& s, double& e) {
    s = a + b;
    const double bb = s - a;
    e = (a - (s - bb)) + (b - bb);
}

inline void quick_two_sum(double a, double b, double& s, double& e) {
    s = a + b;
    e = b - (s - a);
}

inline void add_dd(DD& d, double bhi, double blo) {
    double s1, s2, t1, t2;
    two_sum(d.hi, bhi, s1, s2);
    two_sum(d.lo, blo, t1, t2);
    s2 += t1;
    quick_two_sum(s1, s2, s1, s2);
    s2 += t2;
    quick_two_sum(s1, s2, d.hi, d.lo);
}

inline void add_prod(DD& d, double a, double b) {
    const double p = a * b;
    const double e = std::fma(a, b, -p);
    add_dd(d, p, e);
}

// ---- whole-file read (regular files in parallel; pipes as a stream; a
// directory opens and has no lines, as with std::ifstream)
bool read_all(const char* path, std::vector<char>& buf, int threads) {
    const int fd = ::open(path, O_RDONLY);
    if (fd < 0) return false;
    struct stat st;
    if (::fstat(fd, &st) != 0) {
        ::close(fd);
        return false;
    }
    constexpr size_t kPad = 64;
    if (!S_ISREG(st.st_mode)) {
        buf.clear();
        if (!S_ISDIR(st.st_mode)) {
            std::vector<char> tmp(size_t(1) << 16);
            for (;;) {
                const ssize_t r = ::read(fd, tmp.data(), tmp.size());
                if (r < 0 && errno == EINTR) continue;
                if (r <= 0) break;
                buf.insert(buf.end(), tmp.data(), tmp.data() + r);
            }
        }
        ::close(fd);
        buf.resize(buf.size() + kPad, '\n');
        return true;
    }
    const size_t size = size_t(st.st_size);
    buf.resize(size + kPad);
    std::memset(buf.data() + size, '\n', kPad);
    const int nt = int(std::max<size_t>(1, std::min<size_t>(size_t(threads), size / (size_t(8) << 20) + 1)));
    std::vector<size_t> got(static_cast<size_t>(nt), 0);
    run_threads(nt, [&](int k) {
        size_t off = size * size_t(k) / size_t(nt);
        const size_t end = size * size_t(k + 1) / size_t(nt);
        while (off < end) {
            const ssize_t r = ::pread(fd, buf.data() + off, end - off, off_t(off));
            if (r < 0 && errno == EINTR) continue;
            if (r <= 0) break;  // a file that shrank: what was read is what there is
            off += size_t(r);
            got[size_t(k)] += size_t(r);
        }
    });
    ::close(fd);
    size_t total = 0;
    for (size_t g : got) total += g;
    if (total != size) {  // keep the bytes as an ifstream would see them: up to the short read
        size_t keep = 0;
        for (int k = 0; k < nt; ++k) {
            const size_t want = size * size_t(k + 1) / size_t(nt) - size * size_t(k) / size_t(nt);
            keep += got[size_t(k)];
            if (got[size_t(k)] != want) break;
        }
        std::memset(buf.data() + keep, '\n', size + kPad - keep);
        buf.resize(keep + kPad);
    }
    return true;
}

// `istream >> double` in the C locale (libstdc++'s num_get::_M_extract_float
// followed by its strtod conversion): the longest prefix that fits
// [sign] digits [. digits] [(e|E) [sign] digits] -- an exponent only after
// a mantissa digit -- converted by strtod; the extraction fails when that
// prefix does not convert completely or converts to an infinity.
bool extract_double(const char* p, const char* e, double& v) {
    while (p < e && is_space(*p)) ++p;
    if (p == e) return false;
    char small[128];
    std::string big;
    size_t n = 0;
    auto put = [&](char c) {
        if (n + 1 < sizeof(small)) {
            small[n++] = c;
        } else {
            if (big.empty()) big.assign(small, n);
            big += c;
            ++n;
        }
    };
    const char* q = p;
    if (q < e && (*q == '+' || *q == '-')) put(*q++);
    bool mantissa = false, dec = false, sci = false;
    while (q < e && *q == '0') {
        if (!mantissa) {
            put('0');
            mantissa = true;
        }
        ++q;
    }
    while (q < e) {
        const char c = *q;
        if (c >= '0' && c <= '9') {
            put(c);
            mantissa = true;
        } else if (c == '.' && !dec && !sci) {
            put('.');
            dec = true;
        } else if ((c == 'e' || c == 'E') && !sci && mantissa) {
            put('e');
            sci = true;
            if (++q == e) break;
            if (*q == '+' || *q == '-') put(*q);
            else continue;
        } else {
            break;
        }
        ++q;
    }
    const char* s;
    if (big.empty()) {
        small[n] = 0;
        s = small;
    } else {
        s = big.c_str();
    }
    if (n == 0) return false;
    if (nir::decimal::parse_decimal(s, n, v)) return true;  // a finite, exactly rounded value
    char* end = nullptr;
    v = std::strtod(s, &end);
    if (end == s || *end != '\0') return false;
    if (std::isinf(v)) return false;
    return true;
}

struct Names {
    const char* const* given;
    int64_t n;
    const char* get(int64_t i, char* tmp) const {
        if (i < n) return given[i];
        std::snprintf(tmp, 32, "C%lld", (long long)i);
        return tmp;
    }
};

}  // namespace

extern "C" {

int nir_sol_write(const char* path, const char* status_text, double objective, double gap, int32_t ncol,
                  const double* x, int64_t nx, const char* const* col_names, int64_t n_names, int32_t threads) {
    if (!path || (nx > 0 && !x) || (n_names > 0 && !col_names)) return 12;
    const int64_t cols = std::min<int64_t>(ncol, nx);
    const Names nm{col_names, n_names};
    std::string head = std::string("# status ") + (status_text ? status_text : "") + "\n";
    char b[256];
    std::snprintf(b, sizeof(b), "# objective %.17g\n", objective);
    head += b;
    std::snprintf(b, sizeof(b), "# gap %.6e\n", gap);
    head += b;
    const int nt = int(std::max<int64_t>(1, std::min<int64_t>(hw(threads), cols / 8192 + 1)));
    std::vector<std::string> chunk(static_cast<size_t>(nt) + 1);
    chunk[0] = head;
    run_threads(nt, [&](int k) {
        std::string& out = chunk[size_t(k) + 1];
        const int64_t a = cols * k / nt, e = cols * (k + 1) / nt;
        out.reserve(size_t(e - a) * 32);
        char line[256], tmp[32];
        for (int64_t j = a; j < e; ++j) {
            const int r = std::snprintf(line, sizeof(line), "%s %.17g\n", nm.get(j, tmp), x[j]);
            if (r > 0) out.append(line, size_t(std::min(r, int(sizeof(line)) - 1)));
        }
    });
    const int fd = ::open(path, O_WRONLY | O_CREAT | O_TRUNC, 0666);
    if (fd < 0) return 14;
    std::vector<size_t> off(chunk.size() + 1, 0);
    for (size_t c = 0; c < chunk.size(); ++c) off[c + 1] = off[c] + chunk[c].size();
    std::vector<int> fail(chunk.size(), 0);
    run_threads(int(chunk.size()), [&](int c) {
        size_t done = 0;
        while (done < chunk[size_t(c)].size()) {
            const ssize_t w = ::pwrite(fd, chunk[size_t(c)].data() + done, chunk[size_t(c)].size() - done,
                                       off_t(off[size_t(c)] + done));
            if (w < 0 && errno == EINTR) continue;
            if (w <= 0) {
                fail[size_t(c)] = 1;
                return;
            }
            done += size_t(w);
        }
    });
    const bool closed = ::close(fd) == 0;
    for (int f : fail)
        if (f || !closed) return 14;
    return 0;
}

int nir_sol_read(const char* path, int32_t ncol, const char* const* col_names, int32_t threads, double* x_out,
                 double* objective, int32_t* n_objective_lines) {
    g_obj_tokens.clear();
    if (!path || ncol < 0 || (ncol > 0 && (!col_names || !x_out))) return 12;
    const int T = hw(threads);
    std::vector<char> buf;
    if (!read_all(path, buf, T)) return 14;
    for (int32_t j = 0; j < ncol; ++j) x_out[j] = 0.0;
    // the model's names; a name given twice maps to its last column
    NameMap names;
    names.reserve(size_t(ncol));
    for (int32_t j = 0; j < ncol; ++j) names.assign(col_names[j], std::strlen(col_names[j]), j);
    const size_t size = buf.size() - 64;
    const char* B = buf.data();
    // runs of whole lines
    const int nt = int(std::max<size_t>(1, std::min<size_t>(size_t(T), size / (size_t(1) << 18) + 1)));
    std::vector<size_t> at(static_cast<size_t>(nt) + 1, size);
    at[0] = 0;
    for (int k = 1; k < nt; ++k) {
        size_t x = size * size_t(k) / size_t(nt);
        if (x > 0 && B[x - 1] != '\n') {
            const void* q = std::memchr(B + x, '\n', size - x);
            x = q ? size_t(static_cast<const char*>(q) - B) + 1 : size;
        }
        at[size_t(k)] = std::max(at[size_t(k) - 1], x);
    }
    struct Set {
        int32_t j;
        double v;
    };
    std::vector<std::vector<Set>> sets(static_cast<size_t>(nt));
    std::vector<std::vector<std::string>> objs(static_cast<size_t>(nt));
    run_threads(nt, [&](int k) {
        std::vector<Tok> tk;
        auto& out = sets[size_t(k)];
        for (size_t lb = at[size_t(k)]; lb < at[size_t(k) + 1];) {
            const char* nlp = static_cast<const char*>(std::memchr(B + lb, '\n', size + 1 - lb));
            const size_t le = size_t(nlp - B);  // getline: split on '\n' only
            const size_t b = lb;
            lb = le + 1;
            if (le == b) continue;
            if (B[b] == '#') {
                tokenize(B + b, B + le, tk);
                if (tk.size() >= 2 && tk[1].n == 9 && std::memcmp(tk[1].p, "objective", 9) == 0)
                    objs[size_t(k)].emplace_back(tk.size() >= 3 ? std::string(tk[2].p, tk[2].n) : std::string());
                continue;
            }
            // the name: the first token
            const char* p = B + b;
            const char* e = B + le;
            while (p < e && is_space(*p)) ++p;
            if (p == e) continue;
            const char* s = p;
            while (p < e && !is_space(*p)) ++p;
            double v = 0.0;
            if (!extract_double(p, e, v)) continue;
            const int32_t j = names.find(s, size_t(p - s));
            if (j >= 0) out.push_back({j, v});
        }
    });
    for (const auto& r : sets)
        for (const Set& q : r) x_out[q.j] = q.v;
    int status = 0;
    double obj = 0.0;
    for (const auto& r : objs)
        for (const std::string& t : r) {
            g_obj_tokens.push_back(t);
            if (status) continue;
            // std::stod: the longest prefix strtod converts; none, or ERANGE, throws
            errno = 0;
            char* end = nullptr;
            const double v = std::strtod(t.c_str(), &end);
            if (end == t.c_str() || errno == ERANGE) status = 12;
            else obj = v;
        }
    if (objective) *objective = obj;
    if (n_objective_lines) *n_objective_lines = int32_t(g_obj_tokens.size());
    return status;
}

const char* nir_sol_objective_token(int32_t k) {
    if (k < 0 || size_t(k) >= g_obj_tokens.size()) return nullptr;
    return g_obj_tokens[size_t(k)].c_str();
}

double nir_eval_objective(const nir_lp_view* lp, int64_t qnnz, const int64_t* q_start, const int32_t* q_index,
                          const double* q_value, const double* x) {
    DD sum{lp->obj_offset, 0.0};
    for (int32_t j = 0; j < lp->ncol; ++j)
        if (lp->cost[j] != 0.0 && x[j] != 0.0) add_prod(sum, lp->cost[j], x[j]);
    if (qnnz > 0) {
        DD q;
        for (int32_t j = 0; j < lp->ncol; ++j) {
            const double xj = x[j];
            if (xj == 0.0) continue;
            for (int64_t k = q_start[j]; k < q_start[j + 1]; ++k) {
                const int32_t i = q_index[k];
                const double qij = q_value[k];
                if (i == j) add_prod(q, 0.5 * qij, xj * xj);
                else if (i < j) add_prod(q, qij, x[i] * xj);
            }
        }
        add_dd(sum, q.hi, q.lo);
    }
    return sum.hi + sum.lo;
}

int nir_verify_solution(const nir_lp_view* lp, const int8_t* vartype, int64_t qnnz, const int64_t* q_start,
                        const int32_t* q_index, const double* q_value, const double* x, int64_t nx,
                        double claimed_obj, double tol, int32_t threads, nir_verify_report* out) {
    if (!lp || !out) return 12;
    nir_verify_report rep{1, 0, -1, 0.0, 0.0, 0.0, 0.0, 0.0};
    const int32_t n = lp->ncol, m = lp->nrow;
    if (nx != n) {
        rep.passed = 0;
        rep.worst_kind = 1;
        *out = rep;
        return 0;
    }
    const int T = hw(threads);
    // the first non-finite value ends the check there (the maxima then
    // cover the columns before it only)
    int64_t first_bad = n;
    {
        const int nt = int(std::max<int64_t>(1, std::min<int64_t>(T, n / 16384 + 1)));
        std::vector<int64_t> fb(static_cast<size_t>(nt), n);
        run_threads(nt, [&](int k) {
            for (int64_t j = int64_t(n) * k / nt; j < int64_t(n) * (k + 1) / nt; ++j)
                if (!std::isfinite(x[j])) {
                    fb[size_t(k)] = j;
                    return;
                }
        });
        for (int64_t f : fb) first_bad = std::min(first_bad, f);
    }
    // A record: a value and the position of the check that first reached it
    // (columns: 3j lower bound, 3j+1 upper bound, 3j+2 integrality; rows: 2i
    // lower, 2i+1 upper).  The reference's loops change the worst item at
    // each new maximum above tol, so the item named last is the later of the
    // categories' first maxima.
    struct Rec {
        double v = 0.0;
        int64_t pos = -1;
        int kind = 0;
        void see(double x, int64_t p, int k) {
            if (x > v) {
                v = x;
                pos = p;
                kind = k;
            }
        }
        void merge(const Rec& o) {  // o covers later positions
            if (o.v > v) *this = o;
        }
    };
    const int64_t ncheck = first_bad;
    const int nc = int(std::max<int64_t>(1, std::min<int64_t>(T, ncheck / 16384 + 1)));
    std::vector<Rec> bnd(static_cast<size_t>(nc)), itg(static_cast<size_t>(nc));
    run_threads(nc, [&](int k) {
        Rec b, g;
        for (int64_t j = ncheck * k / nc; j < ncheck * (k + 1) / nc; ++j) {
            const double v = x[j];
            if (fin(lp->collo[j])) b.see(std::max(0.0, lp->collo[j] - v) / (1.0 + std::abs(lp->collo[j])), 3 * j, 3);
            if (fin(lp->colup[j])) b.see(std::max(0.0, v - lp->colup[j]) / (1.0 + std::abs(lp->colup[j])), 3 * j + 1, 4);
            if (vartype && (vartype[j] == 1 || vartype[j] == 2)) g.see(std::abs(v - std::round(v)), 3 * j + 2, 5);
        }
        bnd[size_t(k)] = b;
        itg[size_t(k)] = g;
    });
    Rec B, G;
    for (int k = 0; k < nc; ++k) {
        B.merge(bnd[size_t(k)]);
        G.merge(itg[size_t(k)]);
    }
    rep.max_bound_viol = B.v;
    rep.max_int_viol = G.v;
    // the worst item after the column loop: the later of the two records
    // that exceed tol
    const Rec* worst = nullptr;
    if (B.v > tol) worst = &B;
    if (G.v > tol && (!worst || G.pos > worst->pos)) worst = &G;
    if (worst) {
        rep.worst_kind = worst->kind;
        rep.worst_index = worst->pos / 3;
    }
    if (first_bad < n) {
        rep.passed = 0;
        rep.worst_kind = 2;
        rep.worst_index = first_bad;
        *out = rep;
        return 0;
    }
    // rows in double-double: thread k owns a range of rows and scans the
    // columns with x != 0 in order, adding the entries that fall in its
    // range.  Every row's terms thus arrive in ascending column order, the
    // order of the reference's column loop, and each thread's accumulators
    // stay in its own cache.  With more than one thread allowed, one more
    // thread evaluates the objective meanwhile.
    {
        const int64_t nnz = lp->nnz;
        const int nr = int(std::max<int64_t>(1, std::min<int64_t>(T, 1 + nnz / 131072)));
        std::vector<Rec> rows(static_cast<size_t>(nr));
        double obj = 0.0;
        const bool obj_thread = T > 1;  // with one thread the objective follows the rows
        run_threads(nr + (obj_thread ? 1 : 0), [&](int k) {
            if (k == nr) {
                obj = nir_eval_objective(lp, qnnz, q_start, q_index, q_value, x);
                return;
            }
            const int32_t lo = int32_t(int64_t(m) * k / nr), hi = int32_t(int64_t(m) * (k + 1) / nr);
            const uint32_t span = uint32_t(hi - lo);
            if (span == 0) return;
            std::vector<DD> acc(span);
            for (int32_t j = 0; j < n; ++j) {
                const double xj = x[j];
                if (xj == 0.0) continue;
                for (int64_t q = lp->col_start[j]; q < lp->col_start[j + 1]; ++q) {
                    const uint32_t i = uint32_t(lp->row_index[q] - lo);  // rows below lo wrap past span
                    if (i < span) add_prod(acc[i], lp->value[q], xj);
                }
            }
            Rec r;
            for (uint32_t i = 0; i < span; ++i) {
                const int64_t g = int64_t(lo) + i;
                const double a = acc[i].hi + acc[i].lo;
                if (fin(lp->rowlo[g])) r.see(std::max(0.0, lp->rowlo[g] - a) / (1.0 + std::abs(lp->rowlo[g])), 2 * g, 6);
                if (fin(lp->rowup[g])) r.see(std::max(0.0, a - lp->rowup[g]) / (1.0 + std::abs(lp->rowup[g])), 2 * g + 1, 7);
            }
            rows[size_t(k)] = r;
        });
        Rec R;
        for (int k = 0; k < nr; ++k) R.merge(rows[size_t(k)]);
        rep.max_row_viol = R.v;
        if (R.v > tol) {
            rep.worst_kind = R.kind;
            rep.worst_index = R.pos / 2;
        }
        rep.computed_obj = obj_thread ? obj : nir_eval_objective(lp, qnnz, q_start, q_index, q_value, x);
    }
    if (std::isfinite(claimed_obj))
        rep.obj_rel_err = std::abs(rep.computed_obj - claimed_obj) / (1.0 + std::abs(rep.computed_obj));
    if (rep.max_bound_viol > tol || rep.max_row_viol > tol || rep.max_int_viol > tol || rep.obj_rel_err > 1e-5)
        rep.passed = 0;
    *out = rep;
    return 0;
}

}  // extern "C"
