// Multi-threaded MPS reader (C ABI: include/nir_mps.h).
//
// The model is the one sov::MpsReader::read builds (src/io/mps_reader.hpp:
// 15-304), followed by CscMatrix::from_triplets (src/core/csc_matrix.hpp:
// 30-96) and Model::validate (src/model/model.hpp:117-178).  What differs is
// how the work is done:
//   * the file is read by all threads (pread of one slice each);
//   * the threads find the header lines (a keyword in column 0); the section
//     state machine then walks the headers in file order, with the
//     reference's rules for each header line;
//   * the data lines between two headers form one range.  ROWS and the
//     quadratic block are handled line by line on one thread.  COLUMNS,
//     RHS, RANGES and BOUNDS ranges are cut into one run of lines per
//     thread; each thread tokenises its lines, converts the numbers and
//     looks the names up in tables that nobody writes while the runs last;
//   * the runs are then applied in file order on one thread -- columns are
//     created in order of first appearance with the integer-marker state of
//     that moment, objective entries summed in file order, bounds applied in
//     file order -- so the model is the sequential one; the matrix triplets
//     are written back in parallel at offsets known from the runs;
//   * the CSC is bucketed in triplet order and each column's entries are
//     sorted by row (stably) and merged, in parallel over columns.
// Numbers: the exact fast conversion of decimal.hpp, with strtod (as
// std::stod calls it) wherever that conversion declines.
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "decimal.hpp"
#include "nir_mps.h"
#include "text.hpp"

namespace {

using namespace nir::text;

thread_local std::string g_err;
thread_local double g_times[6] = {0, 0, 0, 0, 0, 0};

constexpr double kInf = std::numeric_limits<double>::infinity();
constexpr double kInfInput = 1e20;  // src/core/types.hpp:16

enum VarType : int8_t { kContinuous = 0, kInteger = 1, kBinary = 2 };
enum RowType : int8_t { kRowL = 0, kRowG = 1, kRowE = 2 };

struct InputError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct InfeasibleError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

double now() { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); }

std::string upper(const Tok& t) {
    std::string s(t.p, t.n);
    for (char& c : s) c = char(std::toupper((unsigned char)c));
    return s;
}

bool contains(const Tok& t, const char* needle, size_t n) {
    if (t.n < n) return false;
    for (size_t i = 0; i + n <= t.n; ++i)
        if (t.p[i] == needle[0] && std::memcmp(t.p + i, needle, n) == 0) return true;
    return false;
}

// std::stod on the token with D/d read as E (src/io/mps_reader.hpp:57-62).
// Returns false where stod would throw (nothing converted, or ERANGE).
bool parse_number(const Tok& t, double& v) {
    if (nir::decimal::parse_decimal(t.p, t.n, v)) return true;
    char buf[128];
    std::string big;
    char* s = buf;
    if (t.n < sizeof(buf)) {
        std::memcpy(buf, t.p, t.n);
        buf[t.n] = 0;
    } else {
        big.assign(t.p, t.n);
        s = &big[0];
    }
    for (char* q = s; *q; ++q)
        if (*q == 'D' || *q == 'd') *q = 'E';
    errno = 0;
    char* end = nullptr;
    v = std::strtod(s, &end);
    return end != s && errno != ERANGE;
}

std::string number_error(const Tok& t) {
    double v;
    char buf[128];
    const size_t n = std::min<size_t>(t.n, sizeof(buf) - 1);
    std::memcpy(buf, t.p, n);
    buf[n] = 0;
    for (size_t k = 0; k < n; ++k)
        if (buf[k] == 'D' || buf[k] == 'd') buf[k] = 'E';
    errno = 0;
    char* end = nullptr;
    v = std::strtod(buf, &end);
    (void)v;
    return std::string(end == buf ? "invalid number '" : "number out of range '") + std::string(t.p, t.n) + "'";
}

struct Triplets {
    uvector<int32_t> row, col;
    uvector<double> val;
    size_t size() const { return val.size(); }
    void push(int32_t r, int32_t c, double v) {
        row.push_back(r);
        col.push_back(c);
        val.push_back(v);
    }
    void resize(size_t n) {
        row.resize(n);
        col.resize(n);
        val.resize(n);
    }
};

}  // namespace

struct nir_mps {
    int32_t nrow = 0, ncol = 0;
    int32_t sense = 1;
    double obj_offset = 0.0;
    std::vector<double> cost, collo, colup, rowlo, rowup;
    std::vector<int8_t> vartype;
    std::vector<int64_t> start{0};
    nir::text::uvector<int32_t> index;
    nir::text::uvector<double> value;
    std::vector<int64_t> qstart{0};
    nir::text::uvector<int32_t> qindex;
    nir::text::uvector<double> qvalue;
    std::string name = "mps_model";
    std::vector<char> col_chars, row_chars;  // names, packed
    std::vector<int64_t> col_off{0}, row_off{0};
};

namespace {

// CscMatrix::from_triplets: entries with a row or column out of range or
// a zero value are dropped, the rest bucketed by column in input order, each
// column sorted by row and duplicates summed; sums that come to zero are
// dropped.  The sort is stable here.
void from_triplets(int32_t nrow, int32_t ncol, const Triplets& t, std::vector<int64_t>& start,
                   uvector<int32_t>& index, uvector<double>& value, int threads) {
    const size_t T = t.size();
    auto keep = [&](size_t k) {
        return t.row[k] >= 0 && t.row[k] < nrow && t.col[k] >= 0 && t.col[k] < ncol && t.val[k] != 0.0;
    };
    // stable counting sort by column: thread k counts its slice of the
    // triplets per column, then writes them after the slices before it
    const int ns = int(std::max<size_t>(1, std::min<size_t>(size_t(threads), T / 65536 + 1)));
    std::vector<std::vector<int64_t>> pos(static_cast<size_t>(ns));
    run_threads(ns, [&](int k) {
        std::vector<int64_t>& c = pos[size_t(k)];
        c.assign(size_t(ncol), 0);
        for (size_t q = T * size_t(k) / size_t(ns); q < T * size_t(k + 1) / size_t(ns); ++q)
            if (keep(q)) ++c[size_t(t.col[q])];
    });
    std::vector<int64_t> cnt(size_t(ncol) + 1, 0);
    for (int32_t j = 0; j < ncol; ++j) {
        int64_t s = 0;
        for (int k = 0; k < ns; ++k) s += pos[size_t(k)][size_t(j)];
        cnt[size_t(j) + 1] = cnt[size_t(j)] + s;
    }
    {
        const int nc = std::max(1, std::min(threads, int(ncol / 4096) + 1));
        run_threads(nc, [&](int q) {
            for (int32_t j = int32_t(int64_t(ncol) * q / nc); j < int32_t(int64_t(ncol) * (q + 1) / nc); ++j) {
                int64_t off = cnt[size_t(j)];
                for (int k = 0; k < ns; ++k) {
                    const int64_t c = pos[size_t(k)][size_t(j)];
                    pos[size_t(k)][size_t(j)] = off;
                    off += c;
                }
            }
        });
    }
    uvector<int32_t> ri(size_t(cnt[ncol]));
    uvector<double> rv(size_t(cnt[ncol]));
    run_threads(ns, [&](int k) {
        std::vector<int64_t>& w = pos[size_t(k)];
        for (size_t q = T * size_t(k) / size_t(ns); q < T * size_t(k + 1) / size_t(ns); ++q)
            if (keep(q)) {
                const int64_t p = w[size_t(t.col[q])]++;
                ri[size_t(p)] = t.row[q];
                rv[size_t(p)] = t.val[q];
            }
    });
    // per column: sort (stable) and merge in place; merged count per column
    std::vector<int64_t> kept(size_t(ncol), 0);
    auto work = [&](int32_t j0, int32_t j1) {
        std::vector<std::pair<int32_t, double>> buf;
        for (int32_t j = j0; j < j1; ++j) {
            const int64_t s = cnt[j], e = cnt[j + 1];
            if (s == e) continue;
            bool sorted = true;
            for (int64_t k = s + 1; k < e && sorted; ++k) sorted = ri[k - 1] < ri[k];
            if (sorted) {
                kept[j] = e - s;
                continue;
            }
            buf.clear();
            for (int64_t k = s; k < e; ++k) buf.push_back({ri[k], rv[k]});
            std::stable_sort(buf.begin(), buf.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
            int64_t w = s;
            int32_t cur_r = buf[0].first;
            double cur_v = buf[0].second;
            for (size_t k = 1; k < buf.size(); ++k) {
                if (buf[k].first == cur_r) {
                    cur_v += buf[k].second;
                } else {
                    if (cur_v != 0.0) {
                        ri[w] = cur_r;
                        rv[w] = cur_v;
                        ++w;
                    }
                    cur_r = buf[k].first;
                    cur_v = buf[k].second;
                }
            }
            if (cur_v != 0.0) {
                ri[w] = cur_r;
                rv[w] = cur_v;
                ++w;
            }
            kept[j] = w - s;
        }
    };
    const int nt = std::max(1, std::min(threads, int(ncol / 1024) + 1));
    // column ranges with about equal numbers of entries
    std::vector<int32_t> jb(size_t(nt) + 1, ncol);
    jb[0] = 0;
    for (int k = 1; k < nt; ++k) {
        const int64_t target = cnt[ncol] * k / nt;
        jb[k] = int32_t(std::lower_bound(cnt.begin(), cnt.end(), target) - cnt.begin());
        jb[k] = std::max(jb[k - 1], std::min(jb[k], ncol));
    }
    run_threads(nt, [&](int k) { work(jb[k], jb[k + 1]); });
    bool merged = false;  // some column lost entries to merging
    for (int32_t c = 0; c < ncol && !merged; ++c) merged = kept[c] != cnt[c + 1] - cnt[c];
    if (!merged) {  // the usual case: the bucketed arrays are the CSC
        start.swap(cnt);
        index.swap(ri);
        value.swap(rv);
        return;
    }
    start.assign(size_t(ncol) + 1, 0);
    for (int32_t c = 0; c < ncol; ++c) start[c + 1] = start[c] + kept[c];
    index.resize(size_t(start[ncol]));
    value.resize(size_t(start[ncol]));
    run_threads(nt, [&](int k) {
        for (int32_t c = jb[k]; c < jb[k + 1]; ++c) {
            std::memcpy(index.data() + start[c], ri.data() + cnt[c], size_t(kept[c]) * sizeof(int32_t));
            std::memcpy(value.data() + start[c], rv.data() + cnt[c], size_t(kept[c]) * sizeof(double));
        }
    });
}

// ---- per-run records of the parallel sections

// COLUMNS, per run.  A group is a stretch of consecutive entry lines of one
// column (a marker line ends it); the pairs with a known row are kept in
// the run's arrays group after group, objective pairs on their own list.
struct ColGroup {
    uint64_t hash;   // of the name
    const char* p;   // name in the file buffer
    uint32_t n;
    int32_t col;     // filled in by the ordered pass
    uint64_t t0;     // first pair of the group in trow / tval
    char key[16];    // first 16 bytes of the name
};

struct ColRun {
    std::vector<int32_t> events;  // in file order: group index, or -1 INTEND / -2 INTORG
    std::vector<ColGroup> groups;
    std::vector<int32_t> trow;    // pairs with a known row: row index
    std::vector<double> tval;     //   and value
    std::vector<std::pair<uint32_t, double>> obj;  // objective pairs: (group, value)
    size_t trip0 = 0;             // offset of this run's triplets
    std::string error;
    size_t error_at = SIZE_MAX;   // byte offset of the failing line
};

// RHS / RANGES: one record per pair
struct PairRec {
    int32_t code;  // row index, -2 objective, -1 unknown row
    double val;
};

// BOUNDS: one record per line
enum BoundKind : int8_t { kLO, kUP, kFX, kFR, kMI, kPL, kBV, kLI, kUI, kSC, kOther };
struct BoundRec {
    int8_t kind;
    int32_t col;
    double val;
};

template <class Rec>
struct Run {
    std::vector<Rec> recs;
    std::string error;
    size_t error_at = SIZE_MAX;
};

struct Header {
    size_t at;   // line start
    int kind;
};

struct Reader {
    static constexpr size_t kPad = 64;
    std::unique_ptr<char[]> store;
    const char* buf = nullptr;
    size_t size = 0;  // bytes of the file; buf[size] == '\n'
    int threads = 1;

    nir_mps* m = nullptr;
    std::string obj_row;
    NameMap rows, cols;
    std::vector<Tok> row_name, col_name;  // views into the file buffer
    std::vector<RowType> row_type;
    std::vector<double> rhs, range;
    std::vector<char> has_range;
    Triplets trip, qtrip;
    bool in_int = false;
    double t_parse = 0, t_apply = 0, t_other = 0;

    enum Sec { NONE, NAME, OBJSENSE, OBJNAME, ROWS, COLUMNS, RHS, RANGES, BOUNDS, QUADOBJ, QMATRIX, SOS, END };

    // ---- lines
    size_t line_end(size_t b) const {  // the '\n' ending the line at b
        return size_t(static_cast<const char*>(std::memchr(buf + b, '\n', size + 1 - b)) - buf);
    }
    // [b, e) without the one '\r' getline + pop_back would drop
    size_t trimmed(size_t b, size_t nl) const { return (nl > b && buf[nl - 1] == '\r') ? nl - 1 : nl; }
    bool skipped(size_t b, size_t e) const { return e == b || buf[b] == '*'; }
    size_t line_number(size_t at) const {
        size_t n = 1;
        for (size_t i = 0; i < at; ++i) n += buf[i] == '\n';
        return n;
    }

    // Header kind of the line [b, e) (first byte not white space and a known
    // first word, compared upper-cased), else NONE.
    Sec header(size_t b, size_t e) const {
        if (b == e || is_space(buf[b]) || buf[b] == '*') return NONE;
        size_t w = b;
        while (w < e && !is_space(buf[w])) ++w;
        const size_t n = w - b;
        if (n < 3 || n > 8) return NONE;
        char u[9];
        for (size_t k = 0; k < n; ++k) u[k] = char(std::toupper((unsigned char)buf[b + k]));
        u[n] = 0;
        if (!std::strcmp(u, "NAME")) return NAME;
        if (!std::strcmp(u, "OBJSENSE")) return OBJSENSE;
        if (!std::strcmp(u, "OBJNAME")) return OBJNAME;
        if (!std::strcmp(u, "ROWS")) return ROWS;
        if (!std::strcmp(u, "COLUMNS")) return COLUMNS;
        if (!std::strcmp(u, "RHS")) return RHS;
        if (!std::strcmp(u, "RANGES")) return RANGES;
        if (!std::strcmp(u, "BOUNDS")) return BOUNDS;
        if (!std::strcmp(u, "QUADOBJ") || !std::strcmp(u, "QSECTION")) return QUADOBJ;
        if (!std::strcmp(u, "QMATRIX")) return QMATRIX;
        if (!std::strcmp(u, "SOS")) return SOS;
        if (!std::strcmp(u, "ENDATA")) return END;
        return NONE;
    }

    // first line start at or after x (x itself when a line starts there)
    size_t line_start_from(size_t x, size_t lo, size_t hi) const {
        if (x <= lo) return lo;
        if (x >= hi) return hi;
        if (buf[x - 1] == '\n') return x;
        const void* q = std::memchr(buf + x, '\n', hi - x);
        return q ? size_t(static_cast<const char*>(q) - buf) + 1 : hi;
    }
    // nt runs of whole lines over [a, b); about `grain` bytes each at least
    std::vector<size_t> cut(size_t a, size_t b, int& nt, size_t grain = size_t(1) << 18) const {
        nt = int(std::max<size_t>(1, std::min<size_t>(size_t(threads), (b - a) / grain + 1)));
        std::vector<size_t> at(size_t(nt) + 1);
        at[0] = a;
        at[size_t(nt)] = b;
        for (int k = 1; k < nt; ++k) at[k] = line_start_from(a + (b - a) * size_t(k) / size_t(nt), a, b);
        return at;
    }

    void read_file(const char* path) {
        const int fd = ::open(path, O_RDONLY);
        if (fd < 0) throw InputError(std::string("Cannot open MPS file: ") + path);
        struct stat st;
        if (::fstat(fd, &st) != 0) {
            ::close(fd);
            throw InputError(std::string("Cannot open MPS file: ") + path);
        }
        if (!S_ISREG(st.st_mode)) {
            // a pipe or a device is read as a stream, as std::ifstream reads
            // it; a directory opens but yields no line, so the model is empty
            std::vector<char> v;
            if (!S_ISDIR(st.st_mode)) {
                std::vector<char> tmp(size_t(1) << 16);
                for (;;) {
                    const ssize_t r = ::read(fd, tmp.data(), tmp.size());
                    if (r < 0 && errno == EINTR) continue;
                    if (r <= 0) break;
                    v.insert(v.end(), tmp.data(), tmp.data() + r);
                }
            }
            ::close(fd);
            size = v.size();
            store.reset(new char[size + kPad]);
            if (size) std::memcpy(store.get(), v.data(), size);
            std::memset(store.get() + size, '\n', kPad);
            buf = store.get();
            return;
        }
        size = size_t(st.st_size);
        // one '\n' after the file, then padding for the 16-byte loads
        store.reset(new char[size + kPad]);
        char* dst = store.get();
        std::memset(dst + size, '\n', kPad);
        int nt = int(std::max<size_t>(1, std::min<size_t>(size_t(threads), size / (size_t(8) << 20) + 1)));
        std::vector<int> fail(size_t(nt), 0);
        run_threads(nt, [&](int k) {
            size_t off = size * size_t(k) / size_t(nt);
            const size_t end = size * size_t(k + 1) / size_t(nt);
            while (off < end) {
                const ssize_t r = ::pread(fd, dst + off, end - off, off_t(off));
                if (r <= 0) {
                    if (r < 0 && errno == EINTR) continue;
                    fail[size_t(k)] = 1;
                    return;
                }
                off += size_t(r);
            }
        });
        ::close(fd);
        for (int f : fail)
            if (f) throw InputError(std::string("Cannot read MPS file: ") + path);
        buf = dst;
    }

    std::vector<Header> find_headers() const {
        int nt;
        const std::vector<size_t> at = cut(0, size, nt, size_t(4) << 20);
        std::vector<std::vector<Header>> part(static_cast<size_t>(nt));
        run_threads(nt, [&](int k) {
            for (size_t b = at[k]; b < at[k + 1];) {
                const size_t nl = line_end(b);
                const size_t e = trimmed(b, nl);
                const Sec h = header(b, e);
                if (h != NONE) part[size_t(k)].push_back({b, int(h)});
                b = nl + 1;
            }
        });
        std::vector<Header> out;
        for (auto& p : part) out.insert(out.end(), p.begin(), p.end());
        return out;
    }

    int32_t ensure_col(const ColGroup& g) {
        const int32_t j = m->ncol;
        const int32_t old = cols.insert_h(g.hash, g.n <= 16 ? g.key : g.p, g.p, g.n, j);
        if (old >= 0) return old;
        m->ncol++;
        col_name.push_back({g.p, g.n});
        m->cost.push_back(0.0);
        m->collo.push_back(0.0);
        m->colup.push_back(kInf);
        m->vartype.push_back(in_int ? kInteger : kContinuous);
        return j;
    }

    bool is_obj(const Tok& t) const {
        return !obj_row.empty() && t.n == obj_row.size() && std::memcmp(t.p, obj_row.data(), t.n) == 0;
    }
    // -2 objective, row index, or -1
    int32_t row_code(const Tok& t) const { return is_obj(t) ? -2 : rows.find(t.p, t.n); }

    [[noreturn]] void fail_number(const Tok& t, size_t at) const {
        throw InputError(number_error(t) + " at line " + std::to_string(line_number(at)));
    }

    // ---- COLUMNS
    void columns(size_t a, size_t b) {
        double t0 = now();
        int nt;
        const std::vector<size_t> at = cut(a, b, nt);
        std::vector<ColRun> run(static_cast<size_t>(nt));
        run_threads(nt, [&](int k) {
            ColRun& r = run[size_t(k)];
            std::vector<Tok> tk;
            std::vector<uint64_t> hs;
            std::vector<double> vals;
            bool open = false;  // a group is open (no marker since its last line)
            const size_t bytes = at[k + 1] - at[k];
            r.groups.reserve(bytes / 128 + 16);
            r.trow.reserve(bytes / 24 + 16);
            r.tval.reserve(bytes / 24 + 16);
            for (size_t lb = at[k]; lb < at[k + 1];) {
                const size_t nl = line_end(lb);
                const size_t le = trimmed(lb, nl);
                const size_t this_line = lb;
                lb = nl + 1;
                if (skipped(this_line, le)) continue;
                tokenize(buf + this_line, buf + le, tk);
                if (tk.empty()) continue;
                int marker = -1;
                if (std::memchr(buf + this_line, 'I', le - this_line)) {  // both markers hold an I
                    for (const Tok& t : tk) {
                        if (contains(t, "INTORG", 6)) marker = 1;
                        else if (contains(t, "INTEND", 6)) marker = 0;
                    }
                }
                if (marker >= 0) {
                    r.events.push_back(marker == 1 ? -2 : -1);
                    open = false;
                    continue;
                }
                if (tk.size() < 3) continue;
                // hash the row names and prefetch their slots, then convert
                // the numbers while those loads are in flight
                const size_t np = (tk.size() - 1) / 2;
                hs.resize(np);
                vals.resize(np);
                for (size_t q = 0; q < np; ++q) {
                    const Tok& rn = tk[1 + 2 * q];
                    hs[q] = hash_name(rn.p, rn.n);
                    __builtin_prefetch(rows.slot_for(hs[q]));
                }
                const Tok& cn = tk[0];
                if (!open || r.groups.back().n != cn.n || std::memcmp(r.groups.back().p, cn.p, cn.n) != 0) {
                    ColGroup g;
                    g.hash = hash_name(cn.p, cn.n);
                    g.p = cn.p;
                    g.n = cn.n;
                    g.col = -1;
                    g.t0 = r.trow.size();
                    std::memcpy(g.key, cn.p, std::min<size_t>(cn.n, 16));
                    r.events.push_back(int32_t(r.groups.size()));
                    r.groups.push_back(g);
                    open = true;
                }
                const uint32_t gi = uint32_t(r.groups.size() - 1);
                for (size_t q = 0; q < np; ++q) {
                    if (!parse_number(tk[2 + 2 * q], vals[q])) {
                        r.error = number_error(tk[2 + 2 * q]);
                        r.error_at = this_line;
                        return;
                    }
                }
                for (size_t q = 0; q < np; ++q) {
                    const Tok& rn = tk[1 + 2 * q];
                    const double v = vals[q];
                    if (is_obj(rn)) {
                        r.obj.push_back({gi, v});
                        continue;
                    }
                    const int32_t code = rows.find_h(hs[q], rn.p, rn.n);
                    if (code < 0) continue;  // unknown rows are ignored
                    r.trow.push_back(code);
                    r.tval.push_back(v);
                }
            }
        });
        t_parse += now() - t0;
        t0 = now();
        // the first error in file order, as the sequential reader meets it
        for (const ColRun& r : run)
            if (!r.error.empty()) throw InputError(r.error + " at line " + std::to_string(line_number(r.error_at)));
        // ordered pass: columns in order of first appearance with the marker
        // state of that moment, then the run's objective sums in file order
        size_t ngroups = 0;
        for (const ColRun& r : run) ngroups += r.groups.size();
        cols.reserve(cols.count + ngroups);
        const ColGroup* last = nullptr;
        int32_t last_col = -1;
        size_t base = trip.size();
        for (ColRun& r : run) {
            r.trip0 = base;
            base += r.trow.size();
            const size_t G = r.groups.size();
            for (const int32_t ev : r.events) {
                if (ev < 0) {
                    in_int = ev == -2;
                    continue;
                }
                if (size_t(ev) + 32 < G) __builtin_prefetch(cols.slot_for(r.groups[size_t(ev) + 32].hash));
                ColGroup& g = r.groups[size_t(ev)];
                if (last && last->n == g.n &&
                    (g.n <= 16 ? std::memcmp(last->key, g.key, g.n) : std::memcmp(last->p, g.p, g.n)) == 0) {
                    g.col = last_col;
                } else {
                    g.col = ensure_col(g);
                }
                last = &g;
                last_col = g.col;
            }
            for (const auto& o : r.obj) m->cost[r.groups[o.first].col] += o.second;
        }
        // triplets in file order, written in parallel
        trip.resize(base);
        run_threads(nt, [&](int k) {
            const ColRun& r = run[size_t(k)];
            const size_t G = r.groups.size();
            for (size_t g = 0; g < G; ++g) {
                const size_t s = r.groups[g].t0, e = g + 1 < G ? r.groups[g + 1].t0 : r.trow.size();
                const int32_t c = r.groups[g].col;
                for (size_t t = s; t < e; ++t) {
                    trip.row[r.trip0 + t] = r.trow[t];
                    trip.col[r.trip0 + t] = c;
                    trip.val[r.trip0 + t] = r.tval[t];
                }
            }
        });
        t_apply += now() - t0;
    }

    // ---- RHS / RANGES
    void rhs_ranges(size_t a, size_t b, bool is_rhs) {
        double t0 = now();
        int nt;
        const std::vector<size_t> at = cut(a, b, nt);
        std::vector<Run<PairRec>> run(static_cast<size_t>(nt));
        run_threads(nt, [&](int k) {
            Run<PairRec>& r = run[size_t(k)];
            std::vector<Tok> tk;
            for (size_t lb = at[k]; lb < at[k + 1];) {
                const size_t nl = line_end(lb);
                const size_t le = trimmed(lb, nl);
                const size_t this_line = lb;
                lb = nl + 1;
                if (skipped(this_line, le)) continue;
                tokenize(buf + this_line, buf + le, tk);
                if (tk.empty()) continue;
                const size_t s0 = (tk.size() % 2 == 1) ? 1 : 0;
                for (size_t pos = s0; pos + 1 < tk.size(); pos += 2) {
                    double v;
                    if (!parse_number(tk[pos + 1], v)) {
                        r.error = number_error(tk[pos + 1]);
                        r.error_at = this_line;
                        return;
                    }
                    // RANGES never treats the objective row specially
                    const int32_t code = is_rhs ? row_code(tk[pos]) : rows.find(tk[pos].p, tk[pos].n);
                    r.recs.push_back({code, v});
                }
            }
        });
        t_parse += now() - t0;
        t0 = now();
        for (const auto& r : run) {
            for (const PairRec& p : r.recs) {
                if (p.code == -2) {
                    m->obj_offset = -p.val;  // MPS convention: objective offset = -RHS
                } else if (p.code >= 0) {
                    if (is_rhs) {
                        rhs[p.code] = p.val;
                    } else {
                        range[p.code] = p.val;
                        has_range[p.code] = 1;
                    }
                }
            }
            if (!r.error.empty()) throw InputError(r.error + " at line " + std::to_string(line_number(r.error_at)));
        }
        t_apply += now() - t0;
    }

    // ---- BOUNDS
    static int8_t bound_kind(const Tok& t) {
        if (t.n != 2) return kOther;
        const char a = char(std::toupper((unsigned char)t.p[0])), b = char(std::toupper((unsigned char)t.p[1]));
        const struct {
            char a, b;
            int8_t k;
        } tab[] = {{'L', 'O', kLO}, {'U', 'P', kUP}, {'F', 'X', kFX}, {'F', 'R', kFR}, {'M', 'I', kMI},
                   {'P', 'L', kPL}, {'B', 'V', kBV}, {'L', 'I', kLI}, {'U', 'I', kUI}, {'S', 'C', kSC}};
        for (const auto& e : tab)
            if (e.a == a && e.b == b) return e.k;
        return kOther;
    }

    void bounds(size_t a, size_t b) {
        double t0 = now();
        int nt;
        const std::vector<size_t> at = cut(a, b, nt);
        std::vector<Run<BoundRec>> run(static_cast<size_t>(nt));
        run_threads(nt, [&](int k) {
            Run<BoundRec>& r = run[size_t(k)];
            std::vector<Tok> tk;
            for (size_t lb = at[k]; lb < at[k + 1];) {
                const size_t nl = line_end(lb);
                const size_t le = trimmed(lb, nl);
                const size_t this_line = lb;
                lb = nl + 1;
                if (skipped(this_line, le)) continue;
                tokenize(buf + this_line, buf + le, tk);
                if (tk.size() < 3) continue;
                const int8_t kind = bound_kind(tk[0]);
                const bool has_val = kind == kLO || kind == kUP || kind == kFX || kind == kLI || kind == kUI ||
                                     kind == kSC;
                Tok cn = tk[2];
                double v = 0.0;
                if (has_val) {
                    const Tok& vt = tk.size() >= 4 ? tk[3] : tk[2];
                    if (tk.size() < 4) cn = tk[1];
                    if (!parse_number(vt, v)) {
                        r.error = number_error(vt);
                        r.error_at = this_line;
                        return;
                    }
                }
                const int32_t j = cols.find(cn.p, cn.n);
                if (j < 0) {
                    r.error = "Unknown column in BOUNDS: " + std::string(cn.p, cn.n);
                    r.error_at = SIZE_MAX;  // the reference's message has no line number
                    return;
                }
                r.recs.push_back({kind, j, v});
            }
        });
        t_parse += now() - t0;
        t0 = now();
        for (const auto& r : run) {
            for (const BoundRec& q : r.recs) apply_bound(q);
            if (!r.error.empty()) {
                if (r.error_at == SIZE_MAX) throw InputError(r.error);
                throw InputError(r.error + " at line " + std::to_string(line_number(r.error_at)));
            }
        }
        t_apply += now() - t0;
    }

    void apply_bound(const BoundRec& q) {
        const int32_t j = q.col;
        const double v = q.val;
        switch (q.kind) {
            case kLO: m->collo[j] = v; break;
            case kUP:
                if (v < 0.0 && m->collo[j] == 0.0) m->collo[j] = -kInf;  // the negative UP rule
                m->colup[j] = v;
                break;
            case kFX:
                m->collo[j] = v;
                m->colup[j] = v;
                break;
            case kFR:
                m->collo[j] = -kInf;
                m->colup[j] = kInf;
                break;
            case kMI: m->collo[j] = -kInf; break;
            case kPL: m->colup[j] = kInf; break;
            case kBV:
                m->vartype[j] = kBinary;
                m->collo[j] = 0.0;
                m->colup[j] = 1.0;
                break;
            case kLI:
                m->vartype[j] = kInteger;
                m->collo[j] = v;
                break;
            case kUI:
                m->vartype[j] = kInteger;
                m->colup[j] = v;
                break;
            default: break;  // SC and unknown types change nothing
        }
    }

    // ---- ROWS: lines tokenised in parallel, rows numbered on one thread in
    // order of appearance
    struct RowRec {
        uint64_t hash;
        const char* p;
        uint32_t n;
        char type;  // upper-cased first letter of the type token
        char key[16];
        size_t line;
    };

    void rows_section(size_t a, size_t b) {
        int nt;
        const std::vector<size_t> at = cut(a, b, nt);
        std::vector<std::vector<RowRec>> run(static_cast<size_t>(nt));
        run_threads(nt, [&](int k) {
            std::vector<Tok> tk;
            std::vector<RowRec>& r = run[size_t(k)];
            r.reserve((at[k + 1] - at[k]) / 16 + 16);
            for (size_t lb = at[k]; lb < at[k + 1];) {
                const size_t nl = line_end(lb);
                const size_t le = trimmed(lb, nl);
                const size_t this_line = lb;
                lb = nl + 1;
                if (skipped(this_line, le)) continue;
                tokenize(buf + this_line, buf + le, tk);
                if (tk.size() < 2) continue;
                RowRec q;
                q.hash = hash_name(tk[1].p, tk[1].n);
                q.p = tk[1].p;
                q.n = tk[1].n;
                q.type = char(std::toupper((unsigned char)tk[0].p[0]));
                std::memcpy(q.key, tk[1].p, std::min<size_t>(tk[1].n, 16));
                q.line = this_line;
                r.push_back(q);
            }
        });
        size_t total = 0;
        for (const auto& r : run) total += r.size();
        rows.reserve(rows.count + total);
        row_name.reserve(row_name.size() + total);
        for (const auto& r : run) {
            for (size_t i = 0; i < r.size(); ++i) {
                if (i + 8 < r.size()) __builtin_prefetch(rows.slot_for(r[i + 8].hash));
                const RowRec& q = r[i];
                if (q.type == 'N') {
                    if (obj_row.empty()) obj_row.assign(q.p, q.n);
                    continue;  // further free rows are dropped
                }
                const int32_t idx = m->nrow;
                if (rows.insert_h(q.hash, q.n <= 16 ? q.key : q.p, q.p, q.n, idx) >= 0)
                    throw InputError("Duplicate row name at line " + std::to_string(line_number(q.line)));
                m->nrow++;
                row_name.push_back({q.p, q.n});
                row_type.push_back(q.type == 'L' ? kRowL : (q.type == 'G' ? kRowG : kRowE));
                rhs.push_back(0.0);
                range.push_back(0.0);
                has_range.push_back(0);
            }
        }
    }

    // ---- QUADOBJ / QMATRIX
    void quadratic(size_t a, size_t b, bool qmatrix) {
        std::vector<Tok> tk;
        for (size_t lb = a; lb < b;) {
            const size_t nl = line_end(lb);
            const size_t le = trimmed(lb, nl);
            const size_t this_line = lb;
            lb = nl + 1;
            if (skipped(this_line, le)) continue;
            tokenize(buf + this_line, buf + le, tk);
            if (tk.size() < 3) continue;
            int32_t i = cols.find(tk[0].p, tk[0].n), j = cols.find(tk[1].p, tk[1].n);
            if (i < 0 || j < 0) continue;
            double v;
            if (!parse_number(tk[2], v)) fail_number(tk[2], this_line);
            if (qmatrix) {
                if (i <= j) qtrip.push(i, j, v);
            } else {
                if (i > j) std::swap(i, j);
                qtrip.push(i, j, v);
            }
        }
    }

    // the first data line of [a, b) with a token, or false
    bool first_data_line(size_t a, size_t b, std::vector<Tok>& tk) const {
        for (size_t lb = a; lb < b;) {
            const size_t nl = line_end(lb);
            const size_t le = trimmed(lb, nl);
            const size_t this_line = lb;
            lb = nl + 1;
            if (skipped(this_line, le)) continue;
            tokenize(buf + this_line, buf + le, tk);
            if (!tk.empty()) return true;
        }
        return false;
    }

    void parse(const char* path) {
        double t0 = now();
        read_file(path);
        g_times[0] = now() - t0;
        t0 = now();
        const std::vector<Header> hdr = find_headers();
        g_times[1] = now() - t0;
        const double t_all = now();
        double t_csc = 0;

        Sec sec = NONE;
        bool sense_wait = false;
        std::vector<Tok> tk;
        // data lines before the first header belong to no section
        for (size_t h = 0; h < hdr.size(); ++h) {
            const size_t hb = hdr[h].at;
            const size_t hnl = line_end(hb);
            tokenize(buf + hb, buf + trimmed(hb, hnl), tk);
            const Sec kind = Sec(hdr[h].kind);
            if (kind == END) break;
            if (kind == NAME) {
                if (tk.size() >= 2) m->name.assign(tk[1].p, tk[1].n);
                sec = NAME;
            } else if (kind == OBJSENSE) {
                if (tk.size() >= 2) {
                    m->sense = upper(tk[1]).rfind("MAX", 0) == 0 ? -1 : 1;
                } else {
                    sense_wait = true;
                    sec = OBJSENSE;
                }
            } else if (kind == OBJNAME) {
                if (tk.size() >= 2) obj_row.assign(tk[1].p, tk[1].n);
                else sec = OBJNAME;
            } else {
                sec = kind;
            }
            // the data lines up to the next header
            const size_t a = hnl + 1;
            const size_t b = h + 1 < hdr.size() ? hdr[h + 1].at : size;
            if (a >= b) continue;
            if (sec == OBJSENSE && sense_wait) {
                if (first_data_line(a, b, tk)) {
                    m->sense = upper(tk[0]).rfind("MAX", 0) == 0 ? -1 : 1;
                    sense_wait = false;
                }
                continue;  // the section's other lines are ignored
            }
            if (sec == OBJNAME && obj_row.empty()) {
                if (first_data_line(a, b, tk)) obj_row.assign(tk[0].p, tk[0].n);
                continue;
            }
            switch (sec) {
                case ROWS: rows_section(a, b); break;
                case COLUMNS: columns(a, b); break;
                case RHS: rhs_ranges(a, b, true); break;
                case RANGES: rhs_ranges(a, b, false); break;
                case BOUNDS: bounds(a, b); break;
                case QUADOBJ: quadratic(a, b, false); break;
                case QMATRIX: quadratic(a, b, true); break;
                default: break;  // NAME, SOS, NONE: data lines ignored
            }
        }
        t0 = now();
        from_triplets(m->nrow, m->ncol, trip, m->start, m->index, m->value, threads);
        from_triplets(m->ncol, m->ncol, qtrip, m->qstart, m->qindex, m->qvalue, threads);
        t_csc = now() - t0;
        assemble_rows();
        validate();
        pack_names(col_name, m->col_chars, m->col_off);
        pack_names(row_name, m->row_chars, m->row_off);
        g_times[2] = t_parse;
        g_times[3] = t_apply;
        g_times[4] = t_csc;
        g_times[5] = (now() - t_all) - t_parse - t_apply - t_csc;
    }

    // names as one character array with offsets (n + 1), copied in parallel
    void pack_names(const std::vector<Tok>& nm, std::vector<char>& chars, std::vector<int64_t>& off) const {
        const size_t n = nm.size();
        off.assign(n + 1, 0);
        for (size_t i = 0; i < n; ++i) off[i + 1] = off[i] + nm[i].n;
        chars.resize(size_t(off[n]));
        const int nt = int(std::max<size_t>(1, std::min<size_t>(size_t(threads), n / 65536 + 1)));
        run_threads(nt, [&](int k) {
            for (size_t i = n * size_t(k) / size_t(nt); i < n * size_t(k + 1) / size_t(nt); ++i)
                std::memcpy(chars.data() + off[i], nm[i].p, nm[i].n);
        });
    }

    void assemble_rows() {
        m->rowlo.resize(size_t(m->nrow));
        m->rowup.resize(size_t(m->nrow));
        for (int32_t i = 0; i < m->nrow; ++i) {
            const double b = rhs[i];
            if (!has_range[i]) {
                if (row_type[i] == kRowL) {
                    m->rowlo[i] = -kInf;
                    m->rowup[i] = b;
                } else if (row_type[i] == kRowG) {
                    m->rowlo[i] = b;
                    m->rowup[i] = kInf;
                } else {
                    m->rowlo[i] = b;
                    m->rowup[i] = b;
                }
            } else {
                const double R = range[i];
                if (row_type[i] == kRowG) {
                    m->rowlo[i] = b;
                    m->rowup[i] = b + std::abs(R);
                } else if (row_type[i] == kRowL) {
                    m->rowlo[i] = b - std::abs(R);
                    m->rowup[i] = b;
                } else if (R >= 0.0) {
                    m->rowlo[i] = b;
                    m->rowup[i] = b + R;
                } else {
                    m->rowlo[i] = b + R;
                    m->rowup[i] = b;
                }
            }
        }
    }

    static bool finite_bound(double b) { return std::isfinite(b) && std::abs(b) < kInfInput; }
    static double san_lo(double b) { return (!std::isfinite(b) || b <= -kInfInput) ? -kInf : b; }
    static double san_up(double b) { return (!std::isfinite(b) || b >= kInfInput) ? kInf : b; }

    // Model::validate (src/model/model.hpp:117-178), repairs included
    void validate() {
        for (int32_t j = 0; j < m->ncol; ++j) {
            if (!std::isfinite(m->cost[j]))
                throw InputError("Non-finite objective coefficient on column " + std::to_string(j));
            double& lo = m->collo[j];
            double& up = m->colup[j];
            lo = san_lo(lo);
            up = san_up(up);
            if (m->vartype[j] == kBinary) {
                lo = std::max(0.0, lo);
                up = std::min(1.0, up);
            }
            if (m->vartype[j] == kInteger || m->vartype[j] == kBinary) {
                if (finite_bound(lo)) lo = std::ceil(lo - 1e-9);
                if (finite_bound(up)) up = std::floor(up + 1e-9);
            }
            if (lo > up) {
                if (lo <= up + 1e-9 * (1.0 + std::abs(up))) lo = up;
                else
                    throw InfeasibleError("Infeasible column bounds on variable " +
                                          std::string(col_name[j].p, col_name[j].n));
            }
            if (m->vartype[j] == kInteger && lo >= 0.0 && up <= 1.0) m->vartype[j] = kBinary;
        }
        for (int32_t i = 0; i < m->nrow; ++i) {
            double& lo = m->rowlo[i];
            double& up = m->rowup[i];
            lo = san_lo(lo);
            up = san_up(up);
            if (lo > up) {
                if (lo <= up + 1e-9 * (1.0 + std::abs(up))) lo = up;
                else
                    throw InfeasibleError("Infeasible row bounds on row " +
                                          std::string(row_name[i].p, row_name[i].n));
            }
        }
        for (double v : m->value)
            if (!std::isfinite(v)) throw InputError("Non-finite matrix entry");
    }
};

}  // namespace

namespace nir {
__attribute__((visibility("hidden"))) void set_mps_error(const std::string& msg) { g_err = msg; }
}  // namespace nir

extern "C" {

int nir_mps_read(const char* path, int32_t threads, nir_mps** out) {
    if (!path || !out) {
        g_err = "null argument";
        return 12;
    }
    *out = nullptr;
    auto m = std::make_unique<nir_mps>();
    try {
        Reader r;
        r.m = m.get();
        const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
        r.threads = threads > 0 ? threads : int(hw);
        r.parse(path);
    } catch (const InfeasibleError& e) {
        g_err = e.what();
        return 1;
    } catch (const InputError& e) {
        g_err = e.what();
        return 12;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 14;
    }
    *out = m.release();
    return 0;
}

int nir_mps_view(const nir_mps* m, nir_lp_view* v, int32_t* sense) {
    if (!m || !v) return 12;
    v->nrow = m->nrow;
    v->ncol = m->ncol;
    v->nnz = m->start.back();
    v->col_start = m->start.data();
    v->row_index = m->index.data();
    v->value = m->value.data();
    v->cost = m->cost.data();
    v->collo = m->collo.data();
    v->colup = m->colup.data();
    v->rowlo = m->rowlo.data();
    v->rowup = m->rowup.data();
    v->obj_offset = m->obj_offset;
    if (sense) *sense = m->sense;
    return 0;
}

const int8_t* nir_mps_vartypes(const nir_mps* m) { return m ? m->vartype.data() : nullptr; }

const char* nir_mps_model_name(const nir_mps* m) { return m ? m->name.c_str() : nullptr; }

int nir_mps_names(const nir_mps* m, int32_t of_rows, const char** chars, const int64_t** offsets) {
    if (!m) return 12;
    if (chars) *chars = of_rows ? m->row_chars.data() : m->col_chars.data();
    if (offsets) *offsets = of_rows ? m->row_off.data() : m->col_off.data();
    return 0;
}

int nir_mps_quadratic(const nir_mps* m, int64_t* nnz, const int64_t** col_start, const int32_t** row_index,
                      const double** value) {
    if (!m) return 12;
    if (nnz) *nnz = m->qstart.back();
    if (col_start) *col_start = m->qstart.data();
    if (row_index) *row_index = m->qindex.data();
    if (value) *value = m->qvalue.data();
    return 0;
}

int nir_mps_timings(double* out6) {
    if (!out6) return 12;
    for (int k = 0; k < 6; ++k) out6[k] = g_times[k];
    return 0;
}

void nir_mps_free(nir_mps* m) { delete m; }

const char* nir_mps_last_error(void) { return g_err.c_str(); }

}  // extern "C"
