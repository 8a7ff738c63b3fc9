// Checks nir::decimal::parse_decimal against strtod: wherever the fast path
// accepts a token, its double must have strtod's bit pattern.  Usage:
//   decimal_harness <cases> <seed>
// Prints "checked N accepted A fallback F mismatches X" and exits 1 on any
// mismatch.
#include <cinttypes>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>

#include "../../nirnaya_b200/csrc/decimal.hpp"

static uint64_t g_checked = 0, g_acc = 0, g_mis = 0;

static void check(const std::string& s) {
    ++g_checked;
    double fast;
    if (!nir::decimal::parse_decimal(s.data(), s.size(), fast)) return;
    ++g_acc;
    std::string t = s;
    for (char& c : t)
        if (c == 'd' || c == 'D') c = 'E';
    const double ref = std::strtod(t.c_str(), nullptr);
    if (std::memcmp(&fast, &ref, 8) != 0) {
        if (g_mis < 20) std::printf("MISMATCH %s fast=%a strtod=%a\n", s.c_str(), fast, ref);
        ++g_mis;
    }
}

int main(int argc, char** argv) {
    const long cases = argc > 1 ? std::atol(argv[1]) : 1000000;
    const unsigned seed = argc > 2 ? unsigned(std::atoi(argv[2])) : 1;
    std::mt19937_64 rng(seed);
    char buf[128];
    // fixed tokens: signs, zeros, exponent letters, edges of the fast path
    const char* fixed[] = {"0", "-0", "+0", "0.0", ".5", "5.", "-.25e1", "1e0", "1E+2", "1d-3", "2D4", "007",
                           "0.000123", "1e308", "1.7976931348623157e308", "2.2250738585072014e-308",
                           "4.9406564584124654e-324", "1e-342", "9007199254740993", "9007199254740995",
                           "18014398509481985", "1234567890123456789", "9999999999999999999",
                           "0.30000000000000004", "1.5", "-2.75e-10", "123456789e-30", "1e22", "1e23"};
    for (const char* f : fixed) check(f);
    std::uniform_int_distribution<int> ndig(1, 19), e10(-360, 330), esmall(-30, 30), kind(0, 5);
    for (long i = 0; i < cases; ++i) {
        const int k = kind(rng);
        if (k == 0) {  // %.17g of a random finite double (all binades)
            uint64_t b = rng();
            double d;
            std::memcpy(&d, &b, 8);
            if (!(d == d) || d - d != 0) continue;
            std::snprintf(buf, sizeof buf, "%.17g", d);
            check(buf);
        } else if (k == 1) {  // %.17g / %.15g of a double near 1
            const double d = std::ldexp(double(rng() >> 11), -53) * std::pow(10.0, esmall(rng));
            std::snprintf(buf, sizeof buf, (rng() & 1) ? "%.17g" : "%.15g", d);
            check(buf);
        } else if (k == 2 || k == 3) {  // random digit strings with random exponents
            const int nd = ndig(rng);
            std::string s;
            if (rng() & 1) s += '-';
            const int dot = int(rng() % (nd + 1));
            for (int j = 0; j < nd; ++j) {
                if (j == dot) s += '.';
                s += char('0' + rng() % 10);
            }
            const int ex = k == 2 ? e10(rng) : esmall(rng);
            s += "eEdD"[rng() & 3];
            s += std::to_string(ex);
            check(s);
        } else if (k == 4) {  // exact ties: odd integers in [2^53, 2^64) with scale 10^0..10^-3
            const uint64_t v = (rng() | (uint64_t(1) << 53)) | 1;
            std::snprintf(buf, sizeof buf, "%" PRIu64, v);
            std::string s = buf;
            if (s.size() > 19) s = s.substr(0, 19);
            const int sh = int(rng() % 4);
            if (sh) s += "e-" + std::to_string(sh);
            check(s);
        } else {  // midpoints between neighbouring doubles, printed with 17-19 digits
            uint64_t b = (rng() & 0x7FEFFFFFFFFFFFFFull) | 0x0010000000000000ull;
            double lo, hi;
            std::memcpy(&lo, &b, 8);
            ++b;
            std::memcpy(&hi, &b, 8);
            const long double mid = (static_cast<long double>(lo) + static_cast<long double>(hi)) / 2;
            std::snprintf(buf, sizeof buf, "%.*Lg", 17 + int(rng() % 3), mid);
            check(buf);
        }
    }
    std::printf("checked %" PRIu64 " accepted %" PRIu64 " fallback %" PRIu64 " mismatches %" PRIu64 "\n", g_checked,
                g_acc, g_checked - g_acc, g_mis);
    return g_mis ? 1 : 0;
}
