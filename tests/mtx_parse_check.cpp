// Host build of the Matrix Market token parser (csrc/mtx_parse.cuh) checked
// against the C library: every value the parser converts itself must carry
// exactly strtod's bits, and every index exactly strtol's value.  Random
// tokens of many shapes (digit counts, point positions, exponents, signs,
// leading zeros, exact halfway cases between neighbouring doubles) plus
// fixed hard cases.  Prints "ok <converted> <handed-to-host>" or the first
// mismatch and exits 1.
#include <cinttypes>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>

#include "mtx_parse.cuh"

static long long g_ok = 0, g_host = 0;

static bool check(const std::string &t) {
    double v = 0;
    long long end = 0;
    const int rc = mtxp::parse_real((const unsigned char *)t.data(), (long long)t.size(), 0, v, end);
    if (end != (long long)t.size()) {
        printf("token end mismatch for '%s'\n", t.c_str());
        return false;
    }
    if (rc == mtxp::PARSE_HOST) {
        ++g_host;
        return true;
    }
    char *e = nullptr;
    const double r = strtod(t.c_str(), &e);
    uint64_t a, b;
    memcpy(&a, &v, 8);
    memcpy(&b, &r, 8);
    if (rc != mtxp::PARSE_OK || *e != '\0' || a != b) {
        printf("mismatch '%s': parser %.17g (%016" PRIx64 ") rc %d, strtod %.17g (%016" PRIx64 ")\n", t.c_str(), v, a,
               rc, r, b);
        return false;
    }
    ++g_ok;
    return true;
}

static std::string digits(std::mt19937_64 &g, int n, bool lead_nonzero) {
    std::string s;
    for (int i = 0; i < n; ++i) s += char('0' + ((i == 0 && lead_nonzero) ? 1 + g() % 9 : g() % 10));
    return s;
}

int main(int argc, char **argv) {
    const long long count = argc > 1 ? atoll(argv[1]) : 2000000;
    std::mt19937_64 g(12345);
    const char *fixed[] = {"0", "-0", "+0", "0.0", "1", "-1", "1.", ".5", "-.5", "1e0", "1E+0", "1e-0", "0e5",
                           "9007199254740993", "9007199254740995", "9007199254740992.5", "1.7976931348623157e308",
                           "2.2250738585072014e-308", "4.9e-324", "1e27", "1e-27", "1e28", "1e-28", "123456789012345678",
                           "1234567890123456789", "12345678901234567890", "0.1", "0.2", "0.3", "3.14159265358979323846",
                           "2.718281828459045", "1e22", "1e23", "8.98846567431158e307", "0.000000000000000000000000001",
                           "00000000000000000000000000000123.456", "1.00000000000000000000000000000", "5e-20",
                           "9.999999999999999e26", "-2.5e-27", "inf", "nan", "0x1p3", "1e", "1e+", "+", "-", ".", "1.2.3",
                           "1d5", "7.0e-10", "4.35", "0.1e1", "100e-2"};
    for (const char *t : fixed)
        if (!check(t)) return 1;
    // exact halfway points between neighbouring doubles (ties to even)
    for (int i = 0; i < 200000; ++i) {
        const uint64_t m = (1ULL << 53) + (g() & ((1ULL << 53) - 1));
        const int sh = (int)(g() % 11);
        const unsigned long long half = ((m << 1) | 1) << sh;  // (2m+1) * 2^sh, 54+sh bits
        if (sh > 9) continue;
        if (!check(std::to_string(half))) return 1;
    }
    for (long long i = 0; i < count; ++i) {
        std::string t;
        const int shape = (int)(g() % 7);
        if (g() % 3 == 0) t += (g() & 1) ? "-" : "+";
        if (shape == 0) {  // %.17g-like: d.ddddde[+-]xx
            t += digits(g, 1, true) + "." + digits(g, 1 + g() % 18, false);
            t += "e" + std::string(g() & 1 ? "-" : "+") + std::to_string(g() % 30);
        } else if (shape == 1) {  // plain decimals
            t += digits(g, 1 + g() % 12, g() & 1) + "." + digits(g, g() % 12, false);
        } else if (shape == 2) {  // integers of up to 20 digits
            t += digits(g, 1 + g() % 20, true);
        } else if (shape == 3) {  // leading zeros and exponents
            t += "0." + std::string(g() % 12, '0') + digits(g, 1 + g() % 17, true) + "e" + std::to_string((long long)(g() % 40) - 12);
        } else if (shape == 4) {  // printf round trips of random doubles
            uint64_t b = g();
            double d;
            memcpy(&d, &b, 8);
            if (!std::isfinite(d)) continue;
            char buf[64];
            snprintf(buf, sizeof buf, (g() & 1) ? "%.17g" : "%.16e", d);
            t = buf;
        } else if (shape == 5) {  // %.17g of values between 1e-45 and 1e45
            const double d = std::pow(10.0, -45.0 + 90.0 * (double)(g() >> 11) / 9007199254740992.0);
            char buf[64];
            snprintf(buf, sizeof buf, (g() & 1) ? "%.17g" : "%.16e", d);
            t = buf;
        } else {  // values of moderate size printed at every precision
            const double d = std::ldexp((double)(g() >> 11), (int)(g() % 120) - 110);
            char buf[64];
            snprintf(buf, sizeof buf, "%.*g", (int)(1 + g() % 17), d);
            t = buf;
        }
        if (!check(t)) return 1;
    }
    // indices
    const char *ints[] = {"1", "0", "-7", "+42", "2147483647", "-2147483648", "007"};
    for (const char *t : ints) {
        int v = 0;
        long long end = 0;
        if (mtxp::parse_int((const unsigned char *)t, (long long)strlen(t), 0, v, end) != mtxp::PARSE_OK ||
            v != (int)strtol(t, nullptr, 10)) {
            printf("int mismatch '%s'\n", t);
            return 1;
        }
    }
    const char *bad_ints[] = {"2147483648", "-2147483649", "1.5", "x", "+", "12a"};
    for (const char *t : bad_ints) {
        int v = 0;
        long long end = 0;
        if (mtxp::parse_int((const unsigned char *)t, (long long)strlen(t), 0, v, end) != mtxp::PARSE_BAD) {
            printf("int accepted '%s'\n", t);
            return 1;
        }
    }
    printf("ok %lld %lld\n", g_ok, g_host);
    return 0;
}
