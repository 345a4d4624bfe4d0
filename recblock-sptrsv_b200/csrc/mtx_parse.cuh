// mtx_parse.cuh -- token parsing for the Matrix Market reader, shared by
// the device kernels (mtx.cu) and host-compiled tests.
//
// The reference reads entries with fscanf("%d %d %lg") (mmio_highlevel.h:
// 187-205): whitespace-separated tokens, indices as C ints, values converted
// by the C library's correctly rounded decimal-to-binary conversion.  Here a
// value token in plain decimal form (sign, digits, optional point and
// fraction, optional exponent) whose significant digits fit in 19 decimal
// digits (w < 10^19) and whose decimal exponent e lies in [-54, 54] is
// converted exactly with integer arithmetic:
//   e >= 0: w * 5^e is an exact product of at most 190 bits (5^54 < 2^126),
//           scaled by 2^e;
//   e <  0: w / 5^|e| by bit-serial long division to 64 quotient bits plus a
//           sticky bit from the remainder (64-bit divisor for |e| <= 27,
//           128-bit beyond), scaled by 2^e;
// then rounded once to 53 bits, ties to even -- the correctly rounded double,
// i.e. the same bits strtod gives.  Every other token (more significant
// digits, exponents outside the window, inf/nan/hexadecimal forms, stray
// characters) is reported as PARSE_HOST and converted by strtod on the host.
#pragma once

#include <stdint.h>

#if defined(__CUDACC__)
#define MTX_HD __host__ __device__ __forceinline__
#else
#define MTX_HD inline
#endif

namespace mtxp {

enum { PARSE_OK = 0, PARSE_HOST = 1, PARSE_BAD = 2 };

// C-locale isspace: space, \t \n \v \f \r
MTX_HD bool is_space(unsigned char c) { return c == ' ' || (c >= 9 && c <= 13); }

MTX_HD int clz64(uint64_t x) {  // x != 0
#if defined(__CUDA_ARCH__)
    return __clzll((long long)x);
#else
    return __builtin_clzll(x);
#endif
}

MTX_HD double bits_to_double(uint64_t b) {
#if defined(__CUDA_ARCH__)
    return __longlong_as_double((long long)b);
#else
    double d;
    __builtin_memcpy(&d, &b, 8);
    return d;
#endif
}

typedef unsigned __int128 u128;

MTX_HD u128 pow5(int k) {  // 0 <= k <= 54 (5^54 < 2^126)
    u128 p = 1;
    for (int i = 0; i < k; ++i) p *= 5;
    return p;
}

// (w2 * 2^128 + w1 * 2^64 + w0 + s) * 2^bexp rounded to the nearest double,
// ties to even, where s in (0, 1) stands for nonzero bits below w0 when
// sticky is set.  The caller guarantees a nonzero value in the normal range.
MTX_HD double round_pack(uint64_t w2, uint64_t w1, uint64_t w0, int bexp, bool sticky, bool neg) {
    for (int i = 0; i < 2 && w2 == 0; ++i) {
        w2 = w1;
        w1 = w0;
        w0 = 0;
        bexp -= 64;
    }
    const int z = clz64(w2);
    const uint64_t top = z ? (w2 << z) | (w1 >> (64 - z)) : w2;
    sticky = sticky || (z ? (w1 << z) : w1) != 0 || w0 != 0;
    const int e = bexp + 128 - z;
    // value = top * 2^e (+ sticky), bit 63 of top set
    uint64_t mant = top >> 11;
    const uint64_t rb = top & 0x7FF;
    if (rb > 0x400 || (rb == 0x400 && (sticky || (mant & 1)))) ++mant;
    int e2 = e + 11;
    if (mant >> 53) {
        mant >>= 1;
        ++e2;
    }
    const uint64_t biased = (uint64_t)(e2 + 52 + 1023);
    return bits_to_double(((uint64_t)neg << 63) | (biased << 52) | (mant & ((1ULL << 52) - 1)));
}

// w * 10^e10 (w != 0) correctly rounded; PARSE_HOST outside [-54, 54]
MTX_HD int decimal_to_double(uint64_t w, long long e10, bool neg, double &v) {
    if (e10 > 54 || e10 < -54) return PARSE_HOST;
    if (e10 >= 0) {
        const u128 p = pow5((int)e10);
        const u128 a = (u128)w * (uint64_t)p, b = (u128)w * (uint64_t)(p >> 64);
        const u128 t = (a >> 64) + (uint64_t)b;
        v = round_pack((uint64_t)(b >> 64) + (uint64_t)(t >> 64), (uint64_t)t, (uint64_t)a, (int)e10, false, neg);
        return PARSE_OK;
    }
    // w / 5^k * 2^-k, k = -e10: the quotient of w * 2^sh by 5^k, sh chosen
    // so that it lies in [2^62, 2^64), by restoring division over the bits
    // of w followed by sh zero bits
    const int k = (int)-e10;
    const int lw = 64 - clz64(w);
    uint64_t q = 0;
    bool rem = false;
    int sh;
    if (k <= 27) {
        const uint64_t D = (uint64_t)pow5(k);  // < 2^63, so 2r + 1 never overflows
        sh = 63 + (64 - clz64(D)) - lw;
        uint64_t r = 0;
        for (int bit = lw - 1; bit >= 0; --bit) {
            r = (r << 1) | ((w >> bit) & 1);
            q <<= 1;
            if (r >= D) {
                r -= D;
                q |= 1;
            }
        }
        for (int i = 0; i < sh; ++i) {
            r <<= 1;
            q <<= 1;
            if (r >= D) {
                r -= D;
                q |= 1;
            }
        }
        rem = r != 0;
    } else {
        const u128 D = pow5(k);  // < 2^126
        const uint64_t dh = (uint64_t)(D >> 64);
        sh = 63 + (128 - clz64(dh)) - lw;
        u128 r = 0;
        for (int bit = lw - 1; bit >= 0; --bit) {
            r = (r << 1) | ((w >> bit) & 1);
            q <<= 1;
            if (r >= D) {
                r -= D;
                q |= 1;
            }
        }
        for (int i = 0; i < sh; ++i) {
            r <<= 1;
            q <<= 1;
            if (r >= D) {
                r -= D;
                q |= 1;
            }
        }
        rem = r != 0;
    }
    v = round_pack(0, 0, q, -(sh + k), rem, neg);
    return PARSE_OK;
}

// Parses the token starting at s[pos] (pos at a non-space byte, token ends at
// the next space or at len) as a C int (fscanf "%d").  Returns PARSE_OK and
// sets v and end (one past the token), or PARSE_BAD.
MTX_HD int parse_int(const unsigned char *s, long long len, long long pos, int &v, long long &end) {
    long long i = pos;
    bool neg = false;
    if (i < len && (s[i] == '+' || s[i] == '-')) {
        neg = s[i] == '-';
        ++i;
    }
    long long acc = 0;
    int nd = 0;
    while (i < len && s[i] >= '0' && s[i] <= '9') {
        acc = acc * 10 + (s[i] - '0');
        if (acc > 2147483648LL) return PARSE_BAD;
        ++nd;
        ++i;
    }
    if (!nd || (i < len && !is_space(s[i]))) return PARSE_BAD;
    if (neg) acc = -acc;
    if (acc > 2147483647LL) return PARSE_BAD;
    v = (int)acc;
    end = i;
    return PARSE_OK;
}

// Parses the token starting at s[pos] as a double (fscanf "%lg").  Returns
// PARSE_OK with the correctly rounded value, or PARSE_HOST when the token is
// outside the exact window above (the host converts it).  end is set to one
// past the token either way.
MTX_HD int parse_real(const unsigned char *s, long long len, long long pos, double &v, long long &end) {
    long long i = pos;
    long long tok_end = pos;
    while (tok_end < len && !is_space(s[tok_end])) ++tok_end;
    end = tok_end;
    bool neg = false;
    if (i < tok_end && (s[i] == '+' || s[i] == '-')) {
        neg = s[i] == '-';
        ++i;
    }
    uint64_t w = 0;
    int ndig = 0;              // significant digits held in w (at most 19)
    long long scale = 0;       // decimal exponent contributed by the mantissa digits
    bool any = false, lost = false;
    for (; i < tok_end && s[i] >= '0' && s[i] <= '9'; ++i) {
        const int d = s[i] - '0';
        any = true;
        if (w == 0 && d == 0) continue;  // leading zero
        if (ndig < 19) {
            w = w * 10 + d;
            ++ndig;
        } else {
            ++scale;  // integer digit beyond the 19th
            lost = lost || d != 0;
        }
    }
    if (i < tok_end && s[i] == '.') {
        for (++i; i < tok_end && s[i] >= '0' && s[i] <= '9'; ++i) {
            const int d = s[i] - '0';
            any = true;
            if (ndig < 19) {
                if (w != 0 || d != 0) {
                    w = w * 10 + d;
                    ++ndig;
                }
                --scale;
            } else {
                lost = lost || d != 0;
            }
        }
    }
    if (!any) return PARSE_HOST;
    long long ex = 0;
    if (i < tok_end && (s[i] == 'e' || s[i] == 'E')) {
        long long j = i + 1;
        bool eneg = false;
        if (j < tok_end && (s[j] == '+' || s[j] == '-')) {
            eneg = s[j] == '-';
            ++j;
        }
        if (!(j < tok_end && s[j] >= '0' && s[j] <= '9')) return PARSE_HOST;
        for (; j < tok_end && s[j] >= '0' && s[j] <= '9'; ++j)
            if (ex < 100000) ex = ex * 10 + (s[j] - '0');
        if (eneg) ex = -ex;
        i = j;
    }
    if (i != tok_end || lost) return PARSE_HOST;
    if (w == 0) {
        v = neg ? -0.0 : 0.0;
        return PARSE_OK;
    }
    return decimal_to_double(w, ex + scale, neg, v);
}

}  // namespace mtxp
