// Number parsing for the device BSR text reader, in host and device code alike.
//
// parse_int: an optional sign and decimal digits (what "%d" accepts after the white space the
// tokeniser removed), range-checked to int.
//
// parse_double: the decimal forms "%le" accepts (sign, digits, optional fraction, optional
// exponent) converted to the nearest binary64 (ties to even), as a correctly rounding strtod gives.
// The conversion is the Eisel-Lemire method (D. Lemire, "Number parsing at a gigabyte per
// second", Software: Practice and Experience 51(8), 2021; N. Mushtak and D. Lemire, "Fast number
// parsing without fallback", 2023): the decimal significand w (up to 19 digits, exact in 64 bits)
// times a 128-bit truncated power of five gives the binary significand and exponent; the table
// (pow5_table.inc) is generated by exact integer arithmetic (make_pow5_table.py).  Tokens outside
// this form (more than 19 significant digits, "inf", "nan", hexadecimal) are reported as
// kParseFallback: the reader converts those few on the host with strtod.
#pragma once

#include <cstdint>

namespace jxcpr {
namespace numparse {

#include "pow5_table.inc"

enum { kParseOk = 0, kParseFallback = 1, kParseBad = 2 };

__host__ __device__ inline bool np_digit(char c) { return c >= '0' && c <= '9'; }

__host__ __device__ inline void mul128(uint64_t a, uint64_t b, uint64_t &hi, uint64_t &lo) {
#ifdef __CUDA_ARCH__
    hi = __umul64hi(a, b);
    lo = a * b;
#else
    const unsigned __int128 p = (unsigned __int128)a * b;
    hi = (uint64_t)(p >> 64);
    lo = (uint64_t)p;
#endif
}

__host__ __device__ inline int clz64(uint64_t x) {
#ifdef __CUDA_ARCH__
    return __clzll((long long)x);
#else
    return __builtin_clzll(x);
#endif
}

__host__ __device__ inline int parse_int(const char *s, int len, int *out) {
    int k = 0;
    bool neg = false;
    if (k < len && (s[k] == '+' || s[k] == '-')) neg = s[k++] == '-';
    if (k >= len) return kParseBad;
    long long v = 0;
    for (; k < len; ++k) {
        if (!np_digit(s[k])) return kParseBad;
        v = v * 10 + (s[k] - '0');
        if (v > 2147483648LL) return kParseBad;
    }
    if (neg) v = -v;
    if (v > 2147483647LL || v < -2147483648LL) return kParseBad;
    *out = (int)v;
    return kParseOk;
}

// w * 10^q (w != 0, q in [-342, 308]) to binary64 bits, sign excluded.
__host__ __device__ inline uint64_t eisel_lemire(uint64_t w, int q, const unsigned long long *table) {
    const int lz = clz64(w);
    w <<= lz;
    const int index = 2 * (q + 342);
    uint64_t hi, lo;
#ifdef __CUDA_ARCH__
    const uint64_t t0 = __ldg(table + index), t1 = __ldg(table + index + 1);
#else
    const uint64_t t0 = table[index], t1 = table[index + 1];
#endif
    mul128(w, t0, hi, lo);
    const uint64_t mask = 0x1FFull;  // 64 - (52 + 3) low bits of the high word
    if ((hi & mask) == mask) {
        uint64_t hi2, lo2;
        mul128(w, t1, hi2, lo2);
        lo += hi2;
        if (hi2 > lo) ++hi;
    }
    const int upperbit = (int)(hi >> 63);
    const int shift = upperbit + 9;
    uint64_t mant = hi >> shift;
    // floor(q log2(10)) + 63 (exact for q in [-342, 308]): the binary exponent of 10^q times 2^63
    int power2 = (((152170 + 65536) * q) >> 16) + 63 + upperbit - lz + 1023;
    if (power2 <= 0) {  // subnormal
        if (-power2 + 1 >= 64) return 0;
        mant >>= -power2 + 1;
        mant += mant & 1;
        mant >>= 1;
        power2 = mant < (1ull << 52) ? 0 : 1;
        return ((uint64_t)power2 << 52) | (mant & ((1ull << 52) - 1));
    }
    // exactly between two doubles: only possible when 5^q is exact in the product (q in [-4, 23])
    if (lo <= 1 && q >= -4 && q <= 23 && (mant & 3) == 1 && (mant << shift) == hi) mant &= ~1ull;
    mant += mant & 1;
    mant >>= 1;
    if (mant >= (2ull << 52)) {
        mant = 1ull << 52;
        ++power2;
    }
    mant &= ~(1ull << 52);
    if (power2 >= 0x7FF) return 0x7FFull << 52;  // infinity
    return ((uint64_t)power2 << 52) | mant;
}

// One token (no white space) to binary64 bits in *bits.
__host__ __device__ inline int parse_double(const char *s, int len, const unsigned long long *table,
                                            uint64_t *bits) {
    int k = 0;
    bool neg = false;
    if (k < len && (s[k] == '+' || s[k] == '-')) neg = s[k++] == '-';
    uint64_t w = 0;
    int nd = 0, dropped = 0;  // significant digits kept; digits beyond 19 (fallback)
    bool any = false;
    long long e10 = 0;
    for (; k < len && np_digit(s[k]); ++k) {
        any = true;
        if (w == 0 && s[k] == '0') continue;  // leading zeros
        if (nd < 19) {
            w = w * 10 + (uint64_t)(s[k] - '0');
            ++nd;
        } else {
            ++dropped;
            ++e10;
        }
    }
    if (k < len && s[k] == '.') {
        ++k;
        for (; k < len && np_digit(s[k]); ++k) {
            any = true;
            if (w == 0 && s[k] == '0') {
                --e10;
                continue;
            }
            if (nd < 19) {
                w = w * 10 + (uint64_t)(s[k] - '0');
                ++nd;
                --e10;
            } else {
                ++dropped;
            }
        }
    }
    if (!any) {
        // inf / nan and other forms strtod knows: the host converts them
        return (k < len && (s[k] == 'i' || s[k] == 'I' || s[k] == 'n' || s[k] == 'N')) ? kParseFallback : kParseBad;
    }
    if (k < len && (s[k] == 'e' || s[k] == 'E')) {
        ++k;
        bool eneg = false;
        if (k < len && (s[k] == '+' || s[k] == '-')) eneg = s[k++] == '-';
        if (k >= len || !np_digit(s[k])) return kParseBad;
        long long ev = 0;
        for (; k < len && np_digit(s[k]); ++k)
            if (ev < 100000) ev = ev * 10 + (s[k] - '0');
        e10 += eneg ? -ev : ev;
    }
    if (k != len) return kParseBad;
    if (dropped) return kParseFallback;  // inexact significand: strtod decides
    uint64_t b;
    if (w == 0 || e10 < -342) b = 0;
    else if (e10 > 308) b = 0x7FFull << 52;
    else b = eisel_lemire(w, (int)e10, table);
    *bits = b | (neg ? (1ull << 63) : 0ull);
    return kParseOk;
}

}  // namespace numparse
}  // namespace jxcpr
