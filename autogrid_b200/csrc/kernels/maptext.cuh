// Map-file text of one value, as the reference's writer prints it
// (main.cpp:3481-3519):
//
//   energy maps      fabs(e) < PRECISION (1e-4, autogrid.h:68) -> "0\n",
//                    else fprintf("%.3f\n", (float)round3dp(e))
//   floating grid    fprintf("%.3f\n", (float)round3dp(r_min))
//   constriction     fprintf("%d\n", c_count)
//
// with round3dp(x) = round(x*1000.0L)/1000.0L (main.cpp:84-86, HAVE_ROUND):
// the product is exact in 80-bit long double (53 + 7 significant bits), round()
// takes halves away from zero, the quotient is rounded to a 64-bit significand
// (nearest, ties to even), and the cast rounds that to float.  "%.3f" then
// prints the float's exact binary value rounded to three decimals, ties to even
// (glibc, round-to-nearest mode).
//
// Everything is integer or correctly rounded IEEE arithmetic, so the same
// functions run on the device and, for the CPU check, on the host.  The fast
// path replaces the 64-bit-significand quotient by the correctly rounded double
// quotient: both give the float nearest the exact quotient unless the double
// quotient lands exactly halfway between two floats (then the 64-bit quotient
// would too, or lies nearer the exact value); that case takes the exact
// long-division path.
#pragma once
#include <stdint.h>
#include <string.h>

#ifdef __CUDACC__
#define AGT_HD __host__ __device__ __forceinline__
#else
#define AGT_HD inline
#endif

namespace agt {

constexpr int kMaxLine = 48;          // "-" + 39 digits + ".000\n" = 45
constexpr double kPrecision = 0.0001; // autogrid.h:68

enum LineKind : int { kEnergy = 0, kFloating = 1, kCount = 2 };

AGT_HD uint64_t dbits(double x)
{
#ifdef __CUDA_ARCH__
    return (uint64_t)__double_as_longlong(x);
#else
    uint64_t u;
    memcpy(&u, &x, 8);
    return u;
#endif
}

AGT_HD uint32_t fbits(float x)
{
#ifdef __CUDA_ARCH__
    return (uint32_t)__float_as_uint(x);
#else
    uint32_t u;
    memcpy(&u, &x, 4);
    return u;
#endif
}

AGT_HD float fromfbits(uint32_t u)
{
#ifdef __CUDA_ARCH__
    return __uint_as_float(u);
#else
    float x;
    memcpy(&x, &u, 4);
    return x;
#endif
}

AGT_HD int clz64(uint64_t x)
{
#ifdef __CUDA_ARCH__
    return __clzll((long long)x);
#else
    return __builtin_clzll(x);
#endif
}

// floor(num / 1000) and num mod 1000 for num = n * 2^k < 2^75 (n < 2^63,
// k <= 74 - bitlength(n)), by long division over 32-bit limbs.
AGT_HD uint64_t div1000_shifted(uint64_t n, int k, uint32_t *rem)
{
    // num as three 32-bit limbs (bits 64..95, 32..63, 0..31)
    uint32_t l[3];
    uint64_t lo, hi;
    if (k >= 64) {
        lo = 0;
        hi = n << (k - 64);
    } else if (k > 0) {
        lo = n << k;
        hi = n >> (64 - k);
    } else {
        lo = n;
        hi = 0;
    }
    l[0] = (uint32_t)hi;
    l[1] = (uint32_t)(lo >> 32);
    l[2] = (uint32_t)lo;
    uint64_t r = 0, q[3];
    for (int i = 0; i < 3; i++) {
        const uint64_t cur = (r << 32) | l[i];
        q[i] = cur / 1000u;
        r = cur % 1000u;
    }
    *rem = (uint32_t)r;
    // callers keep the quotient below 2^64, so the top limb q[0] is zero
    return (q[1] << 32) | q[2];
}

// float(RN64(n / 1000)): the long double quotient of round3dp, rounded to float
// (both roundings to nearest, ties to even), for 0 < n < 2^63.
AGT_HD float quotient_exact(uint64_t n)
{
    const int len = 64 - clz64(n);
    int k = 73 - len;  // n*2^k in [2^72, 2^73): quotient in [2^62.03, 2^63.03)
    uint32_t r;
    uint64_t q = div1000_shifted(n, k, &r);
    if (!(q >> 63)) {
        k++;
        q = div1000_shifted(n, k, &r);
    }
    // 64-bit significand, nearest, ties to even (sticky: the remainder)
    if (2 * r > 1000 || (2 * r == 1000 && (q & 1))) {
        q++;
        if (q == 0) {  // carried out of 64 bits
            q = 1ull << 63;
            k--;
        }
    }
    // then to 24 bits, nearest, ties to even (no sticky: double rounding)
    uint64_t sig = q >> 40;
    const uint64_t low = q & ((1ull << 40) - 1), half = 1ull << 39;
    if (low > half || (low == half && (sig & 1))) {
        sig++;
        if (sig == (1ull << 24)) {
            sig = 1ull << 23;
            k--;
        }
    }
    // value = sig * 2^(40-k); sig < 2^24 and the scale is a power of two, so
    // both conversions are exact
    const int e2 = 40 - k;
    double v = (double)sig;
    // scale by 2^e2 (|e2| < 80) through an exact power of two
    const uint64_t pb = (uint64_t)(1023 + e2) << 52;
    double p;
#ifdef __CUDA_ARCH__
    p = __longlong_as_double((long long)pb);
#else
    memcpy(&p, &pb, 8);
#endif
    return (float)(v * p);
}

// (float)round3dp(e) of main.cpp:84-86.
AGT_HD float round3dp_float(double e)
{
    const uint64_t b = dbits(e);
    const bool neg = (b >> 63) != 0;
    const uint64_t mag = b & 0x7fffffffffffffffull;
    const int ef = (int)(mag >> 52);
    if (ef == 0x7ff) {  // inf and NaN keep their sign
        if (mag & ((1ull << 52) - 1)) return fromfbits(0x7fc00000u | (neg ? 0x80000000u : 0u));
        return fromfbits(0x7f800000u | (neg ? 0x80000000u : 0u));
    }
    if (ef >= 1023 + 53) return (float)e;  // |e| >= 2^53: an integer, round3dp(e) == e
    // |e| = M * 2^E, M < 2^53
    uint64_t M = mag & ((1ull << 52) - 1);
    int E;
    if (ef == 0) {
        E = -1074;
    } else {
        M |= 1ull << 52;
        E = ef - 1075;
    }
    // N = round(|e| * 1000), halves away from zero (exact: M*1000 < 2^63)
    const uint64_t X = M * 1000u;
    uint64_t N;
    if (E >= 0) {
        N = X << E;  // |e| < 2^53 keeps this below 2^63
    } else {
        const int s = -E;
        N = (s >= 64) ? 0 : ((X + (1ull << (s - 1))) >> s);
    }
    float v;
    if (N == 0) {
        v = 0.0f;
    } else if (N < (1ull << 53)) {
        const double A = (double)N / 1000.0;  // correctly rounded
        // halfway between two floats: the low 29 fraction bits are 1 followed by zeros
        if ((dbits(A) & ((1ull << 29) - 1)) == (1ull << 28))
            v = quotient_exact(N);
        else
            v = (float)A;
    } else {
        v = quotient_exact(N);
    }
    return neg ? -v : v;
}

AGT_HD int u64_ndigits(uint64_t x)
{
    int n = 1;
    while (x >= 10u) {
        x /= 10u;
        n++;
    }
    return n;
}

// Decimal digits of x into buf (most significant first); returns the count (>= 1).
AGT_HD int u64_digits(uint64_t x, char *buf)
{
    const int n = u64_ndigits(x);
    for (int i = n - 1; i >= 0; i--) {
        buf[i] = (char)('0' + (int)(x % 10u));
        x /= 10u;
    }
    return n;
}

// Decimal digits of the integer sig * 2^sh (sig < 2^24, 0 <= sh <= 104) into
// buf (or only counted when buf is null), by repeated division by 10^9 over
// 32-bit limbs.
AGT_HD int big_digits(uint32_t sig, int sh, char *buf)
{
    uint32_t l[5] = {0, 0, 0, 0, 0};  // little-endian limbs
    {
        const int w = sh >> 5, bit = sh & 31;
        const uint64_t v = (uint64_t)sig << bit;
        l[w] = (uint32_t)v;
        if (w + 1 < 5) l[w + 1] = (uint32_t)(v >> 32);
    }
    uint32_t chunk[6];
    int nc = 0;
    bool nz = true;
    while (nz) {
        uint64_t r = 0;
        nz = false;
        for (int i = 4; i >= 0; i--) {
            const uint64_t cur = (r << 32) | l[i];
            l[i] = (uint32_t)(cur / 1000000000u);
            r = cur % 1000000000u;
            if (l[i]) nz = true;
        }
        chunk[nc++] = (uint32_t)r;
    }
    // most significant chunk without leading zeros, then 9 digits per chunk
    int n = 0;
    char tmp[20];
    const int lead = u64_digits(chunk[nc - 1], tmp);
    for (int i = 0; i < lead; i++) {
        if (buf) buf[n] = tmp[i];
        n++;
    }
    for (int c = nc - 2; c >= 0; c--) {
        uint32_t v = chunk[c];
        for (int i = 8; i >= 0; i--) {
            if (buf) buf[n + i] = (char)('0' + (int)(v % 10u));
            v /= 10u;
        }
        n += 9;
    }
    return n;
}

// "%.3f\n" of the float v (promoted to double).  Writes to out when out is not
// null; returns the length.
AGT_HD int print_f3(float v, char *out)
{
    const uint32_t b = fbits(v);
    const bool neg = (b >> 31) != 0;
    const uint32_t mag = b & 0x7fffffffu;
    int n = 0;
    if (neg) {
        if (out) out[n] = '-';
        n++;
    }
    if (mag >= 0x7f800000u) {  // glibc prints inf / nan (with the sign for -nan)
        const char *s = (mag == 0x7f800000u) ? "inf\n" : "nan\n";
        for (int i = 0; i < 4; i++) {
            if (out) out[n] = s[i];
            n++;
        }
        return n;
    }
    const double w = (double)fromfbits(mag) * 1000.0;  // exact: 24 + 10 significant bits
    uint64_t ip, fp;
    if (w < 9223372036854775808.0) {
        // nearest integer, ties to even, of an exact value below 2^63
        const uint64_t t = (uint64_t)w;           // floor
        const double frac = w - (double)t;        // exact
        uint64_t D = t + ((frac > 0.5 || (frac == 0.5 && (t & 1))) ? 1 : 0);
        ip = D / 1000u;
        fp = D % 1000u;
        if (out) n += u64_digits(ip, out + n);
        else n += u64_ndigits(ip);
    } else {
        // |v| >= 2^53 / 1000 > 2^24: v is an integer, sig * 2^sh
        const int ex = (int)(mag >> 23);
        const uint32_t sig = (mag & 0x7fffffu) | 0x800000u;
        const int sh = ex - 150;
        n += big_digits(sig, sh, out ? out + n : nullptr);
        fp = 0;
    }
    if (out) {
        out[n] = '.';
        out[n + 1] = (char)('0' + (int)(fp / 100u));
        out[n + 2] = (char)('0' + (int)(fp / 10u % 10u));
        out[n + 3] = (char)('0' + (int)(fp % 10u));
        out[n + 4] = '\n';
    }
    return n + 5;
}

// "%d\n" of a non-negative count below 2^31.
AGT_HD int print_count(double c, char *out)
{
    int64_t k = (int64_t)c;
    int n = 0;
    if (k < 0) {
        if (out) out[n] = '-';
        n++;
        k = -k;
    }
    if (out) n += u64_digits((uint64_t)k, out + n);
    else n += u64_ndigits((uint64_t)k);
    if (out) out[n] = '\n';
    return n + 1;
}

// One line of map text; returns its length, writes it when out is not null.
AGT_HD int format_line(int kind, double e, char *out)
{
    if (kind == kCount) return print_count(e, out);
    if (kind == kEnergy && (e < 0 ? -e : e) < kPrecision) {
        if (out) {
            out[0] = '0';
            out[1] = '\n';
        }
        return 2;
    }
    return print_f3(round3dp_float(e), out);
}

}  // namespace agt
