// Correctly rounded exp for binary64 (round to nearest even), the same code on
// the device and on the host.
//
// Method: P. T. P. Tang's table-driven reduction ("Table-driven implementation
// of the exponential function in IEEE floating-point arithmetic", ACM TOMS
// 15(2), 1989) with A. Ziv's two-step rounding strategy ("Fast evaluation of
// elementary mathematical functions with correctly rounded last bit", ACM TOMS
// 17(3), 1991):
//
//   x = (256 k + j) ln2/256 + r,  |r| <= ln2/512,  exp(x) = 2^k 2^(j/256) e^r.
//
//   fast step:     r and e^r - 1 (degree-8 Taylor polynomial) in double-double
//                  arithmetic, 2^(j/256) from a double-double table; relative
//                  error below 2^-98. When the result rounds to the same double
//                  at both ends of a +-2^-90 interval around it, that double is
//                  exp(x) correctly rounded.
//   accurate step: otherwise (rare), and for subnormal results: r in 128-bit
//                  fixed point from a 192-bit reduction, e^r by a degree-10
//                  Horner scheme in 128-bit fixed point, times 2^(j/256) in
//                  128-bit fixed point: absolute error below 2^-120 on a value
//                  in [1/2, 2), far inside the distance of any binary64 exp
//                  value from a rounding boundary (about 2^-113 relative at
//                  worst: V. Lefevre and J.-M. Muller, "Worst cases for correct
//                  rounding of the elementary functions in double precision",
//                  ARITH 15, 2001), then rounded once.
//
// Every double operation is written out (explicit fused multiply-adds where
// one is meant, plain operations elsewhere; the library builds with FMA
// contraction off), so host and device round alike. Results are correctly
// rounded for every x whose result is a normal double, with +0, +inf and NaN
// at the ends; subnormal results are rounded from the accurate step's value
// (error below 2^-120 of 2^-1022).
#pragma once

#include <cmath>
#include <cstdint>

#include "crexp_tables.h"

#ifdef __CUDACC__
#define BBPD_CREXP_HD __host__ __device__
#else
#define BBPD_CREXP_HD
#endif

namespace bbpd {
namespace crexp_detail {

#ifdef __CUDACC__
static __device__ const double T_DD_D[256][2] = BBPD_CREXP_T_DD;
static __device__ const uint64_t T_FX_D[256][2] = BBPD_CREXP_T_FX;
static __device__ const uint64_t FACT_FX_D[11][2] = BBPD_CREXP_FACT_FX;
#endif
static const double T_DD_H[256][2] = BBPD_CREXP_T_DD;
static const uint64_t T_FX_H[256][2] = BBPD_CREXP_T_FX;
static const uint64_t FACT_FX_H[11][2] = BBPD_CREXP_FACT_FX;

typedef unsigned __int128 u128;

BBPD_CREXP_HD inline double fma_(double a, double b, double c)
{
#ifdef __CUDA_ARCH__
    return __fma_rn(a, b, c);
#else
    return std::fma(a, b, c);
#endif
}

BBPD_CREXP_HD inline double t_dd(int j, int h)
{
#ifdef __CUDA_ARCH__
    return T_DD_D[j][h];
#else
    return T_DD_H[j][h];
#endif
}

BBPD_CREXP_HD inline u128 t_fx(int j)
{
#ifdef __CUDA_ARCH__
    return ((u128)T_FX_D[j][0] << 64) | T_FX_D[j][1];
#else
    return ((u128)T_FX_H[j][0] << 64) | T_FX_H[j][1];
#endif
}

BBPD_CREXP_HD inline u128 fact_fx(int i)
{
#ifdef __CUDA_ARCH__
    return ((u128)FACT_FX_D[i][0] << 64) | FACT_FX_D[i][1];
#else
    return ((u128)FACT_FX_H[i][0] << 64) | FACT_FX_H[i][1];
#endif
}

BBPD_CREXP_HD inline double as_double(uint64_t u)
{
#ifdef __CUDA_ARCH__
    return __longlong_as_double((long long)u);
#else
    double d;
    __builtin_memcpy(&d, &u, 8);
    return d;
#endif
}

BBPD_CREXP_HD inline uint64_t as_bits(double d)
{
#ifdef __CUDA_ARCH__
    return (uint64_t)__double_as_longlong(d);
#else
    uint64_t u;
    __builtin_memcpy(&u, &d, 8);
    return u;
#endif
}

// Double-double helpers (Dekker / Knuth error-free transformations).
BBPD_CREXP_HD inline void two_sum(double a, double b, double &s, double &e)
{
    s = a + b;
    const double bv = s - a;
    e = (a - (s - bv)) + (b - bv);
}

BBPD_CREXP_HD inline void fast_two_sum(double a, double b, double &s, double &e)   // |a| >= |b|
{
    s = a + b;
    e = b - (s - a);
}

BBPD_CREXP_HD inline void dd_mul(double ah, double al, double bh, double bl, double &ph, double &pl)
{
    const double p = ah * bh;
    double e = fma_(ah, bh, -p);
    e = fma_(ah, bl, e);
    e = fma_(al, bh, e);
    fast_two_sum(p, e, ph, pl);
}

BBPD_CREXP_HD inline void dd_add(double ah, double al, double bh, double bl, double &sh, double &sl)
{
    double s, e;
    two_sum(ah, bh, s, e);
    e = e + (al + bl);
    fast_two_sum(s, e, sh, sl);
}

// 2^k as a double, -1022 <= k <= 1023.
BBPD_CREXP_HD inline double pow2(int k)
{
    return as_double((uint64_t)(k + 1023) << 52);
}

// (a * b) >> 125 for 128-bit a, b whose product is below 2^253.
BBPD_CREXP_HD inline u128 mulshift125(u128 a, u128 b)
{
    const uint64_t a0 = (uint64_t)a, a1 = (uint64_t)(a >> 64), b0 = (uint64_t)b, b1 = (uint64_t)(b >> 64);
    const u128 p00 = (u128)a0 * b0, p01 = (u128)a0 * b1, p10 = (u128)a1 * b0, p11 = (u128)a1 * b1;
    u128 t = (p00 >> 64) + (uint64_t)p01 + (uint64_t)p10;
    const uint64_t w1 = (uint64_t)t;
    t = (t >> 64) + (p01 >> 64) + (p10 >> 64) + (uint64_t)p11;
    const uint64_t w2 = (uint64_t)t;
    const uint64_t w3 = (uint64_t)(p11 >> 64) + (uint64_t)(t >> 64);
    const uint64_t lo = (w1 >> 61) | (w2 << 3), hi = (w2 >> 61) | (w3 << 3);
    return ((u128)hi << 64) | lo;
}

// 192-bit two's-complement numbers as three limbs, least significant first.
struct U192 {
    uint64_t l[3];
};

BBPD_CREXP_HD inline U192 neg192(U192 a)
{
    U192 r;
    uint64_t c = 1;
    for (int i = 0; i < 3; i++) {
        const u128 t = (u128)(uint64_t)~a.l[i] + c;
        r.l[i] = (uint64_t)t;
        c = (uint64_t)(t >> 64);
    }
    return r;
}

BBPD_CREXP_HD inline U192 sub192(U192 a, U192 b)
{
    U192 r;
    uint64_t br = 0;
    for (int i = 0; i < 3; i++) {
        const u128 t = (u128)a.l[i] - b.l[i] - br;
        r.l[i] = (uint64_t)t;
        br = (uint64_t)(t >> 64) ? 1 : 0;
    }
    return r;
}

// The accurate step, for |x| >= 2^-60, x in [-745.2, 709.8]; m = the
// reduction's multiple of ln2/256.
BBPD_CREXP_HD inline double accurate(double x, int m)
{
    const int j = m & 255, k = m >> 8;
    // x * 2^145 as a 192-bit integer (exact: x's last bit is >= 2^-112)
    const uint64_t bx = as_bits(x);
    const int ex = (int)((bx >> 52) & 0x7FF);
    const uint64_t mant = (bx & 0xFFFFFFFFFFFFFull) | (1ull << 52);
    const int sh = ex - 1075 + 145;   // 33 .. 102
    U192 X;
    X.l[0] = X.l[1] = X.l[2] = 0;
    {
        const int w = sh >> 6, b = sh & 63;
        X.l[w] = mant << b;
        if (b && w + 1 < 3) X.l[w + 1] = mant >> (64 - b);
    }
    if (bx >> 63) X = neg192(X);
    // m * ln2/256 * 2^145 (mod 2^192)
    const uint64_t am = (uint64_t)(m < 0 ? -m : m);
    U192 P;
    {
        u128 t = (u128)am * crexp_tab::LN2_N_FX0;
        P.l[0] = (uint64_t)t;
        t = (t >> 64) + (u128)am * crexp_tab::LN2_N_FX1;
        P.l[1] = (uint64_t)t;
        t = (t >> 64) + (u128)am * crexp_tab::LN2_N_FX2;
        P.l[2] = (uint64_t)t;
    }
    if (m < 0) P = neg192(P);
    U192 Rr = sub192(X, P);   // r * 2^145, |r| < 2^-9.4
    // r * 2^125, rounded: add 2^19, then the magnitude shifted right by 20
    {
        const u128 t = (u128)Rr.l[0] + (1ull << 19);
        Rr.l[0] = (uint64_t)t;
        const u128 t1 = (u128)Rr.l[1] + (uint64_t)(t >> 64);
        Rr.l[1] = (uint64_t)t1;
        Rr.l[2] += (uint64_t)(t1 >> 64);
    }
    const bool neg = (Rr.l[2] >> 63) != 0;
    if (neg) Rr = neg192(Rr);   // < 2^137
    const u128 ar = ((u128)((Rr.l[2] << 44) | (Rr.l[1] >> 20)) << 64) | ((Rr.l[1] << 44) | (Rr.l[0] >> 20));
    // e^r in 2^-125 units by Horner: acc = 1/i! + r * acc, acc > 0 throughout
    u128 acc = fact_fx(10);
    for (int i = 9; i >= 0; i--) {
        const u128 pr = mulshift125(ar, acc);
        acc = neg ? fact_fx(i) - pr : fact_fx(i) + pr;
    }
    // Y = 2^(j/256) e^r in 2^-126 units: (T * 2^126) (E * 2^125) >> 125
    const u128 Y = mulshift125(t_fx(j), acc);   // in [2^125.99, 2^127)
    // value = Y 2^-126 2^k = 1.f * 2^E2
    const int top = (Y >> 126) ? 126 : 125;
    int E2 = k + top - 126;
    // mantissa bits kept: 53 for a normal result, fewer below 2^-1022
    int keep = 53;
    if (E2 < -1022) keep = 53 - (-1022 - E2);
    if (keep < 0) return 0.0;   // below half the smallest subnormal
    const int cut = top + 1 - keep;   // bits below `cut` are rounded away
    u128 q = Y >> cut;
    const u128 rem = Y & (((u128)1 << cut) - 1), half = (u128)1 << (cut - 1);
    if (rem > half || (rem == half && (q & 1))) q += 1;
    if (keep == 53) {
        if (q >> 53) { q >>= 1; E2 += 1; }   // rounded up to the next power of 2
        if (E2 > 1023) return as_double(0x7FF0000000000000ull);
        return as_double(((uint64_t)(E2 + 1023) << 52) | ((uint64_t)q & 0xFFFFFFFFFFFFFull));
    }
    // subnormal (or rounded up to the smallest normal): q counts units of 2^-1074
    return as_double((uint64_t)q);
}

}  // namespace crexp_detail

// exp(x) correctly rounded to nearest (see the file comment for the range).
BBPD_CREXP_HD inline double cr_exp(double x)
{
    using namespace crexp_detail;
    if (!(x == x)) return x + x;
    if (x > 709.8) return as_double(0x7FF0000000000000ull);
    if (x < -745.2) return 0.0;
    if (::fabs(x) < 0x1p-60) return 1.0 + x;   // no midpoint lies within x^2 of 1 + x here
    const double mf = ::rint(x * crexp_tab::INV_LN2_N);
    const int m = (int)mf;
    const int j = m & 255, k = m >> 8;
    if (k < -1021) return accurate(x, m);   // subnormal range
    // r = x - m ln2/256 as a double-double (three-part constant; the first
    // product and difference are exact)
    const double t1 = fma_(-mf, crexp_tab::LN2_N_1, x);
    const double p2 = mf * crexp_tab::LN2_N_2;
    const double p2e = fma_(mf, crexp_tab::LN2_N_2, -p2);
    double rh, e1;
    two_sum(t1, -p2, rh, e1);
    const double rl0 = (e1 - p2e) - mf * crexp_tab::LN2_N_3;
    double r, rl;
    fast_two_sum(rh, rl0, r, rl);
    // e^r - 1 = r s1, s1 = 1 + r (1/2 + r (1/6 + r (1/24 + r q))),
    // q = 1/120 + r (1/720 + r (1/5040 + r/40320))
    double q = fma_(r, crexp_tab::C8, crexp_tab::C7);
    q = fma_(r, q, crexp_tab::C6);
    q = fma_(r, q, crexp_tab::C5);
    double sh, sl, ph, pl;
    dd_add(crexp_tab::C4H, crexp_tab::C4L, r * q, 0.0, sh, sl);
    dd_mul(r, rl, sh, sl, ph, pl);
    dd_add(crexp_tab::C3H, crexp_tab::C3L, ph, pl, sh, sl);
    dd_mul(r, rl, sh, sl, ph, pl);
    dd_add(0.5, 0.0, ph, pl, sh, sl);
    dd_mul(r, rl, sh, sl, ph, pl);
    dd_add(1.0, 0.0, ph, pl, sh, sl);
    dd_mul(r, rl, sh, sl, ph, pl);   // e^r - 1
    // Y = T (1 + P) = T + T P
    const double th = t_dd(j, 0), tl = t_dd(j, 1);
    double wh, wl, yh, yl;
    dd_mul(th, tl, ph, pl, wh, wl);
    dd_add(th, tl, wh, wl, yh, yl);
    // rounding test: the same double at both ends of +-2^-90 |Y|
    const double eps = ::fabs(yh) * 0x1p-90;
    const double lo = yh + (yl - eps), hi = yh + (yl + eps);
    if (lo != hi) return accurate(x, m);
    if (k == 1024) return (lo * pow2(1023)) * 2.0;
    return lo * pow2(k);
}

}  // namespace bbpd
