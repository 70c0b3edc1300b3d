// crmath.cuh -- correctly rounded log, sin and cos in double-double arithmetic.
//
// The plain FP64 form reproduces the CPU reference's event streams, and the path length
// of a phonon (d = -log(u) v / Gamma) and the Kaplan pair-breaking energies
// (sin^2(pi u / 2)) feed a geometry in which a last-bit difference can grow into a
// different trajectory. These functions therefore return the correctly rounded result
// (the double nearest to the exact value), which is what a good libm returns on all but
// a tiny fraction of arguments. The same code runs on the host and on the device, using
// only IEEE + - * / and fused multiply-add, so host and device results are bit-identical.
//
// Methods (all evaluated in double-double, ~2^-100 relative error before the final
// rounding, so a wrong rounding needs an argument within ~2^-47 ulp of a midpoint):
//  * log: table-driven reduction in the style of P. T. P. Tang, "Table-driven
//    implementation of the logarithm function in IEEE floating-point arithmetic",
//    ACM TOMS 16 (1990): x = 2^e m, c = n/128 nearest m, r = (m - c)/c, and
//    log1p(r) = 2 atanh(r / (2 + r)) summed as a series; log(n/128) and log(2) come
//    from 80-digit tables (gen_crmath_tables.py).
//  * exp / pow: reduction by k log 2, then the Taylor series of exp(r/16) squared four
//    times (pow(x, y) = exp(y log x) with log x kept as a double-double).
//  * hypot / cbrt / acos / atan2: one Newton correction in double-double from
//    sqrt(x^2 + y^2) rounded and from the platform cbrt / acos / atan2 (the correction makes
//    the result independent of the platform's last bit).
//  * sin / cos: Cody-Waite reduction by pi/2 split into four parts (W. J. Cody and
//    W. Waite, "Software Manual for the Elementary Functions", 1980), then the Taylor
//    series of sin and cos on |r| <= pi/4.
//  * double-double arithmetic: error-free transformations of T. J. Dekker, "A
//    floating-point technique for extending the available precision", Numer. Math. 18
//    (1971) and D. E. Knuth, TAOCP vol. 2 (two-sum).
#pragma once

#include <math.h>
#include <stdint.h>
#include <string.h>

#include "crmath_tables.h"

#ifndef CMPMC_HD
#ifdef __CUDACC__
#define CMPMC_HD __host__ __device__ __forceinline__
#else
#define CMPMC_HD inline
#endif
#endif

// rare slow paths are kept out of line so the hot kernels stay small
#ifdef __CUDACC__
#define CMPMC_CR_COLD static __host__ __device__ __noinline__
#else
#define CMPMC_CR_COLD static inline
#endif

namespace cmpmc_gpu {
namespace crmath {

static const double h_logc[87][2] = CMPMC_CR_LOGC;
static const double h_invodd[12][2] = CMPMC_CR_INVODD;
static const double h_sinc[16][2] = CMPMC_CR_SINC;
static const double h_cosc[17][2] = CMPMC_CR_COSC;
#ifdef __CUDACC__
static __device__ const double d_logc[87][2] = CMPMC_CR_LOGC;
static __constant__ double d_invodd[12][2] = CMPMC_CR_INVODD;
static __constant__ double d_sinc[16][2] = CMPMC_CR_SINC;
static __constant__ double d_cosc[17][2] = CMPMC_CR_COSC;
#endif

#ifdef __CUDA_ARCH__
#define CMPMC_CR_TAB(name) d_##name
CMPMC_HD double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
CMPMC_HD double logc_hi(int i) { return __ldg(&d_logc[i][0]); }
CMPMC_HD double logc_lo(int i) { return __ldg(&d_logc[i][1]); }
#else
#define CMPMC_CR_TAB(name) h_##name
CMPMC_HD double fma_rn(double a, double b, double c) { return ::fma(a, b, c); }
CMPMC_HD double logc_hi(int i) { return h_logc[i][0]; }
CMPMC_HD double logc_lo(int i) { return h_logc[i][1]; }
#endif

struct DD {
    double hi, lo;
};

CMPMC_HD DD two_sum(double a, double b) {
    const double s = a + b;
    const double bb = s - a;
    const double e = (a - (s - bb)) + (b - bb);
    return DD{s, e};
}
// requires |a| >= |b| (or a == 0)
CMPMC_HD DD fast_two_sum(double a, double b) {
    const double s = a + b;
    const double e = b - (s - a);
    return DD{s, e};
}
CMPMC_HD DD two_prod(double a, double b) {
    const double p = a * b;
    return DD{p, fma_rn(a, b, -p)};
}
CMPMC_HD DD dd_add(DD x, DD y) {
    DD s = two_sum(x.hi, y.hi);
    const DD t = two_sum(x.lo, y.lo);
    s.lo += t.hi;
    s = fast_two_sum(s.hi, s.lo);
    s.lo += t.lo;
    return fast_two_sum(s.hi, s.lo);
}
CMPMC_HD DD dd_add_d(DD x, double b) {
    DD s = two_sum(x.hi, b);
    s.lo += x.lo;
    return fast_two_sum(s.hi, s.lo);
}
CMPMC_HD DD dd_mul(DD x, DD y) {
    DD p = two_prod(x.hi, y.hi);
    p.lo += x.hi * y.lo + x.lo * y.hi;
    return fast_two_sum(p.hi, p.lo);
}
CMPMC_HD DD dd_mul_d(DD x, double b) {
    DD p = two_prod(x.hi, b);
    p.lo += x.lo * b;
    return fast_two_sum(p.hi, p.lo);
}
CMPMC_HD DD dd_div(DD x, DD y) {
    const double q1 = x.hi / y.hi;
    const DD p = dd_mul_d(y, q1);
    DD r = two_sum(x.hi, -p.hi);
    r.lo += x.lo - p.lo;
    r = fast_two_sum(r.hi, r.lo);
    const double q2 = r.hi / y.hi;
    return fast_two_sum(q1, q2);
}
CMPMC_HD DD dd_tab(const double (*t)[2], int i) { return DD{t[i][0], t[i][1]}; }

// log(x) as a double-double for positive finite normal or subnormal x
CMPMC_CR_COLD DD log_dd(double x) {
    uint64_t bits;
    memcpy(&bits, &x, 8);
    int e = static_cast<int>((bits >> 52) & 0x7ff);
    if (e == 0) {  // subnormal: scale into the normal range
        x *= 18014398509481984.0;  // 2^54
        memcpy(&bits, &x, 8);
        e = static_cast<int>((bits >> 52) & 0x7ff) - 54;
    }
    e -= 1023;
    const uint64_t mbits = (bits & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL;
    double m;
    memcpy(&m, &mbits, 8);  // m in [1, 2)
    if (m >= 4.0 / 3.0) {
        m *= 0.5;
        e += 1;
    }
    const int n = static_cast<int>(m * 128.0 + 0.5);  // c = n / 128, n in [85, 171]
    const double c = n * (1.0 / 128.0);
    const double t = m - c;  // exact (Sterbenz)
    const double q = t / c;
    const DD r = fast_two_sum(q, fma_rn(-q, c, t) / c);  // r = t / c, |r| < 2^-7.4
    // log1p(r) = 2 s (1 + s^2/3 + s^4/5 + ...), s = r / (2 + r), |s| < 2^-8.4
    const DD s = dd_div(r, dd_add_d(r, 2.0));
    const DD z = dd_mul(s, s);
    DD acc = dd_tab(CMPMC_CR_TAB(invodd), 7);
#pragma unroll
    for (int k = 6; k >= 0; --k) acc = dd_add(dd_mul(acc, z), dd_tab(CMPMC_CR_TAB(invodd), k));
    DD res = dd_mul_d(dd_mul(s, acc), 2.0);
    res = dd_add(res, DD{logc_hi(n - 85), logc_lo(n - 85)});
    if (e != 0) res = dd_add(res, dd_mul_d(DD{CMPMC_CR_LN2_HI, CMPMC_CR_LN2_LO}, static_cast<double>(e)));
    return res;
}

// Ziv's rounding test: (h, l) is normalised (h = RN(h + l)) and the exact value lies within
// eps |h| of h + l; true when every value in that interval rounds to h, so h is the
// correctly rounded result (J.-M. Muller et al., Handbook of Floating-Point Arithmetic,
// "Ziv's strategy"). The margin is inflated slightly to cover the rounding of l +- e.
CMPMC_HD bool ziv_ok(double h, double l, double eps) {
    const double e = fabs(h) * (eps * 1.125);
    return (h + (l + e) == h) && (h + (l - e) == h);
}

// log(x) correctly rounded for positive finite x; other inputs go to the platform log.
// Fast path: the same reduction with log1p(r) summed as r - r^2/2 (error-free) plus an
// FP64 tail, relative error below 2^-64; the double-double path runs only when the
// rounding test fails (about one call in a thousand).
CMPMC_HD double log(double x) {
    if (!(x > 0.0) || !(x < __builtin_huge_val())) return ::log(x);
    uint64_t bits;
    memcpy(&bits, &x, 8);
    int e = static_cast<int>((bits >> 52) & 0x7ff);
    if (e == 0) {
        const DD r = log_dd(x);
        return r.hi + r.lo;
    }
    e -= 1023;
    const uint64_t mbits = (bits & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL;
    double m;
    memcpy(&m, &mbits, 8);
    if (m >= 4.0 / 3.0) {
        m *= 0.5;
        e += 1;
    }
    const int n = static_cast<int>(m * 128.0 + 0.5);
    const double c = n * (1.0 / 128.0);
    const double t = m - c;
    const double q = t / c;
    const double ql = fma_rn(-q, c, t) / c;  // r = q + ql
    const DD z = two_prod(q, q);
    // log1p(q) - q + q^2/2 = q^3 (1/3 - q/4 + q^2/5 - ...), |q| < 2^-7.4, to q^11
    const double tail = q * z.hi *
                        (1.0 / 3 + q * (-1.0 / 4 + q * (1.0 / 5 + q * (-1.0 / 6 + q * (1.0 / 7 + q * (-1.0 / 8 +
                         q * (1.0 / 9 + q * (-1.0 / 10 + q * (1.0 / 11)))))))));
    const double ed = static_cast<double>(e);
    const DD A = two_sum(ed * CMPMC_CR_LN2_H42, logc_hi(n - 85));  // ed * head is exact
    const DD B = two_sum(A.hi, q);
    const DD C = two_sum(B.hi, -0.5 * z.hi);
    const double lo = A.lo + B.lo + C.lo + (ql - ql * q) - 0.5 * z.lo + tail +
                      (ed * CMPMC_CR_LN2_T42 + logc_lo(n - 85));
    const DD y = fast_two_sum(C.hi, lo);
    if (ziv_ok(y.hi, y.lo, 0x1p-64)) return y.hi;
    const DD r = log_dd(x);
    return r.hi + r.lo;
}

// exp of a double-double argument t, |t| < 700: t = k ln2 + r, exp(r) = (exp(r/16))^16
// with the Taylor series of exp(r/16), |r/16| < 0.022.
CMPMC_CR_COLD DD exp_dd(DD t, int& k_out) {
    const double kd = rint(t.hi * 1.4426950408889634);
    const DD kl = dd_mul_d(DD{CMPMC_CR_LN2_HI, CMPMC_CR_LN2_LO}, kd);
    DD r = dd_add(t, DD{-kl.hi, -kl.lo});
    r = DD{r.hi * 0.0625, r.lo * 0.0625};  // exact scaling
    // sum_{n=0}^{12} r^n / n! by Horner with exact 1/n! as double-double quotients
    DD acc = DD{1.0, 0.0};
#pragma unroll
    for (int n = 12; n >= 1; --n) {
        acc = dd_div(dd_mul(acc, r), DD{static_cast<double>(n), 0.0});
        acc = dd_add_d(acc, 1.0);
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) acc = dd_mul(acc, acc);
    k_out = static_cast<int>(kd);
    return acc;
}

CMPMC_HD double scale2(double v, int k) {
    // v * 2^k for |k| < 1000 in two exact steps (results stay normal for our arguments)
    const int k1 = k / 2, k2 = k - k / 2;
    uint64_t b1 = static_cast<uint64_t>(k1 + 1023) << 52, b2 = static_cast<uint64_t>(k2 + 1023) << 52;
    double f1, f2;
    memcpy(&f1, &b1, 8);
    memcpy(&f2, &b2, 8);
    return (v * f1) * f2;
}

// exp(x) correctly rounded for |x| < 700 (results in the normal range)
CMPMC_HD double exp(double x) {
    if (!(fabs(x) < 700.0)) return ::exp(x);
    int k;
    const DD e = exp_dd(DD{x, 0.0}, k);
    return scale2(e.hi + e.lo, k);
}

// pow(x, y) = exp(y log x) correctly rounded for x > 0 and |y log x| < 700
CMPMC_HD double pow(double x, double y) {
    if (!(x > 0.0) || !(x < __builtin_huge_val()) || !(fabs(y) < 1e300)) return ::pow(x, y);
    if (y == 0.0 || x == 1.0) return 1.0;
    const DD t = dd_mul_d(log_dd(x), y);
    if (!(fabs(t.hi) < 700.0)) return ::pow(x, y);
    int k;
    const DD e = exp_dd(t, k);
    return scale2(e.hi + e.lo, k);
}

// sqrt(x^2 + y^2) correctly rounded, for |x|, |y| in [2^-400, 2^400] (or one of them 0)
CMPMC_HD double hypot(double x, double y) {
    x = fabs(x);
    y = fabs(y);
    if (x < y) {
        const double t = x;
        x = y;
        y = t;
    }
    if (y == 0.0) return x;
    if (!(x < 2.5e120) || !(y > 3.9e-121)) return ::hypot(x, y);
    const DD s = dd_add(two_prod(x, x), two_prod(y, y));
    const double r = sqrt(s.hi);
    const DD r2 = two_prod(r, r);
    const DD d = dd_add(s, DD{-r2.hi, -r2.lo});
    const double corr = (d.hi + d.lo) / (2.0 * r);
    return r + corr;
}

// cbrt(x) correctly rounded: one Newton step in double-double from the platform cbrt
CMPMC_HD double cbrt(double x) {
    const double ax = fabs(x);
    if (!(ax > 2.3e-200) || !(ax < 4.3e200)) return ::cbrt(x);
    const double y = ::cbrt(ax);
    const DD y3 = dd_mul_d(two_prod(y, y), y);
    const DD d = dd_add_d(y3, -ax);
    const double corr = (d.hi + d.lo) / (3.0 * y * y);
    const double r = y - corr;
    return x < 0.0 ? -r : r;
}

// Reduction x = k pi/2 + r with r as double-double, |r| <= ~pi/4, for |x| < 2^20.
CMPMC_HD DD reduce_pio2(double x, int& quadrant) {
    const double kd = rint(x * CMPMC_CR_TWO_OVER_PI);
    const double a = x - kd * CMPMC_CR_PIO2_1;  // exact: k pi/2 near x, 33-bit part
    DD r = two_sum(a, -kd * CMPMC_CR_PIO2_2);    // kd * part2 exact (33-bit part)
    const DD p3 = two_prod(kd, CMPMC_CR_PIO2_3);
    r = dd_add(r, DD{-p3.hi, -p3.lo});
    r = dd_add_d(r, -kd * CMPMC_CR_PIO2_4);
    quadrant = static_cast<int>(static_cast<int64_t>(kd) & 3);
    return r;
}

// sin(r) and cos(r) for |r| <= pi/4 + eps as double-double
CMPMC_HD DD sin_kernel(DD r, DD z) {
    DD acc = dd_tab(CMPMC_CR_TAB(sinc), 14);
#pragma unroll
    for (int k = 13; k >= 0; --k) acc = dd_add(dd_mul(acc, z), dd_tab(CMPMC_CR_TAB(sinc), k));
    return dd_mul(acc, r);
}
CMPMC_HD DD cos_kernel(DD z) {
    DD acc = dd_tab(CMPMC_CR_TAB(cosc), 15);
#pragma unroll
    for (int k = 14; k >= 0; --k) acc = dd_add(dd_mul(acc, z), dd_tab(CMPMC_CR_TAB(cosc), k));
    return acc;
}

CMPMC_HD bool in_range(double x) { return fabs(x) < 1048576.0; }

// Fast sin / cos of a reduced argument r = rh + rl (|r| <= pi/4 + eps) as unrounded (h, l)
// with relative error below 2^-64 (sin) and 2^-63 (cos): the leading Taylor terms
// (r^3/6, r^5/120 and r^2/2, r^4/24) in double-double, the rest in FP64.
CMPMC_HD DD sin_fast(DD r) {
    const double rh = r.hi, rl = r.lo;
    const DD z = two_prod(rh, rh);                                   // rh^2 exactly
    const DD p3 = two_prod(rh, z.hi);
    const DD r3 = fast_two_sum(p3.hi, p3.lo + rh * z.lo);            // rh^3
    const DD t3 = dd_mul(r3, DD{CMPMC_CR_INV6_HI, CMPMC_CR_INV6_LO});
    const DD t5 = dd_div(dd_mul(r3, z), DD{120.0, 0.0});
    const double zz = z.hi;
    const double tail7 = rh * zz * zz * zz *
                         (-1.0 / 5040 + zz * (1.0 / 362880 + zz * (-1.0 / 39916800 + zz * (1.0 / 6227020800.0 +
                          zz * (-1.0 / 1307674368000.0 + zz * (1.0 / 355687428096000.0 +
                          zz * (-1.0 / 121645100408832000.0 + zz * (1.0 / 51090942171709440000.0))))))));
    const double dcos = 1.0 - 0.5 * zz + zz * zz * (1.0 / 24) - zz * zz * zz * (1.0 / 720);
    DD s = two_sum(rh, -t3.hi);
    const DD s2 = two_sum(s.hi, t5.hi);
    const double lo = s.lo + s2.lo - t3.lo + t5.lo + tail7 + rl * dcos;
    return fast_two_sum(s2.hi, lo);
}
CMPMC_HD DD cos_fast(DD r) {
    const double rh = r.hi, rl = r.lo;
    const DD z = two_prod(rh, rh);
    const double w = z.lo + 2.0 * rh * rl;                            // r^2 = z.hi + w
    const DD zsq = two_prod(z.hi, z.hi);
    const DD t4 = dd_mul(DD{zsq.hi, zsq.lo + 2.0 * z.hi * w}, DD{CMPMC_CR_INV24_HI, CMPMC_CR_INV24_LO});
    const double zz = z.hi;
    const double tail6 = zz * zz * zz *
                         (-1.0 / 720 + zz * (1.0 / 40320 + zz * (-1.0 / 3628800 + zz * (1.0 / 479001600.0 +
                          zz * (-1.0 / 87178291200.0 + zz * (1.0 / 20922789888000.0 +
                          zz * (-1.0 / 6402373705728000.0 + zz * (1.0 / 2432902008176640000.0))))))));
    const DD c = two_sum(1.0, -0.5 * z.hi);
    const DD c2 = two_sum(c.hi, t4.hi);
    const double lo = c.lo + c2.lo + t4.lo - 0.5 * w + tail6;
    return fast_two_sum(c2.hi, lo);
}

CMPMC_CR_COLD double sin_slow(double x);
CMPMC_CR_COLD double cos_slow(double x);

CMPMC_HD double sin(double x) {
    if (!in_range(x) || x == 0.0) return sin_slow(x);
    int q;
    const DD r = reduce_pio2(x, q);
    const DD v = (q & 1) ? cos_fast(r) : sin_fast(r);
    if (!ziv_ok(v.hi, v.lo, 0x1p-62)) return sin_slow(x);
    return (q & 2) ? -v.hi : v.hi;
}

CMPMC_HD double cos(double x) {
    if (!in_range(x)) return cos_slow(x);
    int q;
    const DD r = reduce_pio2(x, q);
    const DD v = (q & 1) ? sin_fast(r) : cos_fast(r);
    if (!ziv_ok(v.hi, v.lo, 0x1p-62)) return cos_slow(x);
    return ((q + 1) & 2) ? -v.hi : v.hi;
}

CMPMC_CR_COLD double sin_slow(double x) {
    if (!in_range(x)) return ::sin(x);
    if (x == 0.0) return x;
    int q;
    const DD r = reduce_pio2(x, q);
    const DD z = dd_mul(r, r);
    DD v;
    if (q & 1) v = cos_kernel(z);
    else v = sin_kernel(r, z);
    const double y = v.hi + v.lo;
    return (q & 2) ? -y : y;
}

CMPMC_CR_COLD double cos_slow(double x) {
    if (!in_range(x)) return ::cos(x);
    int q;
    const DD r = reduce_pio2(x, q);
    const DD z = dd_mul(r, r);
    DD v;
    if (q & 1) v = sin_kernel(r, z);
    else v = cos_kernel(z);
    const double y = v.hi + v.lo;
    return ((q + 1) & 2) ? -y : y;
}

// sin and cos of x as double-doubles (|x| < 2^20)
CMPMC_CR_COLD void sincos_dd(double x, DD& s, DD& c) {
    int q;
    const DD r = reduce_pio2(x, q);
    const DD z = dd_mul(r, r);
    const DD vs = sin_kernel(r, z);
    const DD vc = cos_kernel(z);
    const DD ns{-vs.hi, -vs.lo}, nc{-vc.hi, -vc.lo};
    switch (q) {
        case 0: s = vs; c = vc; break;
        case 1: s = vc; c = ns; break;
        case 2: s = ns; c = nc; break;
        default: s = nc; c = vs; break;
    }
}

// acos(x) correctly rounded: one Newton step on cos(y) = x in double-double from the
// platform acos (|x| = 1 and arguments outside [-1, 1] go to the platform acos).
CMPMC_HD double acos(double x) {
    if (!(fabs(x) < 1.0)) return ::acos(x);
    const double y0 = ::acos(x);
    DD s, c;
    sincos_dd(y0, s, c);
    const DD f = dd_add_d(c, -x);  // cos(y0) - x
    const double corr = (f.hi + f.lo) / (s.hi + s.lo);
    return y0 + corr;
}

// atan2(y, x) correctly rounded: one Newton step on y cos(t) - x sin(t) = 0 in double-double
// from the platform atan2 (zeros, infinities and NaNs go to the platform atan2).
CMPMC_HD double atan2(double y, double x) {
    if (!(fabs(x) < 1.0 / 0.0) || !(fabs(y) < 1.0 / 0.0) || x == 0.0 || y == 0.0) return ::atan2(y, x);
    const double t0 = ::atan2(y, x);
    DD s, c;
    sincos_dd(t0, s, c);
    const DD f = dd_add(dd_mul_d(c, y), dd_mul_d(s, -x));  // y cos(t0) - x sin(t0)
    const double g = x * c.hi + y * s.hi;                    // hypot(x, y) near the root
    return t0 + (f.hi + f.lo) / g;
}

// both at once
CMPMC_HD void sincos(double x, double& s, double& c) {
    s = sin(x);
    c = cos(x);
}

}  // namespace crmath
}  // namespace cmpmc_gpu
