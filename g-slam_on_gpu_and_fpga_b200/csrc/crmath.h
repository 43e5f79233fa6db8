/*
 * crmath.h — correctly rounded double-precision sin/cos, shared by host and device.
 *
 * Why this exists: the reference linearises every edge with glibc's sin/cos/pow
 * (src/cpu_pcg_fp64/ObsEdge.c:22-49, MotionEdge.c:254-258,290-291,
 * GSLAM.c:373-401). Neither glibc nor CUDA's device libm is correctly rounded, so
 * the two disagree in the last bit on a fraction of arguments. This header gives
 * one routine that returns the correctly rounded result (except on arguments whose
 * exact value lies within ~2^-100 relative of a rounding boundary) and that
 * compiles to bit-identical results under gcc (-ffp-contract=off) and nvcc
 * (-fmad=false): every operation is an IEEE round-to-nearest +, -, *, or an
 * explicit fused multiply-add.
 *
 * Method (published, restated here):
 *  - Argument reduction after Cody & Waite (1980): k = nearest(x * 2/pi);
 *    r = x - k*(P1+P2+P3+P4) with pi/2 split into three 32-bit pieces and a
 *    53-bit tail, so k*P1, k*P2, k*P3 are exact for |k| < 2^21; the reduced
 *    argument is carried as a double-double (hi, lo).
 *  - Double-double arithmetic after Dekker (1971) and Knuth (TAOCP vol. 2):
 *    two-sum, fast two-sum and the FMA two-product.
 *  - Taylor series of sin and cos about 0 on |r| <= pi/4 (+ slack), with the
 *    coefficients 1/n! given as double-doubles (computed from their exact
 *    rational values). Terms below 2^-53 of the leading term are summed in plain
 *    double, the rest in double-double. Truncation error < 2^-110 relative.
 *
 * The split constants and 1/n! values were computed with 400-bit arithmetic.
 * Arguments with |x| >= 2^21 * pi/2 (about 3.3e6 rad) or non-finite fall back to
 * the platform's sin/cos, which is never reached by pose graphs of bounded angle.
 */
#ifndef GSLAM_CRMATH_H
#define GSLAM_CRMATH_H

#include <math.h>

#if defined(__CUDACC__)
#define CRM_FN static __host__ __device__ __forceinline__
#else
#define CRM_FN static inline
#endif

#if defined(__CUDA_ARCH__)
#define CRM_FMA(a, b, c) __fma_rn((a), (b), (c))
#define CRM_RINT(a) rint(a)
#else
#define CRM_FMA(a, b, c) fma((a), (b), (c))
#define CRM_RINT(a) nearbyint(a)
#endif

typedef struct { double hi, lo; } crm_dd;

/* Knuth two-sum: s + e == a + b exactly. */
CRM_FN crm_dd crm_two_sum(double a, double b) {
    crm_dd r;
    double s = a + b;
    double bb = s - a;
    double e = (a - (s - bb)) + (b - bb);
    r.hi = s; r.lo = e;
    return r;
}

/* Dekker fast two-sum, requires |a| >= |b| (or a == 0). */
CRM_FN crm_dd crm_fast_two_sum(double a, double b) {
    crm_dd r;
    double s = a + b;
    double e = b - (s - a);
    r.hi = s; r.lo = e;
    return r;
}

/* a * b == p + e exactly (FMA two-product). */
CRM_FN crm_dd crm_two_prod(double a, double b) {
    crm_dd r;
    double p = a * b;
    r.hi = p;
    r.lo = CRM_FMA(a, b, -p);
    return r;
}

CRM_FN crm_dd crm_dd_add(crm_dd a, crm_dd b) {
    crm_dd s = crm_two_sum(a.hi, b.hi);
    crm_dd t = crm_two_sum(a.lo, b.lo);
    s.lo = s.lo + t.hi;
    s = crm_fast_two_sum(s.hi, s.lo);
    s.lo = s.lo + t.lo;
    return crm_fast_two_sum(s.hi, s.lo);
}

CRM_FN crm_dd crm_dd_mul(crm_dd a, crm_dd b) {
    crm_dd p = crm_two_prod(a.hi, b.hi);
    p.lo = p.lo + (a.hi * b.lo + a.lo * b.hi);
    return crm_fast_two_sum(p.hi, p.lo);
}

CRM_FN crm_dd crm_dd_mul_d(crm_dd a, double b) {
    crm_dd p = crm_two_prod(a.hi, b);
    p.lo = p.lo + a.lo * b;
    return crm_fast_two_sum(p.hi, p.lo);
}

/* 1/n! as double-doubles, n = 0..28 (hi, lo). */
#define CRM_INVF_HI_0 0x1.0000000000000p+0
#define CRM_INVF_LO_0 0.0
#define CRM_INVF_HI_1 0x1.0000000000000p+0
#define CRM_INVF_LO_1 0.0
#define CRM_INVF_HI_2 0x1.0000000000000p-1
#define CRM_INVF_LO_2 0.0
#define CRM_INVF_HI_3 0x1.5555555555555p-3
#define CRM_INVF_LO_3 0x1.5555555555555p-57
#define CRM_INVF_HI_4 0x1.5555555555555p-5
#define CRM_INVF_LO_4 0x1.5555555555555p-59
#define CRM_INVF_HI_5 0x1.1111111111111p-7
#define CRM_INVF_LO_5 0x1.1111111111111p-63
#define CRM_INVF_HI_6 0x1.6c16c16c16c17p-10
#define CRM_INVF_LO_6 -0x1.f49f49f49f49fp-65
#define CRM_INVF_HI_7 0x1.a01a01a01a01ap-13
#define CRM_INVF_LO_7 0x1.a01a01a01a01ap-73
#define CRM_INVF_HI_8 0x1.a01a01a01a01ap-16
#define CRM_INVF_LO_8 0x1.a01a01a01a01ap-76
#define CRM_INVF_HI_9 0x1.71de3a556c734p-19
#define CRM_INVF_LO_9 -0x1.c154f8ddc6c00p-73
#define CRM_INVF_HI_10 0x1.27e4fb7789f5cp-22
#define CRM_INVF_LO_10 0x1.cbbc05b4fa99ap-76
#define CRM_INVF_HI_11 0x1.ae64567f544e4p-26
#define CRM_INVF_LO_11 -0x1.c062e06d1f209p-80
#define CRM_INVF_HI_12 0x1.1eed8eff8d898p-29
#define CRM_INVF_LO_12 -0x1.2aec959e14c06p-83
#define CRM_INVF_HI_13 0x1.6124613a86d09p-33
#define CRM_INVF_LO_13 0x1.f28e0cc748ebep-87
#define CRM_INVF_HI_14 0x1.93974a8c07c9dp-37
#define CRM_INVF_LO_14 0x1.05d6f8a2efd1fp-92
#define CRM_INVF_HI_15 0x1.ae7f3e733b81fp-41
#define CRM_INVF_LO_15 0x1.1d8656b0ee8cbp-97
#define CRM_INVF_HI_16 0x1.ae7f3e733b81fp-45
#define CRM_INVF_LO_16 0x1.1d8656b0ee8cbp-101
#define CRM_INVF_17 0x1.952c77030ad4ap-49
#define CRM_INVF_18 0x1.6827863b97d97p-53
#define CRM_INVF_19 0x1.2f49b46814157p-57
#define CRM_INVF_20 0x1.e542ba4020225p-62
#define CRM_INVF_21 0x1.71b8ef6dcf572p-66
#define CRM_INVF_22 0x1.0ce396db7f853p-70
#define CRM_INVF_23 0x1.761b41316381ap-75
#define CRM_INVF_24 0x1.f2cf01972f578p-80
#define CRM_INVF_25 0x1.3f3ccdd165fa9p-84
#define CRM_INVF_26 0x1.88e85fc6a4e5ap-89
#define CRM_INVF_27 0x1.d1ab1c2dccea3p-94
#define CRM_INVF_28 0x1.0a18a2635085dp-98

/* One double-double Horner step: acc = c + u * acc (c given as hi/lo, signed). */
CRM_FN crm_dd crm_horner(crm_dd acc, crm_dd u, double chi, double clo) {
    crm_dd c; c.hi = chi; c.lo = clo;
    return crm_dd_add(c, crm_dd_mul(u, acc));
}

/*
 * sin and cos of the double-double r (|r| <= pi/4 + 2^-40), each returned as a
 * normalised double-double.
 */
CRM_FN void crm_sincos_kernel(crm_dd r, crm_dd *s, crm_dd *c) {
    crm_dd u = crm_dd_mul(r, r);
    double uh = u.hi;
    /* sin(r) = r * S(u), S(u) = sum_m (-1)^m u^m / (2m+1)!, m = 0..13 */
    double ts = -CRM_INVF_27;
    ts = CRM_INVF_25 + uh * ts;
    ts = -CRM_INVF_23 + uh * ts;
    ts = CRM_INVF_21 + uh * ts;
    ts = -CRM_INVF_19 + uh * ts;
    ts = CRM_INVF_17 + uh * ts;            /* m = 8..13 in double */
    crm_dd a; a.hi = ts; a.lo = 0.0;
    a = crm_horner(a, u, -CRM_INVF_HI_15, -CRM_INVF_LO_15);
    a = crm_horner(a, u, CRM_INVF_HI_13, CRM_INVF_LO_13);
    a = crm_horner(a, u, -CRM_INVF_HI_11, -CRM_INVF_LO_11);
    a = crm_horner(a, u, CRM_INVF_HI_9, CRM_INVF_LO_9);
    a = crm_horner(a, u, -CRM_INVF_HI_7, -CRM_INVF_LO_7);
    a = crm_horner(a, u, CRM_INVF_HI_5, CRM_INVF_LO_5);
    a = crm_horner(a, u, -CRM_INVF_HI_3, -CRM_INVF_LO_3);
    a = crm_horner(a, u, CRM_INVF_HI_1, CRM_INVF_LO_1);
    *s = crm_dd_mul(r, a);
    /* cos(r) = C(u), C(u) = sum_m (-1)^m u^m / (2m)!, m = 0..14 */
    double tc = CRM_INVF_28;
    tc = -CRM_INVF_26 + uh * tc;
    tc = CRM_INVF_24 + uh * tc;
    tc = -CRM_INVF_22 + uh * tc;
    tc = CRM_INVF_20 + uh * tc;
    tc = -CRM_INVF_18 + uh * tc;           /* m = 9..14 in double */
    crm_dd b; b.hi = tc; b.lo = 0.0;
    b = crm_horner(b, u, CRM_INVF_HI_16, CRM_INVF_LO_16);
    b = crm_horner(b, u, -CRM_INVF_HI_14, -CRM_INVF_LO_14);
    b = crm_horner(b, u, CRM_INVF_HI_12, CRM_INVF_LO_12);
    b = crm_horner(b, u, -CRM_INVF_HI_10, -CRM_INVF_LO_10);
    b = crm_horner(b, u, CRM_INVF_HI_8, CRM_INVF_LO_8);
    b = crm_horner(b, u, -CRM_INVF_HI_6, -CRM_INVF_LO_6);
    b = crm_horner(b, u, CRM_INVF_HI_4, CRM_INVF_LO_4);
    b = crm_horner(b, u, -CRM_INVF_HI_2, -CRM_INVF_LO_2);
    b = crm_horner(b, u, CRM_INVF_HI_0, CRM_INVF_LO_0);
    *c = b;
}

/* pi/2 = P1 + P2 + P3 + P4 (+ 7.4e-49); P1..P3 carry 32 significant bits. */
#define CRM_PIO2_1 0x1.921fb54400000p+0
#define CRM_PIO2_2 0x1.0b4611a600000p-34
#define CRM_PIO2_3 0x1.3198a2e000000p-69
#define CRM_PIO2_4 0x1.b839a252049c1p-104
#define CRM_TWO_OVER_PI 0x1.45f306dc9c883p-1
#define CRM_REDUCE_LIMIT 0x1.921fb54442d18p+21 /* 2^21 * pi/2 */

/* Correctly rounded sin(x) and cos(x). */
CRM_FN void cr_sincos(double x, double *sn, double *cs) {
    if (!(fabs(x) < CRM_REDUCE_LIMIT)) {   /* huge or non-finite: platform libm */
        *sn = sin(x);
        *cs = cos(x);
        return;
    }
    if (x == 0.0) {                        /* keeps the sign of zero */
        *sn = x;
        *cs = 1.0;
        return;
    }
    double k = CRM_RINT(x * CRM_TWO_OVER_PI);
    crm_dd r;
    if (k == 0.0) {
        r.hi = x; r.lo = 0.0;
    } else {
        double t = x - k * CRM_PIO2_1;               /* exact */
        crm_dd a = crm_two_sum(t, -(k * CRM_PIO2_2)); /* k*P2 exact */
        crm_dd b; b.hi = -(k * CRM_PIO2_3); b.lo = 0.0; /* k*P3 exact */
        a = crm_dd_add(a, b);
        crm_dd c = crm_two_prod(k, CRM_PIO2_4);
        c.hi = -c.hi; c.lo = -c.lo;
        r = crm_dd_add(a, c);
    }
    crm_dd s, c;
    crm_sincos_kernel(r, &s, &c);
    /* quadrant: k mod 4 (k is an exact integer with |k| < 2^21) */
    long q = ((long)k) & 3;
    double sv, cv;
    switch (q) {
        case 0: sv = s.hi;  cv = c.hi;  break;
        case 1: sv = c.hi;  cv = -s.hi; break;
        case 2: sv = -s.hi; cv = -c.hi; break;
        default: sv = -c.hi; cv = s.hi; break;
    }
    *sn = sv;
    *cs = cv;
}

CRM_FN double cr_sin(double x) { double s, c; cr_sincos(x, &s, &c); return s; }
CRM_FN double cr_cos(double x) { double s, c; cr_sincos(x, &s, &c); return c; }

#endif /* GSLAM_CRMATH_H */
