/*
 * se2_dd.c — the SE(2) pose-graph gradient and a position loss in double-double.
 *
 * TEST INFRASTRUCTURE ONLY (built into liboracle.so; nothing in the product links,
 * loads or calls it). It is the checker for the implicit-function adjoint's finite
 * differences: a central difference of a loss of Gauss-Newton's fixed point needs that
 * fixed point far more precisely than FP64 gives it. The fixed point is where
 * xi = -sum_e J_e^T Lambda_e e_e vanishes, and it is known only as precisely as xi is
 * evaluated; in FP64 that noise, divided by 2h, swamps the difference at h = 1e-6.
 * Evaluating xi at double-double poses in double-double arithmetic (Dekker 1971; Knuth,
 * TAOCP vol. 2: about 106-bit significands) lowers that floor by about 16 orders of
 * magnitude, and so does summing the loss in double-double.
 *
 * The factor is the library's SE(2) between-factor (csrc/edge_math.cuh em_se2_edge):
 *   e = [R(th_i)^T (t_j - t_i) - z_t ; wrap(th_j - th_i - z_th)],  Lambda = diag(info),
 *   J_i = [[-c, -s, c dy - s dx], [s, -c, -c dx - s dy], [0, 0, -1]],
 *   J_j = [[c, s, 0], [-s, c, 0], [0, 0, 1]],  c, s = cos, sin(th_i).
 * sin and cos of a double-double angle reuse crmath.h's Cody-Waite reduction (pi/2 in
 * four pieces, 7.4e-49 short of pi/2) and its double-double Taylor kernel (truncation
 * below 2^-110 relative).
 */
#include <math.h>
#include <stddef.h>

#include "crmath.h"

static crm_dd dd(double hi, double lo) { crm_dd r; r.hi = hi; r.lo = lo; return r; }
static crm_dd dd_neg(crm_dd a) { return dd(-a.hi, -a.lo); }
static crm_dd dd_sub(crm_dd a, crm_dd b) { return crm_dd_add(a, dd_neg(b)); }

/* x - m (P1 + P2 + P3 + P4) for an integer m with |m| < 2^21: the Cody-Waite reduction
 * of cr_sincos, carried on a double-double x. */
static crm_dd dd_reduce(crm_dd x, double m) {
    if (m == 0.0) return x;
    crm_dd r = crm_two_sum(x.hi - m * CRM_PIO2_1, -(m * CRM_PIO2_2));   /* both products exact */
    r = crm_dd_add(r, dd(-(m * CRM_PIO2_3), 0.0));
    crm_dd t = crm_two_prod(m, CRM_PIO2_4);
    r = crm_dd_add(r, dd_neg(t));
    return crm_dd_add(r, dd(x.lo, 0.0));
}

/* sin and cos of a double-double angle (|x| well below 2^21 pi/2). */
static void sincos_dd(crm_dd x, crm_dd *sn, crm_dd *cs) {
    const double k = CRM_RINT(x.hi * CRM_TWO_OVER_PI);
    crm_dd s, c;
    crm_sincos_kernel(dd_reduce(x, k), &s, &c);
    switch (((long)k) & 3) {
        case 0: *sn = s; *cs = c; break;
        case 1: *sn = c; *cs = dd_neg(s); break;
        case 2: *sn = dd_neg(s); *cs = dd_neg(c); break;
        default: *sn = dd_neg(c); *cs = s; break;
    }
}

/* a - 2 pi round(a / 2 pi): the angle residual's wrap into [-pi, pi] */
static crm_dd wrap_dd(crm_dd a) {
    const double k = CRM_RINT(a.hi * (0.5 * CRM_TWO_OVER_PI * 0.5));   /* a / (2 pi) */
    return dd_reduce(a, 4.0 * k);
}

static crm_dd dd_madd(crm_dd acc, crm_dd a, crm_dd b) { return crm_dd_add(acc, crm_dd_mul(a, b)); }

/*
 * xi = -sum_e J_e^T Lambda_e e_e at poses (p_hi + p_lo) [3 n_poses], in double-double,
 * edges summed in array order; info[3 e + k] = Lambda_e's diagonal (lambda folded in).
 * Returns 0, or -1 for an edge whose pose index is out of range.
 */
int or_se2_rhs_dd(long n_poses, long n_edges, const unsigned *ei, const unsigned *ej,
                  const double *p_hi, const double *p_lo, const double *meas, const double *info,
                  double *xi_hi, double *xi_lo) {
    for (long q = 0; q < 3 * n_poses; q++) xi_hi[q] = xi_lo[q] = 0.0;
    for (long e = 0; e < n_edges; e++) {
        const long i = ei[e], j = ej[e];
        if (i >= n_poses || j >= n_poses) return -1;
        const crm_dd xi_ = dd(p_hi[3 * i], p_lo[3 * i]), yi = dd(p_hi[3 * i + 1], p_lo[3 * i + 1]);
        const crm_dd ti = dd(p_hi[3 * i + 2], p_lo[3 * i + 2]);
        const crm_dd xj = dd(p_hi[3 * j], p_lo[3 * j]), yj = dd(p_hi[3 * j + 1], p_lo[3 * j + 1]);
        const crm_dd tj = dd(p_hi[3 * j + 2], p_lo[3 * j + 2]);
        crm_dd s, c;
        sincos_dd(ti, &s, &c);
        const crm_dd dx = dd_sub(xj, xi_), dy = dd_sub(yj, yi);
        /* e0 = c dx + s dy - z0, e1 = c dy - s dx - z1, e2 = wrap(th_j - th_i - z2) */
        crm_dd e0 = dd_madd(crm_dd_mul(c, dx), s, dy);
        e0 = crm_dd_add(e0, dd(-meas[3 * e], 0.0));
        crm_dd e1 = dd_sub(crm_dd_mul(c, dy), crm_dd_mul(s, dx));
        e1 = crm_dd_add(e1, dd(-meas[3 * e + 1], 0.0));
        const crm_dd e2 = wrap_dd(crm_dd_add(dd_sub(tj, ti), dd(-meas[3 * e + 2], 0.0)));
        const crm_dd a0 = crm_dd_mul_d(e0, info[3 * e]), a1 = crm_dd_mul_d(e1, info[3 * e + 1]);
        const crm_dd a2 = crm_dd_mul_d(e2, info[3 * e + 2]);
        /* J_i^T a and J_j^T a */
        const crm_dd gi0 = dd_sub(crm_dd_mul(s, a1), crm_dd_mul(c, a0));
        const crm_dd gi1 = dd_neg(crm_dd_add(crm_dd_mul(s, a0), crm_dd_mul(c, a1)));
        const crm_dd jt0 = dd_sub(crm_dd_mul(c, dy), crm_dd_mul(s, dx));        /* d e0 / d th_i */
        const crm_dd jt1 = dd_neg(crm_dd_add(crm_dd_mul(c, dx), crm_dd_mul(s, dy))); /* d e1 / d th_i */
        const crm_dd gi2 = dd_sub(dd_madd(crm_dd_mul(jt0, a0), jt1, a1), a2);
        const crm_dd gj0 = dd_sub(crm_dd_mul(c, a0), crm_dd_mul(s, a1));
        const crm_dd gj1 = crm_dd_add(crm_dd_mul(s, a0), crm_dd_mul(c, a1));
        const crm_dd g[6] = { gi0, gi1, gi2, gj0, gj1, a2 };
        const long at[6] = { 3 * i, 3 * i + 1, 3 * i + 2, 3 * j, 3 * j + 1, 3 * j + 2 };
        for (int q = 0; q < 6; q++) {
            const crm_dd v = dd_sub(dd(xi_hi[at[q]], xi_lo[at[q]]), g[q]);
            xi_hi[at[q]] = v.hi;
            xi_lo[at[q]] = v.lo;
        }
    }
    return 0;
}

/* (hi + lo) += d elementwise, renormalised. */
void or_dd_add_vec(long n, double *hi, double *lo, const double *d) {
    for (long q = 0; q < n; q++) {
        const crm_dd v = crm_dd_add(dd(hi[q], lo[q]), dd(d[q], 0.0));
        hi[q] = v.hi;
        lo[q] = v.lo;
    }
}

/* sum over poses of (x - tx)^2 + (y - ty)^2 at poses (p_hi + p_lo), in double-double;
 * returns the high part and stores the low part in *lo. */
double or_position_loss_dd(long n_poses, const double *p_hi, const double *p_lo, const double *target,
                           double *lo) {
    crm_dd acc = dd(0.0, 0.0);
    for (long i = 0; i < n_poses; i++)
        for (int k = 0; k < 2; k++) {
            const crm_dd d = crm_dd_add(dd(p_hi[3 * i + k], p_lo[3 * i + k]), dd(-target[3 * i + k], 0.0));
            acc = dd_madd(acc, d, d);
        }
    *lo = acc.lo;
    return acc.hi;
}

/* sin and cos of (x_hi + x_lo) as double-doubles (for the tests of this file). */
void or_sincos_dd(double x_hi, double x_lo, double *s_hi, double *s_lo, double *c_hi, double *c_lo) {
    crm_dd s, c;
    sincos_dd(dd(x_hi, x_lo), &s, &c);
    *s_hi = s.hi; *s_lo = s.lo; *c_hi = c.hi; *c_lo = c.lo;
}
