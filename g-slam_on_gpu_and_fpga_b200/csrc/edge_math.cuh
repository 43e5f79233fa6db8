/*
 * edge_math.cuh — per-edge linearisation in the reference's operation order.
 *
 * Compiled with -fmad=false so every product and sum is rounded on its own,
 * exactly as the reference's C (x86-64, no FMA) does. Transcendentals come from
 * crmath.h (correctly rounded), and pow(x, 2.0) is x * x (correctly rounded).
 * With those two substitutions every edge block is bit-identical to the
 * reference's; the substitutions differ from glibc only where glibc misrounds.
 *
 * Reference: src/cpu_pcg_fp64/ObsEdge.c:10-212, MotionEdge.c:9-193,
 * GSLAM.c:373-401 (state_transition), MatrixOps.c:18-159 (tra, inv, dot).
 */
#ifndef GSLAM_EDGE_MATH_CUH
#define GSLAM_EDGE_MATH_CUH

#include "crmath.h"

#define EM_FN static __host__ __device__ __forceinline__

/* dot: res[ay x bx] = a[ay x ax] . b[ax x bx], each entry 0.0 + sum in index order. */
template <int AY, int AX, int BX>
EM_FN void em_dot(double *res, const double *a, const double *b) {
#pragma unroll
    for (int i = 0; i < AY * BX; i++) {
        const int row = i / BX, col = i % BX;
        double acc = 0.0;
#pragma unroll
        for (int j = 0; j < AX; j++) acc = acc + a[row * AX + j] * b[j * BX + col];
        res[i] = acc;
    }
}

/* tra: res[AX x AY] = transpose(m[AY x AX]) */
template <int AY, int AX>
EM_FN void em_tra(double *res, const double *m) {
#pragma unroll
    for (int r = 0; r < AX; r++)
#pragma unroll
        for (int c = 0; c < AY; c++) res[r * AY + c] = m[c * AX + r];
}

/* inv: Gauss-Jordan without pivoting; a zero pivot gives the zero matrix. */
template <int N>
EM_FN void em_inv(double *res, const double *m) {
    double t[N * N];
#pragma unroll
    for (int r = 0; r < N; r++)
#pragma unroll
        for (int c = 0; c < N; c++) {
            t[r * N + c] = m[r * N + c];
            res[r * N + c] = (r == c) ? 1.0 : 0.0;
        }
    bool zero = false;
#pragma unroll
    for (int i = 0; i < N; i++) {
        if (!zero && t[i * N + i] == 0.0) zero = true;
        if (!zero) {
#pragma unroll
            for (int j = 0; j < N; j++) {
                if (j == i) continue;
                const double ratio = t[j * N + i] / t[i * N + i];
#pragma unroll
                for (int k = 0; k < N; k++) {
                    t[j * N + k] = t[j * N + k] - ratio * t[i * N + k];
                    res[j * N + k] = res[j * N + k] - ratio * res[i * N + k];
                }
            }
        }
    }
    if (zero) {
#pragma unroll
        for (int k = 0; k < N * N; k++) res[k] = 0.0;
        return;
    }
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = 0; j < N; j++) res[i * N + j] = res[i * N + j] / t[i * N + i];
}

/*
 * ObsEdge (ObsEdge.c:10-212): poses x1, x2 (x, y, theta), observations z1, z2
 * (range, bearing). out[42] = UL, UR, BL, BR (row-major 3x3), xi_u[3], xi_b[3].
 * cost_out (may be null) receives hat_e^T Omega hat_e with the 2x2 Omega, times the
 * edge's lambda of 1.0: the GSLAM.c:74-87 cost term with the dimensions it meant.
 */
EM_FN void em_obs_edge(const double *x1, const double *x2, const double *z1, const double *z2,
                       double *out, double *cost_out = nullptr) {
    const double snr0 = 0.14, snr1 = 0.05;
    double s1, c1, s2, c2;
    cr_sincos(x1[2] + z1[1], &s1, &c1);
    cr_sincos(x2[2] + z2[1], &s2, &c2);
    double e[2];
    e[0] = x2[0] - x1[0] + z2[0] * c2 - z1[0] * c1;
    e[1] = x2[1] - x1[1] + z2[0] * s2 - z1[0] * s1;
    const double r1s = z1[0] * snr0, r2s = z2[0] * snr0;
    double Q1[4] = { r1s * r1s, 0.0, 0.0, snr1 * snr1 };
    double R1[4] = { -c1, z1[0] * s1, -s1, -z1[0] * c1 };
    double Q2[4] = { r2s * r2s, 0.0, 0.0, snr1 * snr1 };
    double R2[4] = { c2, -z2[0] * s2, s2, z2[0] * c2 };
    double tR1[4], R1Q1[4], S1[4], tR2[4], R2Q2[4], S2[4], Sig[4], Om[4];
    em_tra<2, 2>(tR1, R1);
    em_dot<2, 2, 2>(R1Q1, R1, Q1);
    em_dot<2, 2, 2>(S1, R1Q1, tR1);
    em_tra<2, 2>(tR2, R2);
    em_dot<2, 2, 2>(R2Q2, R2, Q2);
    em_dot<2, 2, 2>(S2, R2Q2, tR2);
#pragma unroll
    for (int i = 0; i < 4; i++) Sig[i] = S1[i] + S2[i];
    em_inv<2>(Om, Sig);
    if (cost_out) {
        double t[2], c;
        em_dot<1, 2, 2>(t, e, Om);
        em_dot<1, 2, 1>(&c, t, e);
        *cost_out = c * 1.0;
    }
    double B1[6] = { -1.0, -0.0, z1[0] * s1, -0.0, -1.0, -z1[0] * c1 };
    double B2[6] = { 1.0, 0.0, -z2[0] * s2, 0.0, 1.0, z2[0] * c2 };
    double tB1[6], tB2[6], tB1Om[6], tB2Om[6];
    em_tra<2, 3>(tB1, B1);
    em_tra<2, 3>(tB2, B2);
    em_dot<3, 2, 2>(tB1Om, tB1, Om);
    em_dot<3, 2, 2>(tB2Om, tB2, Om);
    em_dot<3, 2, 3>(out + 0, tB1Om, B1);
    em_dot<3, 2, 3>(out + 9, tB1Om, B2);
    em_dot<3, 2, 3>(out + 18, tB2Om, B1);
    em_dot<3, 2, 3>(out + 27, tB2Om, B2);
    double v[3];
    em_dot<3, 2, 1>(v, tB1Om, e);
#pragma unroll
    for (int i = 0; i < 3; i++) out[36 + i] = -v[i];
    em_dot<3, 2, 1>(v, tB2Om, e);
#pragma unroll
    for (int i = 0; i < 3; i++) out[39 + i] = -v[i];
}

/*
 * MotionEdge (MotionEdge.c:9-193) between consecutive poses with the control
 * (nu, omega) of the second step. Same 42-double output. cost_out (may be null)
 * receives lambda d^T Omega d with d = x2 - state_transition(x1), the motion term of
 * the cost (the reference stores hat_e = 0 for motion edges, MotionEdge.c:187-190).
 */
EM_FN void em_motion_edge(const double *x1, const double *x2, double nu, double omega,
                          double delta, double lambda, const double *mns, double *out,
                          double *cost_out = nullptr) {
    if (fabs(omega) < 1e-5) omega = 1e-5;
    const double M[4] = { mns[0] * mns[0] * fabs(nu) / delta + mns[1] * mns[1] * fabs(omega) / delta,
                          0.0, 0.0,
                          mns[2] * mns[2] * fabs(nu) / delta + mns[3] * mns[3] * fabs(omega) / delta };
    double st, ct, stw, ctw;
    cr_sincos(x1[2], &st, &ct);
    cr_sincos(x1[2] + omega * delta, &stw, &ctw);
    const double A[6] = {
        stw / omega - st / omega,
        nu / omega * delta * ctw - nu / omega / omega * stw + nu / omega / omega * st,
        ct / omega - ctw / omega,
        nu / omega * delta * stw - nu / omega / omega * ct + nu / omega / omega * ctw,
        0.0, delta };
    double F[9] = { 1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0 };
    F[2] = nu / omega * ctw - nu / omega * ct;
    F[5] = nu / omega * stw - nu / omega * st;
    double tA[6], AM[6], AMtA[9], Sg[9], Om[9];
    em_tra<3, 2>(tA, A);
    em_dot<3, 2, 2>(AM, A, M);
    em_dot<3, 2, 3>(AMtA, AM, tA);
#pragma unroll
    for (int i = 0; i < 9; i++) Sg[i] = AMtA[i] + ((i % 4 == 0) ? 1.0 : 0.0) * 0.0001;
    em_inv<3>(Om, Sg);
    double tF[9], tFOm[9], tFOmF[9], OmF[9];
    em_tra<3, 3>(tF, F);
    em_dot<3, 3, 3>(tFOm, tF, Om);
    em_dot<3, 3, 3>(tFOmF, tFOm, F);
#pragma unroll
    for (int i = 0; i < 9; i++) out[i] = tFOmF[i] * lambda;
#pragma unroll
    for (int i = 0; i < 9; i++) out[9 + i] = tFOm[i] * -lambda;
    em_dot<3, 3, 3>(OmF, Om, F);
#pragma unroll
    for (int i = 0; i < 9; i++) out[18 + i] = OmF[i] * -lambda;
#pragma unroll
    for (int i = 0; i < 9; i++) out[27 + i] = Om[i] * lambda;
    /* state_transition with the reference's unsigned-truncated time (GSLAM.h:13) */
    const double time = (double)(unsigned int)delta;
    double xp[3];
    if (fabs(omega) < 1e-10) {
        double s0, c0;
        cr_sincos(x1[2], &s0, &c0);
        const double v[3] = { nu * c0, nu * s0, omega };
#pragma unroll
        for (int i = 0; i < 3; i++) xp[i] = x1[i] + v[i] * time;
    } else {
        double sw = stw, cw = ctw;
        if (time != delta) cr_sincos(x1[2] + omega * time, &sw, &cw);
        const double v[3] = { nu / omega * sw - nu / omega * st, nu / omega * ct - nu / omega * cw,
                              omega * time };
#pragma unroll
        for (int i = 0; i < 3; i++) xp[i] = x1[i] + v[i];
    }
    double d[3], v[3];
#pragma unroll
    for (int i = 0; i < 3; i++) d[i] = x2[i] - xp[i];
    if (cost_out) {
        double t[3], c;
        em_dot<1, 3, 3>(t, d, Om);
        em_dot<1, 3, 1>(&c, t, d);
        *cost_out = c * lambda;
    }
    em_dot<3, 3, 1>(v, tFOm, d);
#pragma unroll
    for (int i = 0; i < 3; i++) out[36 + i] = v[i] * lambda;
    em_dot<3, 3, 1>(v, Om, d);
#pragma unroll
    for (int i = 0; i < 3; i++) out[39 + i] = v[i] * -lambda;
}

/* Angle wrap to (-pi, pi]: exact fmod-based reduction (fmod is exact in IEEE). */
EM_FN double em_wrap_angle(double t) {
    const double pi = 3.141592653589793, two_pi = 6.283185307179586;
    if (t > pi || t <= -pi) {
        t = fmod(t + pi, two_pi);
        if (t < 0.0) t = t + two_pi;
        t = t - pi;
    }
    return t;
}

/*
 * SE(2) between-factor: e = [R(th_i)^T (t_j - t_i) - z_t ; wrap(th_j - th_i - z_th)],
 * Lambda = diag(info) * lambda. Blocks UL = Ji^T L Ji, UR = Ji^T L Jj, BL = Jj^T L Ji,
 * BR = Jj^T L Jj, xi_u = -Ji^T L e, xi_b = -Jj^T L e (the reference's Omega dx = xi
 * convention). Sums run k = 0, 1, 2 from 0.0 with separate multiply and add.
 */
EM_FN void em_se2_edge(const double *xi, const double *xj, const double *z, const double *info,
                       double lambda, double *out) {
    double s, c;
    cr_sincos(xi[2], &s, &c);
    const double dx = xj[0] - xi[0], dy = xj[1] - xi[1];
    double e[3];
    e[0] = (c * dx + s * dy) - z[0];
    e[1] = (c * dy - s * dx) - z[1];
    e[2] = em_wrap_angle((xj[2] - xi[2]) - z[2]);
    const double Ji[9] = { -c, -s, c * dy - s * dx, s, -c, -(c * dx) - s * dy, 0.0, 0.0, -1.0 };
    const double Jj[9] = { c, s, 0.0, -s, c, 0.0, 0.0, 0.0, 1.0 };
    double L[3], LJi[9], LJj[9], Le[3];
#pragma unroll
    for (int k = 0; k < 3; k++) L[k] = info[k] * lambda;
#pragma unroll
    for (int k = 0; k < 3; k++) {
#pragma unroll
        for (int cc = 0; cc < 3; cc++) {
            LJi[3 * k + cc] = L[k] * Ji[3 * k + cc];
            LJj[3 * k + cc] = L[k] * Jj[3 * k + cc];
        }
        Le[k] = L[k] * e[k];
    }
#pragma unroll
    for (int r = 0; r < 3; r++) {
#pragma unroll
        for (int cc = 0; cc < 3; cc++) {
            double ul = 0.0, ur = 0.0, bl = 0.0, br = 0.0;
#pragma unroll
            for (int k = 0; k < 3; k++) {
                ul = ul + Ji[3 * k + r] * LJi[3 * k + cc];
                ur = ur + Ji[3 * k + r] * LJj[3 * k + cc];
                bl = bl + Jj[3 * k + r] * LJi[3 * k + cc];
                br = br + Jj[3 * k + r] * LJj[3 * k + cc];
            }
            out[3 * r + cc] = ul;
            out[9 + 3 * r + cc] = ur;
            out[18 + 3 * r + cc] = bl;
            out[27 + 3 * r + cc] = br;
        }
        double xu = 0.0, xb = 0.0;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            xu = xu + Ji[3 * k + r] * Le[k];
            xb = xb + Jj[3 * k + r] * Le[k];
        }
        out[36 + r] = -xu;
        out[39 + r] = -xb;
    }
}

#endif
