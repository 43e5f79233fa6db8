/*
 * pcg_mixed.cu — mixed-precision solve of Omega dx = xi: FP32 inner block-Jacobi
 * PCG inside an FP64 iterative-refinement loop, one cooperative launch.
 *
 * Precisions (the reference solves everything in FP64: MatrixOps.c:281-391):
 *   FP64: the outer residual r = xi - Omega x (FP64 matrix), the solution x, every
 *         global dot product (accumulated in FP64), the 3x3 block inverses D^-1
 *         (applied in FP64 and rounded to FP32).
 *   FP32: the inner SpMV (FP32 copy of Omega, staged in shared memory) and the
 *         inner vector updates.
 *
 * Inner iteration (Chronopoulos & Gear 1989, "s-step" CG with s = 1): with
 * s = A p and w = A z carried as recurrences, alpha and beta come from ONE fused
 * reduction of (r.z, w.z, r.r) per iteration instead of the two of standard PCG:
 *     x += alpha_{k-1} p_{k-1};  r_k = r_{k-1} - alpha_{k-1} s_{k-1};  z_k = D^-1 r_k
 *     w_k = A z_k;  gamma = r.z, delta = w.z, rho = r.r            -> grid reduction
 *     beta_k = gamma_k / gamma_{k-1};  alpha_k = gamma_k / (delta_k - beta_k gamma_k / alpha_{k-1})
 *     p_k = z_k + beta_k p_{k-1};  s_k = w_k + beta_k s_{k-1}
 * The SpMV needs z_k of neighbouring rows, which are only final after their own
 * r update; instead of a second grid barrier each row publishes r_k, w_k and
 * s_{k-1} before the reduction, and a neighbour's z_k is recomputed from those
 * (s_{k-1} = w_{k-1} + beta s_{k-2}, r_k = r_{k-1} - alpha s_{k-1}, z_k = D^-1 r_k)
 * with the same device function the owner uses, so it is bit-identical. Rows owned
 * by the same CTA read those values and D^-1 from shared memory; others from L2.
 *
 * Outer step: publish x (FP64), grid barrier, r = xi - Omega x with the FP64
 * matrix, ||r|| -> stop at tol * ||xi||, else restart the inner solve from r.
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "gslam.h"
#include "kernels.cuh"
#include "pcg_common.cuh"
#include "tma_bulk.cuh"

struct F3 { float a, b, c; };

__device__ __forceinline__ F3 ldcgf3(const float *v4, int row) {
    const float4 v = __ldcg(reinterpret_cast<const float4 *>(v4 + 4 * (size_t)row));
    return F3{ v.x, v.y, v.z };
}

__device__ __forceinline__ void stf3(float *v4, int row, F3 v) {
    *reinterpret_cast<float4 *>(v4 + 4 * (size_t)row) = make_float4(v.a, v.b, v.c, 0.f);
}

/* z = D^-1 r in FP64 (dinv rows at stride 32), rounded to FP32. */
__device__ __forceinline__ F3 dinv_apply_f(const double *d, F3 r) {
    const double r0 = r.a, r1 = r.b, r2 = r.c;
    double z0 = 0.0, z1 = 0.0, z2 = 0.0;
    z0 = z0 + d[0] * r0;   z0 = z0 + d[32] * r1;  z0 = z0 + d[64] * r2;
    z1 = z1 + d[96] * r0;  z1 = z1 + d[128] * r1; z1 = z1 + d[160] * r2;
    z2 = z2 + d[192] * r0; z2 = z2 + d[224] * r1; z2 = z2 + d[256] * r2;
    return F3{ (float)z0, (float)z1, (float)z2 };
}

/* The shared recurrence step: from (r_{k-1}, w_{k-1}, s_{k-2}) to (s_{k-1}, r_k). */
__device__ __forceinline__ void step_rs(F3 r_old, F3 w_old, F3 s_old2, float alpha, float beta,
                                        F3 &s_new, F3 &r_new) {
    s_new = F3{ __fmaf_rn(beta, s_old2.a, w_old.a), __fmaf_rn(beta, s_old2.b, w_old.b),
                __fmaf_rn(beta, s_old2.c, w_old.c) };
    r_new = F3{ __fmaf_rn(-alpha, s_new.a, r_old.a), __fmaf_rn(-alpha, s_new.b, r_old.b),
                __fmaf_rn(-alpha, s_new.c, r_old.c) };
}

__device__ __forceinline__ void blk_acc_f(const float *v, F3 p, float &q0, float &q1, float &q2) {
    q0 = __fmaf_rn(v[0], p.a, q0);   q0 = __fmaf_rn(v[32], p.b, q0);  q0 = __fmaf_rn(v[64], p.c, q0);
    q1 = __fmaf_rn(v[96], p.a, q1);  q1 = __fmaf_rn(v[128], p.b, q1); q1 = __fmaf_rn(v[160], p.c, q1);
    q2 = __fmaf_rn(v[192], p.a, q2); q2 = __fmaf_rn(v[224], p.b, q2); q2 = __fmaf_rn(v[256], p.c, q2);
}

/* halo record of one row in shared memory: r, w, s (FP32) */
struct Halo { float r[3], w[3], s[3]; };

template <int BS>
__global__ void __launch_bounds__(BS, 1) k_pcg_mixed(PcgParams P) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ double s_red[3][BS / 32];
    __shared__ double s_bc[4];
    __shared__ int s_ok;
    __shared__ __align__(8) uint64_t s_bar;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int epoch = 0;
    if ((int)blockIdx.x == P.absent_cta) return; /* test hook, see pcg.cu */

    const int s0 = __ldg(P.cta_slice + blockIdx.x), s1 = __ldg(P.cta_slice + blockIdx.x + 1);
    const int row0 = 32 * s0, row1 = 32 * s1;
    const int64_t slot0 = __ldg(P.slice_ptr + s0), slot1 = __ldg(P.slice_ptr + s1);
    const int64_t nval = 9 * (slot1 - slot0);
    const int64_t nsm = nval < P.smem_val_cap ? nval : P.smem_val_cap;
    /* dynamic shared memory: FP32 values | columns | D^-1 of own rows | halo of own rows */
    float *sval = reinterpret_cast<float *>(smem);
    int *scol = reinterpret_cast<int *>(smem + 4 * P.smem_val_cap);
    double *sdinv = reinterpret_cast<double *>(smem + P.smem_dinv_off);
    Halo *shalo = reinterpret_cast<Halo *>(smem + P.smem_halo_off);

    if (threadIdx.x == 0) {
        tma_mbar_init(&s_bar, 1);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned vbytes = (unsigned)(4 * nsm), cbytes = (unsigned)(4 * (slot1 - slot0));
        const unsigned dbytes = (unsigned)(2304 * (s1 - s0));
        tma_mbar_expect_tx(&s_bar, vbytes + cbytes + dbytes);
        if (vbytes) tma_bulk_g2s(sval, P.val32 + 9 * slot0, vbytes, &s_bar);
        if (cbytes) tma_bulk_g2s(scol, P.col + slot0, cbytes, &s_bar);
        if (dbytes) tma_bulk_g2s(sdinv, P.dinv + 288 * (size_t)s0, dbytes, &s_bar);
        int ok = tma_wait(&s_bar, 0, P.spin_limit);
        if (!ok) {
            atomicExch(&P.gs->abort, 1);
            tma_wait(&s_bar, 0, P.spin_limit);
        }
        s_ok = ok;
    }
    __syncthreads();
    if (!s_ok) {
        if (threadIdx.x == 0) { P.res->timeout = 1; P.res->reason = GSLAM_STOP_TIMEOUT; }
        return;
    }

    const int s = s0 + warp;
    const bool own_slice = s < s1;
    const int row = 32 * s + lane;
    const bool mine = own_slice && row < P.n_rows;
    const int len = mine ? __ldg(P.row_len + row) : 0;
    const int64_t lslot = own_slice ? (__ldg(P.slice_ptr + s) - slot0) : 0;
    const float *gval = P.val32 + 9 * slot0;
    const int *cb = scol + lslot + lane;
    const double *my_d = sdinv + 288 * (size_t)warp + lane; /* own row's D^-1 (stride 32) */
    Halo *my_h = shalo + (row - row0);

    /* published halo in global memory, double-buffered by iteration parity */
    /* (selected by parity with ?: so no local-memory array is needed) */
#define HALO_R(par) ((par) ? P.rf4 : P.xf4)
#define HALO_W(par) ((par) ? P.pfa4 : P.zf4)
#define HALO_S(par) ((par) ? P.qf4 : P.pfb4)

    /* ---- ||xi|| ---- */
    double bb[1] = { 0.0 };
    V3 b = { 0.0, 0.0, 0.0 };
    if (mine) {
        b = ldg3(P.b4, row);
        bb[0] = bb[0] + b.a * b.a; bb[0] = bb[0] + b.b * b.b; bb[0] = bb[0] + b.c * b.c;
    }
    if (!grid_allreduce<1, BS>(bb, P.partials, epoch, P.gs, P.spin_limit, s_red, s_bc, &s_ok)) {
        if (threadIdx.x == 0) { P.res->timeout = 1; P.res->reason = GSLAM_STOP_TIMEOUT; }
        return;
    }
    const double bnorm = sqrt(bb[0]);
    const double tol = P.tol_rel * bnorm;

    V3 x = { 0.0, 0.0, 0.0 };   /* FP64 solution */
    V3 r64 = b;                 /* FP64 residual, = b for x = 0 */
    double rnorm = bnorm;
    int total = 0, outer = 0, reason = GSLAM_STOP_MAXIT;
    bool timed_out = false;

    while (true) {
        if (rnorm < tol) { reason = GSLAM_STOP_TOL; break; }
        if (total >= P.max_iter || outer >= P.max_refine) { reason = GSLAM_STOP_MAXIT; break; }
        outer++;
        /* ---- inner FP32 solve of A d = r64, accumulated into x ---- */
        F3 r = { (float)r64.a, (float)r64.b, (float)r64.c };
        F3 z = { 0.f, 0.f, 0.f }, w = { 0.f, 0.f, 0.f }, sv = { 0.f, 0.f, 0.f }, p = { 0.f, 0.f, 0.f };
        /* state "k = -1": r_{-1} = r0, w_{-1} = 0, s_{-2} = 0, alpha = beta = 0 */
        if (mine) {
            const int par = 1; /* readers of iteration 0 use parity (0 - 1) & 1 = 1 */
            stf3(HALO_R(par), row, r);
            stf3(HALO_W(par), row, F3{ 0.f, 0.f, 0.f });
            stf3(HALO_S(par), row, F3{ 0.f, 0.f, 0.f });
            my_h->r[0] = r.a; my_h->r[1] = r.b; my_h->r[2] = r.c;
            my_h->w[0] = my_h->w[1] = my_h->w[2] = 0.f;
            my_h->s[0] = my_h->s[1] = my_h->s[2] = 0.f;
        }
        if (!grid_barrier(P.gs, (unsigned)(++epoch), P.spin_limit, &s_ok)) { timed_out = true; break; }
        float alpha = 0.f, beta = 0.f;
        double gamma_prev = 1.0, alpha_prev = 1.0, rho0 = -1.0;
        int k = 0;
        while (true) {
            const int pr = (k - 1) & 1, pw = k & 1;
            /* own recurrence, identical to what neighbours compute from the halo */
            F3 s_new, r_new;
            step_rs(r, w, sv, alpha, beta, s_new, r_new);
            /* x += alpha p_{k-1} (FP64), p_{k-1} = z_{k-1} + beta p_{k-2} */
            const F3 p_new = { __fmaf_rn(beta, p.a, z.a), __fmaf_rn(beta, p.b, z.b), __fmaf_rn(beta, p.c, z.c) };
            if (k > 0) {
                x.a = x.a + (double)alpha * (double)p_new.a;
                x.b = x.b + (double)alpha * (double)p_new.b;
                x.c = x.c + (double)alpha * (double)p_new.c;
            }
            p = p_new;
            sv = s_new;       /* s_{k-1} */
            r = r_new;        /* r_k */
            z = mine ? dinv_apply_f(my_d, r) : F3{ 0.f, 0.f, 0.f };
            /* w_k = A z_k */
            double part[3] = { 0.0, 0.0, 0.0 };
            if (mine) {
                float q0 = 0.f, q1 = 0.f, q2 = 0.f;
                for (int j = 0; j < len; j++) {
                    const int c = cb[32 * j];
                    F3 zc;
                    if (c == row) {
                        zc = z;
                    } else if (c >= row0 && c < row1) {
                        const Halo *h = shalo + (c - row0);
                        F3 sn, rn;
                        step_rs(F3{ h->r[0], h->r[1], h->r[2] }, F3{ h->w[0], h->w[1], h->w[2] },
                                F3{ h->s[0], h->s[1], h->s[2] }, alpha, beta, sn, rn);
                        const int cl = c - row0;
                        zc = dinv_apply_f(sdinv + 288 * (size_t)(cl >> 5) + (cl & 31), rn);
                    } else {
                        F3 sn, rn;
                        step_rs(ldcgf3(HALO_R(pr), c), ldcgf3(HALO_W(pr), c), ldcgf3(HALO_S(pr), c), alpha, beta,
                                sn, rn);
                        zc = dinv_apply_f(P.dinv + 288 * (size_t)(c >> 5) + (c & 31), rn);
                    }
                    const int64_t o = 9 * lslot + 288 * j;
                    blk_acc_f(o + 288 <= nsm ? sval + o + lane : gval + o + lane, zc, q0, q1, q2);
                }
                w = F3{ q0, q1, q2 };
                const double r0 = r.a, r1 = r.b, r2 = r.c, z0 = z.a, z1 = z.b, z2 = z.c;
                part[0] = r0 * z0 + r1 * z1 + r2 * z2;                            /* gamma */
                part[1] = (double)w.a * z0 + (double)w.b * z1 + (double)w.c * z2; /* delta */
                part[2] = r0 * r0 + r1 * r1 + r2 * r2;                            /* rho */
            }
            /* publish r_k, w_k, s_{k-1} for iteration k + 1 */
            __syncthreads(); /* every local read of the previous halo is done */
            if (mine) {
                stf3(HALO_R(pw), row, r);
                stf3(HALO_W(pw), row, w);
                stf3(HALO_S(pw), row, sv);
                my_h->r[0] = r.a; my_h->r[1] = r.b; my_h->r[2] = r.c;
                my_h->w[0] = w.a; my_h->w[1] = w.b; my_h->w[2] = w.c;
                my_h->s[0] = sv.a; my_h->s[1] = sv.b; my_h->s[2] = sv.c;
            }
            if (!grid_allreduce<3, BS>(part, P.partials, epoch, P.gs, P.spin_limit, s_red, s_bc, &s_ok)) {
                timed_out = true;
                break;
            }
            total++;
            k++;
            const double gamma = part[0], delta = part[1], rho = part[2];
            if (rho0 < 0.0) rho0 = rho;
            double a, bt;
            if (k == 1) { bt = 0.0; a = gamma / delta; }
            else { bt = gamma / gamma_prev; a = gamma / (delta - bt * gamma / alpha_prev); }
            if (!(delta != 0.0) || !(a == a)) { reason = GSLAM_STOP_PQ_ZERO; break; }
            gamma_prev = gamma;
            alpha_prev = a;
            alpha = (float)a;
            beta = (float)bt;
            const bool inner_done = rho <= P.inner_tol * P.inner_tol * rho0 || k >= P.inner_max_iter ||
                                    total >= P.max_iter || sqrt(rho) < tol;
            if (inner_done) {
                /* the last update: x += alpha_k p_k */
                const F3 pf = { __fmaf_rn(beta, p.a, z.a), __fmaf_rn(beta, p.b, z.b), __fmaf_rn(beta, p.c, z.c) };
                x.a = x.a + (double)alpha * (double)pf.a;
                x.b = x.b + (double)alpha * (double)pf.b;
                x.c = x.c + (double)alpha * (double)pf.c;
                break;
            }
        }
        if (timed_out) break;
        /* ---- outer FP64 residual r64 = b - A x ---- */
        if (mine) st3(P.x4, row, x);
        if (!grid_barrier(P.gs, (unsigned)(++epoch), P.spin_limit, &s_ok)) { timed_out = true; break; }
        double rr[1] = { 0.0 };
        if (mine) {
            const int64_t sb = __ldg(P.slice_ptr + s);
            const V3 ax = spmv_row(P.val + 9 * sb + lane, P.col + sb + lane, len, P.x4, P.x4, 0.0, true);
            r64 = V3{ b.a - ax.a, b.b - ax.b, b.c - ax.c };
            rr[0] = rr[0] + r64.a * r64.a; rr[0] = rr[0] + r64.b * r64.b; rr[0] = rr[0] + r64.c * r64.c;
        }
        if (!grid_allreduce<1, BS>(rr, P.partials, epoch, P.gs, P.spin_limit, s_red, s_bc, &s_ok)) {
            timed_out = true;
            break;
        }
        rnorm = sqrt(rr[0]);
        if (reason == GSLAM_STOP_PQ_ZERO) break;
    }
#undef HALO_R
#undef HALO_W
#undef HALO_S
    if (mine) st3(P.x4, row, x);
    if (timed_out && threadIdx.x == 0) {
        P.res->timeout = 1;
        P.res->reason = GSLAM_STOP_TIMEOUT;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && !timed_out) {
        P.res->iterations = total;
        P.res->reason = reason;
        P.res->refinements = outer;
        P.res->timeout = 0;
        P.res->rnorm = rnorm;
        P.res->bnorm = bnorm;
    }
}

template <int BS>
static cudaError_t set_attr_mixed() {
    return cudaFuncSetAttribute((const void *)k_pcg_mixed<BS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                GSLAM_RES_SMEM_MAX);
}

cudaError_t launch_pcg_mixed(cudaStream_t st, const PcgParams &p, int grid, int block, size_t smem_bytes) {
    if (block != 768 && block != 1024) return cudaErrorInvalidValue;
    PcgParams copy = p;
    void *args[] = { &copy };
    const void *fn = block == 768 ? (const void *)k_pcg_mixed<768> : (const void *)k_pcg_mixed<1024>;
    return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(block), args, smem_bytes, st);
}

int pcg_mixed_max_grid(int device, size_t smem_bytes) {
    int n_sm = 0, a = 0, b = 0;
    if (cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return 0;
    if (set_attr_mixed<768>() != cudaSuccess || set_attr_mixed<1024>() != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, (const void *)k_pcg_mixed<768>, 768, smem_bytes) !=
        cudaSuccess)
        return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, (const void *)k_pcg_mixed<1024>, 1024, smem_bytes) !=
        cudaSuccess)
        return 0;
    return std::min(a, b) * n_sm;
}
