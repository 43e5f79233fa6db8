/*
 * pcg_mixed.cu — mixed-precision solve of Omega dx = xi: FP32 inner block-Jacobi
 * PCG inside an FP64 iterative-refinement loop, one cooperative launch.
 *
 * Precisions (the reference solves everything in FP64: MatrixOps.c:281-391):
 *   FP64: the outer residual r = xi - Omega x (FP64 matrix), the solution x, every
 *         global dot product (accumulated in FP64), the 3x3 block inverses D^-1
 *         (stored and applied in FP64, the product rounded to FP32).
 *   FP32: the inner SpMV (FP32 copy of Omega, staged in shared memory), the inner
 *         vector updates and the inner correction d (x += d in FP64 after each
 *         inner solve).
 *
 * Inner iteration (Chronopoulos & Gear 1989, "s-step" CG with s = 1, in the
 * preconditioned form that also carries M^-1 of the recurrence vectors): with
 * s = A p, w = A z, u = M^-1 w and v = M^-1 s, alpha and beta come from ONE
 * fused reduction of (r.z, w.z, r.r) per iteration instead of the two of
 * standard PCG (M = the block diagonal, M^-1 = D^-1):
 *     s_{k-1} = w_{k-1} + beta s_{k-2};   v_{k-1} = u_{k-1} + beta v_{k-2}
 *     r_k = r_{k-1} - alpha s_{k-1};      z_k = z_{k-1} - alpha v_{k-1}
 *     p_{k-1} = z_{k-1} + beta p_{k-2};   d += alpha p_{k-1}
 *     w_k = A z_k;  u_k = D^-1 w_k;  gamma = r.z, delta = w.z, rho = r.r  -> reduction
 *     beta_k = gamma_k / gamma_{k-1};  alpha_k = gamma_k / (delta_k - beta_k gamma_k / alpha_{k-1})
 * (alpha, beta = those of the previous reduction). The SpMV needs z_k of rows
 * other CTAs own, which is only final after the reduction; instead of a second
 * grid barrier every row publishes (z_k, u_k, v_{k-1}) before the reduction and
 * a reader forms v_k and z_{k+1} from them with the same two FP32 FMAs per
 * component the owner uses, so the copies are bit-identical and no reader needs
 * the owner's D^-1.
 *
 * Shared memory holds, per CTA: its FP32 matrix share, CTA-local column indices
 * (own rows first, then the CTA's halo: the other CTAs' rows its blocks touch, a
 * list fixed at setup), its own rows' D^-1, and z of its own and halo rows. Each
 * thread owns one row and keeps r, z, s, v, w, u, p, d in registers; every thread
 * also advances z of (at least) one halo row per iteration. The halo's published
 * values are loaded right after the grid barrier, while warps 0-2 sum the
 * reduction partials, so the two L2 round trips overlap; thread 0 alone then
 * advances the scalar recurrence. The SpMV reads values, columns and z from
 * shared memory only.
 *
 * Outer step: x += d (FP64), grid barrier, r = xi - Omega x with the FP64 matrix,
 * ||r|| -> stop at tol * ||xi||, else restart the inner solve from r; a step that
 * does not halve ||r|| ends the solve with GSLAM_STOP_STAGNATION (the host then
 * solves in FP64).
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

__device__ __forceinline__ F3 ldf3(const float *v4, int row) {
    const float4 v = *reinterpret_cast<const float4 *>(v4 + 4 * (size_t)row);
    return F3{ v.x, v.y, v.z };
}

/* 16-byte asynchronous global -> shared copy through L2 (no registers), and its wait */
__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gsrc) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gsrc) : "memory");
}

__device__ __forceinline__ void cp_async_commit_wait_later() { asm volatile("cp.async.commit_group;" ::: "memory"); }

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

__device__ __forceinline__ void stf3(float *v4, int row, F3 v) {
    *reinterpret_cast<float4 *>(v4 + 4 * (size_t)row) = make_float4(v.a, v.b, v.c, 0.f);
}

/* y = D^-1 x in FP64 (the 9 entries of D^-1 at stride 32 doubles), rounded to FP32. */
__device__ __forceinline__ F3 dinv_apply_f(const double *d, F3 x) {
    const double x0 = x.a, x1 = x.b, x2 = x.c;
    double y0 = 0.0, y1 = 0.0, y2 = 0.0;
    y0 = y0 + d[0] * x0;   y0 = y0 + d[32] * x1;  y0 = y0 + d[64] * x2;
    y1 = y1 + d[96] * x0;  y1 = y1 + d[128] * x1; y1 = y1 + d[160] * x2;
    y2 = y2 + d[192] * x0; y2 = y2 + d[224] * x1; y2 = y2 + d[256] * x2;
    return F3{ (float)y0, (float)y1, (float)y2 };
}

/* a * x + y, one FP32 FMA per component: every inner vector update */
__device__ __forceinline__ F3 axpy_f(float a, F3 x, F3 y) {
    return F3{ __fmaf_rn(a, x.a, y.a), __fmaf_rn(a, x.b, y.b), __fmaf_rn(a, x.c, y.c) };
}

/* v = u + beta v_old; z = z_old - alpha v: the step every copy of a row's z takes */
__device__ __forceinline__ void step_zv(F3 z_old, F3 u, F3 v_old, float alpha, float beta, F3 &z_new,
                                        F3 &v_new) {
    v_new = axpy_f(beta, v_old, u);
    z_new = axpy_f(-alpha, v_new, z_old);
}

__device__ __forceinline__ void blk_acc_f(const float *v, F3 p, float &q0, float &q1, float &q2) {
    q0 = __fmaf_rn(v[0], p.a, q0);   q0 = __fmaf_rn(v[32], p.b, q0);  q0 = __fmaf_rn(v[64], p.c, q0);
    q1 = __fmaf_rn(v[96], p.a, q1);  q1 = __fmaf_rn(v[128], p.b, q1); q1 = __fmaf_rn(v[160], p.c, q1);
    q2 = __fmaf_rn(v[192], p.a, q2); q2 = __fmaf_rn(v[224], p.b, q2); q2 = __fmaf_rn(v[256], p.c, q2);
}

template <int BS>
__global__ void __launch_bounds__(BS, 1) k_pcg_mixed(PcgParams P) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ double s_red[3][BS / 32];
    __shared__ double s_bc[4];
    __shared__ int s_ok;
    __shared__ __align__(8) uint64_t s_bar;
    /* scalar recurrence, kept and advanced by thread 0 only (no registers in the
     * other threads): gamma_{k-1}, alpha_{k-1}, rho_0 of the inner solve, tol, ||xi|| */
    __shared__ double s_sc[5];
    __shared__ float s_ab[2];  /* alpha, beta for the next iteration */
    __shared__ int s_flag;     /* 0 continue, 1 inner solve done, 2 breakdown */
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int epoch = 0;
    if ((int)blockIdx.x == P.absent_cta) return; /* test hook, see pcg.cu */

    const int s0 = __ldg(P.cta_slice + blockIdx.x), s1 = __ldg(P.cta_slice + blockIdx.x + 1);
    const int row0 = 32 * s0, n_loc = 32 * (s1 - s0);
    const int64_t slot0 = __ldg(P.slice_ptr + s0), slot1 = __ldg(P.slice_ptr + s1);
    const int64_t nval = 9 * (slot1 - slot0);
    const int64_t nsm = nval < P.smem_val_cap ? nval : P.smem_val_cap;
    const int h0 = __ldg(P.halo_ptr + blockIdx.x), h1 = __ldg(P.halo_ptr + blockIdx.x + 1);
    /* dynamic shared memory: FP32 values | local columns | D^-1 of own rows | z of own + halo rows */
    float *sval = reinterpret_cast<float *>(smem);
    int *scol = reinterpret_cast<int *>(smem + 4 * P.smem_val_cap);
    double *sdinv = reinterpret_cast<double *>(smem + P.smem_dinv_off);
    float *sz = reinterpret_cast<float *>(smem + P.smem_halo_off);
    float *sstage = reinterpret_cast<float *>(smem + P.smem_stage_off); /* halo u, v: 2 float4 per row */

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
        if (cbytes) tma_bulk_g2s(scol, P.lcol + slot0, cbytes, &s_bar);
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
        if (threadIdx.x == 0) res_mark_timeout(P.res);
        return;
    }

    const int s = s0 + warp;
    const bool own_slice = s < s1;
    const int row = 32 * s + lane;
    const bool mine = own_slice && row < P.n_rows;
    const int len = mine ? __ldg(P.row_len + row) : 0;
    /* 32-bit offsets into this CTA's share: local slot of (j = 0), and how many of the
     * row's blocks have their values in shared memory (the rest are read from L2) */
    const int lslot = own_slice ? (int)(__ldg(P.slice_ptr + s) - slot0) : 0;
    const int j_sm = min(len, max(0, ((int)nsm - 9 * lslot) / 288));
    /* the halo row this thread advances every iteration (more, in a loop, only when
     * the halo has more rows than the CTA has threads) */
    const bool has_h = (int)threadIdx.x < h1 - h0;
    const int hrow = has_h ? __ldg(P.halo_rows + h0 + threadIdx.x) : 0;
    const bool h_extra = h1 - h0 > BS;  /* CTA-uniform */

    /* published (z_k, u_k, v_{k-1}) in global memory, double-buffered by iteration
     * parity (selected with ?: so no local-memory array is needed) */
#define PUB_Z(par) ((par) ? P.rf4 : P.xf4)
#define PUB_U(par) ((par) ? P.pfa4 : P.zf4)
#define PUB_V(par) ((par) ? P.qf4 : P.pfb4)

    /* ---- ||xi|| ---- */
    double bb[1] = { 0.0 };
    if (mine) {
        const V3 b = ldg3(P.b4, row);
        bb[0] = bb[0] + b.a * b.a; bb[0] = bb[0] + b.b * b.b; bb[0] = bb[0] + b.c * b.c;
    }
    if (!grid_allreduce<1, BS>(bb, P.partials, epoch, P.gs, P.spin_limit, s_red, s_bc, &s_ok)) {
        if (threadIdx.x == 0) res_mark_timeout(P.res);
        return;
    }
    if (threadIdx.x == 0) {
        const double tol = P.tol_rel * sqrt(bb[0]);
        s_sc[3] = tol * tol;     /* compared with rho = r.r, so no square root per iteration */
        s_sc[4] = sqrt(bb[0]);
    }

    V3 x = { 0.0, 0.0, 0.0 };   /* FP64 solution (P.x4 holds it during an inner solve) */
    V3 r64 = mine ? ldg3(P.b4, row) : V3{ 0.0, 0.0, 0.0 }; /* FP64 residual, = xi for x = 0 */
    double rnorm = sqrt(bb[0]);
    int total = 0, outer = 0, reason = GSLAM_STOP_MAXIT;
    bool timed_out = false;

    while (true) {
        if (rnorm < P.tol_rel * s_sc[4]) { reason = GSLAM_STOP_TOL; break; }
        if (total >= P.max_iter || outer >= P.max_refine) { reason = GSLAM_STOP_MAXIT; break; }
        outer++;
        /* ---- inner FP32 solve of A d = r64; x += d in FP64 afterwards ---- */
        if (mine) st3(P.x4, row, x);  /* x is not held in registers during the inner solve */
        F3 r = { (float)r64.a, (float)r64.b, (float)r64.c };
        const F3 zero = { 0.f, 0.f, 0.f };
        /* state "k = -1": z_{-1} = D^-1 r_0, and w, u, s, v, p of earlier steps 0, so
         * with alpha = beta = 0 the first step leaves r and z unchanged; readers of
         * iteration 0 use parity (0 - 1) & 1 = 1 */
        F3 z = mine ? dinv_apply_f(sdinv + 288 * warp + lane, r) : zero;
        F3 w = zero, u = zero, sv = zero, v = zero, p = zero, d = zero;
        if (mine) {
            stf3(PUB_Z(1), row, z);
            stf3(PUB_U(1), row, zero);
            stf3(PUB_V(1), row, zero);
        }
        if (!grid_barrier(P.gs, (unsigned)(++epoch), P.spin_limit, &s_ok)) { timed_out = true; break; }
        /* the halo's published (z, u, v) go straight into shared memory (no registers held
         * across the reduction): z into the halo row's z slot, u and v into staging */
        if (has_h) {
            cp_async16(sz + 4 * (n_loc + threadIdx.x), PUB_Z(1) + 4 * (size_t)hrow);
            cp_async16(sstage + 8 * threadIdx.x, PUB_U(1) + 4 * (size_t)hrow);
            cp_async16(sstage + 8 * threadIdx.x + 4, PUB_V(1) + 4 * (size_t)hrow);
            cp_async_commit_wait_later();
        }
        float alpha = 0.f, beta = 0.f;
        int k = 0;
        while (true) {
            const int pr = (k - 1) & 1, pw = k & 1;
            /* z_k of the halo rows (first: frees the prefetched registers) */
            if (has_h) {
                cp_async_wait_all();
                F3 zn, vn;
                step_zv(ldf3(sz, n_loc + threadIdx.x), ldf3(sstage, 2 * threadIdx.x), ldf3(sstage, 2 * threadIdx.x + 1),
                        alpha, beta, zn, vn);
                stf3(sz, n_loc + (int)threadIdx.x, zn);
            }
            if (h_extra) {
                /* halo rows beyond the CTA's thread count (bounds re-read: rare path) */
                const int e0 = __ldg(P.halo_ptr + blockIdx.x), e1 = __ldg(P.halo_ptr + blockIdx.x + 1);
                for (int h = e0 + (int)threadIdx.x + BS; h < e1; h += BS) {
                    const int c = __ldg(P.halo_rows + h);
                    F3 zn, vn;
                    step_zv(ldcgf3(PUB_Z(pr), c), ldcgf3(PUB_U(pr), c), ldcgf3(PUB_V(pr), c), alpha, beta, zn, vn);
                    stf3(sz, n_loc + (h - e0), zn);
                }
            }
            /* own row: s_{k-1}, r_k, p_{k-1}, d, then v_{k-1}, z_k */
            sv = axpy_f(beta, sv, w);
            r = axpy_f(-alpha, sv, r);
            p = axpy_f(beta, p, z);
            if (k > 0) d = axpy_f(alpha, p, d);
            step_zv(z, u, v, alpha, beta, z, v);
            if (mine) {
                stf3(sz, row - row0, z);
                /* z_k and v_{k-1} are final here: publish them now, so only u_k's stores
                 * are still in flight when the CTA arrives at the barrier */
                stf3(PUB_Z(pw), row, z);
                stf3(PUB_V(pw), row, v);
            }
            __syncthreads();
            /* w_k = A z_k from shared memory, u_k = D^-1 w_k */
            double part[3] = { 0.0, 0.0, 0.0 };
            float q0 = 0.f, q1 = 0.f, q2 = 0.f;
            if (mine) {
                const int *cb = scol + lslot + lane;
                const int jend = len;
                const int jsm = j_sm;
                int j = 0;
                /* four blocks at a time: their column and z loads are in flight together
                 * (a row's blocks are still added in ascending column order) */
                const float *sv0 = sval + 9 * lslot + lane;
                /* the diagonal block's z is this thread's own (no shared-memory load) */
                const int lrow = row - row0;
                for (; j + 3 < jsm; j += 4) {
                    const int c0 = cb[32 * j], c1 = cb[32 * (j + 1)], c2 = cb[32 * (j + 2)], c3 = cb[32 * (j + 3)];
                    const F3 z0 = c0 == lrow ? z : ldf3(sz, c0), z1 = c1 == lrow ? z : ldf3(sz, c1);
                    const F3 z2 = c2 == lrow ? z : ldf3(sz, c2), z3 = c3 == lrow ? z : ldf3(sz, c3);
                    blk_acc_f(sv0 + 288 * j, z0, q0, q1, q2);
                    blk_acc_f(sv0 + 288 * (j + 1), z1, q0, q1, q2);
                    blk_acc_f(sv0 + 288 * (j + 2), z2, q0, q1, q2);
                    blk_acc_f(sv0 + 288 * (j + 3), z3, q0, q1, q2);
                }
                for (; j < jsm; j++) {
                    const int c0 = cb[32 * j];
                    blk_acc_f(sv0 + 288 * j, c0 == lrow ? z : ldf3(sz, c0), q0, q1, q2);
                }
                if (j < jend) {
                    /* blocks beyond the shared-memory share: values from L2 */
                    const float *gv = P.val32 + 9 * __ldg(P.slice_ptr + s) + lane;
                    for (; j < jend; j++) blk_acc_f(gv + 288 * j, ldf3(sz, cb[32 * j]), q0, q1, q2);
                }
            }
            if (mine) {
                w = F3{ q0, q1, q2 };
                u = dinv_apply_f(sdinv + 288 * warp + lane, w); /* own row's D^-1 (stride 32) */
                const double r0 = r.a, r1 = r.b, r2 = r.c, z0 = z.a, z1 = z.b, z2 = z.c;
                part[0] = r0 * z0 + r1 * z1 + r2 * z2;                            /* gamma */
                part[1] = (double)w.a * z0 + (double)w.b * z1 + (double)w.c * z2; /* delta */
                part[2] = r0 * r0 + r1 * r1 + r2 * r2;                            /* rho */
                /* publish u_k for iteration k + 1 (z_k and v_{k-1} went out before the SpMV) */
                stf3(PUB_U(pw), row, u);
            }
            if (!grid_reduce_arrive<3, BS>(part, P.partials, epoch, P.gs, P.spin_limit, s_red, &s_ok)) {
                timed_out = true;
                break;
            }
            /* the halo's values for iteration k + 1, in flight while the partials are summed
             * (every read of the halo z slots in this iteration's SpMV precedes the barrier) */
            if (has_h) {
                cp_async16(sz + 4 * (n_loc + threadIdx.x), PUB_Z(pw) + 4 * (size_t)hrow);
                cp_async16(sstage + 8 * threadIdx.x, PUB_U(pw) + 4 * (size_t)hrow);
                cp_async16(sstage + 8 * threadIdx.x + 4, PUB_V(pw) + 4 * (size_t)hrow);
                cp_async_commit_wait_later();
            }
            grid_reduce_sum<3>(P.partials, epoch, s_bc);
            total++;
            k++;
            if (threadIdx.x == 0) {
                /* alpha_k = gamma / (delta - beta_k gamma / alpha_{k-1}) = gamma g / (delta g - gamma^2)
                 * with g = gamma_{k-1} alpha_{k-1}: one FP64 division on the critical path (beta's
                 * runs beside it); both rounded to FP32 for the vector updates */
                const double gamma = s_bc[0], delta = s_bc[1], rho = s_bc[2];
                if (k == 1) s_sc[2] = rho;
                double a, bt;
                if (k == 1) { bt = 0.0; a = gamma / delta; }
                else {
                    const double g = s_sc[0] * s_sc[1];
                    bt = gamma / s_sc[0];
                    a = (gamma * g) / (delta * g - gamma * gamma);
                }
                int flag = 0;
                if (!(delta != 0.0) || !(a == a) || isinf(a)) flag = 2;
                else if (rho <= P.inner_tol * P.inner_tol * s_sc[2] || k >= P.inner_max_iter ||
                         total >= P.max_iter || rho < s_sc[3])
                    flag = 1;
                s_sc[0] = gamma;
                s_sc[1] = a;
                s_ab[0] = (float)a;
                s_ab[1] = (float)bt;
                s_flag = flag;
            }
            __syncthreads();
            const int flag = s_flag;
            if (flag == 2) { reason = GSLAM_STOP_PQ_ZERO; break; }
            alpha = s_ab[0];
            beta = s_ab[1];
            if (flag == 1) {
                /* the last update: d += alpha_k p_k, p_k = z_k + beta_k p_{k-1} */
                p = axpy_f(beta, p, z);
                d = axpy_f(alpha, p, d);
                break;
            }
        }
        if (timed_out) break;
        /* ---- x += d in FP64, then the outer FP64 residual r64 = xi - A x ---- */
        if (mine) {
            x = ld3(P.x4, row);
            x = V3{ x.a + (double)d.a, x.b + (double)d.b, x.c + (double)d.c };
            st3(P.x4, row, x);
        }
        if (!grid_barrier(P.gs, (unsigned)(++epoch), P.spin_limit, &s_ok)) { timed_out = true; break; }
        double rr[1] = { 0.0 };
        if (mine) {
            const int64_t sb = __ldg(P.slice_ptr + s);
            const V3 ax = spmv_row(P.val + 9 * sb + lane, P.col + sb + lane, len, P.x4, P.x4, 0.0, true);
            const V3 b = ldg3(P.b4, row);
            r64 = V3{ b.a - ax.a, b.b - ax.b, b.c - ax.c };
            rr[0] = rr[0] + r64.a * r64.a; rr[0] = rr[0] + r64.b * r64.b; rr[0] = rr[0] + r64.c * r64.c;
        }
        if (!grid_allreduce<1, BS>(rr, P.partials, epoch, P.gs, P.spin_limit, s_red, s_bc, &s_ok)) {
            timed_out = true;
            break;
        }
        const double rnorm_prev = rnorm;
        rnorm = sqrt(rr[0]);
        if (reason == GSLAM_STOP_PQ_ZERO) break;
        /* iterative refinement must shrink the true residual; when a step gains less than a
         * factor 2 the FP32 inner solve cannot resolve this system (cond x eps32 >> 1) */
        if (rnorm >= P.tol_rel * s_sc[4] && total < P.max_iter && outer < P.max_refine &&
            rnorm > 0.5 * rnorm_prev) {
            reason = GSLAM_STOP_STAGNATION;
            break;
        }
    }
#undef PUB_Z
#undef PUB_U
#undef PUB_V
    /* P.x4 already holds x: stored at the start of every refinement step and after it */
    if (timed_out && threadIdx.x == 0) {
        res_mark_timeout(P.res);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && !timed_out) {
        res_finish(P.res, P.gs, total, reason, outer, rnorm, s_sc[4]);
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
