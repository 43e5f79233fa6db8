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
 *
 * The same kernel with T = double is the FP64 one-reduction solver (GSLAM_PREC_FP64_CG):
 * one inner solve in FP64 (FP64 values staged in shared memory as far as they fit, the
 * rest read from L2; D^-1 read from global memory, where it stays in L2) to the outer
 * tolerance and iteration cap, no refinement. It stops on the recurrence residual, as the
 * reference's loop does (MatrixOps.c:345-347), and reports the true residual; its
 * iterates are the reference's PCG in exact arithmetic, with other rounding (20
 * Gauss-Newton rounds of a 100k-pose graph at 1e-6 / 500: 9.5e-10 from the reference
 * recurrence's poses, as close as a different summation order of that recurrence, 9.7e-10).
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "gslam.h"
#include "kernels.cuh"
#include "pcg_common.cuh"
#include "tma_bulk.cuh"

/* a row's three components in the inner precision T; rows are padded to 4 elements
 * (16 B in FP32, 32 B in FP64) */
template <typename T> struct T3 { T a, b, c; };

__device__ __forceinline__ T3<float> ldt3(const float *v4, int row) {
    const float4 v = *reinterpret_cast<const float4 *>(v4 + 4 * (size_t)row);
    return { v.x, v.y, v.z };
}
__device__ __forceinline__ T3<double> ldt3(const double *v4, int row) {
    const V3 v = ld3(v4, row);
    return { v.a, v.b, v.c };
}
__device__ __forceinline__ T3<float> ldcgt3(const float *v4, int row) {
    const float4 v = __ldcg(reinterpret_cast<const float4 *>(v4 + 4 * (size_t)row));
    return { v.x, v.y, v.z };
}
__device__ __forceinline__ T3<double> ldcgt3(const double *v4, int row) {
    const V3 v = ldcg3(v4, row);
    return { v.a, v.b, v.c };
}
__device__ __forceinline__ void stt3(float *v4, int row, T3<float> v) {
    *reinterpret_cast<float4 *>(v4 + 4 * (size_t)row) = make_float4(v.a, v.b, v.c, 0.f);
}
__device__ __forceinline__ void stt3(double *v4, int row, T3<double> v) { st3(v4, row, V3{ v.a, v.b, v.c }); }

/* 16-byte asynchronous global -> shared copy through L2 (no registers), and its wait */
__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gsrc) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gsrc) : "memory");
}

__device__ __forceinline__ void cp_async_commit_wait_later() { asm volatile("cp.async.commit_group;" ::: "memory"); }

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

/* one padded row of T (4 elements) global -> shared, asynchronously */
template <typename T>
__device__ __forceinline__ void cp_async_row(T *smem_dst, const T *gsrc) {
#pragma unroll
    for (int c = 0; c < (int)(4 * sizeof(T)) / 16; c++) cp_async16(smem_dst + c * (16 / sizeof(T)), gsrc + c * (16 / sizeof(T)));
}

/* a * b + c in one rounding */
__device__ __forceinline__ float fma_t(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_t(double a, double b, double c) { return __fma_rn(a, b, c); }

/* y = D^-1 x in FP64 (the 9 entries of D^-1 at stride 32 doubles), rounded to T. */
template <typename T>
__device__ __forceinline__ T3<T> dinv_apply_t(const double *d, T3<T> x) {
    const double x0 = x.a, x1 = x.b, x2 = x.c;
    double y0 = 0.0, y1 = 0.0, y2 = 0.0;
    y0 = y0 + d[0] * x0;   y0 = y0 + d[32] * x1;  y0 = y0 + d[64] * x2;
    y1 = y1 + d[96] * x0;  y1 = y1 + d[128] * x1; y1 = y1 + d[160] * x2;
    y2 = y2 + d[192] * x0; y2 = y2 + d[224] * x1; y2 = y2 + d[256] * x2;
    return T3<T>{ (T)y0, (T)y1, (T)y2 };
}

/* a * x + y, one FMA per component: every inner vector update */
template <typename T>
__device__ __forceinline__ T3<T> axpy_t(T a, T3<T> x, T3<T> y) {
    return T3<T>{ fma_t(a, x.a, y.a), fma_t(a, x.b, y.b), fma_t(a, x.c, y.c) };
}

/* v = u + beta v_old; z = z_old - alpha v: the step every copy of a row's z takes */
template <typename T>
__device__ __forceinline__ void step_zv(T3<T> z_old, T3<T> u, T3<T> v_old, T alpha, T beta, T3<T> &z_new,
                                        T3<T> &v_new) {
    v_new = axpy_t(beta, v_old, u);
    z_new = axpy_t(-alpha, v_new, z_old);
}

template <typename T>
__device__ __forceinline__ void blk_acc_t(const T *v, T3<T> p, T &q0, T &q1, T &q2) {
    q0 = fma_t(v[0], p.a, q0);   q0 = fma_t(v[32], p.b, q0);  q0 = fma_t(v[64], p.c, q0);
    q1 = fma_t(v[96], p.a, q1);  q1 = fma_t(v[128], p.b, q1); q1 = fma_t(v[160], p.c, q1);
    q2 = fma_t(v[192], p.a, q2); q2 = fma_t(v[224], p.b, q2); q2 = fma_t(v[256], p.c, q2);
}

/* the inner solve's buffers for T: the matrix copy and the published (z, u, v) of both
 * iteration parities. FP32: the FP32 copy and six FP32 vectors. FP64: the FP64 matrix and
 * six FP64 vectors (r4 .. q4 and w4; x4 holds the solution). */
template <typename T> struct Inner;
template <> struct Inner<float> {
    static __device__ const float *val(const PcgParams &P) { return P.val32; }
    static __device__ float *pz(const PcgParams &P, int par) { return par ? P.rf4 : P.xf4; }
    static __device__ float *pu(const PcgParams &P, int par) { return par ? P.pfa4 : P.zf4; }
    static __device__ float *pv(const PcgParams &P, int par) { return par ? P.qf4 : P.pfb4; }
};
template <> struct Inner<double> {
    static __device__ const double *val(const PcgParams &P) { return P.val; }
    static __device__ double *pz(const PcgParams &P, int par) { return par ? P.r4 : P.z4; }
    static __device__ double *pu(const PcgParams &P, int par) { return par ? P.p4a : P.p4b; }
    static __device__ double *pv(const PcgParams &P, int par) { return par ? P.q4 : P.w4; }
};

/* T = float: the mixed solver; T = double: the FP64 one-reduction solver (one inner
 * solve, D^-1 from global memory) */
template <int BS, typename T>
__global__ void __launch_bounds__(BS, 1) k_pcg_mixed(PcgParams P) {
    constexpr bool F64 = sizeof(T) == 8;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ double s_red[3][BS / 32];
    __shared__ double s_bc[4];
    __shared__ int s_ok;
    __shared__ __align__(8) uint64_t s_bar;
    /* scalar recurrence, kept and advanced by thread 0 only (no registers in the
     * other threads): gamma_{k-1}, alpha_{k-1}, rho_0 of the inner solve, tol, ||xi|| */
    __shared__ double s_sc[5];
    __shared__ T s_ab[2];      /* alpha, beta for the next iteration */
    __shared__ int s_flag;     /* 0 continue, 1 inner solve done, 2 breakdown */
    __shared__ int s_conv;     /* the inner solve ended on its residual tolerance */
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int epoch = 0;
    if ((int)blockIdx.x == P.absent_cta) return; /* test hook, see pcg.cu */

    const int s0 = __ldg(P.cta_slice + blockIdx.x), s1 = __ldg(P.cta_slice + blockIdx.x + 1);
    const int row0 = 32 * s0, n_loc = 32 * (s1 - s0);
    const int64_t slot0 = __ldg(P.slice_ptr + s0), slot1 = __ldg(P.slice_ptr + s1);
    const int64_t nval = 9 * (slot1 - slot0);
    const int h0 = __ldg(P.halo_ptr + blockIdx.x), h1 = __ldg(P.halo_ptr + blockIdx.x + 1);
    /* dynamic shared memory, laid out per CTA from its own sizes (mixed_smem_layout, the
     * host's feasibility check uses the same function): T values as far as they fit |
     * local columns | D^-1 of own rows (FP32 only) | z of own + halo rows | halo u, v
     * (8 T per row, the first BS halo rows) */
    const MixedSmem ml = mixed_smem_layout(sizeof(T), F64, slot1 - slot0, s1 - s0, h1 - h0, BS, P.smem_budget);
    const int64_t nsm = nval < ml.val_cap ? nval : ml.val_cap;
    T *sval = reinterpret_cast<T *>(smem);
    int *scol = reinterpret_cast<int *>(smem + ml.col_off);
    double *sdinv = reinterpret_cast<double *>(smem + ml.dinv_off);
    T *sz = reinterpret_cast<T *>(smem + ml.halo_off);
    T *sstage = reinterpret_cast<T *>(smem + ml.stage_off);

    if (threadIdx.x == 0) {
        tma_mbar_init(&s_bar, 1);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned vbytes = (unsigned)(sizeof(T) * nsm), cbytes = (unsigned)(4 * (slot1 - slot0));
        const unsigned dbytes = F64 ? 0u : (unsigned)(2304 * (s1 - s0));
        tma_mbar_expect_tx(&s_bar, vbytes + cbytes + dbytes);
        if (vbytes) tma_bulk_g2s(sval, Inner<T>::val(P) + 9 * slot0, vbytes, &s_bar);
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
#define PUB_Z(par) Inner<T>::pz(P, par)
#define PUB_U(par) Inner<T>::pu(P, par)
#define PUB_V(par) Inner<T>::pv(P, par)
    /* this thread's own row's D^-1 (stride 32 doubles): staged in shared memory (FP32), or
     * in global memory, where it stays in L2 (FP64: the shared memory holds values) */
    const double *my_dinv = F64 ? P.dinv + 288 * (size_t)s + lane : sdinv + 288 * warp + lane;

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
        T3<T> r = { (T)r64.a, (T)r64.b, (T)r64.c };
        const T3<T> zero = { (T)0, (T)0, (T)0 };
        /* state "k = -1": z_{-1} = D^-1 r_0, and w, u, s, v, p of earlier steps 0, so
         * with alpha = beta = 0 the first step leaves r and z unchanged; readers of
         * iteration 0 use parity (0 - 1) & 1 = 1 */
        T3<T> z = mine ? dinv_apply_t<T>(my_dinv, r) : zero;
        T3<T> w = zero, u = zero, sv = zero, v = zero, p = zero, d = zero;
        if (mine) {
            stt3(PUB_Z(1), row, z);
            stt3(PUB_U(1), row, zero);
            stt3(PUB_V(1), row, zero);
        }
        if (!grid_barrier(P.gs, (unsigned)(++epoch), P.spin_limit, &s_ok)) { timed_out = true; break; }
        /* the halo's published (z, u, v) go straight into shared memory (no registers held
         * across the reduction): z into the halo row's z slot, u and v into staging */
        if (has_h) {
            cp_async_row(sz + 4 * (n_loc + threadIdx.x), PUB_Z(1) + 4 * (size_t)hrow);
            cp_async_row(sstage + 8 * threadIdx.x, PUB_U(1) + 4 * (size_t)hrow);
            cp_async_row(sstage + 8 * threadIdx.x + 4, PUB_V(1) + 4 * (size_t)hrow);
            cp_async_commit_wait_later();
        }
        T alpha = (T)0, beta = (T)0;
        int k = 0;
        while (true) {
            const int pr = (k - 1) & 1, pw = k & 1;
            /* z_k of the halo rows (first: frees the prefetched registers) */
            if (has_h) {
                cp_async_wait_all();
                T3<T> zn, vn;
                step_zv(ldt3(sz, n_loc + threadIdx.x), ldt3(sstage, 2 * threadIdx.x), ldt3(sstage, 2 * threadIdx.x + 1),
                        alpha, beta, zn, vn);
                stt3(sz, n_loc + (int)threadIdx.x, zn);
            }
            if (h_extra) {
                /* halo rows beyond the CTA's thread count (bounds re-read: rare path) */
                const int e0 = __ldg(P.halo_ptr + blockIdx.x), e1 = __ldg(P.halo_ptr + blockIdx.x + 1);
                for (int h = e0 + (int)threadIdx.x + BS; h < e1; h += BS) {
                    const int c = __ldg(P.halo_rows + h);
                    T3<T> zn, vn;
                    step_zv(ldcgt3(PUB_Z(pr), c), ldcgt3(PUB_U(pr), c), ldcgt3(PUB_V(pr), c), alpha, beta, zn, vn);
                    stt3(sz, n_loc + (h - e0), zn);
                }
            }
            /* own row: s_{k-1}, r_k, p_{k-1}, d, then v_{k-1}, z_k */
            sv = axpy_t(beta, sv, w);
            r = axpy_t(-alpha, sv, r);
            p = axpy_t(beta, p, z);
            if (k > 0) d = axpy_t(alpha, p, d);
            step_zv(z, u, v, alpha, beta, z, v);
            if (mine) {
                stt3(sz, row - row0, z);
                /* z_k and v_{k-1} are final here: publish them now, so only u_k's stores
                 * are still in flight when the CTA arrives at the barrier */
                stt3(PUB_Z(pw), row, z);
                stt3(PUB_V(pw), row, v);
            }
            __syncthreads();
            /* w_k = A z_k from shared memory, u_k = D^-1 w_k */
            double part[3] = { 0.0, 0.0, 0.0 };
            T q0 = (T)0, q1 = (T)0, q2 = (T)0;
            if (mine) {
                const int *cb = scol + lslot + lane;
                const int jend = len;
                const int jsm = j_sm;
                int j = 0;
                /* four blocks at a time: their column and z loads are in flight together
                 * (a row's blocks are still added in ascending column order) */
                const T *sv0 = sval + 9 * lslot + lane;
                /* the diagonal block's z is this thread's own (no shared-memory load) */
                const int lrow = row - row0;
                for (; j + 3 < jsm; j += 4) {
                    const int c0 = cb[32 * j], c1 = cb[32 * (j + 1)], c2 = cb[32 * (j + 2)], c3 = cb[32 * (j + 3)];
                    const T3<T> z0 = c0 == lrow ? z : ldt3(sz, c0), z1 = c1 == lrow ? z : ldt3(sz, c1);
                    const T3<T> z2 = c2 == lrow ? z : ldt3(sz, c2), z3 = c3 == lrow ? z : ldt3(sz, c3);
                    blk_acc_t(sv0 + 288 * j, z0, q0, q1, q2);
                    blk_acc_t(sv0 + 288 * (j + 1), z1, q0, q1, q2);
                    blk_acc_t(sv0 + 288 * (j + 2), z2, q0, q1, q2);
                    blk_acc_t(sv0 + 288 * (j + 3), z3, q0, q1, q2);
                }
                for (; j < jsm; j++) {
                    const int c0 = cb[32 * j];
                    blk_acc_t(sv0 + 288 * j, c0 == lrow ? z : ldt3(sz, c0), q0, q1, q2);
                }
                if (j < jend) {
                    /* blocks beyond the shared-memory share: values from L2, four blocks' loads
                     * in flight together (still added in ascending column order) */
                    const T *gv = Inner<T>::val(P) + 9 * __ldg(P.slice_ptr + s) + lane;
                    for (; j + 3 < jend; j += 4) {
                        T vb[4][9];
#pragma unroll
                        for (int u4 = 0; u4 < 4; u4++)
#pragma unroll
                            for (int e = 0; e < 9; e++) vb[u4][e] = __ldg(gv + 288 * (j + u4) + 32 * e);
#pragma unroll
                        for (int u4 = 0; u4 < 4; u4++) {
                            const T3<T> zc = ldt3(sz, cb[32 * (j + u4)]);
                            q0 = fma_t(vb[u4][0], zc.a, q0); q0 = fma_t(vb[u4][1], zc.b, q0); q0 = fma_t(vb[u4][2], zc.c, q0);
                            q1 = fma_t(vb[u4][3], zc.a, q1); q1 = fma_t(vb[u4][4], zc.b, q1); q1 = fma_t(vb[u4][5], zc.c, q1);
                            q2 = fma_t(vb[u4][6], zc.a, q2); q2 = fma_t(vb[u4][7], zc.b, q2); q2 = fma_t(vb[u4][8], zc.c, q2);
                        }
                    }
                    for (; j < jend; j++) blk_acc_t(gv + 288 * j, ldt3(sz, cb[32 * j]), q0, q1, q2);
                }
            }
            if (mine) {
                w = T3<T>{ q0, q1, q2 };
                u = dinv_apply_t<T>(my_dinv, w); /* own row's D^-1 (stride 32) */
                const double r0 = r.a, r1 = r.b, r2 = r.c, z0 = z.a, z1 = z.b, z2 = z.c;
                part[0] = r0 * z0 + r1 * z1 + r2 * z2;                            /* gamma */
                part[1] = (double)w.a * z0 + (double)w.b * z1 + (double)w.c * z2; /* delta */
                part[2] = r0 * r0 + r1 * r1 + r2 * r2;                            /* rho */
                /* publish u_k for iteration k + 1 (z_k and v_{k-1} went out before the SpMV) */
                stt3(PUB_U(pw), row, u);
            }
            if (!grid_reduce_arrive<3, BS>(part, P.partials, epoch, P.gs, P.spin_limit, s_red, &s_ok)) {
                timed_out = true;
                break;
            }
            /* the halo's values for iteration k + 1, in flight while the partials are summed
             * (every read of the halo z slots in this iteration's SpMV precedes the barrier) */
            if (has_h) {
                cp_async_row(sz + 4 * (n_loc + threadIdx.x), PUB_Z(pw) + 4 * (size_t)hrow);
                cp_async_row(sstage + 8 * threadIdx.x, PUB_U(pw) + 4 * (size_t)hrow);
                cp_async_row(sstage + 8 * threadIdx.x + 4, PUB_V(pw) + 4 * (size_t)hrow);
                cp_async_commit_wait_later();
            }
            grid_reduce_sum<3>(P.partials, epoch, s_bc);
            total++;
            k++;
            if (threadIdx.x == 0) {
                /* alpha_k = gamma / (delta - beta_k gamma / alpha_{k-1}) = gamma g / (delta g - gamma^2)
                 * with g = gamma_{k-1} alpha_{k-1}: one FP64 division on the critical path (beta's
                 * runs beside it); both rounded to T for the vector updates */
                const double gamma = s_bc[0], delta = s_bc[1], rho = s_bc[2];
                if (k == 1) s_sc[2] = rho;
                double a, bt;
                if (k == 1) { bt = 0.0; a = gamma / delta; }
                else {
                    const double g = s_sc[0] * s_sc[1];
                    bt = gamma / s_sc[0];
                    a = (gamma * g) / (delta * g - gamma * gamma);
                }
                int flag = 0, conv = 0;
                if (!(delta != 0.0) || !(a == a) || isinf(a)) flag = 2;
                else if (rho <= P.inner_tol * P.inner_tol * s_sc[2] || rho < s_sc[3])
                    flag = conv = 1;
                else if (k >= P.inner_max_iter || total >= P.max_iter)
                    flag = 1;
                s_conv = conv;
                s_sc[0] = gamma;
                s_sc[1] = a;
                s_ab[0] = (T)a;
                s_ab[1] = (T)bt;
                s_flag = flag;
            }
            __syncthreads();
            const int flag = s_flag;
            if (flag == 2) { reason = GSLAM_STOP_PQ_ZERO; break; }
            alpha = s_ab[0];
            beta = s_ab[1];
            if (flag == 1) {
                /* the last update: d += alpha_k p_k, p_k = z_k + beta_k p_{k-1}. The FP64
                 * solve that met its tolerance ends without it, at the solution whose
                 * residual met the test (the reference's loop stops there); its step count is
                 * one less than its reductions. */
                if (F64 && s_conv) {
                    total--;
                } else {
                    p = axpy_t(beta, p, z);
                    d = axpy_t(alpha, p, d);
                }
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
        if (F64) {
            /* one FP64 solve: TOL if its recurrence residual met the tolerance, else the
             * iteration cap */
            reason = s_conv ? GSLAM_STOP_TOL : GSLAM_STOP_MAXIT;
            break;
        }
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

template <int BS, typename T>
static cudaError_t set_attr_mixed() {
    return cudaFuncSetAttribute((const void *)k_pcg_mixed<BS, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                GSLAM_RES_SMEM_MAX);
}

cudaError_t launch_pcg_mixed(cudaStream_t st, const PcgParams &p, int grid, int block, size_t smem_bytes, bool fp64) {
    if (block != 768 && block != 1024) return cudaErrorInvalidValue;
    PcgParams copy = p;
    void *args[] = { &copy };
    const void *fn = fp64 ? (block == 768 ? (const void *)k_pcg_mixed<768, double> : (const void *)k_pcg_mixed<1024, double>)
                          : (block == 768 ? (const void *)k_pcg_mixed<768, float> : (const void *)k_pcg_mixed<1024, float>);
    return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(block), args, smem_bytes, st);
}

int pcg_mixed_max_grid(int device, size_t smem_bytes) {
    int n_sm = 0, a = 0, b = 0, c = 0, d = 0;
    if (cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return 0;
    if (set_attr_mixed<768, float>() != cudaSuccess || set_attr_mixed<1024, float>() != cudaSuccess ||
        set_attr_mixed<768, double>() != cudaSuccess || set_attr_mixed<1024, double>() != cudaSuccess)
        return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, (const void *)k_pcg_mixed<768, float>, 768, smem_bytes) !=
            cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, (const void *)k_pcg_mixed<1024, float>, 1024, smem_bytes) !=
            cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c, (const void *)k_pcg_mixed<768, double>, 768, smem_bytes) !=
            cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d, (const void *)k_pcg_mixed<1024, double>, 1024, smem_bytes) !=
            cudaSuccess)
        return 0;
    return std::min(std::min(a, b), std::min(c, d)) * n_sm;
}
