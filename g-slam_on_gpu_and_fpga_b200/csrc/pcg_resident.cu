/*
 * pcg_resident.cu — the block-Jacobi PCG solver with the matrix resident in
 * shared memory (reference algorithm: src/cpu_pcg_fp64/MatrixOps.c:281-391).
 *
 * The solver's matrix does not change during a solve, and at the sizes this
 * back-end targets it fits in the GPU's aggregate shared memory (148 SMs x
 * 227 KB): N = 100,000 poses is ~211 KB of FP64 blocks per SM. So each CTA of a
 * cooperative launch (one per SM) copies its contiguous, slot-balanced share of
 * the sliced matrix into shared memory once, with one TMA bulk copy
 * (cp.async.bulk, completion on an mbarrier), and every PCG iteration after that
 * reads values and column indices from shared memory. A share that does not fit
 * reads its tail blocks from global memory (L2) instead.
 *
 * Each thread owns one block row for the whole solve and keeps that row's x, r,
 * z and p in registers. Only what other CTAs need crosses L2 each iteration: p
 * (phase A) and z (phase B). Column indices are staged as CTA-local indices: a
 * CTA's own rows first, then its halo (the other CTAs' rows its blocks touch, a
 * list fixed at setup). Right after each phase-B grid barrier every thread loads
 * the z and previous p of one halo row from L2 while the reduction partials are
 * summed (the two round trips overlap); in phase A every owner writes its p to
 * shared memory and every thread the p of its halo row, so the SpMV reads values
 * and p from shared memory only. Thread 0 alone advances the scalars (alpha,
 * beta, the stopping test) and hands them to the CTA through shared memory. Phases and reductions are those of pcg.cu:
 *   A: p = z + beta p; q = A p (neighbours' p recomputed from their z and old p,
 *      bit-identically); partial p.q                      -> grid reduction
 *   B: x += alpha p; r -= alpha q; z = D^-1 r; partial r.r, r.z -> grid reduction
 * Summation orders are unchanged: each scalar row of q adds its blocks in
 * ascending original column order with separate multiply and add.
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "gslam.h"
#include "kernels.cuh"
#include "pcg_common.cuh"
#include "tma_bulk.cuh"

template <int BS>
__global__ void __launch_bounds__(BS, 1) k_pcg64_res(PcgParams P) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ double s_red[3][BS / 32];
    __shared__ double s_bc[4];
    __shared__ int s_ok;
    /* scalars, advanced by thread 0 only: r.z, r.r, tol; alpha or beta; stop flag */
    __shared__ double s_sc[3];
    __shared__ double s_coef;
    __shared__ int s_flag;
    __shared__ __align__(8) uint64_t s_bar;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int epoch = 0;
    if ((int)blockIdx.x == P.absent_cta) return; /* test hook, see pcg.cu */

    const int s0 = __ldg(P.cta_slice + blockIdx.x), s1 = __ldg(P.cta_slice + blockIdx.x + 1);
    const int64_t slot0 = __ldg(P.slice_ptr + s0), slot1 = __ldg(P.slice_ptr + s1);
    const int64_t nval = 9 * (slot1 - slot0);
    const int n_loc = 32 * (s1 - s0), row0 = 32 * s0;
    const int h0 = __ldg(P.halo_ptr + blockIdx.x), h1 = __ldg(P.halo_ptr + blockIdx.x + 1);
    /* this CTA's own layout (resident_smem_layout; the host checked that it fits): values as
     * far as they fit | local column indices | p of own + halo rows */
    const ResidentSmem ml = resident_smem_layout(slot1 - slot0, s1 - s0, h1 - h0, P.smem_budget);
    const int64_t nsm = nval < ml.val_cap ? nval : ml.val_cap; /* multiple of 288 */
    double *sval = reinterpret_cast<double *>(smem);
    int *scol = reinterpret_cast<int *>(smem + ml.col_off);
    double *sp = reinterpret_cast<double *>(smem + ml.p_off);

    /* ---- stage this CTA's matrix share ---- */
    if (threadIdx.x == 0) {
        tma_mbar_init(&s_bar, 1);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned vbytes = (unsigned)(8 * nsm), cbytes = (unsigned)(4 * (slot1 - slot0));
        tma_mbar_expect_tx(&s_bar, vbytes + cbytes);
        if (vbytes) tma_bulk_g2s(sval, P.val + 9 * slot0, vbytes, &s_bar);
        if (cbytes) tma_bulk_g2s(scol, P.lcol + slot0, cbytes, &s_bar);
        int ok = tma_wait(&s_bar, 0, P.spin_limit);
        if (!ok) {
            atomicExch(&P.gs->abort, 1);
            tma_wait(&s_bar, 0, P.spin_limit); /* let the copy finish before the CTA leaves */
        }
        s_ok = ok;
    }
    __syncthreads();
    if (!s_ok) {
        if (threadIdx.x == 0) res_mark_timeout(P.res);
        return;
    }

    /* ---- this thread's row ---- */
    const int s = s0 + warp;
    const bool own_slice = s < s1;
    const int row = 32 * s + lane;
    const bool mine = own_slice && row < P.n_rows;
    const bool pub = mine && __ldg(P.row_export + row); /* another CTA reads this row */
    const int len = mine ? __ldg(P.row_len + row) : 0;
    const int lslot = own_slice ? (int)(__ldg(P.slice_ptr + s) - slot0) : 0; /* local slot of (j=0) */
    /* how many of the row's blocks have their values in shared memory */
    const int j_sm = min(len, max(0, ((int)nsm - 9 * lslot) / 288));
    const double *gval = P.val + 9 * slot0;  /* global copy of this CTA's share */
    const int *cb = scol + lslot + lane;

    /* the halo row whose z and previous p this thread prefetches after each phase-B
     * barrier (rows beyond the CTA's thread count are read in phase A instead) */
    const int hh = h0 + (int)threadIdx.x;
    const bool has_h = hh < h1;
    const int hrow = has_h ? __ldg(P.halo_rows + hh) : 0;
    V3 hz = { 0.0, 0.0, 0.0 }, hp = { 0.0, 0.0, 0.0 };

    V3 x = { 0.0, 0.0, 0.0 }, r = { 0.0, 0.0, 0.0 }, z = { 0.0, 0.0, 0.0 }, pn = { 0.0, 0.0, 0.0 };
    double acc2[2] = { 0.0, 0.0 };
    if (mine) {
        r = ldg3(P.b4, row);
        z = apply_dinv(P.dinv, row, r);
        if (pub) st3(P.z4, row, z);
        acc2[0] = acc2[0] + r.a * z.a; acc2[0] = acc2[0] + r.b * z.b; acc2[0] = acc2[0] + r.c * z.c;
        acc2[1] = acc2[1] + r.a * r.a; acc2[1] = acc2[1] + r.b * r.b; acc2[1] = acc2[1] + r.c * r.c;
    }
    if (!grid_reduce_arrive<2, BS>(acc2, P.partials, epoch, P.gs, P.spin_limit, s_red, &s_ok)) {
        if (threadIdx.x == 0) res_mark_timeout(P.res);
        return;
    }
    if (has_h) hz = ldcg3(P.z4, hrow);
    grid_reduce_collect<2, BS>(acc2, P.partials, epoch, s_bc);
    const double bnorm = sqrt(acc2[1]);
    if (threadIdx.x == 0) { s_sc[0] = acc2[0]; s_sc[1] = acc2[1]; s_sc[2] = P.tol_rel * bnorm; }
    double beta = 0.0;
    int k = 0, reason = GSLAM_STOP_MAXIT;

    while (true) {
        if (k >= P.max_iter) { reason = GSLAM_STOP_MAXIT; break; }
        const bool first = (k == 0);
        double *pnew = (k & 1) ? P.p4b : P.p4a;
        const double *pold = (k & 1) ? P.p4a : P.p4b;
        /* ---- phase A: p of own rows (registers -> shared + global for other CTAs),
         *      p of halo rows staged from L2 by all threads, then q = A p from shared ---- */
        double pq[1] = { 0.0 };
        V3 q = { 0.0, 0.0, 0.0 };
        if (mine) {
            pn = first ? z : V3{ z.a + beta * pn.a, z.b + beta * pn.b, z.c + beta * pn.c };
            if (pub) st3(pnew, row, pn);
            st3(sp, row - row0, pn);
        }
        if (has_h)
            st3(sp, n_loc + (int)threadIdx.x,
                first ? hz : V3{ hz.a + beta * hp.a, hz.b + beta * hp.b, hz.c + beta * hp.c });
        for (int h = hh + BS; h < h1; h += BS)
            st3(sp, n_loc + (h - h0), p_of(P.z4, pold, __ldg(P.halo_rows + h), beta, first));
        __syncthreads();
        if (mine) {
            double q0 = 0.0, q1 = 0.0, q2 = 0.0;
            /* blocks with values in shared memory, four at a time (their column and p
             * loads in flight together), then the share's tail from L2, two at a time;
             * a row's blocks are added in ascending column order either way */
            const double *sv0 = sval + 9 * lslot + lane;
            int j = 0;
            for (; j + 3 < j_sm; j += 4) {
                const int c0 = cb[32 * j], c1 = cb[32 * (j + 1)], c2 = cb[32 * (j + 2)], c3 = cb[32 * (j + 3)];
                const V3 p0 = ld3(sp, c0), p1 = ld3(sp, c1), p2 = ld3(sp, c2), p3 = ld3(sp, c3);
                blk_acc_any(sv0 + 288 * j, p0, q0, q1, q2);
                blk_acc_any(sv0 + 288 * (j + 1), p1, q0, q1, q2);
                blk_acc_any(sv0 + 288 * (j + 2), p2, q0, q1, q2);
                blk_acc_any(sv0 + 288 * (j + 3), p3, q0, q1, q2);
            }
            for (; j < j_sm; j++) blk_acc_any(sv0 + 288 * j, ld3(sp, cb[32 * j]), q0, q1, q2);
            if (j < len) {
                const double *gv = gval + 9 * lslot + lane;
                for (; j + 1 < len; j += 2) {
                    const V3 p0 = ld3(sp, cb[32 * j]), p1 = ld3(sp, cb[32 * (j + 1)]);
                    blk_acc(gv + 288 * j, p0, q0, q1, q2);
                    blk_acc(gv + 288 * (j + 1), p1, q0, q1, q2);
                }
                if (j < len) blk_acc(gv + 288 * j, ld3(sp, cb[32 * j]), q0, q1, q2);
            }
            q = V3{ q0, q1, q2 };
            pq[0] = pq[0] + pn.a * q.a; pq[0] = pq[0] + pn.b * q.b; pq[0] = pq[0] + pn.c * q.c;
        }
        if (!grid_reduce_arrive<1, BS>(pq, P.partials, epoch, P.gs, P.spin_limit, s_red, &s_ok)) {
            reason = GSLAM_STOP_TIMEOUT;
            break;
        }
        grid_reduce_sum<1>(P.partials, epoch, s_bc);
        if (threadIdx.x == 0) {
            s_flag = s_bc[0] == 0.0;
            s_coef = s_sc[0] / s_bc[0];
        }
        __syncthreads();
        if (s_flag) { reason = GSLAM_STOP_PQ_ZERO; break; }
        const double alpha = s_coef;
        /* ---- phase B ---- */
        double rs[2] = { 0.0, 0.0 };
        if (mine) {
            x.a = x.a + alpha * pn.a; x.b = x.b + alpha * pn.b; x.c = x.c + alpha * pn.c;
            r.a = r.a - alpha * q.a;  r.b = r.b - alpha * q.b;  r.c = r.c - alpha * q.c;
            rs[0] = rs[0] + r.a * r.a; rs[0] = rs[0] + r.b * r.b; rs[0] = rs[0] + r.c * r.c;
            z = apply_dinv(P.dinv, row, r);
            if (pub) st3(P.z4, row, z);
            rs[1] = rs[1] + r.a * z.a; rs[1] = rs[1] + r.b * z.b; rs[1] = rs[1] + r.c * z.c;
        }
        if (!grid_reduce_arrive<2, BS>(rs, P.partials, epoch, P.gs, P.spin_limit, s_red, &s_ok)) {
            reason = GSLAM_STOP_TIMEOUT;
            break;
        }
        /* the partials' loads first, then the halo's z_{k+1} and p_k, in flight while
         * the partials are summed */
        {
            double tp[GSLAM_SUM_UNROLL];
            grid_reduce_sum_issue<2>(P.partials, epoch, tp);
            if (has_h) { hz = ldcg3(P.z4, hrow); hp = ldcg3(pnew, hrow); }
            grid_reduce_sum_finish<2>(P.partials, epoch, tp, s_bc);
        }
        k++;
        if (threadIdx.x == 0) {
            const double rr = s_bc[0], rz_new = s_bc[1];
            s_sc[1] = rr;
            s_flag = sqrt(rr) < s_sc[2];
            s_coef = rz_new / s_sc[0];
            s_sc[0] = rz_new;
        }
        __syncthreads();
        if (s_flag) { reason = GSLAM_STOP_TOL; break; }
        beta = s_coef;
    }
    if (mine) st3(P.x4, row, x);
    if (reason == GSLAM_STOP_TIMEOUT && threadIdx.x == 0) {
        res_mark_timeout(P.res);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && reason != GSLAM_STOP_TIMEOUT) {
        res_finish(P.res, P.gs, k, reason, 0, sqrt(s_sc[1]), bnorm);
    }
}

/* 768 threads (24 slices per CTA, up to 85 registers) when the slices fit, else 1024;
 * the host's slice partition uses the same cap (one slice per warp). */
template <int BS>
static cudaError_t set_smem_attr() {
    return cudaFuncSetAttribute((const void *)k_pcg64_res<BS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                GSLAM_RES_SMEM_MAX);
}

cudaError_t launch_pcg_resident(cudaStream_t st, const PcgParams &p, int grid, int block,
                                size_t smem_bytes) {
    if (block != 768 && block != 1024) return cudaErrorInvalidValue;
    /* the attribute is per function and process: set once (pcg_resident_max_grid sets it
     * before any layout chooses this solver) */
    PcgParams copy = p;
    void *args[] = { &copy };
    const void *fn = block == 768 ? (const void *)k_pcg64_res<768> : (const void *)k_pcg64_res<1024>;
    return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(block), args, smem_bytes, st);
}

int pcg_resident_max_grid(int device, size_t smem_bytes) {
    int n_sm = 0, a = 0, b = 0;
    if (cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return 0;
    if (set_smem_attr<768>() != cudaSuccess || set_smem_attr<1024>() != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, (const void *)k_pcg64_res<768>, 768, smem_bytes) !=
        cudaSuccess)
        return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, (const void *)k_pcg64_res<1024>, 1024, smem_bytes) !=
        cudaSuccess)
        return 0;
    return std::min(a, b) * n_sm;
}
