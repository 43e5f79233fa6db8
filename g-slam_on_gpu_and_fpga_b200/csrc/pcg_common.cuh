/* pcg_common.cuh — device pieces shared by the solver kernels (internal). */
#ifndef GSLAM_PCG_COMMON_CUH
#define GSLAM_PCG_COMMON_CUH

#include <cuda_runtime.h>
#include <stdint.h>

#include "gslam.h"
#include "kernels.cuh"

/* largest dynamic shared memory the resident solver asks for (sm_100: 227 KB per block) */
#define GSLAM_RES_SMEM_MAX (225 * 1024)

__device__ __forceinline__ unsigned ld_relaxed_u32(const unsigned *p) {
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned atom_add_release_u32(unsigned *p, unsigned v) {
    unsigned old;
    asm volatile("atom.add.release.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

__device__ __forceinline__ int ld_relaxed_s32(const int *p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

/*
 * Grid barrier on a monotonic arrival counter: barrier number `epoch` (1, 2, ...)
 * is complete when the counter reaches epoch * gridDim.x. One release atomic per
 * CTA (it orders the CTA's prior writes, made visible to thread 0 by a CTA
 * barrier before it), then polling: each poll reads the counter and the abort flag
 * with relaxed loads that are in flight together (one L2 round trip per poll), and
 * a fence.acq_rel after the counter is seen complete gives the acquire side. The
 * counter is zeroed before every launch, so 2^32 / gridDim.x barriers fit in one
 * solve. grid_barrier_t0 is thread 0's part alone (the caller has already made the
 * CTA's writes visible to thread 0 and publishes *s_ok after it); grid_barrier is
 * the whole-CTA form. Both report false when the solve must be abandoned (this wait
 * ran out of time, or another CTA's did).
 */
__device__ __forceinline__ void grid_barrier_t0(GridSync *gs, unsigned epoch, long long spin_limit, int *s_ok) {
    int ok = 1;
    const unsigned target = epoch * gridDim.x;
    const unsigned arrived = atom_add_release_u32(&gs->count, 1u) + 1u;
    if (arrived < target) {
        const long long t0 = clock64();
        while (true) {
            const unsigned c = ld_relaxed_u32(&gs->count);
            const int ab = ld_relaxed_s32(&gs->abort);
            if (c >= target) break;
            if (ab) { ok = 0; break; }
            if (clock64() - t0 > spin_limit) {
                atomicExch(&gs->abort, 1);
                ok = 0;
                break;
            }
        }
        asm volatile("fence.acq_rel.gpu;" ::: "memory");
    }
    *s_ok = ok;
}

__device__ __forceinline__ bool grid_barrier(GridSync *gs, unsigned epoch, long long spin_limit,
                                             int *s_ok) {
    __syncthreads();
    if (threadIdx.x == 0) grid_barrier_t0(gs, epoch, spin_limit, s_ok);
    __syncthreads();
    return *s_ok != 0;
}

/*
 * The solve's status record (PcgResult). The host zeroes it before every launch and
 * the kernel only ever RAISES `timeout`: a CTA that gave up at a barrier has already
 * arrived there, so the other CTAs can complete that barrier and finish normally while
 * its rows of x stay behind. Block 0 must then not report success, whichever of the two
 * writes lands last.
 *   res_mark_timeout: any CTA that gave up (or saw another CTA give up);
 *   res_finish:       block 0, thread 0, at the end of a solve its own CTA completed:
 *                     counts and norms, then the reason, or a timeout when any CTA has
 *                     raised the abort flag by then (one that gives up later raises
 *                     `timeout` itself).
 */
__device__ __forceinline__ void res_mark_timeout(PcgResult *res) {
    atomicOr(&res->timeout, 1);
    atomicExch(&res->reason, GSLAM_STOP_TIMEOUT);
}

__device__ __forceinline__ void res_finish(PcgResult *res, const GridSync *gs, int iterations, int reason,
                                           int refinements, double rnorm, double bnorm) {
    res->iterations = iterations;
    res->refinements = refinements;
    res->rnorm = rnorm;
    res->bnorm = bnorm;
    res->reason = reason;
    if (ld_relaxed_s32(&gs->abort)) res_mark_timeout(res);
}

/*
 * Deterministic all-reduce of NV (<= 4) doubles across the grid, in pieces so that
 * a caller can issue loads of data the other CTAs published before the barrier
 * while the partials are summed, and can derive scalars from the totals in one
 * thread instead of all of them:
 *   grid_reduce_arrive:  block sum of each thread's v[] (warp shuffles, then warp 0
 *                        over the warps), one partial per CTA, grid barrier
 *                        (false: the solve must be abandoned);
 *   grid_reduce_sum:     warp i < NV sums the CTAs' partials of value i into
 *                        s_bc[i] (a lane's loads all in flight together, a fixed
 *                        order: lane-strided, then a shuffle tree), then a
 *                        barrier among those NV warps, so thread 0 sees every total;
 *   grid_reduce_collect: grid_reduce_sum, CTA barrier, v[] = the totals everywhere.
 * Two partial buffers alternate: a CTA can be at most one reduction ahead of the
 * slowest reader, so it never overwrites partials still being summed.
 */
#define GSLAM_SUM_UNROLL 5 /* partial loads per lane issued together (grids up to 160 CTAs) */

template <int NV, int BS>
__device__ __forceinline__ bool grid_reduce_arrive(const double (&v)[NV], double *partials_base, int &epoch,
                                                   GridSync *gs, long long spin_limit,
                                                   double (*s_red)[BS / 32], int *s_ok) {
    static_assert(NV <= 4 && BS / 32 <= 32, "reduction shape");
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double *partials = partials_base + (epoch & 1) * 4 * gridDim.x;
    epoch++;                                   /* this reduction's barrier number */
#pragma unroll
    for (int i = 0; i < NV; i++) {
        double a = v[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) a = a + __shfl_down_sync(0xffffffffu, a, o);
        if (lane == 0) s_red[i][warp] = a;
    }
    __syncthreads();
    if (warp == 0) {
        /* warp 0 sums every value's per-warp partials (the trees interleave), and
         * its lane 0 stores them and arrives: no second CTA barrier before the
         * arrival, since the one above already ordered every thread's writes */
        double a[NV];
#pragma unroll
        for (int i = 0; i < NV; i++) a[i] = lane < BS / 32 ? s_red[i][lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
            for (int i = 0; i < NV; i++) a[i] = a[i] + __shfl_down_sync(0xffffffffu, a[i], o);
        }
        if (lane == 0) {
#pragma unroll
            for (int i = 0; i < NV; i++) partials[i * gridDim.x + blockIdx.x] = a[i];
            grid_barrier_t0(gs, (unsigned)epoch, spin_limit, s_ok);
        }
    }
    __syncthreads();
    return *s_ok != 0;
}

/* the partial loads of grid_reduce_sum alone (warps < NV), so a caller can issue them
 * ahead of its own loads and finish with grid_reduce_sum_finish */
template <int NV>
__device__ __forceinline__ void grid_reduce_sum_issue(const double *partials_base, int epoch,
                                                      double (&t)[GSLAM_SUM_UNROLL]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (warp >= NV) return;
    const int G = (int)gridDim.x;
    const double *pp = partials_base + ((epoch - 1) & 1) * 4 * G + warp * G;
#pragma unroll
    for (int u = 0; u < GSLAM_SUM_UNROLL; u++) {
        const int c = lane + 32 * u;
        t[u] = c < G ? __ldcg(pp + c) : 0.0;
    }
}

template <int NV>
__device__ __forceinline__ void grid_reduce_sum_finish(const double *partials_base, int epoch,
                                                       const double (&t)[GSLAM_SUM_UNROLL], double *s_bc) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (warp >= NV) return;
    const int G = (int)gridDim.x;
    const double *pp = partials_base + ((epoch - 1) & 1) * 4 * G + warp * G;
    double s = t[0];
#pragma unroll
    for (int u = 1; u < GSLAM_SUM_UNROLL; u++) s = s + t[u];
    for (int c = lane + 32 * GSLAM_SUM_UNROLL; c < G; c += 32) s = s + __ldcg(pp + c);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s = s + __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) s_bc[warp] = s;
    if (NV > 1) asm volatile("bar.sync 1, %0;" ::"r"(NV * 32) : "memory");
}

template <int NV>
__device__ __forceinline__ void grid_reduce_sum(const double *partials_base, int epoch, double *s_bc) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (warp >= NV) return;
    const int G = (int)gridDim.x;
    const double *pp = partials_base + ((epoch - 1) & 1) * 4 * G + warp * G;
    double t[GSLAM_SUM_UNROLL];
#pragma unroll
    for (int u = 0; u < GSLAM_SUM_UNROLL; u++) {
        const int c = lane + 32 * u;
        t[u] = c < G ? __ldcg(pp + c) : 0.0;
    }
    double s = t[0];
#pragma unroll
    for (int u = 1; u < GSLAM_SUM_UNROLL; u++) s = s + t[u];
    for (int c = lane + 32 * GSLAM_SUM_UNROLL; c < G; c += 32) s = s + __ldcg(pp + c);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s = s + __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) s_bc[warp] = s;
    if (NV > 1) asm volatile("bar.sync 1, %0;" ::"r"(NV * 32) : "memory");
}

template <int NV, int BS>
__device__ __forceinline__ void grid_reduce_collect(double (&v)[NV], const double *partials_base, int epoch,
                                                    double *s_bc) {
    grid_reduce_sum<NV>(partials_base, epoch, s_bc);
    __syncthreads();
#pragma unroll
    for (int i = 0; i < NV; i++) v[i] = s_bc[i];
}

template <int NV, int BS>
__device__ __forceinline__ bool grid_allreduce(double (&v)[NV], double *partials_base, int &epoch,
                                               GridSync *gs, long long spin_limit,
                                               double (*s_red)[BS / 32], double *s_bc, int *s_ok) {
    if (!grid_reduce_arrive<NV, BS>(v, partials_base, epoch, gs, spin_limit, s_red, s_ok)) return false;
    grid_reduce_collect<NV, BS>(v, partials_base, epoch, s_bc);
    return true;
}

struct V3 { double a, b, c; };

__device__ __forceinline__ V3 ld3(const double *v4, int row) {
    const double2 lo = *reinterpret_cast<const double2 *>(v4 + 4 * (size_t)row);
    const double hi = v4[4 * (size_t)row + 2];
    return V3{ lo.x, lo.y, hi };
}

/* L2-only loads for data other CTAs write during the kernel (z, p, partials): never
 * served from this SM's L1, so correctness does not depend on L1 invalidation. */
__device__ __forceinline__ V3 ldcg3(const double *v4, int row) {
    const double2 lo = __ldcg(reinterpret_cast<const double2 *>(v4 + 4 * (size_t)row));
    const double hi = __ldcg(v4 + 4 * (size_t)row + 2);
    return V3{ lo.x, lo.y, hi };
}

/* read-only (non-coherent path) variant for data no CTA writes during the kernel */
__device__ __forceinline__ V3 ldg3(const double *v4, int row) {
    const double2 lo = __ldg(reinterpret_cast<const double2 *>(v4 + 4 * (size_t)row));
    const double hi = __ldg(v4 + 4 * (size_t)row + 2);
    return V3{ lo.x, lo.y, hi };
}

__device__ __forceinline__ void st3(double *v4, int row, V3 v) {
    *reinterpret_cast<double2 *>(v4 + 4 * (size_t)row) = make_double2(v.a, v.b);
    v4[4 * (size_t)row + 2] = v.c;
}

/* p_new = z + beta * p_old exactly as MatrixOps.c:382 (first iteration: p = z). */
__device__ __forceinline__ V3 p_of(const double *z4, const double *pold4, int row, double beta,
                                   bool first) {
    V3 z = ldcg3(z4, row);
    if (first) return z;
    V3 p = ldcg3(pold4, row);
    return V3{ z.a + beta * p.a, z.b + beta * p.b, z.c + beta * p.c };
}

/* z = D^-1 r: z_i = ((0 + d_i0 r0) + d_i1 r1) + d_i2 r2 (MatrixOps.c:369-377). */
__device__ __forceinline__ V3 apply_dinv(const double *dinv, int row, V3 r) {
    const double *d = dinv + 288 * (size_t)(row >> 5) + (row & 31);
    double z0 = 0.0, z1 = 0.0, z2 = 0.0;
    z0 = z0 + __ldg(d + 0) * r.a;   z0 = z0 + __ldg(d + 32) * r.b;  z0 = z0 + __ldg(d + 64) * r.c;
    z1 = z1 + __ldg(d + 96) * r.a;  z1 = z1 + __ldg(d + 128) * r.b; z1 = z1 + __ldg(d + 160) * r.c;
    z2 = z2 + __ldg(d + 192) * r.a; z2 = z2 + __ldg(d + 224) * r.b; z2 = z2 + __ldg(d + 256) * r.c;
    return V3{ z0, z1, z2 };
}

/* q += block (3x3, slot layout at v) * p, each scalar row in column order. */
__device__ __forceinline__ void blk_acc(const double *v, V3 p, double &q0, double &q1, double &q2) {
    q0 = q0 + __ldg(v + 0) * p.a;   q0 = q0 + __ldg(v + 32) * p.b;  q0 = q0 + __ldg(v + 64) * p.c;
    q1 = q1 + __ldg(v + 96) * p.a;  q1 = q1 + __ldg(v + 128) * p.b; q1 = q1 + __ldg(v + 160) * p.c;
    q2 = q2 + __ldg(v + 192) * p.a; q2 = q2 + __ldg(v + 224) * p.b; q2 = q2 + __ldg(v + 256) * p.c;
}

/* Same as blk_acc for values that may live in shared or global memory. */
__device__ __forceinline__ void blk_acc_any(const double *v, V3 p, double &q0, double &q1, double &q2) {
    q0 = q0 + v[0] * p.a;   q0 = q0 + v[32] * p.b;  q0 = q0 + v[64] * p.c;
    q1 = q1 + v[96] * p.a;  q1 = q1 + v[128] * p.b; q1 = q1 + v[160] * p.c;
    q2 = q2 + v[192] * p.a; q2 = q2 + v[224] * p.b; q2 = q2 + v[256] * p.c;
}

/*
 * One row of q = A p with p formed on the fly from z and the previous p. Two
 * blocks per step so both columns' gathers are in flight together; blocks are
 * still added in ascending column order.
 */
__device__ __forceinline__ V3 spmv_row(const double *vb, const int *cb, int len, const double *z4,
                                       const double *pold, double beta, bool first) {
    double q0 = 0.0, q1 = 0.0, q2 = 0.0;
    int j = 0;
    for (; j + 1 < len; j += 2) {
        const int c0 = __ldg(cb + 32 * j), c1 = __ldg(cb + 32 * (j + 1));
        const V3 p0 = p_of(z4, pold, c0, beta, first);
        const V3 p1 = p_of(z4, pold, c1, beta, first);
        blk_acc(vb + 288 * j, p0, q0, q1, q2);
        blk_acc(vb + 288 * (j + 1), p1, q0, q1, q2);
    }
    if (j < len) {
        const int c0 = __ldg(cb + 32 * j);
        blk_acc(vb + 288 * j, p_of(z4, pold, c0, beta, first), q0, q1, q2);
    }
    return V3{ q0, q1, q2 };
}

#endif
