/*
 * batch.cu — many independent pose graphs solved in one persistent launch.
 *
 * Not in the reference (its programs solve one graph per process; its README
 * sweeps lambda with a shell loop over runs). A batch is one block-diagonal system:
 * graph g owns the rows [pose_off[g], pose_off[g + 1]), padded to whole slices of
 * 32 rows (padding rows carry an identity-scaled diagonal and a zero right-hand
 * side, so they stay 0). The row-sorting windows restart at every graph, so each
 * slice belongs to exactly one graph (slice_graph).
 *
 * Solver: the reference's block-Jacobi PCG (MatrixOps.c:281-391) run for every
 * graph at once with the graph's own alpha, beta and stopping test. The matrix
 * streams from L2 / HBM (a batch can exceed the aggregate shared memory). CTAs own
 * contiguous slice ranges balanced by slot count, so a CTA touches a handful of
 * graphs and a graph spans a contiguous range of CTAs. Each iteration has the two
 * grid barriers of the single-graph solver; the dot products are per graph:
 *   every warp reduces each of its slices into a per-slice partial in shared memory;
 *   thread t < (graphs of this CTA) adds its graph's slice partials in slice order (the
 *   graph's contiguous slice range, found once per launch) into the CTA's slot of that
 *   graph's partial array; after the grid barrier warp t
 *   sums the graph's CTA partials in CTA order (lane-strided, shuffle tree) and
 *   lane 0 advances that graph's scalars in shared memory.
 * Every CTA that owns rows of a graph computes the same scalars from the same sums
 * (deterministic, no atomics in the arithmetic). A converged graph's rows stop
 * changing; the graph's first CTA records its result and decrements a count of
 * active graphs, which every CTA reads after the next phase-A barrier (all
 * decrements of the previous iteration precede it), so all CTAs leave together.
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "gslam.h"
#include "kernels.cuh"
#include "pcg_common.cuh"

#define BATCH_LG_MAX 32 /* graphs one CTA may touch */

/* ---- row-vector access for either precision of the inner solve ----
 * T = double: the reference's FP64 PCG; T = float: the inner solve of the mixed
 * batch (FP32 values and vectors, FP64 D^-1 and dot products). Rows are padded to
 * 4 elements. */
template <typename T> struct TV { T a, b, c; };

__device__ __forceinline__ TV<double> tv_ld(const double *v4, int row) { const V3 v = ld3(v4, row); return { v.a, v.b, v.c }; }
__device__ __forceinline__ TV<double> tv_ldg(const double *v4, int row) { const V3 v = ldg3(v4, row); return { v.a, v.b, v.c }; }
__device__ __forceinline__ TV<double> tv_ldcg(const double *v4, int row) { const V3 v = ldcg3(v4, row); return { v.a, v.b, v.c }; }
__device__ __forceinline__ void tv_st(double *v4, int row, TV<double> v) { st3(v4, row, V3{ v.a, v.b, v.c }); }
__device__ __forceinline__ TV<float> tv_ld(const float *v4, int row) {
    const float4 v = *reinterpret_cast<const float4 *>(v4 + 4 * (size_t)row);
    return { v.x, v.y, v.z };
}
__device__ __forceinline__ TV<float> tv_ldg(const float *v4, int row) {
    const float4 v = __ldg(reinterpret_cast<const float4 *>(v4 + 4 * (size_t)row));
    return { v.x, v.y, v.z };
}
__device__ __forceinline__ TV<float> tv_ldcg(const float *v4, int row) {
    const float4 v = __ldcg(reinterpret_cast<const float4 *>(v4 + 4 * (size_t)row));
    return { v.x, v.y, v.z };
}
__device__ __forceinline__ void tv_st(float *v4, int row, TV<float> v) {
    *reinterpret_cast<float4 *>(v4 + 4 * (size_t)row) = make_float4(v.a, v.b, v.c, 0.f);
}

/* ---- loads of data that each iteration streams once (block values, column indices,
 * D^-1): read-only, marked evict-first in L2 by a cache policy, so that a batch whose
 * matrix is larger than L2 streams it without pushing out the solve's vectors (p, z, q,
 * r, x: gathered by neighbours and reread in the same iteration) ---- */
__device__ __forceinline__ uint64_t l2_evict_first_policy() {
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ double ld_stream(const double *p, uint64_t pol) {
    double v;
    asm volatile("ld.global.nc.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ float ld_stream(const float *p, uint64_t pol) {
    float v;
    asm volatile("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ int ld_stream(const int *p, uint64_t pol) {
    int v;
    asm volatile("ld.global.nc.L2::cache_hint.s32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
    return v;
}

/* p = z + beta p_old (first iteration: p = z), as MatrixOps.c:382, for a neighbour row */
template <typename T>
__device__ __forceinline__ TV<T> tv_p_of(const T *z4, const T *pold4, int row, T beta, bool first) {
    const TV<T> z = tv_ldcg(z4, row);
    if (first) return z;
    const TV<T> p = tv_ldcg(pold4, row);
    return { z.a + beta * p.a, z.b + beta * p.b, z.c + beta * p.c };
}

/* z = D^-1 r with the FP64 block (apply_dinv's arithmetic, the block streamed), rounded
 * to T */
template <typename T>
__device__ __forceinline__ TV<T> tv_dinv(const double *dinv, int row, TV<T> rv, uint64_t pol) {
    const double *d = dinv + 288 * (size_t)(row >> 5) + (row & 31);
    const double ra = rv.a, rb = rv.b, rc = rv.c;
    double z0 = 0.0, z1 = 0.0, z2 = 0.0;
    z0 = z0 + ld_stream(d + 0, pol) * ra;   z0 = z0 + ld_stream(d + 32, pol) * rb;  z0 = z0 + ld_stream(d + 64, pol) * rc;
    z1 = z1 + ld_stream(d + 96, pol) * ra;  z1 = z1 + ld_stream(d + 128, pol) * rb; z1 = z1 + ld_stream(d + 160, pol) * rc;
    z2 = z2 + ld_stream(d + 192, pol) * ra; z2 = z2 + ld_stream(d + 224, pol) * rb; z2 = z2 + ld_stream(d + 256, pol) * rc;
    return { (T)z0, (T)z1, (T)z2 };
}

/* q = A p for one row, blocks in ascending column order (spmv_row for either type) */
template <typename T>
__device__ __forceinline__ TV<T> tv_spmv_row(const T *vb, const int *cb, int len, const T *z4, const T *pold,
                                              T beta, bool first, uint64_t pol) {
    T q0 = 0, q1 = 0, q2 = 0;
    int j = 0;
    /* four blocks at a time: their column and neighbour loads are in flight together (the
     * blocks are still added one after another in ascending column order) */
    for (; j + 3 < len; j += 4) {
        const int c0 = ld_stream(cb + 32 * j, pol), c1 = ld_stream(cb + 32 * (j + 1), pol);
        const int c2 = ld_stream(cb + 32 * (j + 2), pol), c3 = ld_stream(cb + 32 * (j + 3), pol);
        const TV<T> p0 = tv_p_of(z4, pold, c0, beta, first), p1 = tv_p_of(z4, pold, c1, beta, first);
        const TV<T> p2 = tv_p_of(z4, pold, c2, beta, first), p3 = tv_p_of(z4, pold, c3, beta, first);
        const TV<T> pp[4] = { p0, p1, p2, p3 };
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const T *v0 = vb + 288 * (j + u);
            const TV<T> pu = pp[u];
            q0 = q0 + ld_stream(v0, pol) * pu.a;       q0 = q0 + ld_stream(v0 + 32, pol) * pu.b;  q0 = q0 + ld_stream(v0 + 64, pol) * pu.c;
            q1 = q1 + ld_stream(v0 + 96, pol) * pu.a;  q1 = q1 + ld_stream(v0 + 128, pol) * pu.b; q1 = q1 + ld_stream(v0 + 160, pol) * pu.c;
            q2 = q2 + ld_stream(v0 + 192, pol) * pu.a; q2 = q2 + ld_stream(v0 + 224, pol) * pu.b; q2 = q2 + ld_stream(v0 + 256, pol) * pu.c;
        }
    }
    for (; j + 1 < len; j += 2) {
        const int c0 = ld_stream(cb + 32 * j, pol), c1 = ld_stream(cb + 32 * (j + 1), pol);
        const TV<T> p0 = tv_p_of(z4, pold, c0, beta, first), p1 = tv_p_of(z4, pold, c1, beta, first);
        const T *v0 = vb + 288 * j, *v1 = v0 + 288;
        q0 = q0 + ld_stream(v0, pol) * p0.a;       q0 = q0 + ld_stream(v0 + 32, pol) * p0.b;  q0 = q0 + ld_stream(v0 + 64, pol) * p0.c;
        q1 = q1 + ld_stream(v0 + 96, pol) * p0.a;  q1 = q1 + ld_stream(v0 + 128, pol) * p0.b; q1 = q1 + ld_stream(v0 + 160, pol) * p0.c;
        q2 = q2 + ld_stream(v0 + 192, pol) * p0.a; q2 = q2 + ld_stream(v0 + 224, pol) * p0.b; q2 = q2 + ld_stream(v0 + 256, pol) * p0.c;
        q0 = q0 + ld_stream(v1, pol) * p1.a;       q0 = q0 + ld_stream(v1 + 32, pol) * p1.b;  q0 = q0 + ld_stream(v1 + 64, pol) * p1.c;
        q1 = q1 + ld_stream(v1 + 96, pol) * p1.a;  q1 = q1 + ld_stream(v1 + 128, pol) * p1.b; q1 = q1 + ld_stream(v1 + 160, pol) * p1.c;
        q2 = q2 + ld_stream(v1 + 192, pol) * p1.a; q2 = q2 + ld_stream(v1 + 224, pol) * p1.b; q2 = q2 + ld_stream(v1 + 256, pol) * p1.c;
    }
    if (j < len) {
        const int c0 = ld_stream(cb + 32 * j, pol);
        const TV<T> p0 = tv_p_of(z4, pold, c0, beta, first);
        const T *v0 = vb + 288 * j;
        q0 = q0 + ld_stream(v0, pol) * p0.a;       q0 = q0 + ld_stream(v0 + 32, pol) * p0.b;  q0 = q0 + ld_stream(v0 + 64, pol) * p0.c;
        q1 = q1 + ld_stream(v0 + 96, pol) * p0.a;  q1 = q1 + ld_stream(v0 + 128, pol) * p0.b; q1 = q1 + ld_stream(v0 + 160, pol) * p0.c;
        q2 = q2 + ld_stream(v0 + 192, pol) * p0.a; q2 = q2 + ld_stream(v0 + 224, pol) * p0.b; q2 = q2 + ld_stream(v0 + 256, pol) * p0.c;
    }
    return { q0, q1, q2 };
}

/* the solve's vectors for either precision */
template <typename T> struct BVec;
template <> struct BVec<double> {
    const double *val, *b; double *x, *r, *z, *pa, *pb, *q;
    __device__ BVec(const PcgParams &P, const BatchParams &) : val(P.val), b(P.b4), x(P.x4), r(P.r4), z(P.z4),
        pa(P.p4a), pb(P.p4b), q(P.q4) {}
};
template <> struct BVec<float> {
    const float *val, *b; float *x, *r, *z, *pa, *pb, *q;
    __device__ BVec(const PcgParams &P, const BatchParams &B) : val(P.val32), b(B.bf4), x(P.xf4), r(P.rf4),
        z(P.zf4), pa(P.pfa4), pb(P.pfb4), q(P.qf4) {}
};

/* launch bound of two CTAs per SM: 512-thread CTAs fit in 64 registers without spills, so
 * the tuner's ctas_per_sm = 2 gives 32 warps per SM to hide the gathers' latency (one CTA
 * of 128-register threads left the kernel waiting on memory with 16 warps per SM) */
template <int BS, typename T>
__global__ void __launch_bounds__(BS, 2) k_pcg_batch(PcgParams P, BatchParams B) {
    const BVec<T> V(P, B);
    const uint64_t pol = l2_evict_first_policy();
    extern __shared__ __align__(16) double s_part[]; /* [slices of this CTA][2] */
    __shared__ double s_rz[BATCH_LG_MAX], s_rr[BATCH_LG_MAX], s_bn[BATCH_LG_MAX];
    __shared__ double s_alpha[BATCH_LG_MAX], s_beta[BATCH_LG_MAX];
    __shared__ int s_done[BATCH_LG_MAX], s_iter[BATCH_LG_MAX], s_cnt[BATCH_LG_MAX];
    __shared__ double s_tot[2][BATCH_LG_MAX];
    __shared__ int s_ok, s_exit;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int W = BS / 32;
    const int c = blockIdx.x;
    const int s0 = __ldg(B.cta_slice + c), s1 = __ldg(B.cta_slice + c + 1), ns = s1 - s0;
    const int g0 = __ldg(B.cta_g0 + c);
    const int nlg = ns > 0 ? __ldg(B.cta_g1 + c) - g0 + 1 : 0;
    int epoch = 0;
    if (c == P.absent_cta) return; /* test hook, see pcg.cu */
    /* thread t < nlg: the range of this CTA's slices that belong to its graph g0 + t (a
     * graph's slices are contiguous), found once, and its slot in the graph's partials */
    int my_lo = 0, my_hi = 0, my_slot = 0;
    if ((int)threadIdx.x < nlg) {
        const int g = g0 + threadIdx.x;
        int sl = 0;
        while (sl < ns && __ldg(B.slice_graph + s0 + sl) < g) sl++;
        my_lo = sl;
        while (sl < ns && __ldg(B.slice_graph + s0 + sl) == g) sl++;
        my_hi = sl;
        my_slot = __ldg(B.part_off + g) + (c - __ldg(B.graph_cta0 + g));
    }

    /* per-slice partials -> this CTA's slot of each graph's partial array, then the
     * grid barrier, then the graph totals into tot[v][t] (shared) */
    auto reduce_graphs = [&](int nv, double (*tot)[BATCH_LG_MAX]) -> bool {
        __syncthreads();
        double *part = B.partials + (size_t)(epoch & 1) * 2 * B.total_parts;
        if ((int)threadIdx.x < nlg) {
            double a0 = 0.0, a1 = 0.0;
            for (int sl = my_lo; sl < my_hi; sl++) {
                a0 = a0 + s_part[2 * sl];
                a1 = a1 + s_part[2 * sl + 1];
            }
            part[my_slot] = a0;
            if (nv > 1) part[B.total_parts + my_slot] = a1;
        }
        epoch++;
        if (!grid_barrier(P.gs, (unsigned)epoch, P.spin_limit, &s_ok)) return false;
        for (int t = warp; t < nlg; t += W) {
            const int g = g0 + t;
            const int off = __ldg(B.part_off + g), n = __ldg(B.graph_ncta + g);
            double a0 = 0.0, a1 = 0.0;
            for (int j = lane; j < n; j += 32) {
                a0 = a0 + __ldcg(part + off + j);
                if (nv > 1) a1 = a1 + __ldcg(part + B.total_parts + off + j);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                a0 = a0 + __shfl_down_sync(0xffffffffu, a0, o);
                a1 = a1 + __shfl_down_sync(0xffffffffu, a1, o);
            }
            if (lane == 0) { tot[0][t] = a0; tot[1][t] = a1; }
        }
        __syncthreads();
        return true;
    };
    /* thread t < nlg: the graph's first CTA counts it out of the active graphs once */
    auto count_done = [&](int t) {
        if (s_done[t] && !s_cnt[t] && c == __ldg(B.graph_cta0 + g0 + t)) {
            atomicSub(B.active, 1);
            s_cnt[t] = 1;
        }
    };

    /* ---- x = 0, r = b, z = D^-1 r; per graph r.z and r.r ---- */
    for (int sl = warp; sl < ns; sl += W) {
        const int row = 32 * (s0 + sl) + lane;
        double rz = 0.0, rr = 0.0;
        const bool skipped = B.skip != nullptr && __ldg(B.skip + __ldg(B.slice_graph + s0 + sl)) != 0;
        if (row < P.n_rows && !skipped) {
            const TV<T> b = tv_ldg(V.b, row);
            tv_st(V.x, row, TV<T>{ 0, 0, 0 });
            tv_st(V.r, row, b);
            const TV<T> z = tv_dinv(P.dinv, row, b, pol);
            tv_st(V.z, row, z);
            const double b0 = b.a, b1 = b.b, b2 = b.c;
            rz = rz + b0 * (double)z.a; rz = rz + b1 * (double)z.b; rz = rz + b2 * (double)z.c;
            rr = rr + b0 * b0; rr = rr + b1 * b1; rr = rr + b2 * b2;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            rz = rz + __shfl_down_sync(0xffffffffu, rz, o);
            rr = rr + __shfl_down_sync(0xffffffffu, rr, o);
        }
        if (lane == 0) { s_part[2 * sl] = rz; s_part[2 * sl + 1] = rr; }
    }
    bool timed_out = !reduce_graphs(2, s_tot);
    if (!timed_out && (int)threadIdx.x < nlg) {
        const int t = threadIdx.x;
        s_rz[t] = s_tot[0][t];
        s_rr[t] = s_tot[1][t];
        s_bn[t] = sqrt(s_tot[1][t]);
        s_beta[t] = 0.0;
        s_iter[t] = 0;
        s_cnt[t] = 0;
        s_done[t] = s_bn[t] == 0.0 ? GSLAM_STOP_TOL + 1 : 0; /* zero right-hand side: x = 0 */
        count_done(t);
    }
    __syncthreads();

    int k = 0;
    while (!timed_out) {
        if (k >= P.max_iter) break;
        const bool first = (k == 0);
        T *pnew = (k & 1) ? V.pb : V.pa;
        const T *pold = (k & 1) ? V.pa : V.pb;
        /* ---- phase A: p = z + beta p, q = A p, per-graph p.q ---- */
        for (int sl = warp; sl < ns; sl += W) {
            const int s = s0 + sl;
            const int t = __ldg(B.slice_graph + s) - g0;
            const int row = 32 * s + lane;
            double pq = 0.0;
            if (!s_done[t] && row < P.n_rows) {
                const T beta = (T)s_beta[t];
                const TV<T> pn = tv_p_of(V.z, pold, row, beta, first);
                tv_st(pnew, row, pn);
                const int64_t sb = __ldg(P.slice_ptr + s);
                const TV<T> q = tv_spmv_row(V.val + 9 * sb + lane, P.col + sb + lane, __ldg(P.row_len + row), V.z,
                                            pold, beta, first, pol);
                tv_st(V.q, row, q);
                pq = pq + (double)pn.a * (double)q.a; pq = pq + (double)pn.b * (double)q.b;
                pq = pq + (double)pn.c * (double)q.c;
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) pq = pq + __shfl_down_sync(0xffffffffu, pq, o);
            if (lane == 0) { s_part[2 * sl] = pq; s_part[2 * sl + 1] = 0.0; }
        }
        if (!reduce_graphs(1, s_tot)) { timed_out = true; break; }
        if (threadIdx.x == 0) {
            /* every decrement of the previous iteration precedes this barrier */
            asm volatile("fence.acq_rel.gpu;" ::: "memory");
            s_exit = ld_relaxed_s32(B.active) == 0;
        }
        if ((int)threadIdx.x < nlg) {
            const int t = threadIdx.x;
            if (!s_done[t]) {
                if (s_tot[0][t] == 0.0) {
                    s_done[t] = GSLAM_STOP_PQ_ZERO + 1;
                    s_alpha[t] = 0.0;
                } else {
                    s_alpha[t] = s_rz[t] / s_tot[0][t];
                }
            }
        }
        __syncthreads();
        if (s_exit) break;
        /* ---- phase B: x += alpha p, r -= alpha q, z = D^-1 r; per-graph r.r, r.z ---- */
        for (int sl = warp; sl < ns; sl += W) {
            const int s = s0 + sl;
            const int t = __ldg(B.slice_graph + s) - g0;
            const int row = 32 * s + lane;
            double rr = 0.0, rz = 0.0;
            if (!s_done[t] && row < P.n_rows) {
                const T alpha = (T)s_alpha[t];
                const TV<T> pn = tv_ld(pnew, row), q = tv_ld(V.q, row);
                TV<T> x = tv_ld(V.x, row), r = tv_ld(V.r, row);
                x.a = x.a + alpha * pn.a; x.b = x.b + alpha * pn.b; x.c = x.c + alpha * pn.c;
                r.a = r.a - alpha * q.a;  r.b = r.b - alpha * q.b;  r.c = r.c - alpha * q.c;
                tv_st(V.x, row, x);
                tv_st(V.r, row, r);
                const double r0 = r.a, r1 = r.b, r2 = r.c;
                rr = rr + r0 * r0; rr = rr + r1 * r1; rr = rr + r2 * r2;
                const TV<T> z = tv_dinv(P.dinv, row, r, pol);
                tv_st(V.z, row, z);
                rz = rz + r0 * (double)z.a; rz = rz + r1 * (double)z.b; rz = rz + r2 * (double)z.c;
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                rr = rr + __shfl_down_sync(0xffffffffu, rr, o);
                rz = rz + __shfl_down_sync(0xffffffffu, rz, o);
            }
            if (lane == 0) { s_part[2 * sl] = rr; s_part[2 * sl + 1] = rz; }
        }
        if (!reduce_graphs(2, s_tot)) { timed_out = true; break; }
        k++;
        if ((int)threadIdx.x < nlg) {
            const int t = threadIdx.x;
            if (!s_done[t]) {
                s_iter[t] = k;
                s_rr[t] = s_tot[0][t];
                if (sqrt(s_tot[0][t]) < P.tol_rel * s_bn[t]) {
                    s_done[t] = GSLAM_STOP_TOL + 1;
                } else {
                    s_beta[t] = s_tot[1][t] / s_rz[t];
                    s_rz[t] = s_tot[1][t];
                    if (B.cap != nullptr && k >= __ldg(B.cap + g0 + t)) s_done[t] = GSLAM_STOP_MAXIT + 1;
                }
            }
            count_done(t);
        }
        __syncthreads();
    }
    /* results: each graph's first CTA */
    if ((int)threadIdx.x < nlg) {
        const int t = threadIdx.x, g = g0 + t;
        if (c == __ldg(B.graph_cta0 + g)) {
            PcgResult r;
            r.iterations = s_iter[t];
            r.reason = s_done[t] ? s_done[t] - 1 : GSLAM_STOP_MAXIT;
            r.refinements = 0;
            r.timeout = timed_out ? 1 : 0;
            r.rnorm = sqrt(s_rr[t]);
            r.bnorm = s_bn[t];
            B.res[g] = r;
        }
    }
    if (timed_out && threadIdx.x == 0) {
        res_mark_timeout(P.res);
    }
}

template <typename T>
static const void *batch_kernel(int block) {
    switch (block) {
    case 256: return (const void *)k_pcg_batch<256, T>;
    case 512: return (const void *)k_pcg_batch<512, T>;
    case 1024: return (const void *)k_pcg_batch<1024, T>;
    default: return nullptr;
    }
}

cudaError_t launch_pcg_batch(cudaStream_t st, const PcgParams &p, const BatchParams &b, int grid, int block,
                             size_t smem_bytes, bool fp32) {
    const void *fn = fp32 ? batch_kernel<float>(block) : batch_kernel<double>(block);
    if (!fn) return cudaErrorInvalidValue;
    PcgParams pc = p;
    BatchParams bc = b;
    void *args[] = { &pc, &bc };
    return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(block), args, smem_bytes, st);
}

int pcg_batch_max_grid(int block, size_t smem_bytes, int device) {
    const void *f64 = batch_kernel<double>(block), *f32 = batch_kernel<float>(block);
    if (!f64 || !f32) return 0;
    int n_sm = 0, a = 0, b = 0;
    if (cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, f64, block, smem_bytes) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, f32, block, smem_bytes) != cudaSuccess) return 0;
    return std::min(a, b) * n_sm;
}

int pcg_batch_lg_max() { return BATCH_LG_MAX; }

/* ---- helpers of a batch round ---- */

/* adds `anchor[q]` to the three diagonal entries of block slot `slots[q]` (FP64 values) */
__global__ void k_add_diag(int n, const int64_t *__restrict__ slots, const double *__restrict__ anchor,
                           double *__restrict__ val) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3 * n) return;
    const int q = t / 3, d = t - 3 * q;
    const int64_t slot = slots[q];
    const int e = 4 * d; /* entries 0, 4, 8 of the 3x3 block */
    double *v = val + 288 * (slot / 32) + 32 * e + (slot % 32);
    *v = *v + anchor[q];
}

/*
 * Per-graph sums of squares over the batch's vectors, spread over (chunk, graph) CTAs
 * so a large graph does not walk its rows in one CTA: k_batch_sumsq sums chunk c of
 * graph g (BATCH_CHUNK elements, a fixed order: thread-strided, shuffle tree, warps in
 * order) into part[g * max_chunks + c]; k_batch_sumsq_finish adds a graph's chunk sums
 * in chunk order (one warp per graph). Deterministic.
 *   RESID: r4 = b4 - q4 over the graph's padded rows, sum of r^2 (the mixed batch's
 *          FP64 refinement residual);
 *   else:  sum of dx^2 over the graph's real poses (the update norm).
 */
#define BATCH_CHUNK 2048

template <bool RESID>
__global__ void __launch_bounds__(256) k_batch_sumsq(const int *__restrict__ pose_off, const int *__restrict__ n_real,
                                                     const double *__restrict__ a, const double *__restrict__ q4,
                                                     double *__restrict__ r4, double *__restrict__ part, int max_chunks) {
    __shared__ double sh[8];
    const int g = blockIdx.y, c = blockIdx.x;
    const int p0 = pose_off[g];
    const int n = RESID ? pose_off[g + 1] - p0 : n_real[g];
    const int e0 = c * BATCH_CHUNK, e1 = min(3 * n, e0 + BATCH_CHUNK);
    double acc = 0.0;
    for (int i = e0 + (int)threadIdx.x; i < e1; i += 256) {
        if (RESID) {
            const int row = p0 + i / 3, comp = i - 3 * (i / 3);
            const size_t k = 4 * (size_t)row + comp;
            const double r = a[k] - q4[k];
            r4[k] = r;
            acc = acc + r * r;
        } else {
            const double d = a[3 * (size_t)p0 + i];
            acc = acc + d * d;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc = acc + __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < 8; w++) s = s + sh[w];
        part[(size_t)g * max_chunks + c] = s;
    }
}

__global__ void k_batch_sumsq_finish(int n_graphs, const int *__restrict__ pose_off, const int *__restrict__ n_real,
                                     const double *__restrict__ part, int max_chunks, int diff,
                                     double *__restrict__ out) {
    const int g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (g >= n_graphs) return;
    const int n = diff ? n_real[g] : pose_off[g + 1] - pose_off[g];
    const int nc = min(max_chunks, (3 * n + BATCH_CHUNK - 1) / BATCH_CHUNK);
    double s = 0.0;
    for (int c = lane; c < nc; c += 32) s = s + part[(size_t)g * max_chunks + c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s = s + __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) out[g] = diff ? (n > 0 ? sqrt(s / (3.0 * n)) : 0.0) : s;
}

int batch_max_chunks(int max_graph_rows) { return std::max(1, (3 * max_graph_rows + BATCH_CHUNK - 1) / BATCH_CHUNK); }

void launch_add_diag(cudaStream_t st, int n, const int64_t *slots, const double *anchor, double *val) {
    if (n > 0) k_add_diag<<<(3 * n + 255) / 256, 256, 0, st>>>(n, slots, anchor, val);
}

void launch_batch_diff(cudaStream_t st, int n_graphs, const int *pose_off, const int *n_real, const double *dx,
                       double *out, double *part, int max_chunks) {
    if (n_graphs <= 0) return;
    k_batch_sumsq<false><<<dim3(max_chunks, n_graphs), 256, 0, st>>>(pose_off, n_real, dx, nullptr, nullptr, part,
                                                                     max_chunks);
    k_batch_sumsq_finish<<<(n_graphs + 7) / 8, 256, 0, st>>>(n_graphs, pose_off, n_real, part, max_chunks, 1, out);
}

/* ---- the mixed batch's refinement steps (FP64) ---- */

/* rhs of the FP32 inner solve: bf4 = (float) r4 for rows of active graphs, else 0 */
__global__ void k_batch_rhs32(int n_rows, const int *__restrict__ slice_graph, const int *__restrict__ active,
                              const double *__restrict__ r4, float *__restrict__ bf4) {
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= n_rows) return;
    const bool on = active[slice_graph[row >> 5]] != 0;
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (on) v = make_float4((float)r4[4 * (size_t)row], (float)r4[4 * (size_t)row + 1], (float)r4[4 * (size_t)row + 2], 0.f);
    reinterpret_cast<float4 *>(bf4)[row] = v;
}

/* x4 += xf4 (the FP32 correction, accumulated in FP64) */
__global__ void k_batch_add_x(int n_rows, const float *__restrict__ xf4, double *__restrict__ x4) {
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= n_rows) return;
    const float4 d = reinterpret_cast<const float4 *>(xf4)[row];
    double *x = x4 + 4 * (size_t)row;
    x[0] = x[0] + (double)d.x;
    x[1] = x[1] + (double)d.y;
    x[2] = x[2] + (double)d.z;
}

void launch_batch_rhs32(cudaStream_t st, int n_rows, const int *slice_graph, const int *active, const double *r4,
                        float *bf4) {
    k_batch_rhs32<<<(n_rows + 255) / 256, 256, 0, st>>>(n_rows, slice_graph, active, r4, bf4);
}

void launch_batch_add_x(cudaStream_t st, int n_rows, const float *xf4, double *x4) {
    k_batch_add_x<<<(n_rows + 255) / 256, 256, 0, st>>>(n_rows, xf4, x4);
}

void launch_batch_resid(cudaStream_t st, int n_graphs, const int *pose_off, const double *b4, const double *q4,
                        double *r4, double *out, double *part, int max_chunks) {
    if (n_graphs <= 0) return;
    k_batch_sumsq<true><<<dim3(max_chunks, n_graphs), 256, 0, st>>>(pose_off, nullptr, b4, q4, r4, part, max_chunks);
    k_batch_sumsq_finish<<<(n_graphs + 7) / 8, 256, 0, st>>>(n_graphs, pose_off, nullptr, part, max_chunks, 0, out);
}
