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
 *   thread t < (graphs of this CTA) adds its graph's slice partials in slice order
 *   into the CTA's slot of that graph's partial array; after the grid barrier warp t
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

template <int BS>
__global__ void __launch_bounds__(BS, 1) k_pcg_batch(PcgParams P, BatchParams B) {
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

    /* per-slice partials -> this CTA's slot of each graph's partial array, then the
     * grid barrier, then the graph totals into tot[v][t] (shared) */
    auto reduce_graphs = [&](int nv, double (*tot)[BATCH_LG_MAX]) -> bool {
        __syncthreads();
        double *part = B.partials + (size_t)(epoch & 1) * 2 * B.total_parts;
        if ((int)threadIdx.x < nlg) {
            const int g = g0 + threadIdx.x;
            double a0 = 0.0, a1 = 0.0;
            for (int sl = 0; sl < ns; sl++) {
                if (__ldg(B.slice_graph + s0 + sl) != g) continue;
                a0 = a0 + s_part[2 * sl];
                a1 = a1 + s_part[2 * sl + 1];
            }
            const int slot = __ldg(B.part_off + g) + (c - __ldg(B.graph_cta0 + g));
            part[slot] = a0;
            if (nv > 1) part[B.total_parts + slot] = a1;
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
        if (row < P.n_rows) {
            const V3 b = ldg3(P.b4, row);
            st3(P.x4, row, V3{ 0.0, 0.0, 0.0 });
            st3(P.r4, row, b);
            const V3 z = apply_dinv(P.dinv, row, b);
            st3(P.z4, row, z);
            rz = rz + b.a * z.a; rz = rz + b.b * z.b; rz = rz + b.c * z.c;
            rr = rr + b.a * b.a; rr = rr + b.b * b.b; rr = rr + b.c * b.c;
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
        double *pnew = (k & 1) ? P.p4b : P.p4a;
        const double *pold = (k & 1) ? P.p4a : P.p4b;
        /* ---- phase A: p = z + beta p, q = A p, per-graph p.q ---- */
        for (int sl = warp; sl < ns; sl += W) {
            const int s = s0 + sl;
            const int t = __ldg(B.slice_graph + s) - g0;
            const int row = 32 * s + lane;
            double pq = 0.0;
            if (!s_done[t] && row < P.n_rows) {
                const double beta = s_beta[t];
                const V3 pn = p_of(P.z4, pold, row, beta, first);
                st3(pnew, row, pn);
                const int64_t sb = __ldg(P.slice_ptr + s);
                const V3 q = spmv_row(P.val + 9 * sb + lane, P.col + sb + lane, __ldg(P.row_len + row), P.z4,
                                      pold, beta, first);
                st3(P.q4, row, q);
                pq = pq + pn.a * q.a; pq = pq + pn.b * q.b; pq = pq + pn.c * q.c;
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
                const double alpha = s_alpha[t];
                const V3 pn = ld3(pnew, row), q = ld3(P.q4, row);
                V3 x = ld3(P.x4, row), r = ld3(P.r4, row);
                x.a = x.a + alpha * pn.a; x.b = x.b + alpha * pn.b; x.c = x.c + alpha * pn.c;
                r.a = r.a - alpha * q.a;  r.b = r.b - alpha * q.b;  r.c = r.c - alpha * q.c;
                st3(P.x4, row, x);
                st3(P.r4, row, r);
                rr = rr + r.a * r.a; rr = rr + r.b * r.b; rr = rr + r.c * r.c;
                const V3 z = apply_dinv(P.dinv, row, r);
                st3(P.z4, row, z);
                rz = rz + r.a * z.a; rz = rz + r.b * z.b; rz = rz + r.c * z.c;
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
        P.res->timeout = 1;
        P.res->reason = GSLAM_STOP_TIMEOUT;
    }
}

template <int BS>
static const void *batch_fn() { return (const void *)k_pcg_batch<BS>; }

static const void *batch_kernel(int block) {
    switch (block) {
    case 256: return batch_fn<256>();
    case 512: return batch_fn<512>();
    case 1024: return batch_fn<1024>();
    default: return nullptr;
    }
}

cudaError_t launch_pcg_batch(cudaStream_t st, const PcgParams &p, const BatchParams &b, int grid, int block,
                             size_t smem_bytes) {
    const void *fn = batch_kernel(block);
    if (!fn) return cudaErrorInvalidValue;
    PcgParams pc = p;
    BatchParams bc = b;
    void *args[] = { &pc, &bc };
    return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(block), args, smem_bytes, st);
}

int pcg_batch_max_grid(int block, size_t smem_bytes, int device) {
    const void *fn = batch_kernel(block);
    if (!fn) return 0;
    int n_sm = 0, per = 0;
    if (cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, block, smem_bytes) != cudaSuccess) return 0;
    return per * n_sm;
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

/* per-graph update norm: sqrt(sum dx^2 / (3 n_real)), one CTA per graph */
__global__ void k_batch_diff(const int *__restrict__ pose_off, const int *__restrict__ n_real,
                             const double *__restrict__ dx, double *__restrict__ out) {
    __shared__ double sh[32];
    const int g = blockIdx.x;
    const int p0 = pose_off[g], n = n_real[g];
    double acc = 0.0;
    for (int i = threadIdx.x; i < 3 * n; i += blockDim.x) {
        const double d = dx[3 * (size_t)p0 + i];
        acc = acc + d * d;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc = acc + __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) s = s + sh[w];
        out[g] = n > 0 ? sqrt(s / (3.0 * n)) : 0.0;
    }
}

void launch_add_diag(cudaStream_t st, int n, const int64_t *slots, const double *anchor, double *val) {
    if (n > 0) k_add_diag<<<(3 * n + 255) / 256, 256, 0, st>>>(n, slots, anchor, val);
}

void launch_batch_diff(cudaStream_t st, int n_graphs, const int *pose_off, const int *n_real, const double *dx,
                       double *out) {
    if (n_graphs > 0) k_batch_diff<<<n_graphs, 256, 0, st>>>(pose_off, n_real, dx, out);
}
