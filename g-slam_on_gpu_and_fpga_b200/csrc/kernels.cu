/*
 * kernels.cu — per-round device kernels other than the solver:
 *   linearisation  (reference ObsEdge.c:10-212, MotionEdge.c:9-193),
 *   assembly       (MatrixOps.c:223-272, as a gather in edge order, no atomics),
 *   block-Jacobi   (MatrixOps.c:284-315, cofactor inverse of each diagonal block),
 *   pose update    (GSLAM.c:98-105, plus ||dx||).
 * All FP64, compiled with -fmad=false: results are bit-identical to the
 * reference's arithmetic on the same inputs (transcendentals: see crmath.h).
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include "edge_math.cuh"
#include "gslam.h"
#include "kernels.cuh"

/* ------------------------------------------------------------------------ */
/* linearisation                                                             */
/* ------------------------------------------------------------------------ */

__global__ void k_obs_edges(int64_t n_obs_edges, const unsigned *__restrict__ pair_j,
                            const unsigned *__restrict__ pair_k,
                            const unsigned *__restrict__ z_step, const double *__restrict__ z_rb,
                            const double *__restrict__ poses, double *__restrict__ blocks) {
    int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_obs_edges) return;
    const unsigned a = pair_j[e], b = pair_k[e];
    const unsigned s1 = z_step[a], s2 = z_step[b];
    double x1[3], x2[3], z1[2], z2[2], out[42];
#pragma unroll
    for (int i = 0; i < 3; i++) { x1[i] = poses[3 * (size_t)s1 + i]; x2[i] = poses[3 * (size_t)s2 + i]; }
    z1[0] = z_rb[2 * (size_t)a]; z1[1] = z_rb[2 * (size_t)a + 1];
    z2[0] = z_rb[2 * (size_t)b]; z2[1] = z_rb[2 * (size_t)b + 1];
    em_obs_edge(x1, x2, z1, z2, out);
    double *dst = blocks + 42 * (size_t)e;
#pragma unroll
    for (int i = 0; i < 42; i++) dst[i] = out[i];
}

__global__ void k_motion_edges(int n_poses, int64_t first_edge, const double *__restrict__ controls,
                               double delta, double lambda, double m0, double m1, double m2,
                               double m3, const double *__restrict__ poses,
                               double *__restrict__ blocks) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_poses - 1) return;
    const double mns[4] = { m0, m1, m2, m3 };
    double x1[3], x2[3], out[42];
#pragma unroll
    for (int k = 0; k < 3; k++) { x1[k] = poses[3 * (size_t)i + k]; x2[k] = poses[3 * (size_t)(i + 1) + k]; }
    const double nu = controls[2 * (size_t)(i + 1)], om = controls[2 * (size_t)(i + 1) + 1];
    em_motion_edge(x1, x2, nu, om, delta, lambda, mns, out);
    double *dst = blocks + 42 * (size_t)(first_edge + i);
#pragma unroll
    for (int k = 0; k < 42; k++) dst[k] = out[k];
}

/*
 * SE(2) between-factor (odometry / loop closure), information diag(info) * lambda.
 * Not in the reference; same 42-double block layout and Omega dx = xi convention.
 */
__global__ void k_se2_edges(int64_t n, int64_t first_edge, const unsigned *__restrict__ ei,
                            const unsigned *__restrict__ ej, const double *__restrict__ meas,
                            const double *__restrict__ info, double lambda,
                            const double *__restrict__ poses, double *__restrict__ blocks) {
    int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const unsigned i = ei[e], j = ej[e];
    double xi[3], xj[3], z[3], w[3], out[42];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        xi[k] = poses[3 * (size_t)i + k];
        xj[k] = poses[3 * (size_t)j + k];
        z[k] = meas[3 * (size_t)e + k];
        w[k] = info[3 * (size_t)e + k];
    }
    em_se2_edge(xi, xj, z, w, lambda, out);
    double *dst = blocks + 42 * (size_t)(first_edge + e);
#pragma unroll
    for (int k = 0; k < 42; k++) dst[k] = out[k];
}

/* ------------------------------------------------------------------------ */
/* assembly                                                                  */
/* ------------------------------------------------------------------------ */

/*
 * One thread per (slot, entry), entry fastest: the 9 threads of a slot read the
 * 9 consecutive values of each contributing sub-block. The sum starts at +0.0,
 * adds the 1e6 anchor on the diagonal of block (0,0) first, then every
 * contribution in edge order: the reference's per-entry order.
 */
__global__ void k_assemble(int64_t n_slots, const int64_t *__restrict__ ctr_ptr,
                           const int64_t *__restrict__ ctr, const double *__restrict__ blocks,
                           int64_t anchor_slot, double anchor, double *__restrict__ val,
                           float *__restrict__ val32, const int64_t *__restrict__ slot_csr,
                           const int *__restrict__ chunk_slice, const int *__restrict__ row_len,
                           double *__restrict__ csr_vals) {
    int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= 9 * n_slots) return;
    const int64_t slot = gid / 9;
    const int e = (int)(gid - 9 * slot);
    double acc = 0.0;
    if (slot == anchor_slot && (e == 0 || e == 4 || e == 8)) acc = acc + anchor;
    const int64_t c0 = ctr_ptr[slot], c1 = ctr_ptr[slot + 1];
    for (int64_t c = c0; c < c1; c++) {
        const int64_t code = ctr[c];
        acc = acc + blocks[42 * (code >> 2) + 9 * (code & 3) + e];
    }
    const int64_t chunk = slot >> 5;
    const int lane = (int)(slot & 31);
    const int64_t vpos = 288 * chunk + 32 * e + lane;
    val[vpos] = acc;
    if (val32) val32[vpos] = (float)acc;
    if (csr_vals) {
        const int64_t base = slot_csr[slot];
        const int r = e / 3, cc = e % 3;
        if (base >= 0) {
            const int len = row_len[32 * chunk_slice[chunk] + lane];
            csr_vals[base + (int64_t)r * 3 * len + cc] = acc;
        } else if (base == -2 && r == cc) {
            csr_vals[r] = acc; /* bare anchor: rows 0..2 hold only (d, d) */
        }
    }
}

/* xi per (new row, component), edge order, upper before bottom within an edge. */
__global__ void k_assemble_xi(int n_rows, const int64_t *__restrict__ xi_ptr,
                              const int64_t *__restrict__ xi_ctr, const double *__restrict__ blocks,
                              double *__restrict__ b4, const int *__restrict__ perm,
                              double *__restrict__ xi_orig) {
    int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= 3 * (int64_t)n_rows) return;
    const int row = (int)(gid / 3), r = (int)(gid - 3 * (int64_t)row);
    double acc = 0.0;
    for (int64_t c = xi_ptr[row]; c < xi_ptr[row + 1]; c++) {
        const int64_t code = xi_ctr[c];
        acc = acc + blocks[42 * (code >> 1) + 36 + 3 * (code & 1) + r];
    }
    b4[4 * (size_t)row + r] = acc;
    if (xi_orig) xi_orig[3 * (size_t)perm[row] + r] = acc;
}

/* Caller-provided CSR values -> internal layout (the drop-in solve reads d_csr_vals). */
__global__ void k_csr_to_sell(int64_t n_slots, const int64_t *__restrict__ slot_csr,
                              const int *__restrict__ chunk_slice, const int *__restrict__ row_len,
                              const double *__restrict__ csr_vals, double *__restrict__ val,
                              float *__restrict__ val32) {
    int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= 9 * n_slots) return;
    const int64_t slot = gid / 9;
    const int e = (int)(gid - 9 * slot);
    const int64_t chunk = slot >> 5;
    const int lane = (int)(slot & 31);
    const int64_t base = slot_csr[slot];
    const int r = e / 3, cc = e % 3;
    double v = 0.0;
    if (base >= 0) {
        const int len = row_len[32 * chunk_slice[chunk] + lane];
        v = csr_vals[base + (int64_t)r * 3 * len + cc];
    } else if (base == -2) {
        v = (r == cc) ? csr_vals[r] : 0.0;
    }
    const int64_t vpos = 288 * chunk + 32 * e + lane;
    val[vpos] = v;
    if (val32) val32[vpos] = (float)v;
}

/* Internal layout -> the reference's scalar CSR values (inverse of k_csr_to_sell). */
__global__ void k_sell_to_csr(int64_t n_slots, const int64_t *__restrict__ slot_csr,
                              const int *__restrict__ chunk_slice, const int *__restrict__ row_len,
                              const double *__restrict__ val, double *__restrict__ csr_vals) {
    int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= 9 * n_slots) return;
    const int64_t slot = gid / 9;
    const int e = (int)(gid - 9 * slot);
    const int64_t chunk = slot >> 5;
    const int lane = (int)(slot & 31);
    const int64_t base = slot_csr[slot];
    const int r = e / 3, cc = e % 3;
    const double v = val[288 * chunk + 32 * e + lane];
    if (base >= 0) {
        const int len = row_len[32 * chunk_slice[chunk] + lane];
        csr_vals[base + (int64_t)r * 3 * len + cc] = v;
    } else if (base == -2 && r == cc) {
        csr_vals[r] = v;
    }
}

/* FP64 values -> FP32 copy (same layout), for a mixed solve of values assembled in FP64 mode. */
__global__ void k_val_to_f32(int64_t n, const double *__restrict__ val, float *__restrict__ val32) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) val32[i] = (float)val[i];
}

/* Original-order vector [3N] -> padded new-order vector [4N]. */
__global__ void k_gather_vec(int n_rows, const int *__restrict__ perm, const double *__restrict__ src,
                             double *__restrict__ dst4) {
    int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= 4 * (int64_t)n_rows) return;
    const int row = (int)(gid >> 2), c = (int)(gid & 3);
    dst4[gid] = (c < 3) ? src[3 * (size_t)perm[row] + c] : 0.0;
}

/* Padded new-order vector [4N] -> original-order vector [3N]. */
__global__ void k_scatter_vec(int n_rows, const int *__restrict__ perm, const double *__restrict__ src4,
                              double *__restrict__ dst) {
    int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= 3 * (int64_t)n_rows) return;
    const int row = (int)(gid / 3), c = (int)(gid - 3 * (int64_t)row);
    dst[3 * (size_t)perm[row] + c] = src4[4 * (size_t)row + c];
}

/* ------------------------------------------------------------------------ */
/* block-Jacobi preconditioner                                               */
/* ------------------------------------------------------------------------ */

/*
 * Cofactor inverse of each diagonal block, det == 0 -> 1e-30, in the exact
 * expression order of MatrixOps.c:301-314. dinv uses the slot layout: entry e of
 * new row n at 288 * (n / 32) + 32 * e + n % 32.
 */
__global__ void k_diag_inv(int n_rows, const int *__restrict__ diag_slot,
                           const double *__restrict__ val, double *__restrict__ dinv) {
    int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= n_rows) return;
    double a[9];
    const int ds = diag_slot[n];
#pragma unroll
    for (int e = 0; e < 9; e++)
        a[e] = (ds >= 0) ? val[288 * (int64_t)(ds >> 5) + 32 * e + (ds & 31)] : 0.0;
    double det = a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
                 a[2] * (a[3] * a[7] - a[4] * a[6]);
    if (det == 0.0) det = 1e-30;
    double v[9];
    v[0] = (a[4] * a[8] - a[5] * a[7]) / det;
    v[1] = (a[2] * a[7] - a[1] * a[8]) / det;
    v[2] = (a[1] * a[5] - a[2] * a[4]) / det;
    v[3] = (a[5] * a[6] - a[3] * a[8]) / det;
    v[4] = (a[0] * a[8] - a[2] * a[6]) / det;
    v[5] = (a[2] * a[3] - a[0] * a[5]) / det;
    v[6] = (a[3] * a[7] - a[4] * a[6]) / det;
    v[7] = (a[1] * a[6] - a[0] * a[7]) / det;
    v[8] = (a[0] * a[4] - a[1] * a[3]) / det;
    const int64_t base = 288 * (int64_t)(n >> 5) + (n & 31);
#pragma unroll
    for (int e = 0; e < 9; e++) dinv[base + 32 * e] = v[e];
}

/* ------------------------------------------------------------------------ */
/* pose update and ||dx||                                                    */
/* ------------------------------------------------------------------------ */


/*
 * poses[old] += x[new] (GSLAM.c:98-102) and dx[old] = x[new]; each block writes
 * the sum of dx^2 over its poses (in pose order per thread, then a fixed tree).
 */
/* guard (may be null): the solver's result; when it timed out or stagnated the poses
 * stay as they are (a captured round, whose host decides afterwards) */
__global__ void k_pose_update(int n_rows, const int *__restrict__ iperm, const double *__restrict__ x4,
                              double *__restrict__ poses, double *__restrict__ dx, int wrap,
                              double *__restrict__ block_sums, const PcgResult *__restrict__ guard) {
    __shared__ double sh[32];
    if (guard && (guard->timeout || guard->reason == GSLAM_STOP_STAGNATION)) {
        if (threadIdx.x == 0) block_sums[blockIdx.x] = 0.0;
        return;
    }
    double acc = 0.0;
    for (int old = blockIdx.x * blockDim.x + threadIdx.x; old < n_rows;
         old += gridDim.x * blockDim.x) {
        const int n = iperm[old];
        double d[3];
#pragma unroll
        for (int c = 0; c < 3; c++) d[c] = x4[4 * (size_t)n + c];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            double p = poses[3 * (size_t)old + c] + d[c];
            if (c == 2 && wrap) p = em_wrap_angle(p);
            poses[3 * (size_t)old + c] = p;
            dx[3 * (size_t)old + c] = d[c];
            acc = acc + d[c] * d[c];
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc = acc + __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) s = s + sh[w];
        block_sums[blockIdx.x] = s;
    }
}

/* sum of n values by one warp in a fixed order (lane-strided, then a shuffle tree): the
 * loads of a lane are independent, so they overlap instead of one L2 round trip each */
__device__ __forceinline__ double warp_ordered_sum(int n, const double *__restrict__ v) {
    const int lane = threadIdx.x & 31;
    double s = 0.0;
#pragma unroll 8
    for (int i = lane; i < n; i += 32) s = s + v[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s = s + __shfl_down_sync(0xffffffffu, s, o);
    return s;
}

/* diff = sqrt(sum of the block sums) / sqrt(dim); one warp */
__global__ void k_finish_diff(int n_blocks, const double *__restrict__ block_sums, double dim,
                              double *__restrict__ diff_out) {
    const double s = warp_ordered_sum(n_blocks, block_sums);
    if (threadIdx.x == 0) *diff_out = sqrt(s) / sqrt(dim);
}

/*
 * Round cost (GSLAM.c:74-87 with the intended dimensions): one thread per edge in the
 * reference's array order (observation edges, then motion edges), the edge's term
 * computed by the linearisation's own arithmetic, stored per edge and summed per block
 * (warp tree, then warps in order); k_finish_cost adds the block sums in a fixed order.
 */
__global__ void k_edge_costs(int64_t n_obs_edges, int n_poses, const unsigned *__restrict__ pair_j,
                             const unsigned *__restrict__ pair_k, const unsigned *__restrict__ z_step,
                             const double *__restrict__ z_rb, const double *__restrict__ controls,
                             double delta, double lambda, double m0, double m1, double m2, double m3,
                             const double *__restrict__ poses, double *__restrict__ edge_cost,
                             double *__restrict__ block_sums) {
    __shared__ double sh[32];
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t n_edges = n_obs_edges + (n_poses > 1 ? n_poses - 1 : 0);
    double c = 0.0, out[42];
    if (e < n_obs_edges) {
        const unsigned a = pair_j[e], b = pair_k[e];
        const unsigned s1 = z_step[a], s2 = z_step[b];
        double x1[3], x2[3], z1[2], z2[2];
#pragma unroll
        for (int i = 0; i < 3; i++) { x1[i] = poses[3 * (size_t)s1 + i]; x2[i] = poses[3 * (size_t)s2 + i]; }
        z1[0] = z_rb[2 * (size_t)a]; z1[1] = z_rb[2 * (size_t)a + 1];
        z2[0] = z_rb[2 * (size_t)b]; z2[1] = z_rb[2 * (size_t)b + 1];
        em_obs_edge(x1, x2, z1, z2, out, &c);
    } else if (e < n_edges) {
        const int i = (int)(e - n_obs_edges);
        const double mns[4] = { m0, m1, m2, m3 };
        double x1[3], x2[3];
#pragma unroll
        for (int k = 0; k < 3; k++) { x1[k] = poses[3 * (size_t)i + k]; x2[k] = poses[3 * (size_t)(i + 1) + k]; }
        const double nu = controls[2 * (size_t)(i + 1)], om = controls[2 * (size_t)(i + 1) + 1];
        em_motion_edge(x1, x2, nu, om, delta, lambda, mns, out, &c);
    }
    if (e < n_edges) edge_cost[e] = c;
    double acc = c;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc = acc + __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) s = s + sh[w];
        block_sums[blockIdx.x] = s;
    }
}

__global__ void k_finish_cost(int n_blocks, const double *__restrict__ block_sums, double *__restrict__ out) {
    const double s = warp_ordered_sum(n_blocks, block_sums);
    if (threadIdx.x == 0) *out = s;
}

/* ------------------------------------------------------------------------ */
/* launch helpers                                                            */
/* ------------------------------------------------------------------------ */

static inline unsigned blocks_for(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

void launch_obs_edges(cudaStream_t st, int64_t n, const unsigned *pj, const unsigned *pk,
                      const unsigned *z_step, const double *z_rb, const double *poses,
                      double *blocks) {
    if (n > 0) k_obs_edges<<<blocks_for(n, 128), 128, 0, st>>>(n, pj, pk, z_step, z_rb, poses, blocks);
}

void launch_motion_edges(cudaStream_t st, int n_poses, int64_t first_edge, const double *controls,
                         double delta, double lambda, const double *mns, const double *poses,
                         double *blocks) {
    if (n_poses > 1)
        k_motion_edges<<<blocks_for(n_poses - 1, 128), 128, 0, st>>>(
            n_poses, first_edge, controls, delta, lambda, mns[0], mns[1], mns[2], mns[3], poses, blocks);
}

void launch_assemble(cudaStream_t st, int64_t n_slots, const int64_t *ctr_ptr, const int64_t *ctr,
                     const double *blocks, int64_t anchor_slot, double anchor, double *val,
                     float *val32, const int64_t *slot_csr, const int *chunk_slice,
                     const int *row_len, double *csr_vals) {
    k_assemble<<<blocks_for(9 * n_slots, 256), 256, 0, st>>>(n_slots, ctr_ptr, ctr, blocks, anchor_slot,
                                                            anchor, val, val32, slot_csr, chunk_slice,
                                                            row_len, csr_vals);
}

void launch_sell_to_csr(cudaStream_t st, int64_t n_slots, const int64_t *slot_csr,
                        const int *chunk_slice, const int *row_len, const double *val,
                        double *csr_vals) {
    k_sell_to_csr<<<blocks_for(9 * n_slots, 256), 256, 0, st>>>(n_slots, slot_csr, chunk_slice,
                                                               row_len, val, csr_vals);
}

void launch_se2_edges(cudaStream_t st, int64_t n, int64_t first_edge, const unsigned *ei,
                      const unsigned *ej, const double *meas, const double *info, double lambda,
                      const double *poses, double *blocks) {
    if (n > 0)
        k_se2_edges<<<blocks_for(n, 128), 128, 0, st>>>(n, first_edge, ei, ej, meas, info, lambda,
                                                        poses, blocks);
}

void launch_assemble_xi(cudaStream_t st, int n_rows, const int64_t *xi_ptr, const int64_t *xi_ctr,
                        const double *blocks, double *b4, const int *perm, double *xi_orig) {
    k_assemble_xi<<<blocks_for(3 * (int64_t)n_rows, 256), 256, 0, st>>>(n_rows, xi_ptr, xi_ctr,
                                                                        blocks, b4, perm, xi_orig);
}

void launch_csr_to_sell(cudaStream_t st, int64_t n_slots, const int64_t *slot_csr,
                        const int *chunk_slice, const int *row_len, const double *csr_vals,
                        double *val, float *val32) {
    k_csr_to_sell<<<blocks_for(9 * n_slots, 256), 256, 0, st>>>(n_slots, slot_csr, chunk_slice,
                                                               row_len, csr_vals, val, val32);
}

void launch_val_to_f32(cudaStream_t st, int64_t n, const double *val, float *val32) {
    if (n > 0) k_val_to_f32<<<blocks_for(n, 256), 256, 0, st>>>(n, val, val32);
}

void launch_gather_vec(cudaStream_t st, int n_rows, const int *perm, const double *src, double *dst4) {
    k_gather_vec<<<blocks_for(4 * (int64_t)n_rows, 256), 256, 0, st>>>(n_rows, perm, src, dst4);
}

void launch_scatter_vec(cudaStream_t st, int n_rows, const int *perm, const double *src4, double *dst) {
    k_scatter_vec<<<blocks_for(3 * (int64_t)n_rows, 256), 256, 0, st>>>(n_rows, perm, src4, dst);
}

void launch_diag_inv(cudaStream_t st, int n_rows, const int *diag_slot, const double *val,
                     double *dinv) {
    k_diag_inv<<<blocks_for(n_rows, 128), 128, 0, st>>>(n_rows, diag_slot, val, dinv);
}

void launch_pose_update(cudaStream_t st, int n_rows, const int *iperm, const double *x4,
                        double *poses, double *dx, int wrap, double *block_sums, int n_blocks,
                        double *diff_out, const PcgResult *guard) {
    k_pose_update<<<n_blocks, 256, 0, st>>>(n_rows, iperm, x4, poses, dx, wrap, block_sums, guard);
    k_finish_diff<<<1, 32, 0, st>>>(n_blocks, block_sums, 3.0 * n_rows, diff_out);
}

/* ------------------------------------------------------------------------ */
/* landmark map (GSLAM.c:141-196, MapEdge.c:7-32, vec_mean MatrixOps.c:161-171) */
/* ------------------------------------------------------------------------ */

/* one thread per landmark: mean over its observations (z order, sums from 0.0) of
 * (x + r cos(theta + phi), y + r sin(theta + phi)) at the observing pose */
__global__ void k_landmark_map(int n_groups, const int64_t *__restrict__ ptr, const unsigned *__restrict__ members,
                               const unsigned *__restrict__ z_step, const double *__restrict__ z_rb,
                               const double *__restrict__ poses, double *__restrict__ ms) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n_groups) return;
    double m0 = 0.0, m1 = 0.0;
    const int64_t a = ptr[g], b = ptr[g + 1];
    for (int64_t q = a; q < b; q++) {
        const unsigned z = members[q];
        const double *x = poses + 3 * (size_t)z_step[z];
        double s, c;
        cr_sincos(x[2] + z_rb[2 * (size_t)z + 1], &s, &c);
        m0 = m0 + (x[0] + z_rb[2 * (size_t)z] * c);
        m1 = m1 + (x[1] + z_rb[2 * (size_t)z] * s);
    }
    ms[2 * g] = m0 / (double)(b - a);
    ms[2 * g + 1] = m1 / (double)(b - a);
}

void launch_landmark_map(cudaStream_t st, int n_groups, const int64_t *ptr, const unsigned *members,
                         const unsigned *z_step, const double *z_rb, const double *poses, double *ms) {
    if (n_groups > 0)
        k_landmark_map<<<blocks_for(n_groups, 128), 128, 0, st>>>(n_groups, ptr, members, z_step, z_rb, poses, ms);
}

int edge_cost_blocks(int64_t n_edges) { return (int)blocks_for(n_edges > 0 ? n_edges : 1, 128); }

void launch_edge_costs(cudaStream_t st, int64_t n_obs_edges, int n_poses, const unsigned *pj, const unsigned *pk,
                       const unsigned *z_step, const double *z_rb, const double *controls, double delta,
                       double lambda, const double *mns, const double *poses, double *edge_cost,
                       double *block_sums, double *total) {
    const int64_t n_edges = n_obs_edges + (n_poses > 1 ? n_poses - 1 : 0);
    const int nb = edge_cost_blocks(n_edges);
    k_edge_costs<<<nb, 128, 0, st>>>(n_obs_edges, n_poses, pj, pk, z_step, z_rb, controls, delta, lambda,
                                     mns[0], mns[1], mns[2], mns[3], poses, edge_cost, block_sums);
    k_finish_cost<<<1, 32, 0, st>>>(nb, block_sums, total);
}
