/*
 * pcg.cu — the persistent block-Jacobi PCG solver (reference MatrixOps.c:281-391,
 * GPU twin device_graph.cu:842-913) and standalone SpMV kernels.
 *
 * One cooperative launch runs the whole solve. Each warp owns whole slices of
 * 32 block rows (one row per lane) for the entire solve, so a row's q, p, x, r,
 * z never leave the thread that owns them between phases. Per iteration:
 *   phase A: p = z + beta p (own rows; gathered columns recompute it from z and
 *            the previous p, identically), q = A p, partial p.q
 *            -> grid reduction 1
 *   phase B: alpha = rz / pq; x += alpha p; r -= alpha q; z = D^-1 r;
 *            partial r.r and r.z -> grid reduction 2
 * Two grid-wide synchronisations per iteration and no host round trip, where the
 * reference GPU twin issues ~8 launches and 3 blocking scalar reads.
 *
 * Determinism: every reduction sums per-thread partials in row order, then a
 * fixed shuffle tree, then warps in order, then CTAs in order; every CTA
 * computes the same scalars. Row sums of the SpMV add in ascending original
 * column order with separate multiply and add (compiled -fmad=false): q is
 * bit-identical to the reference's sequential SpMV (MatrixOps.c:349-353).
 *
 * Waits are bounded: a barrier that spins longer than spin_limit cycles raises
 * a shared abort flag; every CTA then leaves the solve and the host reports
 * GSLAM_ERR_DEVICE_TIMEOUT.
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "gslam.h"
#include "kernels.cuh"
#include "pcg_common.cuh"

/* ------------------------------------------------------------------------ */
/* grid barrier                                                              */
/* ------------------------------------------------------------------------ */

/* ------------------------------------------------------------------------ */
/* FP64 persistent PCG                                                       */
/* ------------------------------------------------------------------------ */

/*
 * ONE: every warp owns at most one slice, so a row's p and q stay in registers
 * from phase A to phase B; otherwise they go through memory.
 */
template <int BS, bool ONE>
__global__ void __launch_bounds__(BS, 1) k_pcg64(PcgParams P) {
    __shared__ double s_red[3][BS / 32];
    __shared__ double s_bc[4];
    __shared__ int s_ok;
    const int lane = threadIdx.x & 31;
    const int gw = blockIdx.x * (BS / 32) + (threadIdx.x >> 5);
    const int TW = gridDim.x * (BS / 32);
    int epoch = 0;
    /* Test hook for the bounded wait: this CTA leaves without arriving, so every
     * other CTA's first barrier runs out of time and the solve reports a timeout. */
    if ((int)blockIdx.x == P.absent_cta) return;

    /* x = 0, r = b, z = D^-1 r (MatrixOps.c:322-345) */
    double acc2[2] = { 0.0, 0.0 };
    for (int s = gw; s < P.n_slices; s += TW) {
        const int row = 32 * s + lane;
        if (row >= P.n_rows) continue;
        const V3 b = ldg3(P.b4, row);
        st3(P.x4, row, V3{ 0.0, 0.0, 0.0 });
        st3(P.r4, row, b);
        const V3 z = apply_dinv(P.dinv, row, b);
        st3(P.z4, row, z);
        acc2[0] = acc2[0] + b.a * z.a; acc2[0] = acc2[0] + b.b * z.b; acc2[0] = acc2[0] + b.c * z.c;
        acc2[1] = acc2[1] + b.a * b.a; acc2[1] = acc2[1] + b.b * b.b; acc2[1] = acc2[1] + b.c * b.c;
    }
    if (!grid_allreduce<2, BS>(acc2, P.partials, epoch, P.gs, P.spin_limit, s_red, s_bc, &s_ok)) {
        if (threadIdx.x == 0) res_mark_timeout(P.res);
        return;
    }
    double rz = acc2[0];
    const double bnorm = sqrt(acc2[1]);
    const double tol = P.tol_rel * bnorm;
    double beta = 0.0, rr = acc2[1];
    int k = 0, reason = GSLAM_STOP_MAXIT;

    /* ONE-path row state */
    const int my_row = 32 * gw + lane;
    const bool mine = ONE && gw < P.n_slices && my_row < P.n_rows;
    int my_len = 0;
    const double *my_vb = nullptr;
    const int *my_cb = nullptr;
    if (mine) {
        my_len = __ldg(P.row_len + my_row);
        const int64_t sb = __ldg(P.slice_ptr + gw);
        my_vb = P.val + 9 * sb + lane;
        my_cb = P.col + sb + lane;
    }
    V3 pn_r = { 0.0, 0.0, 0.0 }, q_r = { 0.0, 0.0, 0.0 };

    while (true) {
        if (k >= P.max_iter) { reason = GSLAM_STOP_MAXIT; break; }
        const bool first = (k == 0);
        double *pnew = (k & 1) ? P.p4b : P.p4a;
        const double *pold = (k & 1) ? P.p4a : P.p4b;
        /* ---- phase A: p, q = A p, p.q ---- */
        double pq[1] = { 0.0 };
        if (ONE) {
            if (mine) {
                pn_r = p_of(P.z4, pold, my_row, beta, first);
                st3(pnew, my_row, pn_r);
                q_r = spmv_row(my_vb, my_cb, my_len, P.z4, pold, beta, first);
                pq[0] = pq[0] + pn_r.a * q_r.a; pq[0] = pq[0] + pn_r.b * q_r.b; pq[0] = pq[0] + pn_r.c * q_r.c;
            }
        } else {
            for (int s = gw; s < P.n_slices; s += TW) {
                const int row = 32 * s + lane;
                if (row >= P.n_rows) continue;
                const V3 pn = p_of(P.z4, pold, row, beta, first);
                st3(pnew, row, pn);
                const int64_t sb = __ldg(P.slice_ptr + s);
                const V3 q = spmv_row(P.val + 9 * sb + lane, P.col + sb + lane, __ldg(P.row_len + row),
                                      P.z4, pold, beta, first);
                st3(P.q4, row, q);
                pq[0] = pq[0] + pn.a * q.a; pq[0] = pq[0] + pn.b * q.b; pq[0] = pq[0] + pn.c * q.c;
            }
        }
        if (!grid_allreduce<1, BS>(pq, P.partials, epoch, P.gs, P.spin_limit, s_red, s_bc, &s_ok)) {
            reason = GSLAM_STOP_TIMEOUT;
            break;
        }
        if (pq[0] == 0.0) { reason = GSLAM_STOP_PQ_ZERO; break; }
        const double alpha = rz / pq[0];
        /* ---- phase B: x, r, z, r.r, r.z ---- */
        double rs[2] = { 0.0, 0.0 };
        for (int s = gw; s < (ONE ? min(gw + 1, P.n_slices) : P.n_slices); s += TW) {
            const int row = 32 * s + lane;
            if (row >= P.n_rows) continue;
            const V3 pn = ONE ? pn_r : ld3(pnew, row);
            const V3 q = ONE ? q_r : ld3(P.q4, row);
            V3 x = ld3(P.x4, row), r = ld3(P.r4, row);
            x.a = x.a + alpha * pn.a; x.b = x.b + alpha * pn.b; x.c = x.c + alpha * pn.c;
            r.a = r.a - alpha * q.a;  r.b = r.b - alpha * q.b;  r.c = r.c - alpha * q.c;
            st3(P.x4, row, x);
            st3(P.r4, row, r);
            rs[0] = rs[0] + r.a * r.a; rs[0] = rs[0] + r.b * r.b; rs[0] = rs[0] + r.c * r.c;
            const V3 z = apply_dinv(P.dinv, row, r);
            st3(P.z4, row, z);
            rs[1] = rs[1] + r.a * z.a; rs[1] = rs[1] + r.b * z.b; rs[1] = rs[1] + r.c * z.c;
        }
        if (!grid_allreduce<2, BS>(rs, P.partials, epoch, P.gs, P.spin_limit, s_red, s_bc, &s_ok)) {
            reason = GSLAM_STOP_TIMEOUT;
            break;
        }
        k++;
        rr = rs[0];
        if (sqrt(rr) < tol) { reason = GSLAM_STOP_TOL; break; }
        beta = rs[1] / rz;
        rz = rs[1];
    }
    if (reason == GSLAM_STOP_TIMEOUT && threadIdx.x == 0) {
        res_mark_timeout(P.res);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && reason != GSLAM_STOP_TIMEOUT) {
        res_finish(P.res, P.gs, k, reason, 0, sqrt(rr), bnorm);
    }
}

/* ------------------------------------------------------------------------ */
/* standalone SpMV                                                           */
/* ------------------------------------------------------------------------ */

__global__ void k_spmv64(int n_rows, int n_slices, const int64_t *__restrict__ slice_ptr,
                         const int *__restrict__ row_len, const int *__restrict__ col,
                         const double *__restrict__ val, const double *__restrict__ x4,
                         double *__restrict__ y4) {
    const int lane = threadIdx.x & 31;
    const int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (s >= n_slices) return;
    const int row = 32 * s + lane;
    if (row >= n_rows) return;
    const int len = __ldg(row_len + row);
    const int64_t sb = __ldg(slice_ptr + s);
    /* p_of with first = true reads x4 only: q = A x */
    st3(y4, row, spmv_row(val + 9 * sb + lane, col + sb + lane, len, x4, x4, 0.0, true));
}

__global__ void k_spmv32(int n_rows, int n_slices, const int64_t *__restrict__ slice_ptr,
                         const int *__restrict__ row_len, const int *__restrict__ col,
                         const float *__restrict__ val, const float *__restrict__ x4,
                         float *__restrict__ y4) {
    const int lane = threadIdx.x & 31;
    const int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (s >= n_slices) return;
    const int row = 32 * s + lane;
    if (row >= n_rows) return;
    const int len = row_len[row];
    const int64_t sb = slice_ptr[s];
    const float *vb = val + 9 * sb + lane;
    const int *cb = col + sb + lane;
    float q0 = 0.f, q1 = 0.f, q2 = 0.f;
    for (int j = 0; j < len; j++) {
        const int c = cb[32 * j];
        const float *v = vb + 288 * j;
        const float4 pc = *reinterpret_cast<const float4 *>(x4 + 4 * (size_t)c);
        q0 = __fmaf_rn(v[0], pc.x, q0);   q0 = __fmaf_rn(v[32], pc.y, q0);  q0 = __fmaf_rn(v[64], pc.z, q0);
        q1 = __fmaf_rn(v[96], pc.x, q1);  q1 = __fmaf_rn(v[128], pc.y, q1); q1 = __fmaf_rn(v[160], pc.z, q1);
        q2 = __fmaf_rn(v[192], pc.x, q2); q2 = __fmaf_rn(v[224], pc.y, q2); q2 = __fmaf_rn(v[256], pc.z, q2);
    }
    *reinterpret_cast<float4 *>(y4 + 4 * (size_t)row) = make_float4(q0, q1, q2, 0.f);
}

/* ------------------------------------------------------------------------ */
/* launchers                                                                 */
/* ------------------------------------------------------------------------ */

template <int BS>
static const void *pcg_fn(bool one) {
    return one ? (const void *)k_pcg64<BS, true> : (const void *)k_pcg64<BS, false>;
}

static const void *pcg_kernel(int block, bool one) {
    switch (block) {
        case 256: return pcg_fn<256>(one);
        case 512: return pcg_fn<512>(one);
        case 1024: return pcg_fn<1024>(one);
        default: return nullptr;
    }
}

cudaError_t launch_pcg(cudaStream_t st, const PcgParams &p, int precision, int grid, int block) {
    (void)precision;
    const bool one = (int64_t)grid * (block / 32) >= p.n_slices;
    const void *fn = pcg_kernel(block, one);
    if (!fn) return cudaErrorInvalidValue;
    PcgParams copy = p;
    void *args[] = { &copy };
    return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(block), args, 0, st);
}

int pcg_max_grid(int precision, int block, int device) {
    (void)precision;
    int n_sm = 0, per_sm = 0, per_sm2 = 0;
    if (cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return 0;
    const void *f1 = pcg_kernel(block, true), *f2 = pcg_kernel(block, false);
    if (!f1 || !f2) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, f1, block, 0) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm2, f2, block, 0) != cudaSuccess) return 0;
    return std::min(per_sm, per_sm2) * n_sm;
}

/*
 * Many matrices with one block pattern in one launch (the L2-busting SpMV
 * measurement): warp w handles slice w % n_slices of copy w / n_slices, whose values
 * start at val + copy * stride and whose result goes to y4 + copy * ystride.
 */
template <typename T>
__global__ void k_spmv_multi(int n_copies, int n_rows, int n_slices, const int64_t *__restrict__ slice_ptr,
                             const int *__restrict__ row_len, const int *__restrict__ col,
                             const T *__restrict__ val, int64_t stride, const T *__restrict__ x4,
                             T *__restrict__ y4, int64_t ystride) {
    const int lane = threadIdx.x & 31;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t copy = gw / n_slices;
    const int s = (int)(gw - copy * n_slices);
    if (copy >= n_copies) return;
    const int row = 32 * s + lane;
    if (row >= n_rows) return;
    const int len = __ldg(row_len + row);
    const int64_t sb = __ldg(slice_ptr + s);
    const T *vb = val + copy * stride + 9 * sb + lane;
    const int *cb = col + sb + lane;
    T q0 = 0, q1 = 0, q2 = 0;
    int j = 0;
    for (; j + 1 < len; j += 2) {
        const int c0 = __ldg(cb + 32 * j), c1 = __ldg(cb + 32 * (j + 1));
        const T *p0 = x4 + 4 * (size_t)c0, *p1 = x4 + 4 * (size_t)c1;
        const T a0 = __ldg(p0), a1 = __ldg(p0 + 1), a2 = __ldg(p0 + 2);
        const T b0 = __ldg(p1), b1 = __ldg(p1 + 1), b2 = __ldg(p1 + 2);
        const T *v0 = vb + 288 * j, *v1 = v0 + 288;
        q0 = q0 + __ldg(v0) * a0;       q0 = q0 + __ldg(v0 + 32) * a1;  q0 = q0 + __ldg(v0 + 64) * a2;
        q1 = q1 + __ldg(v0 + 96) * a0;  q1 = q1 + __ldg(v0 + 128) * a1; q1 = q1 + __ldg(v0 + 160) * a2;
        q2 = q2 + __ldg(v0 + 192) * a0; q2 = q2 + __ldg(v0 + 224) * a1; q2 = q2 + __ldg(v0 + 256) * a2;
        q0 = q0 + __ldg(v1) * b0;       q0 = q0 + __ldg(v1 + 32) * b1;  q0 = q0 + __ldg(v1 + 64) * b2;
        q1 = q1 + __ldg(v1 + 96) * b0;  q1 = q1 + __ldg(v1 + 128) * b1; q1 = q1 + __ldg(v1 + 160) * b2;
        q2 = q2 + __ldg(v1 + 192) * b0; q2 = q2 + __ldg(v1 + 224) * b1; q2 = q2 + __ldg(v1 + 256) * b2;
    }
    if (j < len) {
        const int c0 = __ldg(cb + 32 * j);
        const T *p0 = x4 + 4 * (size_t)c0;
        const T a0 = __ldg(p0), a1 = __ldg(p0 + 1), a2 = __ldg(p0 + 2);
        const T *v0 = vb + 288 * j;
        q0 = q0 + __ldg(v0) * a0;       q0 = q0 + __ldg(v0 + 32) * a1;  q0 = q0 + __ldg(v0 + 64) * a2;
        q1 = q1 + __ldg(v0 + 96) * a0;  q1 = q1 + __ldg(v0 + 128) * a1; q1 = q1 + __ldg(v0 + 160) * a2;
        q2 = q2 + __ldg(v0 + 192) * a0; q2 = q2 + __ldg(v0 + 224) * a1; q2 = q2 + __ldg(v0 + 256) * a2;
    }
    T *y = y4 + copy * ystride + 4 * (size_t)row;
    y[0] = q0;
    y[1] = q1;
    y[2] = q2;
}

void launch_spmv_multi64(cudaStream_t st, int n_copies, int n_rows, int n_slices, const int64_t *slice_ptr,
                         const int *row_len, const int *col, const double *val, int64_t stride,
                         const double *x4, double *y4, int64_t ystride) {
    const int64_t nthreads = 32 * (int64_t)n_slices * n_copies;
    k_spmv_multi<double><<<(unsigned)((nthreads + 255) / 256), 256, 0, st>>>(
        n_copies, n_rows, n_slices, slice_ptr, row_len, col, val, stride, x4, y4, ystride);
}

void launch_spmv_multi32(cudaStream_t st, int n_copies, int n_rows, int n_slices, const int64_t *slice_ptr,
                         const int *row_len, const int *col, const float *val, int64_t stride,
                         const float *x4, float *y4, int64_t ystride) {
    const int64_t nthreads = 32 * (int64_t)n_slices * n_copies;
    k_spmv_multi<float><<<(unsigned)((nthreads + 255) / 256), 256, 0, st>>>(
        n_copies, n_rows, n_slices, slice_ptr, row_len, col, val, stride, x4, y4, ystride);
}

void launch_spmv64(cudaStream_t st, int n_rows, int n_slices, const int64_t *slice_ptr,
                   const int *row_len, const int *col, const double *val, const double *x4,
                   double *y4) {
    const int threads = 256;
    const int64_t nthreads = 32 * (int64_t)n_slices;
    k_spmv64<<<(unsigned)((nthreads + threads - 1) / threads), threads, 0, st>>>(
        n_rows, n_slices, slice_ptr, row_len, col, val, x4, y4);
}

void launch_spmv32(cudaStream_t st, int n_rows, int n_slices, const int64_t *slice_ptr,
                   const int *row_len, const int *col, const float *val, const float *x4,
                   float *y4) {
    const int threads = 256;
    const int64_t nthreads = 32 * (int64_t)n_slices;
    k_spmv32<<<(unsigned)((nthreads + threads - 1) / threads), threads, 0, st>>>(
        n_rows, n_slices, slice_ptr, row_len, col, val, x4, y4);
}
