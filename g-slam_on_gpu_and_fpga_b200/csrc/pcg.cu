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

#include "gslam.h"
#include "kernels.cuh"

/* ------------------------------------------------------------------------ */
/* grid barrier                                                              */
/* ------------------------------------------------------------------------ */

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_u32(unsigned *p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ int ld_relaxed_s32(const int *p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

/* Returns false when the solve must be abandoned (timeout here or elsewhere). */
__device__ __forceinline__ bool grid_barrier(GridSync *gs, long long spin_limit, int *s_ok) {
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        __threadfence();
        const unsigned gen = ld_acquire_u32(&gs->gen);
        const unsigned arrived = atomicAdd(&gs->count, 1u) + 1u;
        if (arrived == gridDim.x) {
            atomicExch(&gs->count, 0u);
            __threadfence();
            st_release_u32(&gs->gen, gen + 1u);
        } else {
            const long long t0 = clock64();
            while (ld_acquire_u32(&gs->gen) == gen) {
                if (ld_relaxed_s32(&gs->abort)) { ok = 0; break; }
                if (clock64() - t0 > spin_limit) {
                    atomicExch(&gs->abort, 1);
                    ok = 0;
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
        *s_ok = ok;
    }
    __syncthreads();
    return *s_ok != 0;
}

/*
 * Deterministic all-reduce of NV doubles across the grid. v[] holds this
 * thread's partials on entry and the grid totals on exit.
 */
template <int NV, int BS>
__device__ __forceinline__ bool grid_allreduce(double (&v)[NV], double *partials_base, int &epoch,
                                               GridSync *gs, long long spin_limit,
                                               double (*s_red)[BS / 32], double *s_bc, int *s_ok) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    /* Two partial buffers alternate: a CTA can be at most one reduction ahead of
     * the slowest reader, so it never overwrites partials still being summed. */
    double *partials = partials_base + (epoch & 1) * 4 * gridDim.x;
    epoch++;
#pragma unroll
    for (int i = 0; i < NV; i++) {
        double a = v[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) a = a + __shfl_down_sync(0xffffffffu, a, o);
        if (lane == 0) s_red[i][warp] = a;
    }
    __syncthreads();
    if (threadIdx.x < NV) {
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < BS / 32; w++) s = s + s_red[threadIdx.x][w];
        partials[threadIdx.x * gridDim.x + blockIdx.x] = s;
    }
    if (!grid_barrier(gs, spin_limit, s_ok)) return false;
    if (warp == 0) {
#pragma unroll
        for (int i = 0; i < NV; i++) {
            double s = 0.0;
            for (int c = lane; c < (int)gridDim.x; c += 32) s = s + partials[i * gridDim.x + c];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s = s + __shfl_down_sync(0xffffffffu, s, o);
            if (lane == 0) s_bc[i] = s;
        }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < NV; i++) v[i] = s_bc[i];
    return true;
}

/* ------------------------------------------------------------------------ */
/* FP64 persistent PCG                                                       */
/* ------------------------------------------------------------------------ */

struct V3 { double a, b, c; };

__device__ __forceinline__ V3 ld3(const double *v4, int row) {
    const double2 lo = *reinterpret_cast<const double2 *>(v4 + 4 * (size_t)row);
    const double hi = v4[4 * (size_t)row + 2];
    return V3{ lo.x, lo.y, hi };
}

__device__ __forceinline__ void st3(double *v4, int row, V3 v) {
    *reinterpret_cast<double2 *>(v4 + 4 * (size_t)row) = make_double2(v.a, v.b);
    v4[4 * (size_t)row + 2] = v.c;
}

/* p_new = z + beta * p_old exactly as MatrixOps.c:382 (first iteration: p = z). */
__device__ __forceinline__ V3 p_of(const double *z4, const double *pold4, int row, double beta,
                                   bool first) {
    V3 z = ld3(z4, row);
    if (first) return z;
    V3 p = ld3(pold4, row);
    return V3{ z.a + beta * p.a, z.b + beta * p.b, z.c + beta * p.c };
}

/* z = D^-1 r: z_i = ((0 + d_i0 r0) + d_i1 r1) + d_i2 r2 (MatrixOps.c:369-377). */
__device__ __forceinline__ V3 apply_dinv(const double *dinv, int row, V3 r) {
    const double *d = dinv + 288 * (size_t)(row >> 5) + (row & 31);
    double z0 = 0.0, z1 = 0.0, z2 = 0.0;
    z0 = z0 + d[0] * r.a;   z0 = z0 + d[32] * r.b;  z0 = z0 + d[64] * r.c;
    z1 = z1 + d[96] * r.a;  z1 = z1 + d[128] * r.b; z1 = z1 + d[160] * r.c;
    z2 = z2 + d[192] * r.a; z2 = z2 + d[224] * r.b; z2 = z2 + d[256] * r.c;
    return V3{ z0, z1, z2 };
}

template <int BS>
__global__ void __launch_bounds__(BS) k_pcg64(PcgParams P) {
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

    /* x = 0, r = b, z = D^-1 r, p.. (MatrixOps.c:322-345) */
    double acc2[2] = { 0.0, 0.0 };
    for (int s = gw; s < P.n_slices; s += TW) {
        const int row = 32 * s + lane;
        if (row >= P.n_rows) continue;
        const V3 b = ld3(P.b4, row);
        st3(P.x4, row, V3{ 0.0, 0.0, 0.0 });
        st3(P.r4, row, b);
        const V3 z = apply_dinv(P.dinv, row, b);
        st3(P.z4, row, z);
        acc2[0] = acc2[0] + b.a * z.a; acc2[0] = acc2[0] + b.b * z.b; acc2[0] = acc2[0] + b.c * z.c;
        acc2[1] = acc2[1] + b.a * b.a; acc2[1] = acc2[1] + b.b * b.b; acc2[1] = acc2[1] + b.c * b.c;
    }
    if (!grid_allreduce<2, BS>(acc2, P.partials, epoch, P.gs, P.spin_limit, s_red, s_bc, &s_ok)) {
        if (threadIdx.x == 0) { P.res->timeout = 1; P.res->reason = GSLAM_STOP_TIMEOUT; }
        return;
    }
    double rz = acc2[0];
    const double bnorm = sqrt(acc2[1]);
    const double tol = P.tol_rel * bnorm;
    double beta = 0.0, rr = acc2[1];
    int k = 0, reason = GSLAM_STOP_MAXIT;

    while (true) {
        if (k >= P.max_iter) { reason = GSLAM_STOP_MAXIT; break; }
        const bool first = (k == 0);
        double *pnew = (k & 1) ? P.p4b : P.p4a;
        const double *pold = (k & 1) ? P.p4a : P.p4b;
        /* ---- phase A: p, q = A p, p.q ---- */
        double pq[1] = { 0.0 };
        for (int s = gw; s < P.n_slices; s += TW) {
            const int row = 32 * s + lane;
            if (row >= P.n_rows) continue;
            const V3 pn = p_of(P.z4, pold, row, beta, first);
            st3(pnew, row, pn);
            const int len = P.row_len[row];
            const int64_t sb = P.slice_ptr[s];
            const double *vb = P.val + 9 * sb + lane;
            const int *cb = P.col + sb + lane;
            double q0 = 0.0, q1 = 0.0, q2 = 0.0;
            for (int j = 0; j < len; j++) {
                const int c = cb[32 * j];
                const double *v = vb + 288 * j;
                const V3 pc = p_of(P.z4, pold, c, beta, first);
                q0 = q0 + v[0] * pc.a;   q0 = q0 + v[32] * pc.b;  q0 = q0 + v[64] * pc.c;
                q1 = q1 + v[96] * pc.a;  q1 = q1 + v[128] * pc.b; q1 = q1 + v[160] * pc.c;
                q2 = q2 + v[192] * pc.a; q2 = q2 + v[224] * pc.b; q2 = q2 + v[256] * pc.c;
            }
            st3(P.q4, row, V3{ q0, q1, q2 });
            pq[0] = pq[0] + pn.a * q0; pq[0] = pq[0] + pn.b * q1; pq[0] = pq[0] + pn.c * q2;
        }
        if (!grid_allreduce<1, BS>(pq, P.partials, epoch, P.gs, P.spin_limit, s_red, s_bc, &s_ok)) {
            reason = GSLAM_STOP_TIMEOUT;
            break;
        }
        if (pq[0] == 0.0) { reason = GSLAM_STOP_PQ_ZERO; break; }
        const double alpha = rz / pq[0];
        /* ---- phase B: x, r, z, r.r, r.z ---- */
        double rs[2] = { 0.0, 0.0 };
        for (int s = gw; s < P.n_slices; s += TW) {
            const int row = 32 * s + lane;
            if (row >= P.n_rows) continue;
            const V3 pn = ld3(pnew, row);
            const V3 q = ld3(P.q4, row);
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
        P.res->timeout = 1;
        P.res->reason = GSLAM_STOP_TIMEOUT;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && reason != GSLAM_STOP_TIMEOUT) {
        P.res->iterations = k;
        P.res->reason = reason;
        P.res->refinements = 0;
        P.res->timeout = (reason == GSLAM_STOP_TIMEOUT);
        P.res->rnorm = sqrt(rr);
        P.res->bnorm = bnorm;
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
    const int len = row_len[row];
    const int64_t sb = slice_ptr[s];
    const double *vb = val + 9 * sb + lane;
    const int *cb = col + sb + lane;
    double q0 = 0.0, q1 = 0.0, q2 = 0.0;
    for (int j = 0; j < len; j++) {
        const int c = cb[32 * j];
        const double *v = vb + 288 * j;
        const V3 pc = ld3(x4, c);
        q0 = q0 + v[0] * pc.a;   q0 = q0 + v[32] * pc.b;  q0 = q0 + v[64] * pc.c;
        q1 = q1 + v[96] * pc.a;  q1 = q1 + v[128] * pc.b; q1 = q1 + v[160] * pc.c;
        q2 = q2 + v[192] * pc.a; q2 = q2 + v[224] * pc.b; q2 = q2 + v[256] * pc.c;
    }
    st3(y4, row, V3{ q0, q1, q2 });
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
static cudaError_t launch_pcg_bs(cudaStream_t st, const PcgParams &p, int precision, int grid) {
    PcgParams copy = p;
    void *args[] = { &copy };
    (void)precision;
    return cudaLaunchCooperativeKernel((const void *)k_pcg64<BS>, dim3(grid), dim3(BS), args, 0, st);
}

cudaError_t launch_pcg(cudaStream_t st, const PcgParams &p, int precision, int grid, int block) {
    switch (block) {
        case 128: return launch_pcg_bs<128>(st, p, precision, grid);
        case 256: return launch_pcg_bs<256>(st, p, precision, grid);
        case 512: return launch_pcg_bs<512>(st, p, precision, grid);
        default: return cudaErrorInvalidValue;
    }
}

int pcg_max_grid(int precision, int block, int device) {
    (void)precision;
    int n_sm = 0, per_sm = 0;
    if (cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return 0;
    const void *fn = nullptr;
    switch (block) {
        case 128: fn = (const void *)k_pcg64<128>; break;
        case 256: fn = (const void *)k_pcg64<256>; break;
        case 512: fn = (const void *)k_pcg64<512>; break;
        default: return 0;
    }
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, block, 0) != cudaSuccess) return 0;
    return per_sm * n_sm;
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
