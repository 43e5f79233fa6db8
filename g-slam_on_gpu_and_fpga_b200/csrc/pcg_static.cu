/*
 * pcg_static.cu — block-Jacobi PCG on a caller's device CSR that allocates nothing.
 *
 * Who this is for: callers that cannot allocate device memory at solve time —
 * processes whose device memory is owned by another allocator or budgeted up front
 * (a serving process with a fixed pool, an embedded controller), or a real-time
 * loop that must not call cudaMalloc because it can block or fail. Every other
 * entry point of the library allocates its buffers when a graph is created.
 *
 * The solver's scratch (work vectors, block-Jacobi inverses, reduction partials,
 * barrier counter, status) lives in one file-scope __device__ array of
 * GSLAM_STATIC_SCRATCH_BYTES. Every GPU that loads the library holds that array
 * until the process exits. Host code must not pass the array's name to a kernel
 * (in host code it is only a stand-in symbol): its device address is looked up
 * once per device with cudaGetSymbolAddress, on the first call made with that
 * device current, and cached. That first call should therefore happen before any
 * stream capture begins.
 *
 * All calls share the one array: calls that overlap on the GPU (different streams,
 * or different host threads on the same device) race on it and must be serialised
 * by the caller. The counter and status words are cleared at the start of every
 * call; everything else is written before it is read.
 *
 * The arithmetic is the reference's pcg_solve_sparse (src/cpu_pcg_fp64/MatrixOps.c:
 * 281-391): each scalar row of q = A p sums its CSR entries in stored order, the
 * diagonal 3x3 blocks are inverted by the same cofactor expressions, and a grid of
 * one cooperative launch runs the whole solve with two deterministic reductions per
 * iteration (the streamed solver of pcg.cu, reading the matrix in CSR).
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "gslam.h"
#include "gslam_api_internal.h"
#include "kernels.cuh"
#include "pcg_common.cuh"

#define GSLAM_STATIC_MAX_DEVICES 64
#define STATIC_BLOCK 256

/* the scratch array (see the file comment) */
static __device__ __align__(256) unsigned char g_static_scratch[GSLAM_STATIC_SCRATCH_BYTES];

struct StaticLayout {
    double *r, *z, *pa, *pb, *q, *dinv, *partials;
    GridSync *gs;
    PcgResult *res;
};

/* Carves the scratch for n block rows and `grid` CTAs; false if it does not fit. */
static bool static_layout(unsigned char *base, int64_t nb, int grid, StaticLayout *L) {
    size_t off = 0;
    auto take = [&](size_t bytes) {
        unsigned char *p = base + off;
        off += (bytes + 255) / 256 * 256;
        return p;
    };
    /* status words first, at a fixed offset, so gslam_pcg_static_status finds them
     * without knowing the last call's sizes */
    L->res = (PcgResult *)take(sizeof(PcgResult));
    L->gs = (GridSync *)take(sizeof(GridSync));
    const size_t v = 3 * (size_t)nb * sizeof(double);
    L->r = (double *)take(v);
    L->z = (double *)take(v);
    L->pa = (double *)take(v);
    L->pb = (double *)take(v);
    L->q = (double *)take(v);
    L->dinv = (double *)take(9 * (size_t)nb * sizeof(double));
    L->partials = (double *)take(8 * (size_t)grid * sizeof(double));
    return off <= (size_t)GSLAM_STATIC_SCRATCH_BYTES;
}

struct CsrPcgParams {
    int nb;
    const int *row_ptr;
    const int *col;
    const double *val;
    const double *b;
    double *x;
    double tol_rel;
    int max_iter;
    long long spin_limit;
    StaticLayout S;
};

/* p at scalar index c, formed on the fly exactly as MatrixOps.c:382 writes it. */
__device__ __forceinline__ double p_at(const double *z, const double *pold, int c, double beta,
                                       bool first) {
    const double zc = __ldcg(z + c);
    return first ? zc : zc + beta * __ldcg(pold + c);
}

template <int BS>
__global__ void __launch_bounds__(BS) k_pcg64_csr(CsrPcgParams P) {
    __shared__ double s_red[3][BS / 32];
    __shared__ double s_bc[4];
    __shared__ int s_ok;
    int epoch = 0;
    const int tid = blockIdx.x * BS + threadIdx.x, nthr = gridDim.x * BS;
    StaticLayout &S = P.S;

    /* D^-1 from the CSR diagonal blocks (MatrixOps.c:287-315), x = 0, r = b, z = D^-1 r */
    double acc2[2] = { 0.0, 0.0 };
    for (int I = tid; I < P.nb; I += nthr) {
        const int base = 3 * I;
        double a[9] = { 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0 };
        for (int rr = 0; rr < 3; rr++)
            for (int p = P.row_ptr[base + rr]; p < P.row_ptr[base + rr + 1]; p++) {
                const int c = P.col[p] - base;
                if (c >= 0 && c < 3) a[rr * 3 + c] = P.val[p];
            }
        double det = a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
                     a[2] * (a[3] * a[7] - a[4] * a[6]);
        if (det == 0.0) det = 1e-30;
        double d[9];
        d[0] = (a[4] * a[8] - a[5] * a[7]) / det;
        d[1] = (a[2] * a[7] - a[1] * a[8]) / det;
        d[2] = (a[1] * a[5] - a[2] * a[4]) / det;
        d[3] = (a[5] * a[6] - a[3] * a[8]) / det;
        d[4] = (a[0] * a[8] - a[2] * a[6]) / det;
        d[5] = (a[2] * a[3] - a[0] * a[5]) / det;
        d[6] = (a[3] * a[7] - a[4] * a[6]) / det;
        d[7] = (a[1] * a[6] - a[0] * a[7]) / det;
        d[8] = (a[0] * a[4] - a[1] * a[3]) / det;
        for (int e = 0; e < 9; e++) S.dinv[9 * (size_t)I + e] = d[e];
        double r[3], z[3];
        for (int c = 0; c < 3; c++) {
            r[c] = P.b[base + c];
            P.x[base + c] = 0.0;
            S.r[base + c] = r[c];
        }
        for (int rr = 0; rr < 3; rr++) {
            z[rr] = 0.0;
            for (int c = 0; c < 3; c++) z[rr] = z[rr] + d[rr * 3 + c] * r[c];
            S.z[base + rr] = z[rr];
        }
        for (int c = 0; c < 3; c++) acc2[0] = acc2[0] + r[c] * z[c];
        for (int c = 0; c < 3; c++) acc2[1] = acc2[1] + r[c] * r[c];
    }
    if (!grid_allreduce<2, BS>(acc2, S.partials, epoch, S.gs, P.spin_limit, s_red, s_bc, &s_ok)) {
        if (threadIdx.x == 0) res_mark_timeout(S.res);
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
        double *pnew = (k & 1) ? S.pb : S.pa;
        const double *pold = (k & 1) ? S.pa : S.pb;
        double pq[1] = { 0.0 };
        for (int I = tid; I < P.nb; I += nthr) {
            for (int r3 = 0; r3 < 3; r3++) {
                const int R = 3 * I + r3;
                const double pn = p_at(S.z, pold, R, beta, first);
                pnew[R] = pn;
                double q = 0.0;
                for (int p = P.row_ptr[R]; p < P.row_ptr[R + 1]; p++)
                    q = q + P.val[p] * p_at(S.z, pold, P.col[p], beta, first);
                S.q[R] = q;
                pq[0] = pq[0] + pn * q;
            }
        }
        if (!grid_allreduce<1, BS>(pq, S.partials, epoch, S.gs, P.spin_limit, s_red, s_bc, &s_ok)) {
            reason = GSLAM_STOP_TIMEOUT;
            break;
        }
        if (pq[0] == 0.0) { reason = GSLAM_STOP_PQ_ZERO; break; }
        const double alpha = rz / pq[0];
        double rs[2] = { 0.0, 0.0 };
        for (int I = tid; I < P.nb; I += nthr) {
            const int base = 3 * I;
            double r[3];
            for (int c = 0; c < 3; c++) {
                P.x[base + c] = P.x[base + c] + alpha * pnew[base + c];
                r[c] = S.r[base + c] - alpha * S.q[base + c];
                S.r[base + c] = r[c];
                rs[0] = rs[0] + r[c] * r[c];
            }
            const double *d = S.dinv + 9 * (size_t)I;
            for (int r3 = 0; r3 < 3; r3++) {
                double z = 0.0;
                for (int c = 0; c < 3; c++) z = z + d[r3 * 3 + c] * r[c];
                S.z[base + r3] = z;
                rs[1] = rs[1] + r[r3] * z;
            }
        }
        if (!grid_allreduce<2, BS>(rs, S.partials, epoch, S.gs, P.spin_limit, s_red, s_bc, &s_ok)) {
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
        res_mark_timeout(S.res);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && reason != GSLAM_STOP_TIMEOUT) {
        res_finish(S.res, S.gs, k, reason, 0, sqrt(rr), bnorm);
    }
}

/* per-device device address of the scratch array and launch shape, set up once */
struct StaticDevice {
    bool ready = false;
    unsigned char *base = nullptr;
    int grid = 0;
    int clock_khz = 0;
};
static StaticDevice g_static_dev[GSLAM_STATIC_MAX_DEVICES];
static std::mutex g_static_mu;

/* Copies the status words of the last solve queued on this device into *stats, after
 * the work queued on `st` so far (the solve, when the caller queued it on `st`). */
static int static_read_status(const PcgResult *d_res, cudaStream_t st, gslam_solve_stats *stats) {
    PcgResult h;
    if (cudaMemcpyAsync(&h, d_res, sizeof h, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        gslam_set_last_error("gslam_pcg_solve_static: reading the status failed");
        return GSLAM_ERR_CUDA;
    }
    stats->iterations = h.iterations;
    stats->refinements = 0;
    stats->reason = h.timeout ? GSLAM_STOP_TIMEOUT : h.reason;
    stats->rel_residual = h.bnorm > 0 ? h.rnorm / h.bnorm : 0.0;
    stats->diff = 0.0;
    stats->solve_ms = 0.0;
    stats->round_ms = 0.0;
    if (h.timeout) {
        gslam_set_last_error("gslam_pcg_solve_static: solver barrier wait timed out");
        return GSLAM_ERR_DEVICE_TIMEOUT;
    }
    return GSLAM_OK;
}

extern "C" int gslam_pcg_solve_static(int dim, const int *d_row_ptr, const int *d_col_idx,
                                      const double *d_values, const double *d_b, double *d_x,
                                      double tol, int max_iter, void *stream,
                                      gslam_solve_stats *stats) {
    if (dim <= 0 || dim % 3 != 0 || !d_row_ptr || !d_col_idx || !d_values || !d_b || !d_x ||
        max_iter < 0) {
        gslam_set_last_error("gslam_pcg_solve_static: needs dim % 3 == 0 and non-null device arrays");
        return GSLAM_ERR_BAD_INPUT;
    }
    const int nb = dim / 3;
    if (nb > GSLAM_STATIC_MAX_POSES) {
        gslam_set_last_error("gslam_pcg_solve_static: more poses than the fixed scratch holds "
                             "(GSLAM_STATIC_MAX_POSES = 16384)");
        return GSLAM_ERR_TOO_LARGE;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= GSLAM_STATIC_MAX_DEVICES) {
        gslam_set_last_error("gslam_pcg_solve_static: no current CUDA device");
        return GSLAM_ERR_NO_DEVICE;
    }
    StaticDevice *D = &g_static_dev[dev];
    {
        std::lock_guard<std::mutex> lock(g_static_mu);
        if (!D->ready) {
            void *ptr = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&ptr, g_static_scratch);
            if (e != cudaSuccess || !ptr) {
                gslam_set_last_error("gslam_pcg_solve_static: cudaGetSymbolAddress failed");
                return GSLAM_ERR_CUDA;
            }
            int n_sm = 0, per_sm = 0, khz = 0;
            if (cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)k_pcg64_csr<STATIC_BLOCK>,
                                                              STATIC_BLOCK, 0) != cudaSuccess ||
                per_sm <= 0) {
                gslam_set_last_error("gslam_pcg_solve_static: cooperative launch not possible");
                return GSLAM_ERR_NO_DEVICE;
            }
            if (cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, dev) != cudaSuccess || khz <= 0)
                khz = 2000000;
            D->base = (unsigned char *)ptr;
            D->grid = std::min(per_sm, 2) * n_sm;
            D->clock_khz = khz;
            D->ready = true;
        }
    }
    const int grid = std::max(1, std::min(D->grid, (nb + STATIC_BLOCK - 1) / STATIC_BLOCK));
    CsrPcgParams P;
    if (!static_layout(D->base, nb, grid, &P.S)) {
        gslam_set_last_error("gslam_pcg_solve_static: more poses than the fixed scratch holds "
                             "(GSLAM_STATIC_MAX_POSES = 16384)");
        return GSLAM_ERR_TOO_LARGE;
    }
    if ((2.0 * max_iter + 4.0) * grid >= 4294967295.0) {
        gslam_set_last_error("gslam_pcg_solve_static: max_iter too large");
        return GSLAM_ERR_TOO_LARGE;
    }
    P.nb = nb;
    P.row_ptr = d_row_ptr;
    P.col = d_col_idx;
    P.val = d_values;
    P.b = d_b;
    P.x = d_x;
    P.tol_rel = tol;
    P.max_iter = max_iter;
    P.spin_limit = (long long)(2000.0 * (double)D->clock_khz); /* 2 s */
    cudaStream_t st = (cudaStream_t)stream;
    /* counter, abort flag and status start at zero on every call */
    if (cudaMemsetAsync(P.S.gs, 0, sizeof(GridSync), st) != cudaSuccess ||
        cudaMemsetAsync(P.S.res, 0, sizeof(PcgResult), st) != cudaSuccess) {
        gslam_set_last_error("gslam_pcg_solve_static: clearing the scratch failed");
        return GSLAM_ERR_CUDA;
    }
    void *args[] = { &P };
    cudaError_t e = cudaLaunchCooperativeKernel((const void *)k_pcg64_csr<STATIC_BLOCK>, dim3(grid),
                                                dim3(STATIC_BLOCK), args, 0, st);
    if (e != cudaSuccess) {
        gslam_set_last_error(cudaGetErrorString(e));
        return GSLAM_ERR_CUDA;
    }
    if (stats) return static_read_status(P.S.res, st, stats);
    return GSLAM_OK;
}

extern "C" int gslam_pcg_static_status(void *stream, gslam_solve_stats *stats) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= GSLAM_STATIC_MAX_DEVICES) {
        gslam_set_last_error("gslam_pcg_static_status: no current CUDA device");
        return GSLAM_ERR_NO_DEVICE;
    }
    unsigned char *base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_static_mu);
        if (g_static_dev[dev].ready) base = g_static_dev[dev].base;
    }
    if (!base) {
        gslam_set_last_error("gslam_pcg_static_status: no gslam_pcg_solve_static call on this device yet");
        return GSLAM_ERR_BAD_INPUT;
    }
    gslam_solve_stats local;
    StaticLayout L;
    static_layout(base, 0, 0, &L); /* only the status words, at their fixed offset */
    return static_read_status(L.res, (cudaStream_t)stream, stats ? stats : &local);
}
