/*
 * adjoint.cu — implicit-function adjoint of a converged SE(2) pose graph.
 *
 * Not in the reference (its programs only run Gauss-Newton forward). For the SE(2)
 * between-factors of edge_math.cuh, the converged poses x* satisfy
 *     g(x*, theta) = sum_e J_e^T Lambda_e e_e = 0,   Lambda_e = lambda diag(exp(w_e)),
 * so for a loss L(x*) the implicit-function theorem gives
 *     H mu = dL/dx,  dL/dw_{e,k} = -lambda exp(w_{e,k}) e_{e,k} (J_e mu)_k,
 *     dL/dlambda = (1 / lambda) sum_{e,k} dL/dw_{e,k},
 * where H = dg/dx is the exact Hessian of (1/2) sum_e e^T Lambda e: the Gauss-Newton
 * blocks J^T Lambda J plus the second-order terms sum_k (Lambda e)_k d2 e_k, which for
 * this factor come only from the rotated translation residual (dependence on theta_i
 * alone and on (theta_i, t_i), (theta_i, t_j)). The pose-0 anchor of the forward
 * solve stays on H's first diagonal block, pinning the gauge the same way.
 *
 * The solve reuses the library's block layout, assembly (same contribution lists,
 * per-edge blocks replaced by the exact-Hessian blocks) and the FP64 persistent PCG
 * (H is symmetric). Kernels here: the exact-Hessian edge blocks, the right-hand side
 * scatter into the solver's row order, the gather of mu back to pose order, and one
 * thread per edge for the gradient.
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "edge_math.cuh"
#include "gslam.h"
#include "gslam_api_internal.h"
#include "kernels.cuh"

/* Exact-Hessian blocks of one SE(2) edge: em_se2_edge's Gauss-Newton blocks (UL, UR,
 * BL, BR at out[0..35]) plus the second-order terms; out[36..41] (xi) are zeroed. */
__device__ void se2_hess_edge(const double *xi, const double *xj, const double *z, const double *info,
                              double lambda, double *out) {
    em_se2_edge(xi, xj, z, info, lambda, out);
    double s, c;
    cr_sincos(xi[2], &s, &c);
    const double dx = xj[0] - xi[0], dy = xj[1] - xi[1];
    const double e0 = (c * dx + s * dy) - z[0];
    const double e1 = (c * dy - s * dx) - z[1];
    const double a0 = info[0] * lambda * e0, a1 = info[1] * lambda * e1; /* (Lambda e) of e_t */
    /* sum_k a_k d2 e_k over (x_i, y_i, th_i, x_j, y_j, th_j); only th_i rows/columns */
    const double h_tt = a0 * (-(c * dx) - s * dy) + a1 * (s * dx - c * dy); /* (th_i, th_i) */
    const double h_tx = a0 * s + a1 * c;                                     /* (th_i, x_i) */
    const double h_ty = a1 * s - a0 * c;                                     /* (th_i, y_i) */
    /* UL: row/column 2 of pose i */
    out[3 * 2 + 2] += h_tt;
    out[3 * 2 + 0] += h_tx;
    out[3 * 0 + 2] += h_tx;
    out[3 * 2 + 1] += h_ty;
    out[3 * 1 + 2] += h_ty;
    /* UR (rows of pose i, columns of pose j): (th_i, x_j) = -h_tx, (th_i, y_j) = -h_ty */
    out[9 + 3 * 2 + 0] -= h_tx;
    out[9 + 3 * 2 + 1] -= h_ty;
    /* BL (rows of pose j, columns of pose i): the transpose */
    out[18 + 3 * 0 + 2] -= h_tx;
    out[18 + 3 * 1 + 2] -= h_ty;
#pragma unroll
    for (int k = 36; k < 42; k++) out[k] = 0.0;
}

__global__ void k_se2_hess_edges(int64_t n, const unsigned *__restrict__ ei, const unsigned *__restrict__ ej,
                                 const double *__restrict__ meas, const double *__restrict__ info, double lambda,
                                 const double *__restrict__ poses, double *__restrict__ blocks) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
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
    se2_hess_edge(xi, xj, z, w, lambda, out);
    double *dst = blocks + 42 * (size_t)e;
#pragma unroll
    for (int k = 0; k < 42; k++) dst[k] = out[k];
}

/* b4[row] = rhs[pose perm[row]] (3 values, padded to 4); padding rows get 0 */
__global__ void k_rhs_to_rows(int n_rows, int n_pad, const int *__restrict__ perm, const double *__restrict__ rhs,
                              double *__restrict__ b4) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_pad) return;
#pragma unroll
    for (int c = 0; c < 4; c++) b4[4 * (size_t)r + c] = (r < n_rows && c < 3) ? rhs[3 * (size_t)perm[r] + c] : 0.0;
}

/* mu[pose] = x4[iperm[pose]] */
__global__ void k_rows_to_poses(int n_rows, const int *__restrict__ iperm, const double *__restrict__ x4,
                                double *__restrict__ mu) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n_rows) return;
    const int r = iperm[p];
#pragma unroll
    for (int c = 0; c < 3; c++) mu[3 * (size_t)p + c] = x4[4 * (size_t)r + c];
}

/* dL/dw_{e,k} = -lambda exp(w_{e,k}) e_{e,k} (J_e mu)_k, one thread per edge */
__global__ void k_se2_edge_grad(int64_t n, const unsigned *__restrict__ ei, const unsigned *__restrict__ ej,
                                const double *__restrict__ meas, const double *__restrict__ info, double lambda,
                                const double *__restrict__ poses, const double *__restrict__ mu,
                                double *__restrict__ grad) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const unsigned i = ei[e], j = ej[e];
    const double *xi = poses + 3 * (size_t)i, *xj = poses + 3 * (size_t)j;
    const double *mi = mu + 3 * (size_t)i, *mj = mu + 3 * (size_t)j;
    const double *z = meas + 3 * (size_t)e;
    double s, c;
    cr_sincos(xi[2], &s, &c);
    const double dx = xj[0] - xi[0], dy = xj[1] - xi[1];
    double ev[3];
    ev[0] = (c * dx + s * dy) - z[0];
    ev[1] = (c * dy - s * dx) - z[1];
    ev[2] = em_wrap_angle((xj[2] - xi[2]) - z[2]);
    /* J_e mu = J_i mu_i + J_j mu_j with em_se2_edge's Jacobians */
    double jm[3];
    jm[0] = ((-c * mi[0] - s * mi[1]) + (c * dy - s * dx) * mi[2]) + (c * mj[0] + s * mj[1]);
    jm[1] = ((s * mi[0] - c * mi[1]) + (-(c * dx) - s * dy) * mi[2]) + (-s * mj[0] + c * mj[1]);
    jm[2] = -mi[2] + mj[2];
#pragma unroll
    for (int k = 0; k < 3; k++) grad[3 * (size_t)e + k] = -(info[3 * (size_t)e + k] * lambda) * ev[k] * jm[k];
}

static inline unsigned nblk(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

int gslam_set_se2_weights(gslam_graph *g, double lambda, const double *log_w) {
    if (!g) { gslam_set_last_error("null handle"); return GSLAM_ERR_BAD_INPUT; }
    if (g->factors != GSLAM_FACTORS_SE2 || g->batch) {
        gslam_set_last_error("weights can be replaced on single SE(2) graphs");
        return GSLAM_ERR_BAD_INPUT;
    }
    if (!(lambda > 0.0)) { gslam_set_last_error("lambda must be positive"); return GSLAM_ERR_BAD_INPUT; }
    g->lambda = lambda;
    if (log_w && g->n_edges) {
        std::vector<double> lw(3 * (size_t)g->n_edges);
        for (size_t k = 0; k < lw.size(); k++) lw[k] = std::exp(log_w[k]);
        cudaError_t e = cudaMemcpyAsync(g->d_info, lw.data(), lw.size() * sizeof(double), cudaMemcpyHostToDevice,
                                        g->st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(g->st);
        if (e != cudaSuccess) { gslam_set_last_error(cudaGetErrorString(e)); return GSLAM_ERR_CUDA; }
    }
    return GSLAM_OK;
}

int gslam_adjoint(gslam_graph *g, const double *dL_dposes, double *dL_dlambda, double *dL_dlogw,
                  double *mu_out, gslam_solve_stats *stats) {
    if (!g || !dL_dposes) { gslam_set_last_error("null argument"); return GSLAM_ERR_BAD_INPUT; }
    if (g->factors != GSLAM_FACTORS_SE2 || g->batch) {
        gslam_set_last_error("the adjoint is defined for single SE(2) graphs");
        return GSLAM_ERR_BAD_INPUT;
    }
    const int n = g->n_poses;
    const int64_t ne = g->n_edges;
    cudaError_t ce = cudaSetDevice(g->device);
    if (ce != cudaSuccess) { gslam_set_last_error(cudaGetErrorString(ce)); return GSLAM_ERR_CUDA; }
    if (!g->d_adj) {
        /* rhs, mu (3 N each) and the per-edge gradient (3 E), allocated on first use */
        const size_t cnt = 6 * (size_t)n + 3 * (size_t)(ne > 0 ? ne : 1);
        void *q = nullptr;
        if (cudaMalloc(&q, cnt * sizeof(double)) != cudaSuccess) {
            gslam_set_last_error("out of device memory (adjoint buffers)");
            return GSLAM_ERR_CUDA;
        }
        g->mem.ptrs.push_back(q);
        g->d_adj = (double *)q;
    }
    double *d_rhs = g->d_adj, *d_mu = g->d_adj + 3 * (size_t)n, *d_grad = g->d_adj + 6 * (size_t)n;
#define ACK(x) do { cudaError_t _e = (x); if (_e != cudaSuccess) { gslam_set_last_error(cudaGetErrorString(_e)); return GSLAM_ERR_CUDA; } } while (0)
    ACK(cudaMemcpyAsync(d_rhs, dL_dposes, 3 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice, g->st));
    /* H = exact Hessian at the current poses, assembled into the solver's layout */
    if (ne) k_se2_hess_edges<<<nblk(ne, 128), 128, 0, g->st>>>(ne, g->d_ei, g->d_ej, g->d_meas, g->d_info, g->lambda,
                                                               g->d_poses, g->d_blocks);
    ACK(cudaGetLastError());
    gslam_opts o = g->o;
    o.precision = GSLAM_PREC_FP64;
    const int saved_prec = g->o.precision;
    g->o.precision = GSLAM_PREC_FP64;
    int rc = gslam_assemble_ex(g, g->d_blocks, nullptr, nullptr);
    g->o.precision = saved_prec;
    if (rc != GSLAM_OK) return rc;
    /* the right-hand side replaces the assembled xi */
    const int n_pad = 32 * g->L.n_slices;
    k_rhs_to_rows<<<nblk(n_pad, 256), 256, 0, g->st>>>(n, n_pad, g->L.perm, d_rhs, g->L.b4);
    ACK(cudaGetLastError());
    gslam_solve_stats st;
    memset(&st, 0, sizeof st);
    rc = gslam_layout_solve(&g->L, g->st, o, g->h_res, &st);
    if (stats) *stats = st;
    if (rc != GSLAM_OK) return rc;
    k_rows_to_poses<<<nblk(n, 256), 256, 0, g->st>>>(n, g->L.iperm, g->L.x4, d_mu);
    if (ne) k_se2_edge_grad<<<nblk(ne, 128), 128, 0, g->st>>>(ne, g->d_ei, g->d_ej, g->d_meas, g->d_info, g->lambda,
                                                              g->d_poses, d_mu, d_grad);
    ACK(cudaGetLastError());
    std::vector<double> grad(3 * (size_t)ne);
    if (ne) ACK(cudaMemcpyAsync(grad.data(), d_grad, grad.size() * sizeof(double), cudaMemcpyDeviceToHost, g->st));
    if (mu_out) ACK(cudaMemcpyAsync(mu_out, d_mu, 3 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, g->st));
    ACK(cudaStreamSynchronize(g->st));
#undef ACK
    double sum = 0.0;
    for (size_t k = 0; k < grad.size(); k++) sum = sum + grad[k];
    if (dL_dlambda) *dL_dlambda = sum / g->lambda;
    if (dL_dlogw)
        for (size_t k = 0; k < grad.size(); k++) dL_dlogw[k] = grad[k];
    return GSLAM_OK;
}
