/*
 * gj.cu — blocked Gauss-Jordan inverse of a dense FP64 matrix, the trailing update
 * on the FP64 tensor cores.
 *
 * The reference's dense path (src/cpu_pcg_fp64/MatrixOps.c:29-91 `inv`, its CUDA
 * twin src/gpu_gj_fp64/inv.cu:221-354) inverts Omega by Gauss-Jordan without
 * pivoting and multiplies xi by the inverse; it is kept for small N as a check of
 * the iterative solvers. Here the same elimination (no pivoting) is blocked by
 * b = 64 columns; step k with K = [64k, 64k + 64):
 *   U = A[:, K] (copy of the old block column), P = A[K, K]^-1 (one CTA: recursive
 *   halving down to 16 x 16 Gauss-Jordan in a warp, see inv_block),
 *   A[K, J] = P A[K, J]                 for J != K   (row panel)
 *   A[I, J] = A[I, J] - U[I] A[K, J]    for I, J != K (trailing update, rank 64)
 *   A[I, K] = -U[I] P                   for I != K,   A[K, K] = P.
 * After the last step A holds A^-1. The next step's copy U of its block column is written
 * by this step's row panel and trailing update as they produce it (no copy launch). The row panel, trailing update and column panel
 * are 64x64-tile GEMMs with K = 64 on mma.sync.m8n8k4 FP64 (DMMA): one CTA per
 * output tile, both 64x64 operand tiles staged in shared memory (rows padded to 68
 * doubles against bank conflicts), four warps of 32x32 each (4 x 4 m8n8 tiles).
 * tcgen05 has no FP64 kind, so mma.sync is the FP64 tensor-core path on sm_100a.
 * Operation count: 2 n^3 (the reference's unblocked version does ~4 n^3, updating
 * the full identity side).
 *
 * n is padded to a multiple of 64 with an identity block (the inverse of
 * diag(A, I) is diag(A^-1, I)).
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "gslam.h"
#include "gslam_api_internal.h"

#define GJ_B 64
#define GJ_LD 68 /* padded leading dimension of a staged 64x64 tile */

/* D = A(8x4, row) * B(4x8, col) + C, FP64: lane layout of the PTX ISA m8n8k4 .f64 shape */
__device__ __forceinline__ void dmma_8x8x4(double &d0, double &d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

/* sA, sB: 64x64 tiles in shared memory (row-major, ld GJ_LD); acc[4][4][2] += sA * sB
 * for this warp's 32x32 quadrant (wm, wn) */
__device__ __forceinline__ void tile_mma(const double *sA, const double *sB, int wm, int wn, int lane,
                                         double (&acc)[4][4][2]) {
    const int gid = lane >> 2, tig = lane & 3;
#pragma unroll 4
    for (int k = 0; k < GJ_B; k += 4) {
        double a[4], b[4];
#pragma unroll
        for (int i = 0; i < 4; i++) a[i] = sA[(32 * wm + 8 * i + gid) * GJ_LD + k + tig];
#pragma unroll
        for (int j = 0; j < 4; j++) b[j] = sB[(k + tig) * GJ_LD + 32 * wn + 8 * j + gid];
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) dmma_8x8x4(acc[i][j][0], acc[i][j][1], a[i], b[j]);
    }
}

/* 64x64 tile g (leading dimension ld, a multiple of 2) -> shared s (ld GJ_LD): 16-byte
 * asynchronous copies through L2 (cp.async.cg), all of a thread's in flight together;
 * complete after load_tile_wait (then a CTA barrier before reading other threads' parts) */
__device__ __forceinline__ void load_tile(double *s, const double *g, int ld) {
    for (int t = threadIdx.x; t < GJ_B * GJ_B / 2; t += blockDim.x) {
        const int r = t >> 5, c = 2 * (t & 31);
        const unsigned d = (unsigned)__cvta_generic_to_shared(s + r * GJ_LD + c);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(g + (size_t)r * ld + c) : "memory");
    }
}

__device__ __forceinline__ void load_tile_wait() {
    asm volatile("cp.async.commit_group;" ::: "memory");
    asm volatile("cp.async.wait_group 0;" ::: "memory");
}

/* U = A[:, K] (n x 64, ld 64) */
__global__ void k_gj_copy_col(int n, const double *__restrict__ A, int k0, double *__restrict__ U) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * GJ_B) return;
    const int r = t >> 6, c = t & 63;
    U[t] = A[(size_t)r * n + k0 + c];
}

/*
 * The 64 x 64 pivot-block inverse, blocked recursively so that few steps are serial (by a
 * CTA of 128 threads, the block in shared memory). With M = [A B; C D] in halves and no
 * pivoting (the same pivot order as Gauss-Jordan, src/cpu_pcg_fp64/MatrixOps.c:29-91):
 *   A <- A^-1;  W = A^-1 B;  V = C A^-1;  S = D - C W;  D <- S^-1;
 *   B <- -W S^-1;  C <- -S^-1 V;  A <- A^-1 - W C   (= A^-1 + W S^-1 V),
 * 32 x 32 halves split the same way into 16 x 16 ones, and a 16 x 16 block is inverted by
 * Gauss-Jordan in one warp (two lanes per row, the pivot row by warp shuffles). Serial
 * path: four 16-pivot warp eliminations and a few small GEMMs, instead of 64 pivot steps
 * each behind a CTA barrier.
 */

/* Gauss-Jordan without pivoting of the 16 x 16 block at m (leading dimension ld), by the
 * 32 lanes of one warp: lane l holds row l / 2, columns [8 (l % 2), 8 (l % 2) + 8). Pivot
 * step i: f = T[r][i] from the lane of row r that owns column i; the two lanes of row i
 * form the new pivot row (T[i][i] -> 1, then times 1 / T[i][i]); every lane takes the
 * pivot row's entries of its own columns by shuffles; the other rows subtract f times
 * them with T[r][i] -> 0 first. */
__device__ __forceinline__ void inv16_warp(double *m, int ld) {
    const int lane = threadIdx.x & 31, r = lane >> 1, h = lane & 1;
    double T[8];
#pragma unroll
    for (int j = 0; j < 8; j++) T[j] = m[r * ld + 8 * h + j];
#pragma unroll
    for (int i = 0; i < 16; i++) {
        const int gi = i >> 3, jj = i & 7;
        const double f = __shfl_sync(0xffffffffu, T[jj], 2 * r + gi);
        if (r == i) {
            const double p = 1.0 / f;
#pragma unroll
            for (int j = 0; j < 8; j++) T[j] = ((8 * h + j == i) ? 1.0 : T[j]) * p;
        }
        double q[8];
#pragma unroll
        for (int j = 0; j < 8; j++) q[j] = __shfl_sync(0xffffffffu, T[j], 2 * i + h);
        if (r != i) {
#pragma unroll
            for (int j = 0; j < 8; j++) T[j] = ((8 * h + j == i) ? 0.0 : T[j]) - f * q[j];
        }
    }
#pragma unroll
    for (int j = 0; j < 8; j++) m[r * ld + 8 * h + j] = T[j];
}

/* out = s * (a b) + (add ? out : 0) for N x N blocks in shared memory, by 128 threads:
 * thread t computes rows RB (t / (N / CB)) + [0, RB) and columns CB (t % (N / CB)) + [0, CB),
 * each entry summed over k in order. */
template <int N>
__device__ __forceinline__ void gemm_small(double *out, int ldo, const double *a, int lda, const double *b, int ldb,
                                           double sgn, bool add) {
    constexpr int RB = N / 16, CB = N / 8;
    const int t = threadIdx.x, tr = t / (N / CB), tc = t % (N / CB);
    double acc[RB][CB];
#pragma unroll
    for (int i = 0; i < RB; i++)
#pragma unroll
        for (int j = 0; j < CB; j++) acc[i][j] = 0.0;
#pragma unroll 4
    for (int k = 0; k < N; k++) {
        double av[RB], bv[CB];
#pragma unroll
        for (int i = 0; i < RB; i++) av[i] = a[(RB * tr + i) * lda + k];
#pragma unroll
        for (int j = 0; j < CB; j++) bv[j] = b[k * ldb + CB * tc + j];
#pragma unroll
        for (int i = 0; i < RB; i++)
#pragma unroll
            for (int j = 0; j < CB; j++) acc[i][j] = fma(av[i], bv[j], acc[i][j]);
    }
#pragma unroll
    for (int i = 0; i < RB; i++)
#pragma unroll
        for (int j = 0; j < CB; j++) {
            double *o = out + (RB * tr + i) * ldo + CB * tc + j;
            *o = add ? *o + sgn * acc[i][j] : sgn * acc[i][j];
        }
}

/* in-place inverse of the N x N block at m (ld), N = 32 or 64, by 128 threads; scratch:
 * 2 (N/2)^2 doubles for this level's W and V and the lower levels' after them */
template <int N>
__device__ void inv_block(double *m, int ld, double *scratch) {
    constexpr int H = N / 2;
    double *A = m, *B = m + H, *Cb = m + H * ld, *D = m + H * ld + H;
    double *W = scratch, *V = scratch + H * H, *lower = scratch + 2 * H * H;
    if constexpr (H == 16) {
        if (threadIdx.x < 32) inv16_warp(A, ld);
    } else {
        inv_block<H>(A, ld, lower);
    }
    __syncthreads();
    gemm_small<H>(W, H, A, ld, B, ld, 1.0, false);   /* W = A^-1 B */
    gemm_small<H>(V, H, Cb, ld, A, ld, 1.0, false);  /* V = C A^-1 */
    __syncthreads();
    gemm_small<H>(D, ld, Cb, ld, W, H, -1.0, true);  /* S = D - C W */
    __syncthreads();
    if constexpr (H == 16) {
        if (threadIdx.x < 32) inv16_warp(D, ld);
    } else {
        inv_block<H>(D, ld, lower);
    }
    __syncthreads();
    gemm_small<H>(B, ld, W, H, D, ld, -1.0, false);  /* B = -W S^-1 */
    gemm_small<H>(Cb, ld, D, ld, V, H, -1.0, false); /* C = -S^-1 V */
    __syncthreads();
    gemm_small<H>(A, ld, W, H, Cb, ld, -1.0, true);  /* A = A^-1 - W C */
    __syncthreads();
}

/* scratch doubles inv_block<64> needs: 2 * 32^2 + 2 * 16^2 */
#define GJ_INV_SCRATCH (2 * 32 * 32 + 2 * 16 * 16)

/* P = inv(U[K, :]): the first step's pivot block (later ones are inverted by the update
 * tile that produces them, k_gj_update); 128 threads, the block and its scratch in the
 * same dynamic shared memory as the GEMM kernels */
__global__ void __launch_bounds__(128) k_gj_diag(const double *__restrict__ U, int k0, double *__restrict__ P) {
    extern __shared__ __align__(16) double sm[];
    double *sM = sm, *scr = sm + GJ_B * GJ_LD;
    for (int t = threadIdx.x; t < GJ_B * GJ_B; t += blockDim.x)
        sM[(t >> 6) * GJ_LD + (t & 63)] = U[(size_t)(k0 + (t >> 6)) * GJ_B + (t & 63)];
    __syncthreads();
    inv_block<64>(sM, GJ_LD, scr);
    for (int t = threadIdx.x; t < GJ_B * GJ_B; t += blockDim.x) P[t] = sM[(t >> 6) * GJ_LD + (t & 63)];
}

/* row panel: A[K, J] = P A[K, J] for every 64-column tile J != K (one CTA per tile); the
 * tile of the next pivot column (J = K + 1) also goes to Un, that step's copy of its block
 * column (rows K; the other rows come from the trailing update) */
__global__ void __launch_bounds__(128) k_gj_row_panel(int n, double *__restrict__ A, int k0,
                                                      const double *__restrict__ P, double *__restrict__ Un) {
    extern __shared__ __align__(16) double sm[];
    double *sA = sm, *sB = sm + GJ_B * GJ_LD;
    const int tj = blockIdx.x;
    if (64 * tj == k0) return;
    const bool next = (64 * tj == k0 + GJ_B);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wm = warp >> 1, wn = warp & 1;
    load_tile(sA, P, GJ_B);
    load_tile(sB, A + (size_t)k0 * n + 64 * tj, n);
    load_tile_wait();
    __syncthreads();
    double acc[4][4][2] = {};
    tile_mma(sA, sB, wm, wn, lane, acc);
    const int gid = lane >> 2, tig = lane & 3;
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int r = 32 * wm + 8 * i + gid, c = 32 * wn + 8 * j + 2 * tig;
            double *dst = A + (size_t)(k0 + r) * n + 64 * tj + c;
            dst[0] = acc[i][j][0];
            dst[1] = acc[i][j][1];
            if (next) *reinterpret_cast<double2 *>(Un + (size_t)(k0 + r) * GJ_B + c) = make_double2(acc[i][j][0], acc[i][j][1]);
        }
}

/* trailing update and column panel, one CTA per 64x64 tile (I, J), I != K:
 *   J != K: A[I, J] -= U[I] A[K, J];   J == K: A[I, K] = -U[I] P.
 * Tile (K, K) writes P. The old A[I, J] is loaded into registers before the operand tiles
 * (its latency overlaps theirs); tiles of the next pivot column also go to Un. Tiles are
 * numbered from the next pivot tile (K + 1, K + 1), so that tile is the first block
 * scheduled: it goes on to invert itself into Pn, the next step's pivot inverse, while
 * the other tiles are updated (the inversion is off the step's critical path). */
__global__ void __launch_bounds__(128) k_gj_update(int n, double *__restrict__ A, int k0,
                                                   const double *__restrict__ U, const double *__restrict__ P,
                                                   double *__restrict__ Un, double *__restrict__ Pn) {
    extern __shared__ __align__(16) double sm[];
    double *sA = sm, *sB = sm + GJ_B * GJ_LD;
    const int nt = n / GJ_B, kn = k0 / GJ_B + 1;
    const int ti = ((int)blockIdx.y + kn) % nt, tj = ((int)blockIdx.x + kn) % nt;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wm = warp >> 1, wn = warp & 1;
    const int gid = lane >> 2, tig = lane & 3;
    if (64 * ti == k0) {
        if (64 * tj == k0)
            for (int t = threadIdx.x; t < GJ_B * GJ_B; t += blockDim.x)
                A[(size_t)(k0 + (t >> 6)) * n + k0 + (t & 63)] = P[t];
        return;
    }
    const bool colp = (64 * tj == k0), next = (64 * tj == k0 + GJ_B);
    const bool pivot_next = next && ti == kn;
    double old[4][4][2];
    if (!colp) {
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int r = 32 * wm + 8 * i + gid, c = 32 * wn + 8 * j + 2 * tig;
                const double2 v = *reinterpret_cast<const double2 *>(A + (size_t)(64 * ti + r) * n + 64 * tj + c);
                old[i][j][0] = v.x;
                old[i][j][1] = v.y;
            }
    }
    load_tile(sA, U + (size_t)(64 * ti) * GJ_B, GJ_B);
    load_tile(sB, colp ? P : A + (size_t)k0 * n + 64 * tj, colp ? GJ_B : n);
    load_tile_wait();
    __syncthreads();
    double acc[4][4][2] = {};
    tile_mma(sA, sB, wm, wn, lane, acc);
    if (pivot_next) __syncthreads(); /* sA is reused below */
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int r = 32 * wm + 8 * i + gid, c = 32 * wn + 8 * j + 2 * tig;
            double2 v;
            if (colp) v = make_double2(-acc[i][j][0], -acc[i][j][1]);
            else v = make_double2(old[i][j][0] - acc[i][j][0], old[i][j][1] - acc[i][j][1]);
            *reinterpret_cast<double2 *>(A + (size_t)(64 * ti + r) * n + 64 * tj + c) = v;
            if (next) *reinterpret_cast<double2 *>(Un + (size_t)(64 * ti + r) * GJ_B + c) = v;
            if (pivot_next) *reinterpret_cast<double2 *>(sA + r * GJ_LD + c) = v;
        }
    if (pivot_next) {
        /* the next pivot block (now in sA) inverted in place, sB as scratch */
        __syncthreads();
        inv_block<64>(sA, GJ_LD, sB);
        for (int t = threadIdx.x; t < GJ_B * GJ_B; t += blockDim.x) Pn[t] = sA[(t >> 6) * GJ_LD + (t & 63)];
    }
}

/* pad: B (m x m, m = n rounded up to 64) = diag(A, I) */
__global__ void k_gj_pad(int n, int m, const double *__restrict__ A, int lda, double *__restrict__ B) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)m * m) return;
    const int r = (int)(t / m), c = (int)(t % m);
    B[t] = (r < n && c < n) ? A[(size_t)r * lda + c] : (r == c ? 1.0 : 0.0);
}

__global__ void k_gj_unpad(int n, int m, const double *__restrict__ B, double *__restrict__ A, int lda) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)n * n) return;
    const int r = (int)(t / n), c = (int)(t % n);
    A[(size_t)r * lda + c] = B[(size_t)r * m + c];
}

/* y = A x, one warp per row (A m x m, row-major), summed in a fixed order */
__global__ void k_gemv(int m, const double *__restrict__ A, const double *__restrict__ x, double *__restrict__ y) {
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (row >= m) return;
    double s = 0.0;
    for (int c = lane; c < m; c += 32) s = s + A[(size_t)row * m + c] * x[c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s = s + __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) y[row] = s;
}

static int gj_run(int m, double *d_a, cudaStream_t st, double *scratch) {
    /* scratch: two copies of a block column (m x 64 each, this step's and the next's) then
     * two pivot inverses (64 x 64 each); the first step's copy and inverse are made here,
     * every later one by the previous step's row panel and trailing update */
    double *Ub[2] = { scratch, scratch + (size_t)m * GJ_B };
    double *Pb[2] = { scratch + 2 * (size_t)m * GJ_B, scratch + 2 * (size_t)m * GJ_B + GJ_B * GJ_B };
    const size_t smem = 2 * GJ_B * GJ_LD * sizeof(double);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_gj_row_panel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(k_gj_update, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(k_gj_diag, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr = true;
    }
    const int nt = m / GJ_B;
    k_gj_copy_col<<<(m * GJ_B + 255) / 256, 256, 0, st>>>(m, d_a, 0, Ub[0]);
    k_gj_diag<<<1, 128, smem, st>>>(Ub[0], 0, Pb[0]);
    for (int k = 0; k < nt; k++) {
        const int k0 = GJ_B * k;
        double *U = Ub[k & 1], *Un = Ub[(k + 1) & 1];
        double *P = Pb[k & 1], *Pn = Pb[(k + 1) & 1];
        k_gj_row_panel<<<nt, 128, smem, st>>>(m, d_a, k0, P, Un);
        k_gj_update<<<dim3(nt, nt), 128, smem, st>>>(m, d_a, k0, U, P, Un, Pn);
    }
    return cudaGetLastError() == cudaSuccess ? GSLAM_OK : GSLAM_ERR_CUDA;
}

int gslam_gj_inverse(int n, double *d_a, int lda, void *stream, float *ms) {
    if (n <= 0 || !d_a || lda < n) { gslam_set_last_error("bad dense matrix"); return GSLAM_ERR_BAD_INPUT; }
    cudaStream_t st = (cudaStream_t)stream;
    const int m = (n + GJ_B - 1) / GJ_B * GJ_B;
    double *B = nullptr, *scratch = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = GSLAM_ERR_CUDA;
    if (cudaMalloc(&B, (size_t)m * m * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&scratch, (2 * (size_t)m * GJ_B + 2 * GJ_B * GJ_B) * sizeof(double)) != cudaSuccess ||
        cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        gslam_set_last_error("cudaMalloc failed (dense inverse)");
        goto done;
    }
    k_gj_pad<<<(unsigned)(((size_t)m * m + 255) / 256), 256, 0, st>>>(n, m, d_a, lda, B);
    cudaEventRecord(e0, st);
    rc = gj_run(m, B, st, scratch);
    cudaEventRecord(e1, st);
    if (rc == GSLAM_OK) {
        k_gj_unpad<<<(unsigned)(((size_t)n * n + 255) / 256), 256, 0, st>>>(n, m, B, d_a, lda);
        if (cudaStreamSynchronize(st) != cudaSuccess) { rc = GSLAM_ERR_CUDA; gslam_set_last_error("dense inverse failed"); }
        else if (ms) cudaEventElapsedTime(ms, e0, e1);
    } else {
        gslam_set_last_error("dense inverse launch failed");
    }
done:
    if (B) cudaFree(B);
    if (scratch) cudaFree(scratch);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    return rc;
}

int gslam_gj_solve(int n, const double *d_a, int lda, const double *d_b, double *d_x, void *stream, float *ms) {
    if (n <= 0 || !d_a || !d_b || !d_x || lda < n) { gslam_set_last_error("bad dense system"); return GSLAM_ERR_BAD_INPUT; }
    cudaStream_t st = (cudaStream_t)stream;
    double *A = nullptr;
    if (cudaMalloc(&A, (size_t)n * n * sizeof(double)) != cudaSuccess) {
        gslam_set_last_error("cudaMalloc failed (dense solve)");
        return GSLAM_ERR_CUDA;
    }
    cudaMemcpy2DAsync(A, n * sizeof(double), d_a, lda * sizeof(double), n * sizeof(double), n,
                      cudaMemcpyDeviceToDevice, st);
    int rc = gslam_gj_inverse(n, A, n, stream, ms);
    if (rc == GSLAM_OK) {
        k_gemv<<<(n * 32 + 255) / 256, 256, 0, st>>>(n, A, d_b, d_x);
        if (cudaStreamSynchronize(st) != cudaSuccess) { rc = GSLAM_ERR_CUDA; gslam_set_last_error("dense solve failed"); }
    }
    cudaFree(A);
    return rc;
}

/*
 * FP64 tensor-core throughput (the roofline of the Gauss-Jordan updates): every warp
 * issues `reps` rounds of 8 independent m8n8k4 DMMAs (512 flops each) on register
 * operands, so nothing but the tensor pipe limits it. The accumulators go to `out`
 * so no MMA is dead code.
 */
__global__ void __launch_bounds__(256) k_dmma_peak(int reps, double *__restrict__ out) {
    const double a = 1.0 + 1e-9 * threadIdx.x, b = 1.0 - 1e-9 * threadIdx.x;
    double acc[8][2];
#pragma unroll
    for (int i = 0; i < 8; i++) { acc[i][0] = 1e-3 * i; acc[i][1] = -1e-3 * i; }
    for (int r = 0; r < reps; r++) {
#pragma unroll
        for (int i = 0; i < 8; i++) dmma_8x8x4(acc[i][0], acc[i][1], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < 8; i++) s = s + acc[i][0] + acc[i][1];
    out[(size_t)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

int gslam_dmma_bench(int reps, int ctas_per_sm, double *tflops, float *ms) {
    if (reps <= 0 || ctas_per_sm <= 0 || !tflops) { gslam_set_last_error("bad DMMA bench arguments"); return GSLAM_ERR_BAD_INPUT; }
    int dev = 0, n_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        gslam_set_last_error("no CUDA device");
        return GSLAM_ERR_NO_DEVICE;
    }
    const int grid = n_sm * ctas_per_sm, block = 256;
    double *out = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = GSLAM_ERR_CUDA;
    float t = 0.f;
    if (cudaMalloc(&out, (size_t)grid * block * sizeof(double)) != cudaSuccess ||
        cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        gslam_set_last_error("cudaMalloc failed (DMMA bench)");
        goto done;
    }
    k_dmma_peak<<<grid, block>>>(reps, out); /* warm-up */
    cudaEventRecord(e0);
    k_dmma_peak<<<grid, block>>>(reps, out);
    cudaEventRecord(e1);
    if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&t, e0, e1) != cudaSuccess) {
        gslam_set_last_error("DMMA bench failed");
        goto done;
    }
    *tflops = (double)grid * (block / 32) * (double)reps * 8.0 * 512.0 / (t * 1e-3) / 1e12;
    if (ms) *ms = t;
    rc = GSLAM_OK;
done:
    if (out) cudaFree(out);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    return rc;
}
