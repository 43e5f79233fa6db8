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
 * by this step's row panel and trailing update as they produce it (no copy launch). The
 * row panel, trailing update and column panel
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
__device__ __forceinline__ void cp_async16(double *s, const double *g) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(s);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(g) : "memory");
}

__device__ __forceinline__ void load_tile(double *s, const double *g, int ld) {
    for (int t = threadIdx.x; t < GJ_B * GJ_B / 2; t += blockDim.x) {
        const int r = t >> 5, c = 2 * (t & 31);
        cp_async16(s + r * GJ_LD + c, g + (size_t)r * ld + c);
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
 * Gauss-Jordan in one warp (a lane per column, the pivot column by warp shuffles); the
 * small GEMMs run on the FP64 tensor cores. Serial path: four 16-pivot warp eliminations
 * and eight GEMM phases, instead of 64 pivot steps each behind a CTA barrier.
 */

/* Gauss-Jordan without pivoting of the 16 x 16 block at m (leading dimension ld), in one
 * warp: lane c < 16 holds column c (lanes 16..31 hold a copy of column c - 16 and store
 * nothing). Pivot step i: every lane reads column i (f_r = T[r][i], f_i the pivot) from
 * buf, where lane i wrote it after its previous update (two 16-double halves, used in
 * turn, 16-byte aligned: eight vector stores and eight broadcast loads per step instead of
 * 32 shuffles), and forms p = 1 / f_i itself; lane c != i scales its pivot-row entry
 * a = T[i][c] p and subtracts f_r a from its other rows, lane i's column becomes -f_r p
 * with p on the diagonal (the same update, with a = p and the old entries taken as 0, so
 * the warp does not diverge). */
__device__ __forceinline__ void inv16_warp(double *m, int ld, double *buf) {
    const int lane = threadIdx.x & 31, c = lane & 15;
    double T[16];
#pragma unroll
    for (int r = 0; r < 16; r++) T[r] = m[r * ld + c];
    if (lane == 0) {
#pragma unroll
        for (int r = 0; r < 16; r += 2) *reinterpret_cast<double2 *>(buf + r) = make_double2(T[r], T[r + 1]);
    }
    __syncwarp();
#pragma unroll
    for (int i = 0; i < 16; i++) {
        const double *col = buf + 16 * (i & 1);
        double f[16];
#pragma unroll
        for (int r = 0; r < 16; r += 2) {
            const double2 v = *reinterpret_cast<const double2 *>(col + r);
            f[r] = v.x;
            f[r + 1] = v.y;
        }
        const double p = 1.0 / f[i];
        const bool piv = (c == i);
        const double a = piv ? p : T[i] * p;
#pragma unroll
        for (int r = 0; r < 16; r++)
            if (r != i) T[r] = fma(-f[r], a, piv ? 0.0 : T[r]);
        T[i] = a;
        if (i < 15) {
            if (lane == i + 1) {
                double *nxt = buf + 16 * ((i + 1) & 1);
#pragma unroll
                for (int r = 0; r < 16; r += 2) *reinterpret_cast<double2 *>(nxt + r) = make_double2(T[r], T[r + 1]);
            }
            __syncwarp();
        }
    }
    if (lane < 16) {
#pragma unroll
        for (int r = 0; r < 16; r++) m[r * ld + c] = T[r];
    }
}

/* out = s * (a b) + (add ? out : 0) for N x N blocks (N = 16 or 32) in shared memory on
 * the FP64 tensor cores, by 4 warps: warp w computes the (N/2) x (N/2) quadrant (w / 2,
 * w % 2) as m8n8 tiles, k in steps of 4 (m8n8k4) */
template <int N>
__device__ __forceinline__ void gemm_small(double *out, int ldo, const double *a, int lda, const double *b, int ldb,
                                           double sgn, bool add) {
    constexpr int TW = N / 16; /* m8n8 tiles per warp in each dimension */
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, gid = lane >> 2, tig = lane & 3;
    const int r0 = (N / 2) * (warp >> 1), c0 = (N / 2) * (warp & 1);
    double acc[TW][TW][2];
#pragma unroll
    for (int i = 0; i < TW; i++)
#pragma unroll
        for (int j = 0; j < TW; j++) acc[i][j][0] = acc[i][j][1] = 0.0;
#pragma unroll
    for (int k = 0; k < N; k += 4) {
        double av[TW], bv[TW];
#pragma unroll
        for (int i = 0; i < TW; i++) av[i] = a[(r0 + 8 * i + gid) * lda + k + tig];
#pragma unroll
        for (int j = 0; j < TW; j++) bv[j] = b[(k + tig) * ldb + c0 + 8 * j + gid];
#pragma unroll
        for (int i = 0; i < TW; i++)
#pragma unroll
            for (int j = 0; j < TW; j++) dmma_8x8x4(acc[i][j][0], acc[i][j][1], av[i], bv[j]);
    }
#pragma unroll
    for (int i = 0; i < TW; i++)
#pragma unroll
        for (int j = 0; j < TW; j++)
#pragma unroll
            for (int h = 0; h < 2; h++) {
                double *o = out + (r0 + 8 * i + gid) * ldo + c0 + 8 * j + 2 * tig + h;
                *o = add ? *o + sgn * acc[i][j][h] : sgn * acc[i][j][h];
            }
}

/* in-place inverse of the N x N block at m (ld), N = 32 or 64, by 128 threads; scratch
 * (16-byte aligned): this level's W and V (N/2 x N/2 each, leading dimension N/2 + 4
 * against bank conflicts), the lower levels' after them, and last the warp elimination's
 * 32-double column buffer */
template <int N>
__device__ void inv_block(double *m, int ld, double *scratch) {
    constexpr int H = N / 2, HL = H + 4;
    double *A = m, *B = m + H, *Cb = m + H * ld, *D = m + H * ld + H;
    double *W = scratch, *V = scratch + H * HL, *lower = scratch + 2 * H * HL;
    if constexpr (H == 16) {
        if (threadIdx.x < 32) inv16_warp(A, ld, lower);
    } else {
        inv_block<H>(A, ld, lower);
    }
    __syncthreads();
    gemm_small<H>(W, HL, A, ld, B, ld, 1.0, false);   /* W = A^-1 B */
    gemm_small<H>(V, HL, Cb, ld, A, ld, 1.0, false);  /* V = C A^-1 */
    __syncthreads();
    gemm_small<H>(D, ld, Cb, ld, W, HL, -1.0, true);  /* S = D - C W */
    __syncthreads();
    if constexpr (H == 16) {
        if (threadIdx.x < 32) inv16_warp(D, ld, lower);
    } else {
        inv_block<H>(D, ld, lower);
    }
    __syncthreads();
    gemm_small<H>(B, ld, W, HL, D, ld, -1.0, false);  /* B = -W S^-1 */
    gemm_small<H>(Cb, ld, D, ld, V, HL, -1.0, false); /* C = -S^-1 V */
    __syncthreads();
    gemm_small<H>(A, ld, W, HL, Cb, ld, -1.0, true);  /* A = A^-1 - W C */
    __syncthreads();
}

/* scratch doubles inv_block<64> needs: 2 * 32 * 36 + 2 * 16 * 20 + 32 */
#define GJ_INV_SCRATCH (2 * 32 * 36 + 2 * 16 * 20 + 32)

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

/* row panel: A[K, J] = P A[K, J] for every 64-column tile J != K, by four CTAs per tile,
 * each a 16-column strip (blockIdx.y): it reads only the strip it overwrites, and P (the
 * same 64 x 64 for every CTA) comes from L2, so 4 nt CTAs share the step's row panel
 * instead of nt. The strip of the next pivot column (J = K + 1) also goes to Un, that
 * step's copy of its block column (rows K; the other rows come from the trailing update). */
#define GJ_RP_LD 20 /* padded leading dimension of the staged 64 x 16 strip */
__global__ void __launch_bounds__(128) k_gj_row_panel(int n, double *__restrict__ A, int k0,
                                                      const double *__restrict__ P, double *__restrict__ Un) {
    extern __shared__ __align__(16) double sm[];
    double *sA = sm, *sB = sm + GJ_B * GJ_LD;
    const int tj = blockIdx.x, c0 = 16 * blockIdx.y;
    if (64 * tj == k0) return;
    const bool next = (64 * tj == k0 + GJ_B);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, gid = lane >> 2, tig = lane & 3;
    const double *g = A + (size_t)k0 * n + 64 * tj + c0;
    load_tile(sA, P, GJ_B);
    for (int t = threadIdx.x; t < GJ_B * 8; t += blockDim.x) { /* 64 rows x 8 pairs */
        const int r = t >> 3, c = 2 * (t & 7);
        cp_async16(sB + r * GJ_RP_LD + c, g + (size_t)r * n + c);
    }
    load_tile_wait();
    __syncthreads();
    /* warp w: rows [16 w, 16 w + 16) of the strip, 2 x 2 m8n8 tiles */
    double acc[2][2][2] = {};
#pragma unroll 4
    for (int k = 0; k < GJ_B; k += 4) {
        double a[2], b[2];
#pragma unroll
        for (int i = 0; i < 2; i++) a[i] = sA[(16 * warp + 8 * i + gid) * GJ_LD + k + tig];
#pragma unroll
        for (int j = 0; j < 2; j++) b[j] = sB[(k + tig) * GJ_RP_LD + 8 * j + gid];
#pragma unroll
        for (int i = 0; i < 2; i++)
#pragma unroll
            for (int j = 0; j < 2; j++) dmma_8x8x4(acc[i][j][0], acc[i][j][1], a[i], b[j]);
    }
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 2; j++) {
            const int r = 16 * warp + 8 * i + gid, c = c0 + 8 * j + 2 * tig;
            const double2 v = make_double2(acc[i][j][0], acc[i][j][1]);
            *reinterpret_cast<double2 *>(A + (size_t)(k0 + r) * n + 64 * tj + c) = v;
            if (next) *reinterpret_cast<double2 *>(Un + (size_t)(k0 + r) * GJ_B + c) = v;
        }
}

/* The SM a CTA runs on. */
__device__ __forceinline__ int sm_id() {
    int s;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(s));
    return s;
}

/* Per step of one inverse: the SM of the CTA that inverts the next pivot block (-1 until
 * it has started) and whether that inverse is written. Initialised before the first
 * launch (-1 and 0). */
struct GjPivotSm {
    int *sm;   /* [nt] */
    int *done; /* [nt] */
    long long spin_limit;
};

/* trailing update and column panel, one CTA per 64x64 tile (I, J), I != K:
 *   J != K: A[I, J] -= U[I] A[K, J];   J == K: A[I, K] = -U[I] P.
 * Tile (K, K) writes P. The old A[I, J] is loaded into registers before the operand tiles
 * (its latency overlaps theirs); tiles of the next pivot column also go to Un. Tiles are
 * numbered from the next pivot tile (K + 1, K + 1), so that tile is the first block
 * scheduled: it goes on to invert itself into Pn, the next step's pivot inverse, while
 * the other tiles are updated. The inversion is a chain of dependent FP64 operations and
 * ran 2.6x slower beside other CTAs' DMMA tiles than alone, long enough to end every
 * launch; so that CTA publishes its SM and a CTA that finds itself on that SM (read while
 * its operand copies are in flight) waits, before its DMMAs, until the inverse is written.
 * The wait is bounded and only a matter of speed: at its limit the CTA goes on. */
__global__ void __launch_bounds__(128) k_gj_update(int n, double *__restrict__ A, int k0,
                                                   const double *__restrict__ U, const double *__restrict__ P,
                                                   double *__restrict__ Un, double *__restrict__ Pn, GjPivotSm ps) {
    extern __shared__ __align__(16) double sm[];
    double *sA = sm, *sB = sm + GJ_B * GJ_LD;
    const int nt = n / GJ_B, k = k0 / GJ_B, kn = k + 1;
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
    const int my_sm = sm_id();
    if (pivot_next && threadIdx.x == 0) {
        *(volatile int *)(ps.sm + k) = my_sm;
        __threadfence();
    }
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
    const int piv_sm = (threadIdx.x == 0 && !pivot_next) ? *(volatile int *)(ps.sm + k) : -1;
    load_tile_wait();
    if (piv_sm == my_sm && !*(volatile int *)(ps.done + k)) {
        const long long t0 = clock64();
        while (!*(volatile int *)(ps.done + k) && clock64() - t0 < ps.spin_limit) __nanosleep(1000);
    }
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
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            *(volatile int *)(ps.done + k) = 1;
        }
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
    /* scratch: two copies of a block column (m x 64 each, this step's and the next's), two
     * pivot inverses (64 x 64 each), then 2 m / 64 ints (GjPivotSm); the first step's copy
     * and inverse are made here, every later one by the previous step's row panel and
     * trailing update */
    double *Ub[2] = { scratch, scratch + (size_t)m * GJ_B };
    double *Pb[2] = { scratch + 2 * (size_t)m * GJ_B, scratch + 2 * (size_t)m * GJ_B + GJ_B * GJ_B };
    const int nt = m / GJ_B;
    GjPivotSm ps;
    ps.sm = reinterpret_cast<int *>(scratch + 2 * (size_t)m * GJ_B + 2 * GJ_B * GJ_B);
    ps.done = ps.sm + nt;
    ps.spin_limit = 200000000LL; /* about 0.1 s of SM clock */
    cudaMemsetAsync(ps.sm, 0xff, nt * sizeof(int), st);
    cudaMemsetAsync(ps.done, 0, nt * sizeof(int), st);
    const size_t smem = 2 * GJ_B * GJ_LD * sizeof(double);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_gj_row_panel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(k_gj_update, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(k_gj_diag, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr = true;
    }
    k_gj_copy_col<<<(m * GJ_B + 255) / 256, 256, 0, st>>>(m, d_a, 0, Ub[0]);
    k_gj_diag<<<1, 128, smem, st>>>(Ub[0], 0, Pb[0]);
    for (int k = 0; k < nt; k++) {
        const int k0 = GJ_B * k;
        double *U = Ub[k & 1], *Un = Ub[(k + 1) & 1];
        double *P = Pb[k & 1], *Pn = Pb[(k + 1) & 1];
        k_gj_row_panel<<<dim3(nt, 4), 128, smem, st>>>(m, d_a, k0, P, Un);
        k_gj_update<<<dim3(nt, nt), 128, smem, st>>>(m, d_a, k0, U, P, Un, Pn, ps);
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
        cudaMalloc(&scratch, (2 * (size_t)m * GJ_B + 2 * GJ_B * GJ_B + m / GJ_B + 1) * sizeof(double)) != cudaSuccess ||
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
