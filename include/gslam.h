/*
 * gslam.h — C ABI of libgslam, a B200 (sm_100a) Graph-SLAM back-end.
 *
 * One handle = one pose graph resident on one GPU. Every call returns an int
 * status (GSLAM_OK or a negative GSLAM_ERR_*); arguments are plain pointers and
 * sizes. Pointers named d_* are device pointers on the handle's GPU; all others
 * are host pointers. Calls on one handle must not overlap; different handles are
 * independent (each owns its stream and buffers).
 *
 * The reference (isaacyhe/G-SLAM_on_GPU_and_FPGA) has no handle API: its path is
 * the program in src/cpu_pcg_fp64 (GSLAM.c main, one process = one graph) and
 * the static-state GPU twin src/gpu_pcg_fp64/device_graph.cuh:23-91. The entry
 * points below replace that path; gslam_dropin.h carries the reference's own
 * signatures on top of them.
 */
#ifndef GSLAM_H
#define GSLAM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (the reference only ever exit(1)s: device_graph.cu:99-106) ---- */
#define GSLAM_OK 0
#define GSLAM_ERR_BAD_INPUT -1      /* sizes, indices or values out of range */
#define GSLAM_ERR_CUDA -2           /* a CUDA runtime call failed */
#define GSLAM_ERR_DEVICE_TIMEOUT -3 /* a bounded device wait gave up (kernel returned) */
#define GSLAM_ERR_NOT_CONVERGED -4  /* solver stopped at max_iter above tolerance (informational) */
#define GSLAM_ERR_TOO_LARGE -5      /* exceeds a fixed capacity (32-bit CSR, scratch size) */
#define GSLAM_ERR_NO_DEVICE -6      /* no sm_100 device / cooperative launch unavailable */

/* ---- solver precision ---- */
#define GSLAM_PREC_FP64 0  /* FP64 block-Jacobi PCG (the reference's arithmetic) */
#define GSLAM_PREC_MIXED 1 /* FP32 SpMV / vectors inside FP64 iterative refinement */
#define GSLAM_PREC_FP64_CG 2 /* FP64 block-Jacobi PCG with one grid reduction per iteration
                              * (Chronopoulos-Gear recurrence: the reference's iterates in exact
                              * arithmetic, other rounding); the graph must fit the resident
                              * layout (<= 32 slices per SM). Batches solve it as FP64. */

/* ---- factor families ---- */
#define GSLAM_FACTORS_REFERENCE 0 /* ObsEdge + MotionEdge of src/cpu_pcg_fp64 */
#define GSLAM_FACTORS_SE2 1       /* SE(2) between-factors with diagonal information */

/* PCG termination reasons (gslam_solve_stats.reason) */
#define GSLAM_STOP_TOL 0     /* ||r|| < tol * ||b|| */
#define GSLAM_STOP_MAXIT 1   /* iteration cap reached */
#define GSLAM_STOP_PQ_ZERO 2 /* p.Ap == 0 (MatrixOps.c:357) */
#define GSLAM_STOP_TIMEOUT 3 /* device barrier wait gave up */
#define GSLAM_STOP_STAGNATION 4 /* mixed: a refinement step reduced ||r|| by less than half (the
                                 * FP32 inner solve cannot resolve this system); the library then
                                 * solves in FP64 and reports that solve's reason */

typedef struct gslam_opts {
    int precision;        /* GSLAM_PREC_*; default FP64 */
    double tol;           /* relative residual tolerance; reference 1e-6 (MatrixOps.c:345) */
    int max_iter;         /* PCG iteration cap; reference 500 (MatrixOps.c:347) */
    int sell_window;      /* rows sorted by block count inside windows of this size; 0 = auto */
    int threads_per_cta;  /* persistent PCG block size; 0 = auto */
    int ctas_per_sm;      /* persistent PCG CTAs per SM; 0 = auto (occupancy) */
    int angle_wrap;       /* wrap theta to (-pi, pi] in the pose update; 0 for the reference */
    double inner_tol;     /* mixed: inner FP32 relative tolerance per refinement step */
    int inner_max_iter;   /* mixed: inner iteration cap per refinement step */
    int max_refine;       /* mixed: outer refinement steps cap */
    int device;           /* CUDA device ordinal; -1 = current */
    double barrier_timeout_ms; /* a solver barrier gives up after this long; 0 = 2000 ms */
    int test_absent_cta;  /* test hook: this solver CTA never arrives at its first barrier, so
                             the others time out (checks the bounded wait); -1 = off */
    int disable_resident; /* 1: never stage the matrix in shared memory (streamed solver only) */
    int round_graph;      /* 1: gslam_round replays the whole round (linearise, assemble,
                             block-Jacobi, solve, pose update, read-backs) as one CUDA graph,
                             captured at the second round; one host wait per round. Results
                             are bit-identical to the eagerly launched round. Single graphs. */
} gslam_opts;

typedef struct gslam_solve_stats {
    int iterations;       /* PCG iterations (mixed: total inner iterations) */
    int refinements;      /* mixed: outer FP64 steps (negative: the FP64 solver finished the
                           * solve after the mixed one stagnated at -refinements steps); FP64: 0 */
    int reason;           /* GSLAM_STOP_* */
    double rel_residual;  /* ||b - A x|| / ||b|| as tracked by the solver */
    double diff;          /* ||dx|| / sqrt(dim) (GSLAM.c:104-105) */
    double solve_ms;      /* device time of the solver launch (CUDA events on the graph's stream) */
    double round_ms;      /* gslam_round only: device time of the whole round */
} gslam_solve_stats;

/* Inputs of the reference's factor family, as read_data produces them (GSLAM.c:415-493). */
typedef struct gslam_reference_graph {
    uint32_t n_poses;          /* size_of_hat_xs; dim = 3 * n_poses */
    const double *poses;       /* [3 * n_poses] x, y, theta (initial guess) */
    const double *controls;    /* [2 * n_poses] nu, omega of each step (row 0 unused) */
    double delta;              /* time step */
    double lambda;             /* motion-edge weight (argv[2]) */
    const double *mns;         /* [4] motion noise; NULL = {0.19, 0.001, 0.13, 0.2} */
    uint32_t n_obs;            /* observations */
    const uint32_t *obs_step;  /* [n_obs] pose index of each observation */
    const uint32_t *obs_landmark; /* [n_obs] landmark id */
    const double *obs;         /* [2 * n_obs] range, bearing */
} gslam_reference_graph;

/* SE(2) pose graph: edge e constrains pose j relative to pose i. */
typedef struct gslam_se2_graph {
    uint32_t n_poses;
    const double *poses;       /* [3 * n_poses] initial guess */
    uint32_t n_edges;
    const uint32_t *edge_i;    /* [n_edges] */
    const uint32_t *edge_j;    /* [n_edges] */
    const double *meas;        /* [3 * n_edges] dx, dy, dtheta in the frame of pose i */
    const double *log_w;       /* [3 * n_edges] log information weights (log 1/sigma^2) */
    double lambda;             /* global information scale */
    double anchor;             /* prior weight on pose 0 (1e6 like the reference) */
} gslam_se2_graph;

typedef struct gslam_graph gslam_graph;

/* Fills the defaults: FP64, tol 1e-6, max_iter 500, reference behaviour. */
int gslam_opts_default(gslam_opts *opts);

/* Builds a resident graph of the reference factor family. */
int gslam_create_reference(const gslam_reference_graph *in, const gslam_opts *opts,
                           gslam_graph **out);
/* Builds a resident SE(2) pose graph (odometry + loop closures). */
int gslam_create_se2(const gslam_se2_graph *in, const gslam_opts *opts, gslam_graph **out);
int gslam_destroy(gslam_graph *g);

/* Replaces solver options (precision, tolerances) of an existing graph. */
int gslam_set_opts(gslam_graph *g, const gslam_opts *opts);
/* Sizes: n_poses, n_edges (all factors), nnzb (3x3 blocks), nnz (scalar CSR). */
int gslam_sizes(const gslam_graph *g, int64_t *n_poses, int64_t *n_edges, int64_t *nnzb,
                int64_t *nnz);

/* The CUDA stream (cudaStream_t) every call on this graph runs on. */
int gslam_get_stream(gslam_graph *g, void **stream);

/* Pose state (x, y, theta per pose, original order). */
int gslam_set_poses(gslam_graph *g, const double *poses);
int gslam_get_poses(gslam_graph *g, double *poses);

/*
 * One Gauss-Newton round on the device: linearise every edge, assemble Omega and
 * xi, invert the 3x3 diagonal blocks, solve Omega dx = xi, add dx to the poses.
 * stats may be NULL. Equivalent to one iteration of GSLAM.c:55-139.
 */
int gslam_round(gslam_graph *g, gslam_solve_stats *stats);

/*
 * One round with its input and output in host memory: poses_in (3 doubles per pose, may
 * be NULL to keep the device poses) is copied in, the round runs, and the new poses are
 * copied to poses_out (may be NULL), all on the graph's stream with one wait at the end
 * (round_graph on, after the first round; otherwise the same as gslam_set_poses,
 * gslam_round, gslam_get_poses). Pinned host buffers make the copies asynchronous.
 */
int gslam_round_io(gslam_graph *g, const double *poses_in, double *poses_out, gslam_solve_stats *stats);

/*
 * Up to max_rounds rounds with the reference's stop rules (diff < 0.01, or 20
 * rounds without a new best diff). diffs[max_rounds] (may be NULL) receives the
 * per-round diff; *rounds_done the number executed.
 */
int gslam_run(gslam_graph *g, int max_rounds, double *diffs, int *rounds_done);

/* ---- stages, for callers that drive the round themselves ---- */
int gslam_linearise(gslam_graph *g);                 /* edge blocks from current poses */
int gslam_assemble(gslam_graph *g);                  /* Omega, xi, block-Jacobi inverse */
int gslam_solve(gslam_graph *g, gslam_solve_stats *stats); /* dx = Omega^-1 xi */
int gslam_update(gslam_graph *g, double *diff);      /* poses += dx */

/* Edge blocks in the reference's Edge order: [n_edges][42] = UL, UR, BL, BR, xi_u, xi_b. */
int gslam_get_edge_blocks(gslam_graph *g, double *blocks);
/* Assembles from caller-provided device edge blocks (same layout) instead of linearising. */
int gslam_assemble_from_edges(gslam_graph *g, const double *d_blocks);
/* Omega and xi in the reference's scalar CSR (MatrixOps.h:21-27): row_ptr[3N+1], col_idx[nnz],
 * values[nnz], xi[3N]; any pointer may be NULL. */
int gslam_get_csr(gslam_graph *g, int *row_ptr, int *col_idx, double *values, double *xi);
/* The last solution dx[3N] (original order). */
int gslam_get_dx(gslam_graph *g, double *dx);
/* Block-Jacobi inverses [N][9] (original order). */
int gslam_get_diag_inv(gslam_graph *g, double *dinv);

/* y = Omega x on device pointers in original order [3N] (FP64, row sums in column order). */
int gslam_spmv(gslam_graph *g, const double *d_x, double *d_y);
/*
 * Times FP64 (prec 0) or FP32 (prec 1) SpMVs y = Omega x: each of `reps` launches
 * multiplies n_copies copies of the matrix values (allocated for the call, back to
 * back, one result vector each) by the same x; *ms = mean device milliseconds per
 * matrix. With n_copies * matrix bytes above three L2 sizes every launch streams
 * its values from HBM.
 */
int gslam_spmv_bench(gslam_graph *g, int prec, int reps, int n_copies, float *ms);
/* Algorithmic bytes of one SpMV: values, column indices, x read once, y written once. */
int gslam_spmv_bytes(gslam_graph *g, int prec, int64_t *bytes);

/* ---- host-only utilities (no GPU needed) ---- */
/* Observation-edge order of make_edges (src/cpu_pcg_fp64/GSLAM.c:222-318): pairs of z-list
 * indices (pj[e], pk[e]). Call with cap 0 to get the count in *n_pairs. */
int gslam_obs_edge_order(uint32_t n_obs, const uint32_t *obs_landmark, uint32_t *pj, uint32_t *pk,
                         int64_t cap, int64_t *n_pairs);
/* The reference's scalar CSR pattern (MatrixOps.c:175-221) for edges (t1[e], t2[e]) between
 * n_poses poses plus the anchor on pose 0. Call with col_idx NULL to get *nnz. */
int gslam_csr_pattern(uint32_t n_poses, int64_t n_edges, const uint32_t *t1, const uint32_t *t2,
                      int *row_ptr, int *col_idx, int64_t *nnz);
/*
 * The sliced 3x3-block layout that gslam_create_* uploads for the edges (t1[e], t2[e])
 * between n_poses poses, computed on the host (no counterpart in the reference: it
 * exposes where every block and every edge contribution lands, for tools and tests).
 * sell_window <= 0 takes the library default (1024), 1 skips the row-length sort.
 * segment_starts (n_segments ascending rows, the first 0) marks a batch's graphs: rows
 * keep their order inside their graph's range and the sort windows restart at every
 * start; with n_segments 0 the rows of the one graph are put in Cuthill-McKee order
 * first. diag_rows adds a diagonal block to rows that no edge touches (a batch's padding
 * rows). Every output pointer may be NULL; sizes come back in *info:
 *   perm[n_rows]                          new row -> pose
 *   slice_ptr[n_slices + 1]               first slot of each 32-row slice
 *   col[n_slots]                          new row of each slot's block column, -1 padding
 *   ctr_ptr[n_slots + 1], ctr[4 n_edges]  per slot, 4 e + sub (0..3 = UL UR BL BR) in edge order
 *   xi_ptr[n_rows + 1], xi_ctr[2 n_edges] per new row, 2 e + (0 upper, 1 bottom) in edge order
 *   slot_csr[n_slots]                     position of the slot's entry (0,0) in the reference's
 *                                         scalar CSR (-1 padding, -2 the bare pose-0 anchor)
 */
typedef struct gslam_layout_info {
    int64_t n_rows, n_slices, n_slots, nnzb, csr_nnz, anchor_slot;
    int32_t max_width, bare_anchor;
} gslam_layout_info;
int gslam_layout_plan(uint32_t n_poses, int64_t n_edges, const uint32_t *t1, const uint32_t *t2,
                      int sell_window, uint32_t n_segments, const int32_t *segment_starts,
                      uint32_t n_diag_rows, const int32_t *diag_rows, gslam_layout_info *info,
                      int32_t *perm, int64_t *slice_ptr, int32_t *col, int64_t *ctr_ptr, int64_t *ctr,
                      int64_t *xi_ptr, int64_t *xi_ctr, int64_t *slot_csr);

/* ---- reference log files (src/cpu_pcg_fp64/GSLAM.c:415-493, data/README.md) ---- */
typedef struct gslam_log {
    double delta;
    uint32_t n_u, n_x, n_z;
    uint32_t *u_step;   /* [n_u] */
    double *u;          /* [2 * n_u] nu, omega */
    uint32_t *x_step;   /* [n_x] */
    double *x;          /* [3 * n_x] x, y, theta */
    uint32_t *z_step;   /* [n_z] */
    uint32_t *z_lm;     /* [n_z] */
    double *z;          /* [2 * n_z] range, bearing */
} gslam_log;
/* Parses a log like read_data: space-separated tokens; `u`, `x`, `z` records; any
 * other first token sets delta from the second. Returns GSLAM_ERR_BAD_INPUT for a
 * missing file or a truncated record. Free with gslam_free_log. */
int gslam_read_log(const char *path, gslam_log **out);
void gslam_free_log(gslam_log *log);

/* ---- solve without any device allocation ---- */
/*
 * No counterpart in the reference. For callers that cannot allocate device memory when
 * they solve: processes whose device memory is owned by another allocator or fixed up
 * front, real-time loops in which an allocation could block or fail. Solves the reference's
 * system (scalar CSR of Omega, dim = 3 * poses, columns ascending within a row; all
 * pointers are device memory the caller owns) with block-Jacobi PCG in FP64
 * (||r|| < tol ||b|| or max_iter iterations, x overwritten) on `stream`
 * (a cudaStream_t; NULL = legacy default stream), using a fixed scratch array inside the
 * library: GSLAM_STATIC_SCRATCH_BYTES on every GPU that loads the library, held until
 * the process exits; systems above GSLAM_STATIC_MAX_POSES poses return
 * GSLAM_ERR_TOO_LARGE. It calls no cudaMalloc or cudaFree. The first call on a device
 * looks up the scratch's device address and caches it: make that first call before any
 * stream capture. All calls share the scratch, so calls that overlap on the GPU race:
 * serialise them. stats (host, may be NULL) makes the call wait for the result and
 * report a timed-out solve as GSLAM_ERR_DEVICE_TIMEOUT; without it the call returns as
 * soon as the solve is queued, and gslam_pcg_static_status reads the result later.
 */
#define GSLAM_STATIC_SCRATCH_BYTES (4u << 20)
#define GSLAM_STATIC_MAX_POSES 16384
int gslam_pcg_solve_static(int dim, const int *d_row_ptr, const int *d_col_idx,
                           const double *d_values, const double *d_b, double *d_x, double tol,
                           int max_iter, void *stream, gslam_solve_stats *stats);
/*
 * The status of the last gslam_pcg_solve_static queued on the current device, for a
 * caller that queued it with stats == NULL: waits for the work queued on `stream` so far
 * (queue the read on the solve's stream, or synchronize first), then fills *stats
 * (iterations, reason, relative residual; may be NULL) and returns GSLAM_ERR_DEVICE_TIMEOUT
 * when a barrier wait of that solve gave up (its x is then incomplete). The status lives in
 * the shared scratch: read it before the next call on this device overwrites it.
 * GSLAM_ERR_BAD_INPUT when no solve has been queued on this device. Allocates nothing.
 */
int gslam_pcg_static_status(void *stream, gslam_solve_stats *stats);

/*
 * Round cost of a reference-factor graph at its current poses: the cost that the
 * reference's use_diff = 0 criterion accumulates (GSLAM.c:74-87), with the dimensions
 * that code meant: sum over edges, in the reference's edge order, of
 * hat_e^T Omega hat_e (observation edges: 2-vector, 2x2 Omega, lambda 1.0) and
 * lambda d^T Omega d (motion edges, d = x2 - state_transition(x1)). The reference reads
 * a 3-vector out of its 2-element hat_e and never resets the sum between rounds; this
 * is computed afresh at each call. edge_costs (host, n_edges entries, may be NULL)
 * receives the per-edge terms.
 */
int gslam_cost(gslam_graph *g, double *cost, double *edge_costs);

/*
 * Landmark map of a reference-factor graph at its current poses (GSLAM.c:141-196 with
 * MapEdge_create, MapEdge.c:7-32): for every landmark, in order of first appearance in
 * the observation list, the mean over its observations of
 * (x + r cos(theta + phi), y + r sin(theta + phi)). *n_landmarks receives the count;
 * ids (n entries) and ms (2 per landmark, host) may be NULL to query the count only.
 * (The reference computes this map and frees it; here it is returned.)
 */
int gslam_landmark_map(gslam_graph *g, uint32_t *n_landmarks, uint32_t *ids, double *ms);

/*
 * Batches of independent SE(2) graphs (no counterpart in the reference, which solves
 * one graph per process and sweeps lambda with a shell loop).
 *
 * gslam_create_se2_batch: one handle for n_graphs graphs of any sizes, each with its
 * own lambda and anchor. They are laid out as one block-diagonal graph, each graph's
 * poses padded to a multiple of 32 (padding poses stay at 0). gslam_batch_layout
 * gives the first padded pose of every graph (pose_offset[n_graphs] = total), so
 * gslam_get_poses / gslam_set_poses work on the concatenation.
 *
 * gslam_batch_round: one Gauss-Newton round of every graph; the linear solves run in
 * ONE persistent launch (block-Jacobi PCG with each graph's own alpha, beta and
 * stopping test, tol / max_iter of the handle's options, FP64). per_graph (host,
 * n_graphs entries, may be NULL) receives each graph's iterations, reason, relative
 * residual and update norm diff = ||dx|| / sqrt(3 n_poses). gslam_round on a batch
 * runs the same round and reports the largest iteration count and residual.
 */
int gslam_create_se2_batch(const gslam_se2_graph *graphs, uint32_t n_graphs, const gslam_opts *opts,
                           gslam_graph **out);
int gslam_batch_round(gslam_graph *g, gslam_solve_stats *per_graph);
int gslam_batch_layout(gslam_graph *g, uint32_t *n_graphs, uint32_t *pose_offset);

/*
 * Dense Gauss-Jordan inverse / solve, replacing the reference's dense check path
 * (inv: src/cpu_pcg_fp64/MatrixOps.c:29-91 and its CUDA twin
 * src/gpu_gj_fp64/inv.cu:221-354; Omega^-1 then Omega^-1 xi): elimination without
 * pivoting, blocked by 64 columns, trailing updates on the FP64 tensor cores.
 * Matrices are row-major device memory with leading dimension lda; stream is a
 * cudaStream_t (NULL = legacy default stream). gslam_gj_inverse overwrites d_a with
 * its inverse; gslam_gj_solve leaves d_a unchanged and writes x = A^-1 b to d_x.
 * ms (may be NULL) receives the device time of the elimination. Both allocate their
 * scratch (an n x n copy padded to a multiple of 64) and synchronize the stream.
 */
int gslam_gj_inverse(int n, double *d_a, int lda, void *stream, float *ms);
int gslam_gj_solve(int n, const double *d_a, int lda, const double *d_b, double *d_x, void *stream, float *ms);
/* Measured FP64 tensor-core throughput (the Gauss-Jordan updates' roofline): one launch of
 * ctas_per_sm x (SM count) CTAs of 8 warps, each warp `reps` x 8 independent m8n8k4 DMMAs on
 * register operands, on the current device's legacy default stream; *tflops = 512 flops per
 * DMMA / device time (*ms, may be NULL). Allocates a small output buffer. */
int gslam_dmma_bench(int reps, int ctas_per_sm, double *tflops, float *ms);

/*
 * Differentiation of a converged SE(2) graph (no counterpart in the reference, whose
 * programs only run Gauss-Newton forward).
 *
 * gslam_set_se2_weights: replaces lambda and, when log_w is non-null, the per-edge
 * log information weights (3 per edge, edge order of gslam_create_se2) of an SE(2)
 * graph; the block structure is kept.
 *
 * gslam_adjoint: implicit-function adjoint at the graph's current poses, which should
 * be converged (g(x) = sum_e J_e^T Lambda_e e_e = 0). Solves H mu = dL/dposes with the
 * FP64 persistent PCG (the graph's tol / max_iter; H = the exact Hessian of
 * (1/2) sum_e e^T Lambda_e e, symmetric, pose-0 anchor included), then
 *   dL_dlogw[3e + k] = -lambda exp(w_{e,k}) e_{e,k} (J_e mu)_k   (host, 3 per edge),
 *   *dL_dlambda      = sum of dL_dlogw / lambda                   (host),
 * mu_out (host, 3 N, may be NULL) receives mu. dL_dposes is host memory, 3 N doubles,
 * pose-major. The graph's assembled Omega / xi are overwritten; the next round
 * re-linearises. Reference-factor graphs return GSLAM_ERR_BAD_INPUT.
 */
int gslam_set_se2_weights(gslam_graph *g, double lambda, const double *log_w);
int gslam_adjoint(gslam_graph *g, const double *dL_dposes, double *dL_dlambda, double *dL_dlogw,
                  double *mu_out, gslam_solve_stats *stats);

/* Library version string and the error text of the last failing call on this thread. */
const char *gslam_version(void);
const char *gslam_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
