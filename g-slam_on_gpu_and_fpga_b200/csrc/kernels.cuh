/* kernels.cuh — launchers of libgslam's device kernels (internal). */
#ifndef GSLAM_KERNELS_CUH
#define GSLAM_KERNELS_CUH

#include <cuda_runtime.h>
#include <stdint.h>

void launch_obs_edges(cudaStream_t st, int64_t n, const unsigned *pj, const unsigned *pk,
                      const unsigned *z_step, const double *z_rb, const double *poses,
                      double *blocks);
void launch_motion_edges(cudaStream_t st, int n_poses, int64_t first_edge, const double *controls,
                         double delta, double lambda, const double *mns, const double *poses,
                         double *blocks);
void launch_se2_edges(cudaStream_t st, int64_t n, int64_t first_edge, const unsigned *ei,
                      const unsigned *ej, const double *meas, const double *info, double lambda,
                      const double *poses, double *blocks);
void launch_assemble(cudaStream_t st, int64_t n_slots, const int64_t *ctr_ptr, const int64_t *ctr,
                     const double *blocks, int64_t anchor_slot, double anchor, double *val,
                     float *val32, const int64_t *slot_csr, const int *chunk_slice,
                     const int *row_len, double *csr_vals);
void launch_sell_to_csr(cudaStream_t st, int64_t n_slots, const int64_t *slot_csr,
                        const int *chunk_slice, const int *row_len, const double *val,
                        double *csr_vals);
void launch_assemble_xi(cudaStream_t st, int n_rows, const int64_t *xi_ptr, const int64_t *xi_ctr,
                        const double *blocks, double *b4, const int *perm, double *xi_orig);
void launch_csr_to_sell(cudaStream_t st, int64_t n_slots, const int64_t *slot_csr,
                        const int *chunk_slice, const int *row_len, const double *csr_vals,
                        double *val, float *val32);
void launch_val_to_f32(cudaStream_t st, int64_t n, const double *val, float *val32);
void launch_gather_vec(cudaStream_t st, int n_rows, const int *perm, const double *src, double *dst4);
void launch_scatter_vec(cudaStream_t st, int n_rows, const int *perm, const double *src4, double *dst);
void launch_diag_inv(cudaStream_t st, int n_rows, const int *diag_slot, const double *val,
                     double *dinv);
struct PcgResult;
void launch_pose_update(cudaStream_t st, int n_rows, const int *iperm, const double *x4,
                        double *poses, double *dx, int wrap, double *block_sums, int n_blocks,
                        double *diff_out, const PcgResult *guard = nullptr);

/* ---- solver ---- */

struct GridSync {
    unsigned count;
    unsigned gen;
    int abort;
    int pad;
};

struct PcgResult {
    int iterations;
    int reason;
    int refinements;
    int timeout;
    double rnorm;
    double bnorm;
};

struct PcgParams {
    int n_rows;
    int n_slices;
    const int64_t *slice_ptr;
    const int *row_len;
    const int *col;
    const double *val;     /* FP64 values (slot layout) */
    const float *val32;    /* FP32 copy (mixed) */
    const double *dinv;    /* block-Jacobi inverses (slot layout) */
    const double *b4;      /* right-hand side, padded new order */
    double *x4, *r4, *z4, *p4a, *p4b, *q4;  /* FP64 work vectors */
    double *w4;            /* FP64 one-reduction solver: its sixth published vector */
    float *xf4, *rf4, *zf4, *pfa4, *pfb4, *qf4; /* FP32 work vectors (mixed) */
    double tol_rel;
    int max_iter;
    double inner_tol;
    int inner_max_iter;
    int max_refine;
    double *partials;      /* [2][4 * gridDim.x]: two alternating buffers */
    GridSync *gs;
    PcgResult *res;
    long long spin_limit;  /* clock cycles a barrier may wait */
    int absent_cta;        /* test hook: CTA that leaves before its first barrier, -1 = none */
    const int *cta_slice;  /* resident solver: [grid + 1] first slice of each CTA */
    int64_t smem_val_cap;  /* resident solvers: the smallest CTA's staged values (statistics only) */
    const int *lcol;       /* resident solver: per slot, CTA-local column index (own rows, then halo) */
    const int *halo_ptr;   /* resident solver: [grid + 1] halo list bounds per CTA */
    const int *halo_rows;  /* resident solver: halo rows (new row indices) */
    const unsigned char *row_export; /* 1 for rows in another CTA's halo: only those are published */
    int64_t smem_budget;   /* resident, mixed and FP64 one-reduction solvers: dynamic shared memory per CTA */
};

/* Shared-memory layout of one CTA of the FP64 resident solver, from its own sizes: local
 * columns and p of own and halo rows (32 B each) after the values, and as many values (whole
 * multiples of 288) as the budget leaves (val_cap < 0: the fixed parts alone do not fit). */
struct ResidentSmem {
    int64_t val_cap, col_off, p_off, end;
};
__host__ __device__ inline ResidentSmem resident_smem_layout(int64_t n_slots, int64_t n_slices, int64_t n_halo,
                                                             int64_t budget) {
    auto up = [](int64_t b) { return (b + 127) / 128 * 128; };
    const int64_t col_b = up(4 * n_slots), p_b = 32 * (32 * n_slices + n_halo);
    ResidentSmem m;
    const int64_t fixed = col_b + p_b;
    m.val_cap = budget >= fixed ? (budget - fixed) / 8 / 288 * 288 : -1;
    const int64_t nv = m.val_cap > 9 * n_slots ? 9 * n_slots : m.val_cap;
    m.col_off = up(8 * (nv > 0 ? nv : 0));
    m.p_off = m.col_off + col_b;
    m.end = m.p_off + p_b;
    return m;
}

/* Shared-memory layout of one CTA of the mixed / FP64 one-reduction solver, from its own
 * sizes: the fixed parts (local columns, D^-1 of own rows when staged, z of own and halo
 * rows, the halo's u and v for the first `block` halo rows) after the values, and as many
 * values (whole multiples of 288, one block position of a slice) as the budget leaves.
 * val_cap < 0: the fixed parts alone exceed the budget. */
struct MixedSmem {
    int64_t val_cap, col_off, dinv_off, halo_off, stage_off, end;
};
__host__ __device__ inline MixedSmem mixed_smem_layout(int64_t elem, bool fp64, int64_t n_slots, int64_t n_slices,
                                                       int64_t n_halo, int64_t block, int64_t budget) {
    auto up = [](int64_t b) { return (b + 127) / 128 * 128; };
    const int64_t col_b = up(4 * n_slots);
    const int64_t dinv_b = fp64 ? 0 : 2304 * n_slices;
    const int64_t z_b = up(4 * elem * (32 * n_slices + n_halo));
    const int64_t stage_b = up(8 * elem * (n_halo < block ? n_halo : block));
    MixedSmem m;
    const int64_t fixed = col_b + dinv_b + z_b + stage_b;
    m.val_cap = budget >= fixed ? (budget - fixed) / elem / 288 * 288 : -1;
    const int64_t nv = m.val_cap > 9 * n_slots ? 9 * n_slots : m.val_cap;
    m.col_off = up(elem * (nv > 0 ? nv : 0));
    m.dinv_off = m.col_off + col_b;
    m.halo_off = m.dinv_off + dinv_b;
    m.stage_off = m.halo_off + z_b;
    m.end = m.stage_off + stage_b;
    return m;
}

/* Round cost terms per edge and their total (kernels.cu); block_sums holds
 * edge_cost_blocks(n_edges) doubles. */
int edge_cost_blocks(int64_t n_edges);
void launch_edge_costs(cudaStream_t st, int64_t n_obs_edges, int n_poses, const unsigned *pj, const unsigned *pk,
                       const unsigned *z_step, const double *z_rb, const double *controls, double delta,
                       double lambda, const double *mns, const double *poses, double *edge_cost,
                       double *block_sums, double *total);

void launch_landmark_map(cudaStream_t st, int n_groups, const int64_t *ptr, const unsigned *members,
                         const unsigned *z_step, const double *z_rb, const double *poses, double *ms);

/* SpMV of n_copies matrices sharing one block pattern, in one launch (pcg.cu). */
void launch_spmv_multi64(cudaStream_t st, int n_copies, int n_rows, int n_slices, const int64_t *slice_ptr,
                         const int *row_len, const int *col, const double *val, int64_t stride,
                         const double *x4, double *y4, int64_t ystride);
void launch_spmv_multi32(cudaStream_t st, int n_copies, int n_rows, int n_slices, const int64_t *slice_ptr,
                         const int *row_len, const int *col, const float *val, int64_t stride,
                         const float *x4, float *y4, int64_t ystride);

/* Batched solver (batch.cu): per-graph scalars over a block-diagonal system. */
struct BatchParams {
    int n_graphs;
    const int *cta_slice;    /* [grid + 1] first slice of each CTA */
    const int *slice_graph;  /* [n_slices] graph of each slice */
    const int *cta_g0, *cta_g1; /* [grid] first / last graph of each CTA's slices */
    const int *graph_cta0;   /* [n_graphs] first CTA owning rows of the graph */
    const int *graph_ncta;   /* [n_graphs] CTAs owning rows of the graph */
    const int *part_off;     /* [n_graphs] offset of the graph's CTA partials */
    int total_parts;         /* sum of graph_ncta */
    double *partials;        /* [2 buffers][2 values][total_parts] */
    PcgResult *res;          /* [n_graphs] */
    int *active;             /* graphs still iterating (set to n_graphs before launch) */
    const float *bf4;        /* FP32 inner solve: right-hand side (padded rows) */
    const int *skip;         /* [n_graphs] or null: graphs left exactly as they are (done from the
                              * start, their vectors untouched: the mixed batch's FP64 rerun of
                              * only the graphs that stagnated) */
    const int *cap;          /* [n_graphs] or null: each graph's own iteration cap (at most the
                              * launch's max_iter; the mixed batch's inner passes, each graph
                              * with what is left of its budget) */
};
/* fp32: the inner solve of the mixed batch (FP32 values / vectors in PcgParams' FP32
 * fields, right-hand side bf4); otherwise the FP64 PCG on val / b4. */
cudaError_t launch_pcg_batch(cudaStream_t st, const PcgParams &p, const BatchParams &b, int grid, int block,
                             size_t smem_bytes, bool fp32);
int pcg_batch_max_grid(int block, size_t smem_bytes, int device);
int pcg_batch_lg_max();
void launch_add_diag(cudaStream_t st, int n, const int64_t *slots, const double *anchor, double *val);
void launch_batch_rhs32(cudaStream_t st, int n_rows, const int *slice_graph, const int *active, const double *r4,
                        float *bf4);
void launch_batch_add_x(cudaStream_t st, int n_rows, const float *xf4, double *x4);
/* per-graph ||b - q||^2 (writing r4 = b4 - q4) and update norms, spread over (chunk, graph)
 * CTAs; part holds n_graphs x max_chunks chunk sums, max_chunks = batch_max_chunks(rows of
 * the largest padded graph) */
void launch_batch_resid(cudaStream_t st, int n_graphs, const int *pose_off, const double *b4, const double *q4,
                        double *r4, double *out, double *part, int max_chunks);
void launch_batch_diff(cudaStream_t st, int n_graphs, const int *pose_off, const int *n_real, const double *dx,
                       double *out, double *part, int max_chunks);
int batch_max_chunks(int max_graph_rows);

/* Cooperative launch of the persistent solver; returns the CUDA error. */
cudaError_t launch_pcg(cudaStream_t st, const PcgParams &p, int precision, int grid, int block);
/* Largest co-resident grid for the solver at this block size (0 if unsupported). */
int pcg_max_grid(int precision, int block, int device);

/* Shared-memory-resident solver (pcg_resident.cu). */
cudaError_t launch_pcg_resident(cudaStream_t st, const PcgParams &p, int grid, int block,
                                size_t smem_bytes);
int pcg_resident_max_grid(int device, size_t smem_bytes);

/* Mixed-precision solver (pcg_mixed.cu); fp64: the same kernel as the FP64 one-reduction
 * solver. */
cudaError_t launch_pcg_mixed(cudaStream_t st, const PcgParams &p, int grid, int block, size_t smem_bytes,
                             bool fp64);
int pcg_mixed_max_grid(int device, size_t smem_bytes);

/* Standalone SpMV y = A x on padded new-order vectors (FP64 or FP32 values). */
void launch_spmv64(cudaStream_t st, int n_rows, int n_slices, const int64_t *slice_ptr,
                   const int *row_len, const int *col, const double *val, const double *x4,
                   double *y4);
void launch_spmv32(cudaStream_t st, int n_rows, int n_slices, const int64_t *slice_ptr,
                   const int *row_len, const int *col, const float *val, const float *x4,
                   float *y4);

#endif
