/* gslam_api_internal.h — device-side objects behind the C ABI (internal). */
#ifndef GSLAM_API_INTERNAL_H
#define GSLAM_API_INTERNAL_H

#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "gslam.h"
#include "gslam_internal.h"
#include "kernels.cuh"

/* Device allocations owned by one object, released together. */
struct DevMem {
    std::vector<void *> ptrs;
    void release();
};

/* Device copy of a layout plus the solver's work vectors. */
struct DevLayout {
    DevMem mem;
    int n_rows = 0, n_slices = 0;
    int64_t n_slots = 0;
    int *perm = nullptr, *iperm = nullptr, *row_len = nullptr, *col = nullptr;
    int *diag_slot = nullptr, *chunk_slice = nullptr;
    int64_t *slice_ptr = nullptr, *slot_csr = nullptr;
    double *val = nullptr, *dinv = nullptr;
    float *val32 = nullptr;
    bool val32_fresh = false;      /* val32 holds the current values */
    double *b4 = nullptr, *x4 = nullptr, *r4 = nullptr, *z4 = nullptr;
    double *p4a = nullptr, *p4b = nullptr, *q4 = nullptr;
    float *f[6] = { nullptr, nullptr, nullptr, nullptr, nullptr, nullptr };
    double *partials = nullptr;
    GridSync *gs = nullptr;
    PcgResult *res = nullptr;
    int grid = 0, block = 0, n_sm = 0;
    int clock_khz = 2000000;       /* SM clock, for barrier wait limits */
    int partial_capacity = 0;
    /* shared-memory-resident solver (pcg_resident.cu), when the layout fits */
    bool resident = false;
    int res_grid = 0, res_block = 0;
    int *cta_slice = nullptr;      /* [res_grid + 1] */
    int64_t smem_val_cap = 0;      /* doubles staged by the CTA that stages fewest */
    int *lcol = nullptr, *halo_ptr = nullptr, *halo_rows = nullptr; /* CTA-local columns, halo lists */
    unsigned char *row_export = nullptr; /* rows some other CTA's halo lists */
    size_t smem_bytes = 0;
    bool mixed_ok = false;          /* the mixed solver's shared-memory layout fits */
    int64_t mixed_val_cap = 0;     /* floats staged by the CTA that stages fewest */
    size_t mixed_smem_bytes = 0;   /* dynamic shared memory per launch: the largest CTA layout (mixed_smem_layout) */
    bool cg_ok = false;             /* the FP64 one-reduction solver's layout fits */
    int64_t cg_val_cap = 0;        /* doubles staged by the CTA that stages fewest */
    size_t cg_smem_bytes = 0;
    double *w4 = nullptr;          /* its sixth published vector (made on first use) */
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;   /* brackets the solver launch */
    int max_grid_alloc() const { return partial_capacity; }
};

/* A batch of independent SE(2) graphs as one block-diagonal graph (batch.cu). */
struct BatchState {
    int n_graphs = 0;
    std::vector<int> pose_off;   /* [n_graphs + 1] first (padded) pose of each graph */
    std::vector<int> n_real;     /* [n_graphs] poses of each graph without padding */
    int *d_pose_off = nullptr, *d_n_real = nullptr;
    int n_anchor = 0;
    int64_t *d_anchor_slots = nullptr;
    double *d_anchor_vals = nullptr;
    /* solver partition */
    int grid = 0, block = 0, max_slices = 0;
    size_t smem_bytes = 0;
    int total_parts = 0;
    int *d_cta_slice = nullptr, *d_slice_graph = nullptr, *d_cta_g0 = nullptr, *d_cta_g1 = nullptr;
    int *d_graph_cta0 = nullptr, *d_graph_ncta = nullptr, *d_part_off = nullptr;
    double *d_partials = nullptr, *d_gdiff = nullptr;
    PcgResult *d_res = nullptr, *h_res = nullptr;
    double *h_gdiff = nullptr;
    int *d_active = nullptr;
    /* mixed batches: FP32 right-hand side, per-graph active flags and residual norms */
    float *d_bf4 = nullptr;
    int *d_gactive = nullptr;
    int *d_gcap = nullptr;       /* mixed: each graph's iteration cap for the current inner pass */
    double *d_gres = nullptr, *h_gres = nullptr;
    int *d_skip = nullptr;       /* graphs the FP64 rerun of a stagnated mixed batch leaves alone */
    /* chunk sums of the per-graph norm kernels */
    double *d_chunk_part = nullptr;
    int max_chunks = 1;
};

struct gslam_graph {
    int device = 0;
    cudaStream_t st = nullptr;
    gslam_opts o;
    int factors = GSLAM_FACTORS_REFERENCE;
    gslam_structure S;
    DevLayout L;
    DevMem mem;
    int n_poses = 0;
    int64_t n_obs_edges = 0, n_edges = 0;
    double delta = 1.0, lambda = 1.0, mns[4] = { 0.19, 0.001, 0.13, 0.2 };
    double anchor = 1000000.0;
    /* reference factor inputs */
    double *d_poses = nullptr, *d_controls = nullptr, *d_z_rb = nullptr;
    unsigned *d_z_step = nullptr, *d_pj = nullptr, *d_pk = nullptr;
    /* SE(2) factor inputs */
    unsigned *d_ei = nullptr, *d_ej = nullptr;
    double *d_meas = nullptr, *d_info = nullptr; /* info = exp(log_w) */
    /* per-round buffers */
    double *d_blocks = nullptr;
    int64_t *d_ctr_ptr = nullptr, *d_ctr = nullptr, *d_xi_ptr = nullptr, *d_xi_ctr = nullptr;
    double *d_dx = nullptr, *d_block_sums = nullptr, *d_diff = nullptr;
    int n_upd_blocks = 1;
    double *d_csr_tmp = nullptr, *d_xi_tmp = nullptr;
    double *d_adj = nullptr;   /* adjoint: rhs, mu (3 N each), per-edge gradient (3 E) */
    BatchState *batch = nullptr; /* non-null for a batch of graphs */
    /* landmark groups of the z list (reference graphs) */
    std::vector<unsigned> lm_ids;
    int64_t *d_lm_ptr = nullptr;
    unsigned *d_lm_members = nullptr;
    double *d_lm_ms = nullptr;
    PcgResult *h_res = nullptr;
    double *h_diff = nullptr;
    /* round cost: per-edge terms, block sums, total (allocated on first use) */
    double *d_edge_cost = nullptr, *d_cost_blocks = nullptr, *d_cost = nullptr;
    PcgResult last_res = {};
    cudaEvent_t ev_round0 = nullptr, ev_round1 = nullptr;
    /* gslam_opts.round_graph: the captured round and how many rounds ran eagerly */
    cudaGraphExec_t round_exec = nullptr;
    int eager_rounds = 0;
};

int gslam_layout_upload(DevLayout *L, const gslam_structure &S, cudaStream_t st, int device,
                        const gslam_opts &o);
int gslam_layout_ensure_fp32(DevLayout *L, cudaStream_t st);
int gslam_layout_solve(DevLayout *L, cudaStream_t st, const gslam_opts &o, PcgResult *h_res,
                       gslam_solve_stats *stats);
void gslam_layout_release(DevLayout *L);
/* Assembles Omega / xi from edge blocks; optionally also writes the reference's CSR
 * values (csr_vals) and xi in original order (xi_orig), both device pointers. */
int gslam_assemble_ex(gslam_graph *g, const double *blocks, double *csr_vals, double *xi_orig);
/* gslam_update that also records `done` (may be null) after the update kernels. */
int gslam_update_ex(gslam_graph *g, double *diff, cudaEvent_t done);
/* Records an error message for gslam_last_error(). */
void gslam_set_last_error(const char *msg);
void gslam_set_error(const char *fmt, const char *what, int code);

/* ---- helpers shared by the handle API's translation units (api.cu, batch_api.cu) ---- */

/* a failing CUDA call: record it for gslam_last_error() and return GSLAM_ERR_CUDA */
#define CK(call)                                                                               \
    do {                                                                                       \
        cudaError_t _e = (call);                                                               \
        if (_e != cudaSuccess) {                                                               \
            gslam_set_last_error((std::string(#call) + ": " + cudaGetErrorString(_e)).c_str()); \
            return GSLAM_ERR_CUDA;                                                             \
        }                                                                                      \
    } while (0)

#define BAD(msg)                        \
    do {                                \
        gslam_set_last_error(msg);      \
        return GSLAM_ERR_BAD_INPUT;     \
    } while (0)

/* device allocation owned by m (released with it) */
template <class T>
inline cudaError_t dalloc(DevMem &m, T **p, size_t n) {
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, (n ? n : 1) * sizeof(T));
    if (e != cudaSuccess) return e;
    m.ptrs.push_back(q);
    *p = (T *)q;
    return cudaSuccess;
}

/* device copy of a host vector, owned by m */
template <class T>
inline cudaError_t dupload(DevMem &m, cudaStream_t st, T **p, const std::vector<T> &v) {
    cudaError_t e = dalloc(m, p, v.size());
    if (e != cudaSuccess) return e;
    if (v.empty()) return cudaSuccess;
    return cudaMemcpyAsync(*p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st);
}

/* an event record that a stream capture keeps as a node of the graph */
cudaError_t record_event(cudaEvent_t e, cudaStream_t st);
/* elapsed time between two recorded events, 0 when unavailable */
float elapsed_ms(cudaEvent_t a, cudaEvent_t b);
/* creation steps every handle shares: options, device, stream, pinned status words */
int common_setup(gslam_graph *g, const gslam_opts *opts);
/* structure, layout upload and per-round buffers of a handle with edges (t1, t2) */
int finish_setup(gslam_graph *g, const std::vector<unsigned> &t1, const std::vector<unsigned> &t2,
                 const std::vector<int> *diag_rows = nullptr, const std::vector<int> *segments = nullptr);
/* the batched solve behind gslam_solve / gslam_round on a batch handle (batch_api.cu) */
int batch_solve(gslam_graph *g, gslam_solve_stats *per_graph, gslam_solve_stats *total,
                const int *d_skip = nullptr);

#endif
