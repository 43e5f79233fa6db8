/*
 * dropin.cu — the reference's solver entry points (include/gslam_dropin.h) on
 * top of libgslam's device path.
 *
 *   pcg_solve_sparse      <- src/cpu_pcg_fp64/MatrixOps.c:281-391
 *   device_graph_*        <- src/gpu_pcg_fp64/device_graph.cuh:23-91 / .cu:834-1129
 *
 * Like the reference GPU twin these keep one graph in process-wide state (not
 * re-entrant). Unlike it, the edge order follows the reference CPU program
 * (landmarks in order of first appearance, GSLAM.c:246-261) and the assembly is
 * a deterministic gather, so Omega and xi are bit-identical to the CPU
 * reference's build_csr_from_edges instead of atomics-ordered.
 */
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "gslam.h"
#include "gslam_api_internal.h"
#include "gslam_dropin.h"
#include "gslam_internal.h"
#include "kernels.cuh"

static int s_status = GSLAM_OK;
static gslam_graph *s_graph = nullptr;
static int *s_d_row_ptr = nullptr, *s_d_col_idx = nullptr;

static void dropin_fail(int rc, const char *where) {
    s_status = rc;
    if (getenv("GSLAM_DROPIN_NOEXIT")) return;
    fprintf(stderr, "gslam error at %s: %s\n", where, gslam_last_error());
    exit(1);
}

#define DCK(call, where)                                  \
    do {                                                  \
        cudaError_t _e = (call);                          \
        if (_e != cudaSuccess) {                          \
            gslam_set_last_error(cudaGetErrorString(_e)); \
            dropin_fail(GSLAM_ERR_CUDA, where);           \
            return;                                       \
        }                                                 \
    } while (0)

int gslam_dropin_status(void) { return s_status; }

/* ------------------------------------------------------------------------ */
/* device_graph_* (GPU twin API)                                             */
/* ------------------------------------------------------------------------ */

void device_graph_free(void) {
    if (s_graph) gslam_destroy(s_graph);
    s_graph = nullptr;
    if (s_d_row_ptr) cudaFree(s_d_row_ptr);
    if (s_d_col_idx) cudaFree(s_d_col_idx);
    s_d_row_ptr = s_d_col_idx = nullptr;
}

void device_graph_init(struct Z *zlist, unsigned int n_obs, struct U *us, unsigned int n_poses,
                       unsigned int dim, double delta, double lambda, const double *mns,
                       int *nnz_out) {
    s_status = GSLAM_OK;
    device_graph_free();
    if (dim != 3u * n_poses || n_poses == 0 || (n_obs && !zlist) || !us) {
        gslam_set_last_error("dim must equal 3 * n_poses and the inputs must be non-null");
        dropin_fail(GSLAM_ERR_BAD_INPUT, "device_graph_init");
        return;
    }
    std::vector<double> poses(3 * (size_t)n_poses, 0.0), controls(2 * (size_t)n_poses);
    for (unsigned i = 0; i < n_poses; i++) {
        controls[2 * i] = us[i].nu;
        controls[2 * i + 1] = us[i].omega;
    }
    std::vector<uint32_t> zs(n_obs), zl(n_obs);
    std::vector<double> zrb(2 * (size_t)n_obs);
    for (unsigned i = 0; i < n_obs; i++) {
        zs[i] = zlist[i].step;
        zl[i] = zlist[i].landmark_id;
        zrb[2 * i] = zlist[i].z[0];
        zrb[2 * i + 1] = zlist[i].z[1];
    }
    gslam_reference_graph in;
    memset(&in, 0, sizeof in);
    in.n_poses = n_poses;
    in.poses = poses.data();
    in.controls = controls.data();
    in.delta = delta;
    in.lambda = lambda;
    in.mns = mns;
    in.n_obs = n_obs;
    in.obs_step = zs.data();
    in.obs_landmark = zl.data();
    in.obs = zrb.data();
    int rc = gslam_create_reference(&in, nullptr, &s_graph);
    if (rc != GSLAM_OK) { dropin_fail(rc, "device_graph_init"); return; }
    const gslam_structure &S = s_graph->S;
    const size_t nnz = S.csr_col.size();
    DCK(cudaMalloc(&s_d_row_ptr, S.csr_row_ptr.size() * sizeof(int)), "device_graph_init");
    DCK(cudaMalloc(&s_d_col_idx, (nnz ? nnz : 1) * sizeof(int)), "device_graph_init");
    DCK(cudaMemcpy(s_d_row_ptr, S.csr_row_ptr.data(), S.csr_row_ptr.size() * sizeof(int),
                   cudaMemcpyHostToDevice), "device_graph_init");
    DCK(cudaMemcpy(s_d_col_idx, S.csr_col.data(), nnz * sizeof(int), cudaMemcpyHostToDevice),
        "device_graph_init");
    int lm_active = 0;
    {
        std::vector<unsigned> ids(zl.begin(), zl.end());
        std::sort(ids.begin(), ids.end());
        for (size_t i = 0; i < ids.size();) {
            size_t j = i;
            while (j < ids.size() && ids[j] == ids[i]) j++;
            if (j - i >= 2) lm_active++;
            i = j;
        }
    }
    printf("device_graph_init: dim=%u nnz=%zu obs_edges=%lld lm_active=%d\n", dim, nnz,
           (long long)s_graph->n_obs_edges, lm_active);
    if (nnz_out) *nnz_out = (int)nnz;
}

void device_graph_update(struct HAT_X *hat_xs, unsigned int n_poses, double *d_csr_vals,
                         double *d_xi) {
    s_status = GSLAM_OK;
    if (!s_graph || n_poses != (unsigned)s_graph->n_poses || !hat_xs) {
        gslam_set_last_error("device_graph_update before init or with a different pose count");
        dropin_fail(GSLAM_ERR_BAD_INPUT, "device_graph_update");
        return;
    }
    std::vector<double> flat(3 * (size_t)n_poses);
    for (unsigned i = 0; i < n_poses; i++)
        for (int c = 0; c < 3; c++) flat[3 * i + c] = hat_xs[i].hat_x[c];
    int rc = gslam_set_poses(s_graph, flat.data());
    if (rc == GSLAM_OK) rc = gslam_linearise(s_graph);
    if (rc == GSLAM_OK) rc = gslam_assemble_ex(s_graph, s_graph->d_blocks, d_csr_vals, d_xi);
    if (rc != GSLAM_OK) { dropin_fail(rc, "device_graph_update"); return; }
    DCK(cudaStreamSynchronize(s_graph->st), "device_graph_update");
}

int *device_graph_get_row_ptr(void) { return s_d_row_ptr; }
int *device_graph_get_col_idx(void) { return s_d_col_idx; }

void device_build_diag_inv(int dim) { (void)dim; /* done inside device_pcg_solve, as in the reference */ }

void device_pcg_solve(double *x_h, double *d_csr_vals, double *d_xi, int dim, int nnz,
                      int max_iter) {
    s_status = GSLAM_OK;
    if (!s_graph || dim != 3 * s_graph->n_poses || (size_t)nnz != s_graph->S.csr_col.size() ||
        !x_h || !d_csr_vals || !d_xi) {
        gslam_set_last_error("device_pcg_solve: sizes do not match device_graph_init");
        dropin_fail(GSLAM_ERR_BAD_INPUT, "device_pcg_solve");
        return;
    }
    gslam_graph *g = s_graph;
    launch_csr_to_sell(g->st, g->L.n_slots, g->L.slot_csr, g->L.chunk_slice, g->L.row_len, d_csr_vals,
                       g->L.val, nullptr);
    g->L.val32_fresh = false;
    launch_gather_vec(g->st, g->n_poses, g->L.perm, d_xi, g->L.b4);
    DCK(cudaGetLastError(), "device_pcg_solve");
    gslam_opts o = g->o;
    o.tol = 1e-6; /* device_graph.cu:869 */
    o.max_iter = max_iter;
    o.precision = GSLAM_PREC_FP64;
    int rc = gslam_layout_solve(&g->L, g->st, o, g->h_res, nullptr);
    if (rc != GSLAM_OK) { dropin_fail(rc, "device_pcg_solve"); return; }
    rc = gslam_get_dx(g, x_h);
    if (rc != GSLAM_OK) { dropin_fail(rc, "device_pcg_solve"); return; }
}

/* ------------------------------------------------------------------------ */
/* pcg_solve_sparse (CPU API)                                                */
/* ------------------------------------------------------------------------ */

namespace {
struct CsrCache {
    bool valid = false;
    int dim = 0;
    std::vector<int> rp, ci;
    gslam_structure S;
    DevLayout L;
    std::vector<int64_t> entry_pos; /* [9 * n_slots]: CSR position of (slot, entry) or -1 */
    std::vector<double> hval, hb;
    cudaStream_t st = nullptr;
    PcgResult *h_res = nullptr;
    double *d_x = nullptr;
};
CsrCache s_csr;

void csr_cache_release() {
    if (s_csr.st) cudaStreamSynchronize(s_csr.st);
    gslam_layout_release(&s_csr.L);
    if (s_csr.d_x) cudaFree(s_csr.d_x);
    s_csr.d_x = nullptr;
    s_csr.valid = false;
}

int csr_cache_build(const CSRMatrix *csr) {
    csr_cache_release();
    const int dim = csr->dim;
    const int nb = dim / 3;
    const uint64_t unb = (uint64_t)nb;
    std::vector<uint64_t> keys;
    keys.reserve((size_t)csr->nnz / 3 + 1);
    for (int R = 0; R < dim; R++)
        for (int p = csr->row_ptr[R]; p < csr->row_ptr[R + 1]; p++) {
            const int c = csr->col_idx[p];
            if (c < 0 || c >= dim) return GSLAM_ERR_BAD_INPUT;
            keys.push_back((uint64_t)(R / 3) * unb + (uint64_t)(c / 3));
        }
    keys.push_back(0);
    std::sort(keys.begin(), keys.end());
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    gslam_opts o;
    gslam_opts_default(&o);
    std::vector<int64_t> key_slot;
    int rc = gslam_layout_from_blocks(nb, keys, false, 256, &s_csr.S, &key_slot);
    if (rc != GSLAM_OK) return rc;
    s_csr.entry_pos.assign(9 * (size_t)s_csr.S.n_slots, -1);
    for (int R = 0; R < dim; R++) {
        const uint64_t I = (uint64_t)(R / 3);
        for (int p = csr->row_ptr[R]; p < csr->row_ptr[R + 1]; p++) {
            const int c = csr->col_idx[p];
            const uint64_t key = I * unb + (uint64_t)(c / 3);
            const size_t k = std::lower_bound(keys.begin(), keys.end(), key) - keys.begin();
            s_csr.entry_pos[9 * (size_t)key_slot[k] + 3 * (R % 3) + (c % 3)] = p;
        }
    }
    if (!s_csr.st && cudaStreamCreateWithFlags(&s_csr.st, cudaStreamNonBlocking) != cudaSuccess)
        return GSLAM_ERR_CUDA;
    if (!s_csr.h_res && cudaMallocHost(&s_csr.h_res, sizeof(PcgResult)) != cudaSuccess)
        return GSLAM_ERR_CUDA;
    int dev = 0;
    cudaGetDevice(&dev);
    rc = gslam_layout_upload(&s_csr.L, s_csr.S, s_csr.st, dev, o);
    if (rc != GSLAM_OK) return rc;
    if (cudaMalloc(&s_csr.d_x, 3 * (size_t)nb * sizeof(double)) != cudaSuccess) return GSLAM_ERR_CUDA;
    s_csr.dim = dim;
    s_csr.rp.assign(csr->row_ptr, csr->row_ptr + dim + 1);
    s_csr.ci.assign(csr->col_idx, csr->col_idx + csr->nnz);
    s_csr.hval.assign(9 * (size_t)s_csr.S.n_slots, 0.0);
    s_csr.hb.assign(4 * 32 * (size_t)s_csr.S.n_slices, 0.0);
    s_csr.valid = true;
    return GSLAM_OK;
}
}  // namespace

void pcg_solve_sparse(double *x, CSRMatrix *csr, double *b, unsigned int dim) {
    s_status = GSLAM_OK;
    if (!x || !csr || !b || (int)dim != csr->dim || dim == 0 || dim % 3 != 0 || !csr->row_ptr ||
        (csr->nnz && (!csr->col_idx || !csr->values)) || csr->row_ptr[dim] != csr->nnz) {
        gslam_set_last_error("pcg_solve_sparse: needs a 3x3-block CSR with dim % 3 == 0");
        dropin_fail(GSLAM_ERR_BAD_INPUT, "pcg_solve_sparse");
        return;
    }
    const bool same = s_csr.valid && s_csr.dim == (int)dim && (int)s_csr.ci.size() == csr->nnz &&
                      memcmp(s_csr.rp.data(), csr->row_ptr, (dim + 1) * sizeof(int)) == 0 &&
                      memcmp(s_csr.ci.data(), csr->col_idx, (size_t)csr->nnz * sizeof(int)) == 0;
    if (!same) {
        int rc = csr_cache_build(csr);
        if (rc != GSLAM_OK) {
            gslam_set_last_error("pcg_solve_sparse: cannot build the block layout");
            dropin_fail(rc, "pcg_solve_sparse");
            return;
        }
    }
    CsrCache &C = s_csr;
    const int64_t n_slots = C.S.n_slots;
    for (int64_t slot = 0; slot < n_slots; slot++)
        for (int e = 0; e < 9; e++) {
            const int64_t p = C.entry_pos[9 * slot + e];
            C.hval[288 * (slot >> 5) + 32 * e + (slot & 31)] = p >= 0 ? csr->values[p] : 0.0;
        }
    const int nb = (int)dim / 3;
    for (int nr = 0; nr < nb; nr++)
        for (int c = 0; c < 3; c++) C.hb[4 * (size_t)nr + c] = b[3 * (size_t)C.S.perm[nr] + c];
    DCK(cudaMemcpyAsync(C.L.val, C.hval.data(), C.hval.size() * sizeof(double), cudaMemcpyHostToDevice, C.st),
        "pcg_solve_sparse");
    C.L.val32_fresh = false;
    DCK(cudaMemcpyAsync(C.L.b4, C.hb.data(), C.hb.size() * sizeof(double), cudaMemcpyHostToDevice, C.st),
        "pcg_solve_sparse");
    gslam_opts o;
    gslam_opts_default(&o); /* tol 1e-6, 500 iterations: MatrixOps.c:345-347 */
    int rc = gslam_layout_solve(&C.L, C.st, o, C.h_res, nullptr);
    if (rc != GSLAM_OK) { dropin_fail(rc, "pcg_solve_sparse"); return; }
    launch_scatter_vec(C.st, nb, C.L.perm, C.L.x4, C.d_x);
    DCK(cudaGetLastError(), "pcg_solve_sparse");
    DCK(cudaMemcpyAsync(x, C.d_x, dim * sizeof(double), cudaMemcpyDeviceToHost, C.st), "pcg_solve_sparse");
    DCK(cudaStreamSynchronize(C.st), "pcg_solve_sparse");
}
