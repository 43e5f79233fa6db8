/*
 * api.cu — the handle API of libgslam (include/gslam.h).
 *
 * A gslam_graph owns one stream and every device buffer of one pose graph. The
 * symbolic work (edge order, block pattern, layout, contribution lists) runs
 * once on the host at creation; every round after that is device-only:
 *   linearise -> assemble -> block-Jacobi inverse -> persistent PCG -> update,
 * with one 8-byte (diff) and one 40-byte (solver status) read back per round.
 * The reference rebuilds edges, structure and a 2.3 GB edge array every round
 * (src/cpu_pcg_fp64/GSLAM.c:55-139) and its GPU twin re-uploads poses and
 * downloads dx every round (src/gpu_pcg_fp64/device_graph.cu:1060-1129, :911).
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "gslam.h"
#include "gslam_api_internal.h"
#include "gslam_internal.h"
#include "kernels.cuh"
#include "pcg_common.cuh"

static thread_local std::string g_last_error;

/* GSLAM_TRACE=1: host time of each step of a solve on stderr (diagnostics). */
static bool trace_on() {
    static int on = -1;
    if (on < 0) on = getenv("GSLAM_TRACE") && atoi(getenv("GSLAM_TRACE")) ? 1 : 0;
    return on == 1;
}
struct HostTrace {
    std::chrono::steady_clock::time_point t = std::chrono::steady_clock::now();
    void step(const char *what) {
        if (!trace_on()) return;
        auto n = std::chrono::steady_clock::now();
        fprintf(stderr, "[gslam trace] %-28s %9.1f us\n", what,
                std::chrono::duration<double, std::micro>(n - t).count());
        t = n;
    }
};

void gslam_set_error(const char *fmt, const char *what, int code) {
    char buf[512];
    snprintf(buf, sizeof buf, fmt, what, code);
    g_last_error = buf;
}


/* an event record that a stream capture keeps as a node of the graph (a plain record
 * inside a capture only orders the capture) */
cudaError_t record_event(cudaEvent_t e, cudaStream_t st) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaError_t err = cudaStreamIsCapturing(st, &cs);
    if (err != cudaSuccess) return err;
    return cs == cudaStreamCaptureStatusActive ? cudaEventRecordWithFlags(e, st, cudaEventRecordExternal)
                                               : cudaEventRecord(e, st);
}

/* elapsed time between two recorded events, 0 when unavailable (leaves no error behind) */
float elapsed_ms(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) {
        ms = 0.f;
        cudaGetLastError();
    }
    return ms;
}


void gslam_set_last_error(const char *msg) { g_last_error = msg ? msg : ""; }

const char *gslam_version(void) { return "gslam-b200 0.1 (sm_100a)"; }
const char *gslam_last_error(void) { return g_last_error.c_str(); }

int gslam_opts_default(gslam_opts *o) {
    if (!o) return GSLAM_ERR_BAD_INPUT;
    memset(o, 0, sizeof *o);
    o->precision = GSLAM_PREC_FP64;
    o->tol = 1e-6;
    o->max_iter = 500;
    o->sell_window = 0;
    o->threads_per_cta = 0;
    o->ctas_per_sm = 0;
    o->angle_wrap = 0;
    o->inner_tol = 1e-4;
    o->inner_max_iter = 4000;
    o->max_refine = 64;
    o->device = -1;
    o->barrier_timeout_ms = 0.0;
    o->test_absent_cta = -1;
    o->disable_resident = 0;
    return GSLAM_OK;
}

/* ------------------------------------------------------------------------ */
/* device buffers                                                            */
/* ------------------------------------------------------------------------ */

void DevMem::release() {
    for (void *p : ptrs) cudaFree(p);
    ptrs.clear();
}

int gslam_layout_upload(DevLayout *L, const gslam_structure &S, cudaStream_t st, int device,
                        const gslam_opts &o) {
    DevMem &m = L->mem;
    L->n_rows = S.n_rows;
    L->n_slices = S.n_slices;
    L->n_slots = S.n_slots;
    CK(dupload(m, st, &L->perm, S.perm));
    CK(dupload(m, st, &L->iperm, S.iperm));
    CK(dupload(m, st, &L->row_len, S.row_len));
    CK(dupload(m, st, &L->col, S.col));
    CK(dupload(m, st, &L->diag_slot, S.diag_slot));
    CK(dupload(m, st, &L->chunk_slice, S.chunk_slice));
    CK(dupload(m, st, &L->slice_ptr, S.slice_ptr));
    CK(dupload(m, st, &L->slot_csr, S.slot_csr));
    const size_t nv = 9 * (size_t)S.n_slots;
    CK(dalloc(m, &L->val, nv));
    CK(cudaMemsetAsync(L->val, 0, nv * sizeof(double), st));
    L->val32 = nullptr;
    const size_t nr32 = 32 * (size_t)S.n_slices;
    CK(dalloc(m, &L->dinv, 9 * nr32));
    const size_t nvec = 4 * nr32;
    CK(dalloc(m, &L->b4, nvec));
    CK(dalloc(m, &L->x4, nvec));
    CK(dalloc(m, &L->r4, nvec));
    CK(dalloc(m, &L->z4, nvec));
    CK(dalloc(m, &L->p4a, nvec));
    CK(dalloc(m, &L->p4b, nvec));
    CK(dalloc(m, &L->q4, nvec));
    CK(cudaMemsetAsync(L->b4, 0, nvec * sizeof(double), st));
    CK(cudaMemsetAsync(L->x4, 0, nvec * sizeof(double), st));
    for (int i = 0; i < 6; i++) L->f[i] = nullptr;
    /* solver launch shape */
    int n_sm = 0;
    CK(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, device));
    {
        int khz = 0;   /* this query costs milliseconds: once per layout, not per solve */
        if (cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, device) != cudaSuccess || khz <= 0)
            khz = 2000000;
        L->clock_khz = khz;
    }
    L->block = o.threads_per_cta ? o.threads_per_cta : 1024;
    int maxg = pcg_max_grid(GSLAM_PREC_FP64, L->block, device);
    if (maxg <= 0) {
        g_last_error = "persistent solver cannot be made co-resident at this block size";
        return GSLAM_ERR_NO_DEVICE;
    }
    int cps = o.ctas_per_sm ? o.ctas_per_sm : 1;
    int grid = std::min(maxg, cps * n_sm);
    int warps = L->block / 32;
    int needed = (S.n_slices + warps - 1) / warps;
    L->grid = std::max(1, std::min(grid, needed));
    L->n_sm = n_sm;
    L->partial_capacity = std::max(L->grid, maxg);
    /* resident solvers: contiguous slice ranges per CTA balanced by slot count, at most
     * one slice per warp; the FP64 solver stages FP64 values, the mixed solver FP32
     * values plus its own rows' D^-1 and halo, each up to the shared-memory budget */
    L->resident = false;
    L->mixed_ok = false;
    L->cg_ok = false;
    const int rgrid = std::min(pcg_resident_max_grid(device, GSLAM_RES_SMEM_MAX),
                               pcg_mixed_max_grid(device, GSLAM_RES_SMEM_MAX));
    if (rgrid > 0 && S.n_slices <= 32 * rgrid) {
        const int block = (S.n_slices <= 24 * rgrid) ? 768 : 1024;
        const int cap_sl = block / 32;          /* one slice per warp */
        /* contiguous slice ranges of at most cap_sl slices that minimise the largest
         * slot count of any CTA (the slowest CTA sets the pace of every iteration):
         * binary search on that bound, each probe a greedy fill; feasible at the
         * upper end since n_slices <= cap_sl * rgrid */
        auto fill = [&](int64_t bound, std::vector<int> *out) {
            int used = 1, nsl = 0;
            int64_t cur = 0;
            if (out) (*out)[0] = 0;
            for (int sl = 0; sl < S.n_slices; sl++) {
                const int64_t w = S.slice_ptr[sl + 1] - S.slice_ptr[sl];
                if (nsl > 0 && (cur + w > bound || nsl == cap_sl)) {
                    if (out && used <= rgrid) (*out)[used] = sl;
                    used++;
                    cur = 0;
                    nsl = 0;
                }
                cur += w;
                nsl++;
            }
            if (out)
                for (int i = std::min(used, rgrid); i <= rgrid; i++) (*out)[i] = S.n_slices;
            return used;
        };
        int64_t lo = 0, hi = S.n_slots;
        for (int sl = 0; sl < S.n_slices; sl++) lo = std::max(lo, S.slice_ptr[sl + 1] - S.slice_ptr[sl]);
        while (lo < hi) {
            const int64_t mid = lo + (hi - lo) / 2;
            if (fill(mid, nullptr) <= rgrid) hi = mid;
            else lo = mid + 1;
        }
        std::vector<int> cs(rgrid + 1);
        fill(lo, &cs);
        bool ok = cs[0] == 0 && cs[rgrid] == S.n_slices;
        for (int i = 0; i < rgrid; i++)
            if (cs[i + 1] < cs[i] || cs[i + 1] - cs[i] > cap_sl) ok = false;
        if (ok) {
            L->res_grid = rgrid;
            L->res_block = block;
            CK(dupload(m, st, &L->cta_slice, cs));
            L->partial_capacity = std::max(L->partial_capacity, rgrid);
            /* CTA-local column indices (own rows first, then the CTA's halo) and halo lists */
            std::vector<int> lcol(S.n_slots, 0), hptr(rgrid + 1, 0), hrows;
            /* mixed / FP64 one-reduction solvers: every CTA's own layout must fit */
            bool fit32 = true, fit64 = true, fit_res = true;
            int64_t cap32_min = INT64_MAX, cap64_min = INT64_MAX, cap_res_min = INT64_MAX;
            /* the largest CTA's layout end: the launch asks for no more shared memory than
             * that (shared memory and L1 share the SM's SRAM, and these kernels read D^-1 and
             * row data through L1) */
            int64_t end32 = 0, end64 = 0, end_res = 0;
            for (int i = 0; i < rgrid; i++) {
                const int row0 = 32 * cs[i], row1 = 32 * cs[i + 1], nloc = row1 - row0;
                const int64_t a0 = S.slice_ptr[cs[i]], a1 = S.slice_ptr[cs[i + 1]];
                std::vector<int> rem;
                for (int64_t t = a0; t < a1; t++) {
                    const int c = S.col[t];
                    if (c >= 0 && (c < row0 || c >= row1)) rem.push_back(c);
                }
                std::sort(rem.begin(), rem.end());
                rem.erase(std::unique(rem.begin(), rem.end()), rem.end());
                for (int64_t t = a0; t < a1; t++) {
                    const int c = S.col[t];
                    if (c < 0) lcol[t] = 0;
                    else if (c >= row0 && c < row1) lcol[t] = c - row0;
                    else lcol[t] = nloc + (int)(std::lower_bound(rem.begin(), rem.end(), c) - rem.begin());
                }
                hptr[i + 1] = hptr[i] + (int)rem.size();
                hrows.insert(hrows.end(), rem.begin(), rem.end());
                const MixedSmem l32 = mixed_smem_layout(4, false, a1 - a0, cs[i + 1] - cs[i], (int64_t)rem.size(), block,
                                                        GSLAM_RES_SMEM_MAX);
                const MixedSmem l64 = mixed_smem_layout(8, true, a1 - a0, cs[i + 1] - cs[i], (int64_t)rem.size(), block,
                                                        GSLAM_RES_SMEM_MAX);
                const ResidentSmem lr = resident_smem_layout(a1 - a0, cs[i + 1] - cs[i], (int64_t)rem.size(),
                                                             GSLAM_RES_SMEM_MAX);
                fit_res = fit_res && lr.val_cap >= 0;
                cap_res_min = std::min(cap_res_min, std::min<int64_t>(lr.val_cap, 9 * (a1 - a0)));
                fit32 = fit32 && l32.val_cap >= 0;
                fit64 = fit64 && l64.val_cap >= 0;
                end_res = std::max(end_res, lr.end);
                end32 = std::max(end32, l32.end);
                end64 = std::max(end64, l64.end);
                cap32_min = std::min(cap32_min, std::min<int64_t>(l32.val_cap, 9 * (a1 - a0)));
                cap64_min = std::min(cap64_min, std::min<int64_t>(l64.val_cap, 9 * (a1 - a0)));
            }
            /* FP64: values | local columns | staged p (32 B per own or halo row), each CTA's
             * from its own sizes (resident_smem_layout) */
            if (fit_res && !o.disable_resident) {
                L->resident = true;
                L->smem_val_cap = cap_res_min; /* the smallest CTA's share (statistics only) */
                L->smem_bytes = (size_t)end_res;
            }
            /* mixed: FP32 values | local columns | D^-1 of own rows (2304 B per slice) | z of
             * own and halo rows (16 B each) | u, v of the first `block` halo rows (32 B each,
             * copied in asynchronously); FP64 one-reduction solver: FP64 values | local
             * columns | z (32 B per row) | u, v (64 B per halo row), D^-1 in global memory
             * (L2). Each CTA lays its share out from its own sizes (mixed_smem_layout), so a
             * CTA with a short halo keeps more of its values on chip. */
            if (fit32) {
                L->mixed_ok = true;
                L->mixed_val_cap = cap32_min; /* the smallest CTA's share (statistics only) */
                L->mixed_smem_bytes = (size_t)end32;
            }
            if (fit64) {
                L->cg_ok = true;
                L->cg_val_cap = cap64_min;
                L->cg_smem_bytes = (size_t)end64;
            }
            if (L->resident || L->mixed_ok || L->cg_ok) {
                CK(dupload(m, st, &L->lcol, lcol));
                CK(dupload(m, st, &L->halo_ptr, hptr));
                /* only rows that some CTA reads as halo are published in global memory */
                std::vector<unsigned char> exported((size_t)std::max(32 * L->n_slices, 1), 0);
                for (int r : hrows)
                    if (r >= 0 && (size_t)r < exported.size()) exported[(size_t)r] = 1;
                CK(dupload(m, st, &L->row_export, exported));
                if (hrows.empty()) hrows.push_back(0);
                CK(dupload(m, st, &L->halo_rows, hrows));
            }
        }
    }
    CK(dalloc(m, &L->partials, 8 * (size_t)L->partial_capacity));
    CK(dalloc(m, &L->gs, 1));
    CK(dalloc(m, &L->res, 1));
    CK(cudaEventCreate(&L->ev0));
    CK(cudaEventCreate(&L->ev1));
    return GSLAM_OK;
}

int gslam_layout_ensure_fp32(DevLayout *L, cudaStream_t st) {
    if (L->val32) return GSLAM_OK;
    DevMem &m = L->mem;
    const size_t nv = 9 * (size_t)L->n_slots;
    CK(dalloc(m, &L->val32, nv));
    CK(cudaMemsetAsync(L->val32, 0, nv * sizeof(float), st));
    const size_t nvec = 4 * 32 * (size_t)L->n_slices;
    for (int i = 0; i < 6; i++) {
        CK(dalloc(m, &L->f[i], nvec));
        CK(cudaMemsetAsync(L->f[i], 0, nvec * sizeof(float), st));
    }
    return GSLAM_OK;
}

/* Runs the persistent solver on L->val / L->b4; result in L->x4 (new order). */
/* everything of one solve up to the read-back of its result into h_res, without waiting
 * (also what a captured round records) */
static int layout_solve_enqueue(DevLayout *L, cudaStream_t st, const gslam_opts &o, PcgResult *h_res) {
    const int fused_prec = o.precision;
    if (fused_prec == GSLAM_PREC_MIXED) {
        int rc = gslam_layout_ensure_fp32(L, st);
        if (rc != GSLAM_OK) return rc;
        if (!L->val32_fresh) {
            launch_val_to_f32(st, 9 * L->n_slots, L->val, L->val32);
            L->val32_fresh = true;
        }
    }
    HostTrace tr;
    launch_diag_inv(st, L->n_rows, L->diag_slot, L->val, L->dinv);
    CK(cudaGetLastError());
    tr.step("diag_inv launch");
    PcgParams P;
    memset(&P, 0, sizeof P);
    P.n_rows = L->n_rows;
    P.n_slices = L->n_slices;
    P.slice_ptr = L->slice_ptr;
    P.row_len = L->row_len;
    P.col = L->col;
    P.val = L->val;
    P.val32 = L->val32;
    P.dinv = L->dinv;
    P.b4 = L->b4;
    P.x4 = L->x4; P.r4 = L->r4; P.z4 = L->z4; P.p4a = L->p4a; P.p4b = L->p4b; P.q4 = L->q4;
    P.xf4 = L->f[0]; P.rf4 = L->f[1]; P.zf4 = L->f[2]; P.pfa4 = L->f[3]; P.pfb4 = L->f[4]; P.qf4 = L->f[5];
    P.tol_rel = o.tol;
    P.max_iter = o.max_iter;
    P.inner_tol = o.inner_tol;
    P.inner_max_iter = o.inner_max_iter;
    P.max_refine = o.max_refine;
    P.partials = L->partials;
    P.gs = L->gs;
    P.res = L->res;
    {
        /* barrier wait limit in SM clock cycles (clock rate queried once at setup) */
        const double ms = o.barrier_timeout_ms > 0 ? o.barrier_timeout_ms : 2000.0;
        P.spin_limit = (long long)(ms * (double)L->clock_khz);
    }
    P.absent_cta = o.test_absent_cta;
    CK(cudaMemsetAsync(L->gs, 0, sizeof(GridSync), st));
    CK(cudaMemsetAsync(L->res, 0, sizeof(PcgResult), st));
    const bool mixed = fused_prec == GSLAM_PREC_MIXED;
    const bool cg = fused_prec == GSLAM_PREC_FP64_CG;
    if (mixed && !L->mixed_ok) {
        g_last_error = "mixed precision needs the graph's rows to fit the resident layout (<= 32 slices per SM)";
        return GSLAM_ERR_TOO_LARGE;
    }
    if (cg && !L->cg_ok) {
        g_last_error = "the one-reduction FP64 solver needs the graph's rows to fit the resident layout (<= 32 slices per SM)";
        return GSLAM_ERR_TOO_LARGE;
    }
    if (cg) {
        if (!L->w4) {
            const size_t nvec = 4 * 32 * (size_t)L->n_slices;
            CK(dalloc(L->mem, &L->w4, nvec));
            CK(cudaMemsetAsync(L->w4, 0, nvec * sizeof(double), st));
        }
        P.w4 = L->w4;
        /* one inner solve to the outer tolerance and iteration cap, no refinement */
        P.inner_tol = o.tol;
        P.inner_max_iter = o.max_iter;
        P.max_refine = 1;
    }
    const bool resident = !mixed && !cg && L->resident && !o.disable_resident;
    const int grid = (resident || mixed || cg) ? L->res_grid : L->grid;
    {
        /* 2 barriers per iteration + 1: the arrival counter must not wrap */
        const double barriers = 2.0 * (double)std::max(o.max_iter, 0) + 4.0 * (double)std::max(o.max_refine, 1) + 4.0;
        if (barriers * (double)grid >= 4294967295.0) {
            g_last_error = "max_iter too large for the solver's 32-bit barrier counter";
            return GSLAM_ERR_TOO_LARGE;
        }
    }
    P.cta_slice = L->cta_slice;
    P.smem_val_cap = L->smem_val_cap;
    /* every CTA lays its share out against the full budget, as the host's check did; the
     * launch asks for the largest resulting layout */
    P.smem_budget = GSLAM_RES_SMEM_MAX;
    P.lcol = L->lcol;
    P.halo_ptr = L->halo_ptr;
    P.halo_rows = L->halo_rows;
    P.row_export = L->row_export;
    tr.step("memsets");
    CK(record_event(L->ev0, st));
    if (mixed) CK(launch_pcg_mixed(st, P, grid, L->res_block, L->mixed_smem_bytes, false));
    else if (cg) CK(launch_pcg_mixed(st, P, grid, L->res_block, L->cg_smem_bytes, true));
    else if (resident) CK(launch_pcg_resident(st, P, grid, L->res_block, L->smem_bytes));
    else CK(launch_pcg(st, P, fused_prec, grid, L->block));
    tr.step("solver launch");
    CK(record_event(L->ev1, st));
    CK(cudaMemcpyAsync(h_res, L->res, sizeof(PcgResult), cudaMemcpyDeviceToHost, st));
    return GSLAM_OK;
}

/* after the stream has passed the read-back: statistics, the timeout status and the FP64
 * rerun of a stagnated mixed solve */
static int layout_solve_finish(DevLayout *L, cudaStream_t st, const gslam_opts &o, PcgResult *h_res,
                               gslam_solve_stats *stats) {
    const bool mixed = o.precision == GSLAM_PREC_MIXED;
    float solve_ms = 0.f;
    solve_ms = elapsed_ms(L->ev0, L->ev1);
    if (stats) {
        stats->solve_ms = solve_ms;
        stats->iterations = h_res->iterations;
        stats->refinements = h_res->refinements;
        stats->reason = h_res->reason;
        stats->rel_residual = h_res->bnorm > 0 ? h_res->rnorm / h_res->bnorm : 0.0;
    }
    if (h_res->timeout) {
        if (stats) stats->reason = GSLAM_STOP_TIMEOUT;
        g_last_error = "solver barrier wait timed out";
        return GSLAM_ERR_DEVICE_TIMEOUT;
    }
    if (mixed && h_res->reason == GSLAM_STOP_STAGNATION) {
        /* the FP32 inner solve cannot resolve this system: solve it in FP64 (from x = 0;
         * the right-hand side is untouched) and report both */
        const int refs = h_res->refinements, its = h_res->iterations;
        gslam_opts o64 = o;
        o64.precision = GSLAM_PREC_FP64;
        gslam_solve_stats s64;
        memset(&s64, 0, sizeof s64);
        int rc = gslam_layout_solve(L, st, o64, h_res, &s64);
        if (stats) {
            stats->solve_ms += s64.solve_ms;
            stats->iterations = its + s64.iterations;
            stats->refinements = -refs;
            stats->reason = s64.reason;
            stats->rel_residual = s64.rel_residual;
        }
        return rc;
    }
    return GSLAM_OK;
}

int gslam_layout_solve(DevLayout *L, cudaStream_t st, const gslam_opts &o, PcgResult *h_res,
                       gslam_solve_stats *stats) {
    int rc = layout_solve_enqueue(L, st, o, h_res);
    if (rc != GSLAM_OK) return rc;
    HostTrace tr;
    CK(cudaStreamSynchronize(st));
    tr.step("solver wait");
    return layout_solve_finish(L, st, o, h_res, stats);
}

void gslam_layout_release(DevLayout *L) {
    L->mem.release();
    if (L->ev0) cudaEventDestroy(L->ev0);
    if (L->ev1) cudaEventDestroy(L->ev1);
    L->ev0 = L->ev1 = nullptr;
}

/* ------------------------------------------------------------------------ */
/* graph creation                                                            */
/* ------------------------------------------------------------------------ */

int common_setup(gslam_graph *g, const gslam_opts *opts) {
    if (opts) g->o = *opts; else gslam_opts_default(&g->o);
    if (g->o.sell_window <= 0) g->o.sell_window = 1024;
    if (g->o.device >= 0) CK(cudaSetDevice(g->o.device));
    CK(cudaGetDevice(&g->device));
    CK(cudaStreamCreateWithFlags(&g->st, cudaStreamNonBlocking));
    CK(cudaMallocHost(&g->h_res, sizeof(PcgResult)));
    CK(cudaMallocHost(&g->h_diff, sizeof(double)));
    return GSLAM_OK;
}

int finish_setup(gslam_graph *g, const std::vector<unsigned> &t1, const std::vector<unsigned> &t2,
                 const std::vector<int> *diag_rows, const std::vector<int> *segments) {
    int rc = gslam_build_structure_ex(g->n_poses, (int64_t)t1.size(), t1.data(), t2.data(),
                                      g->o.sell_window, diag_rows, segments, &g->S);
    if (rc != GSLAM_OK) { g_last_error = "bad edge list"; return rc; }
    rc = gslam_layout_upload(&g->L, g->S, g->st, g->device, g->o);
    if (rc != GSLAM_OK) return rc;
    DevMem &m = g->mem;
    CK(dupload(m, g->st, &g->d_ctr_ptr, g->S.ctr_ptr));
    CK(dupload(m, g->st, &g->d_ctr, g->S.ctr));
    CK(dupload(m, g->st, &g->d_xi_ptr, g->S.xi_ptr));
    CK(dupload(m, g->st, &g->d_xi_ctr, g->S.xi_ctr));
    CK(dalloc(m, &g->d_blocks, 42 * (size_t)g->n_edges));
    CK(dalloc(m, &g->d_dx, 3 * (size_t)g->n_poses));
    CK(cudaMemsetAsync(g->d_dx, 0, 3 * (size_t)g->n_poses * sizeof(double), g->st));
    g->n_upd_blocks = std::max(1, std::min(4 * g->L.n_sm, (g->n_poses + 255) / 256));
    CK(dalloc(m, &g->d_block_sums, (size_t)g->n_upd_blocks));
    CK(dalloc(m, &g->d_diff, 1));
    CK(cudaStreamSynchronize(g->st));
    return GSLAM_OK;
}

int gslam_create_reference(const gslam_reference_graph *in, const gslam_opts *opts,
                           gslam_graph **out) {
    if (!in || !out) BAD("null argument");
    *out = nullptr;
    if (in->n_poses == 0 || !in->poses || !in->controls) BAD("n_poses == 0 or missing arrays");
    if (in->n_poses > 0x3fffffffu) { g_last_error = "too many poses"; return GSLAM_ERR_TOO_LARGE; }
    if (in->n_obs && (!in->obs_step || !in->obs_landmark || !in->obs)) BAD("missing observation arrays");
    for (uint32_t i = 0; i < in->n_obs; i++)
        if (in->obs_step[i] >= in->n_poses) BAD("observation step out of range");
    gslam_graph *g = new gslam_graph();
    int rc = common_setup(g, opts);
    if (rc != GSLAM_OK) { gslam_destroy(g); return rc; }
    g->factors = GSLAM_FACTORS_REFERENCE;
    g->n_poses = (int)in->n_poses;
    g->delta = in->delta;
    g->lambda = in->lambda;
    static const double def_mns[4] = { 0.19, 0.001, 0.13, 0.2 };
    memcpy(g->mns, in->mns ? in->mns : def_mns, sizeof g->mns);
    g->anchor = 1000000.0;
    std::vector<unsigned> pj, pk;
    gslam_obs_pairs(in->n_obs, in->obs_landmark, &pj, &pk);
    g->n_obs_edges = (int64_t)pj.size();
    g->n_edges = g->n_obs_edges + (g->n_poses - 1);
    std::vector<unsigned> t1(g->n_edges), t2(g->n_edges);
    for (int64_t e = 0; e < g->n_obs_edges; e++) {
        t1[e] = in->obs_step[pj[e]];
        t2[e] = in->obs_step[pk[e]];
    }
    for (int i = 0; i + 1 < g->n_poses; i++) {
        t1[g->n_obs_edges + i] = (unsigned)i;
        t2[g->n_obs_edges + i] = (unsigned)(i + 1);
    }
    DevMem &m = g->mem;
    auto fail = [&](int code) { gslam_destroy(g); return code; };
    if (dalloc(m, &g->d_poses, 3 * (size_t)g->n_poses) != cudaSuccess ||
        dalloc(m, &g->d_controls, 2 * (size_t)g->n_poses) != cudaSuccess) {
        g_last_error = "cudaMalloc failed";
        return fail(GSLAM_ERR_CUDA);
    }
    cudaMemcpyAsync(g->d_poses, in->poses, 3 * (size_t)g->n_poses * sizeof(double),
                    cudaMemcpyHostToDevice, g->st);
    cudaMemcpyAsync(g->d_controls, in->controls, 2 * (size_t)g->n_poses * sizeof(double),
                    cudaMemcpyHostToDevice, g->st);
    std::vector<unsigned> zs(in->obs_step, in->obs_step + in->n_obs);
    std::vector<double> zrb(in->obs, in->obs + 2 * (size_t)in->n_obs);
    {
        std::vector<int64_t> lptr;
        std::vector<unsigned> lmem;
        gslam_landmark_groups(in->n_obs, in->obs_landmark, &g->lm_ids, &lptr, &lmem);
        if (dupload(m, g->st, &g->d_lm_ptr, lptr) != cudaSuccess ||
            dupload(m, g->st, &g->d_lm_members, lmem) != cudaSuccess ||
            dalloc(m, &g->d_lm_ms, 2 * std::max<size_t>(g->lm_ids.size(), 1)) != cudaSuccess) {
            g_last_error = "upload failed";
            return fail(GSLAM_ERR_CUDA);
        }
    }
    if (dupload(m, g->st, &g->d_z_step, zs) != cudaSuccess ||
        dupload(m, g->st, &g->d_z_rb, zrb) != cudaSuccess ||
        dupload(m, g->st, &g->d_pj, pj) != cudaSuccess ||
        dupload(m, g->st, &g->d_pk, pk) != cudaSuccess) {
        g_last_error = "upload failed";
        return fail(GSLAM_ERR_CUDA);
    }
    rc = finish_setup(g, t1, t2);
    if (rc != GSLAM_OK) return fail(rc);
    *out = g;
    return GSLAM_OK;
}

int gslam_create_se2(const gslam_se2_graph *in, const gslam_opts *opts, gslam_graph **out) {
    if (!in || !out) BAD("null argument");
    *out = nullptr;
    if (in->n_poses == 0 || !in->poses) BAD("n_poses == 0 or missing poses");
    if (in->n_poses > 0x3fffffffu) { g_last_error = "too many poses"; return GSLAM_ERR_TOO_LARGE; }
    if (in->n_edges && (!in->edge_i || !in->edge_j || !in->meas || !in->log_w)) BAD("missing edge arrays");
    for (uint32_t e = 0; e < in->n_edges; e++)
        if (in->edge_i[e] >= in->n_poses || in->edge_j[e] >= in->n_poses) BAD("edge pose out of range");
    gslam_graph *g = new gslam_graph();
    int rc = common_setup(g, opts);
    if (rc != GSLAM_OK) { gslam_destroy(g); return rc; }
    g->factors = GSLAM_FACTORS_SE2;
    g->n_poses = (int)in->n_poses;
    g->lambda = in->lambda;
    g->anchor = in->anchor;
    g->n_obs_edges = 0;
    g->n_edges = in->n_edges;
    std::vector<unsigned> t1(in->edge_i, in->edge_i + in->n_edges), t2(in->edge_j, in->edge_j + in->n_edges);
    std::vector<double> meas(in->meas, in->meas + 3 * (size_t)in->n_edges);
    /* information weights exp(log_w), computed once here; lambda multiplies on device */
    std::vector<double> lw(3 * (size_t)in->n_edges);
    for (size_t k = 0; k < lw.size(); k++) lw[k] = std::exp(in->log_w[k]);
    DevMem &m = g->mem;
    auto fail = [&](int code) { gslam_destroy(g); return code; };
    if (dalloc(m, &g->d_poses, 3 * (size_t)g->n_poses) != cudaSuccess ||
        dupload(m, g->st, &g->d_ei, t1) != cudaSuccess || dupload(m, g->st, &g->d_ej, t2) != cudaSuccess ||
        dupload(m, g->st, &g->d_meas, meas) != cudaSuccess || dupload(m, g->st, &g->d_info, lw) != cudaSuccess) {
        g_last_error = "upload failed";
        return fail(GSLAM_ERR_CUDA);
    }
    cudaMemcpyAsync(g->d_poses, in->poses, 3 * (size_t)g->n_poses * sizeof(double),
                    cudaMemcpyHostToDevice, g->st);
    rc = finish_setup(g, t1, t2);
    if (rc != GSLAM_OK) return fail(rc);
    *out = g;
    return GSLAM_OK;
}

static void round_graph_release(gslam_graph *g);

int gslam_destroy(gslam_graph *g) {
    if (!g) return GSLAM_OK;
    if (g->st) cudaStreamSynchronize(g->st);
    gslam_layout_release(&g->L);
    g->mem.release();
    if (g->h_res) cudaFreeHost(g->h_res);
    if (g->h_diff) cudaFreeHost(g->h_diff);
    if (g->batch) {
        if (g->batch->h_res) cudaFreeHost(g->batch->h_res);
        if (g->batch->h_gdiff) cudaFreeHost(g->batch->h_gdiff);
        if (g->batch->h_gres) cudaFreeHost(g->batch->h_gres);
        delete g->batch;
    }
    round_graph_release(g);
    if (g->ev_round0) cudaEventDestroy(g->ev_round0);
    if (g->ev_round1) cudaEventDestroy(g->ev_round1);
    if (g->st) cudaStreamDestroy(g->st);
    delete g;
    return GSLAM_OK;
}

int gslam_set_opts(gslam_graph *g, const gslam_opts *opts) {
    if (!g || !opts) BAD("null argument");
    const int window = g->o.sell_window;
    const int threads = g->o.threads_per_cta, cps = g->o.ctas_per_sm;
    g->o = *opts;
    g->o.sell_window = window; /* the layout is fixed at creation */
    if ((opts->threads_per_cta && opts->threads_per_cta != threads) ||
        (opts->ctas_per_sm && opts->ctas_per_sm != cps)) {
        int block = opts->threads_per_cta ? opts->threads_per_cta : g->L.block;
        int maxg = pcg_max_grid(g->o.precision, block, g->device);
        if (maxg <= 0) { g_last_error = "unsupported block size"; return GSLAM_ERR_BAD_INPUT; }
        int c = opts->ctas_per_sm ? opts->ctas_per_sm : 1;
        int warps = block / 32;
        int needed = (g->L.n_slices + warps - 1) / warps;
        int grid = std::max(1, std::min(std::min(maxg, c * g->L.n_sm), needed));
        if (grid > g->L.max_grid_alloc()) { g_last_error = "grid exceeds allocation"; return GSLAM_ERR_BAD_INPUT; }
        g->L.block = block;
        g->L.grid = grid;
    }
    g->o.threads_per_cta = g->L.block;
    round_graph_release(g); /* launch parameters may have changed */
    return GSLAM_OK;
}

int gslam_sizes(const gslam_graph *g, int64_t *n_poses, int64_t *n_edges, int64_t *nnzb,
                int64_t *nnz) {
    if (!g) BAD("null handle");
    if (n_poses) *n_poses = g->n_poses;
    if (n_edges) *n_edges = g->n_edges;
    if (nnzb) *nnzb = g->S.nnzb;
    if (nnz) *nnz = (int64_t)g->S.csr_col.size();
    return GSLAM_OK;
}

int gslam_set_poses(gslam_graph *g, const double *poses) {
    if (!g || !poses) BAD("null argument");
    CK(cudaMemcpyAsync(g->d_poses, poses, 3 * (size_t)g->n_poses * sizeof(double),
                       cudaMemcpyHostToDevice, g->st));
    CK(cudaStreamSynchronize(g->st));
    return GSLAM_OK;
}

int gslam_get_poses(gslam_graph *g, double *poses) {
    if (!g || !poses) BAD("null argument");
    CK(cudaMemcpyAsync(poses, g->d_poses, 3 * (size_t)g->n_poses * sizeof(double),
                       cudaMemcpyDeviceToHost, g->st));
    CK(cudaStreamSynchronize(g->st));
    return GSLAM_OK;
}

/* ------------------------------------------------------------------------ */
/* stages                                                                    */
/* ------------------------------------------------------------------------ */

int gslam_linearise(gslam_graph *g) {
    if (!g) BAD("null handle");
    if (g->factors == GSLAM_FACTORS_REFERENCE) {
        launch_obs_edges(g->st, g->n_obs_edges, g->d_pj, g->d_pk, g->d_z_step, g->d_z_rb,
                         g->d_poses, g->d_blocks);
        launch_motion_edges(g->st, g->n_poses, g->n_obs_edges, g->d_controls, g->delta, g->lambda,
                            g->mns, g->d_poses, g->d_blocks);
    } else {
        launch_se2_edges(g->st, g->n_edges, 0, g->d_ei, g->d_ej, g->d_meas, g->d_info, g->lambda,
                         g->d_poses, g->d_blocks);
    }
    CK(cudaGetLastError());
    return GSLAM_OK;
}

int gslam_assemble_ex(gslam_graph *g, const double *blocks, double *csr_vals, double *xi_orig) {
    float *v32 = nullptr;
    if (g->o.precision == GSLAM_PREC_MIXED) {
        int rc = gslam_layout_ensure_fp32(&g->L, g->st);
        if (rc != GSLAM_OK) return rc;
        v32 = g->L.val32;
    }
    launch_assemble(g->st, g->L.n_slots, g->d_ctr_ptr, g->d_ctr, blocks, g->batch ? -1 : g->S.anchor_slot,
                    g->anchor, g->L.val, v32, g->L.slot_csr, g->L.chunk_slice, g->L.row_len, csr_vals);
    g->L.val32_fresh = (v32 != nullptr);
    if (g->batch) {
        /* every graph's first pose and every padding pose: anchor on the diagonal */
        launch_add_diag(g->st, g->batch->n_anchor, g->batch->d_anchor_slots, g->batch->d_anchor_vals, g->L.val);
        g->L.val32_fresh = false;
    }
    launch_assemble_xi(g->st, g->n_poses, g->d_xi_ptr, g->d_xi_ctr, blocks, g->L.b4, g->L.perm,
                       xi_orig);
    CK(cudaGetLastError());
    return GSLAM_OK;
}

int gslam_assemble(gslam_graph *g) {
    if (!g) BAD("null handle");
    return gslam_assemble_ex(g, g->d_blocks, nullptr, nullptr);
}

int gslam_assemble_from_edges(gslam_graph *g, const double *d_blocks) {
    if (!g || !d_blocks) BAD("null argument");
    return gslam_assemble_ex(g, d_blocks, nullptr, nullptr);
}


int gslam_solve(gslam_graph *g, gslam_solve_stats *stats) {
    if (!g) BAD("null handle");
    if (g->batch) return batch_solve(g, nullptr, stats);
    int rc = gslam_layout_solve(&g->L, g->st, g->o, g->h_res, stats);
    g->last_res = *g->h_res;
    return rc;
}

int gslam_update(gslam_graph *g, double *diff) { return gslam_update_ex(g, diff, nullptr); }

int gslam_update_ex(gslam_graph *g, double *diff, cudaEvent_t done) {
    if (!g) BAD("null handle");
    launch_pose_update(g->st, g->n_poses, g->L.iperm, g->L.x4, g->d_poses, g->d_dx, g->o.angle_wrap,
                       g->d_block_sums, g->n_upd_blocks, g->d_diff);
    CK(cudaGetLastError());
    if (done) CK(record_event(done, g->st));
    CK(cudaMemcpyAsync(g->h_diff, g->d_diff, sizeof(double), cudaMemcpyDeviceToHost, g->st));
    CK(cudaStreamSynchronize(g->st));
    if (diff) *diff = *g->h_diff;
    return GSLAM_OK;
}

int gslam_get_stream(gslam_graph *g, void **stream) {
    if (!g || !stream) BAD("null argument");
    *stream = (void *)g->st;
    return GSLAM_OK;
}

/* The round as one stream of work with no host wait: what the CUDA graph records.
 * The pose update is guarded by the solver's result (a timed-out or stagnated solve
 * leaves the poses alone; the host then decides). */
static int round_enqueue(gslam_graph *g) {
    CK(record_event(g->ev_round0, g->st));
    int rc = gslam_linearise(g);
    if (rc != GSLAM_OK) return rc;
    rc = gslam_assemble(g);
    if (rc != GSLAM_OK) return rc;
    rc = layout_solve_enqueue(&g->L, g->st, g->o, g->h_res);
    if (rc != GSLAM_OK) return rc;
    launch_pose_update(g->st, g->n_poses, g->L.iperm, g->L.x4, g->d_poses, g->d_dx, g->o.angle_wrap,
                       g->d_block_sums, g->n_upd_blocks, g->d_diff, g->L.res);
    CK(cudaGetLastError());
    CK(record_event(g->ev_round1, g->st));
    CK(cudaMemcpyAsync(g->h_diff, g->d_diff, sizeof(double), cudaMemcpyDeviceToHost, g->st));
    return GSLAM_OK;
}

static void round_graph_release(gslam_graph *g) {
    if (g->round_exec) cudaGraphExecDestroy(g->round_exec);
    g->round_exec = nullptr;
    g->eager_rounds = 0;
}

/* captures round_enqueue on the graph's stream into an executable graph */
static int round_graph_build(gslam_graph *g) {
    CK(cudaStreamBeginCapture(g->st, cudaStreamCaptureModeThreadLocal));
    const int rc = round_enqueue(g);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(g->st, &graph);
    if (rc != GSLAM_OK || e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        if (rc == GSLAM_OK) g_last_error = std::string("round capture: ") + cudaGetErrorString(e);
        cudaGetLastError();
        return rc != GSLAM_OK ? rc : GSLAM_ERR_CUDA;
    }
    const cudaError_t ei = cudaGraphInstantiate(&g->round_exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) {
        g->round_exec = nullptr;
        g_last_error = std::string("round graph instantiate: ") + cudaGetErrorString(ei);
        return GSLAM_ERR_CUDA;
    }
    return GSLAM_OK;
}

/* one round replayed from the captured graph (gslam_opts.round_graph) */
/* one replay of the captured round; poses_in / poses_out (host, may be NULL) are copied in
 * before it and out after it on the same stream, so the whole step waits once */
static int round_graphed(gslam_graph *g, gslam_solve_stats *stats, const double *poses_in = nullptr,
                         double *poses_out = nullptr) {
    if (!g->round_exec) {
        const int rc = round_graph_build(g);
        if (rc != GSLAM_OK) return rc;
    }
    const size_t pose_bytes = 3 * (size_t)g->n_poses * sizeof(double);
    if (poses_in) CK(cudaMemcpyAsync(g->d_poses, poses_in, pose_bytes, cudaMemcpyHostToDevice, g->st));
    CK(cudaGraphLaunch(g->round_exec, g->st));
    if (poses_out) CK(cudaMemcpyAsync(poses_out, g->d_poses, pose_bytes, cudaMemcpyDeviceToHost, g->st));
    CK(cudaStreamSynchronize(g->st));
    gslam_solve_stats st;
    memset(&st, 0, sizeof st);
    const bool stagnated = g->o.precision == GSLAM_PREC_MIXED && !g->h_res->timeout &&
                           g->h_res->reason == GSLAM_STOP_STAGNATION;
    double diff = *g->h_diff;
    int rc = layout_solve_finish(&g->L, g->st, g->o, g->h_res, &st);
    g->last_res = *g->h_res;
    if (rc == GSLAM_OK && stagnated) {
        /* the FP64 re-solve moved the poses after the copy-out: copy them again */
        rc = gslam_update_ex(g, &diff, g->ev_round1);
        if (rc == GSLAM_OK && poses_out) rc = gslam_get_poses(g, poses_out);
    }
    float ms = 0.f;
    if (rc == GSLAM_OK) ms = elapsed_ms(g->ev_round0, g->ev_round1);
    st.diff = diff;
    st.round_ms = ms;
    if (stats) *stats = st;
    return rc;
}

int gslam_round_io(gslam_graph *g, const double *poses_in, double *poses_out, gslam_solve_stats *stats) {
    if (!g) BAD("null handle");
    if (g->o.round_graph && !g->batch && g->eager_rounds > 0 && g->ev_round0)
        return round_graphed(g, stats, poses_in, poses_out);
    /* the eager round (the first, or without round_graph): the separate calls */
    int rc = GSLAM_OK;
    if (poses_in) rc = gslam_set_poses(g, poses_in);
    if (rc == GSLAM_OK) rc = gslam_round(g, stats);
    if (rc == GSLAM_OK && poses_out) rc = gslam_get_poses(g, poses_out);
    return rc;
}

int gslam_round(gslam_graph *g, gslam_solve_stats *stats) {
    if (!g) BAD("null handle");
    if (!g->ev_round0) {
        CK(cudaEventCreate(&g->ev_round0));
        CK(cudaEventCreate(&g->ev_round1));
    }
    /* the first round runs eagerly: it makes every lazy allocation before a capture */
    if (g->o.round_graph && !g->batch && g->eager_rounds > 0) return round_graphed(g, stats);
    g->eager_rounds++;
    CK(record_event(g->ev_round0, g->st));
    int rc = gslam_linearise(g);
    if (rc != GSLAM_OK) return rc;
    rc = gslam_assemble(g);
    if (rc != GSLAM_OK) return rc;
    gslam_solve_stats st;
    memset(&st, 0, sizeof st);
    rc = gslam_solve(g, &st);
    if (rc != GSLAM_OK) { if (stats) *stats = st; return rc; }
    double diff = 0.0;
    rc = gslam_update_ex(g, &diff, g->ev_round1);
    st.diff = diff;
    float ms = 0.f;
    if (rc == GSLAM_OK) ms = elapsed_ms(g->ev_round0, g->ev_round1);
    st.round_ms = ms;
    if (stats) *stats = st;
    return rc;
}

int gslam_run(gslam_graph *g, int max_rounds, double *diffs, int *rounds_done) {
    if (!g) BAD("null handle");
    double best = 1e30;
    int no_improve = 0, n = 0;
    for (int r = 1; r <= max_rounds; r++) {
        gslam_solve_stats st;
        int rc = gslam_round(g, &st);
        if (rc != GSLAM_OK) { if (rounds_done) *rounds_done = n; return rc; }
        n = r;
        if (diffs) diffs[r - 1] = st.diff;
        if (st.diff < 0.01) break;                   /* GSLAM.c:120 */
        if (st.diff < best) { best = st.diff; no_improve = 0; }
        else if (++no_improve >= 20) break;          /* GSLAM.c:124-129 */
    }
    if (rounds_done) *rounds_done = n;
    return GSLAM_OK;
}

/* ------------------------------------------------------------------------ */
/* read-back helpers                                                         */
/* ------------------------------------------------------------------------ */

int gslam_get_edge_blocks(gslam_graph *g, double *blocks) {
    if (!g || !blocks) BAD("null argument");
    CK(cudaMemcpyAsync(blocks, g->d_blocks, 42 * (size_t)g->n_edges * sizeof(double),
                       cudaMemcpyDeviceToHost, g->st));
    CK(cudaStreamSynchronize(g->st));
    return GSLAM_OK;
}

int gslam_get_csr(gslam_graph *g, int *row_ptr, int *col_idx, double *values, double *xi) {
    if (!g) BAD("null handle");
    const size_t nnz = g->S.csr_col.size(), dim = 3 * (size_t)g->n_poses;
    if (row_ptr) memcpy(row_ptr, g->S.csr_row_ptr.data(), (dim + 1) * sizeof(int));
    if (col_idx) memcpy(col_idx, g->S.csr_col.data(), nnz * sizeof(int));
    if (values || xi) {
        if (!g->d_csr_tmp) {
            CK(dalloc(g->mem, &g->d_csr_tmp, nnz));
            CK(dalloc(g->mem, &g->d_xi_tmp, dim));
        }
        launch_sell_to_csr(g->st, g->L.n_slots, g->L.slot_csr, g->L.chunk_slice, g->L.row_len,
                           g->L.val, g->d_csr_tmp);
        launch_scatter_vec(g->st, g->n_poses, g->L.perm, g->L.b4, g->d_xi_tmp);
        CK(cudaGetLastError());
        if (values) CK(cudaMemcpyAsync(values, g->d_csr_tmp, nnz * sizeof(double), cudaMemcpyDeviceToHost, g->st));
        if (xi) CK(cudaMemcpyAsync(xi, g->d_xi_tmp, dim * sizeof(double), cudaMemcpyDeviceToHost, g->st));
        CK(cudaStreamSynchronize(g->st));
    }
    return GSLAM_OK;
}

int gslam_get_dx(gslam_graph *g, double *dx) {
    if (!g || !dx) BAD("null argument");
    double *tmp = nullptr;
    if (!g->d_xi_tmp) CK(dalloc(g->mem, &g->d_xi_tmp, 3 * (size_t)g->n_poses));
    tmp = g->d_xi_tmp;
    launch_scatter_vec(g->st, g->n_poses, g->L.perm, g->L.x4, tmp);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(dx, tmp, 3 * (size_t)g->n_poses * sizeof(double), cudaMemcpyDeviceToHost, g->st));
    CK(cudaStreamSynchronize(g->st));
    return GSLAM_OK;
}

int gslam_get_diag_inv(gslam_graph *g, double *dinv) {
    if (!g || !dinv) BAD("null argument");
    const size_t n = 9 * 32 * (size_t)g->L.n_slices;
    std::vector<double> h(n);
    CK(cudaMemcpyAsync(h.data(), g->L.dinv, n * sizeof(double), cudaMemcpyDeviceToHost, g->st));
    CK(cudaStreamSynchronize(g->st));
    for (int old = 0; old < g->n_poses; old++) {
        const int nr = g->S.iperm[old];
        for (int e = 0; e < 9; e++) dinv[9 * (size_t)old + e] = h[288 * (size_t)(nr >> 5) + 32 * e + (nr & 31)];
    }
    return GSLAM_OK;
}

int gslam_spmv(gslam_graph *g, const double *d_x, double *d_y) {
    if (!g || !d_x || !d_y) BAD("null argument");
    launch_gather_vec(g->st, g->n_poses, g->L.perm, d_x, g->L.p4a);
    launch_spmv64(g->st, g->n_poses, g->L.n_slices, g->L.slice_ptr, g->L.row_len, g->L.col, g->L.val,
                  g->L.p4a, g->L.q4);
    launch_scatter_vec(g->st, g->n_poses, g->L.perm, g->L.q4, d_y);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(g->st));
    return GSLAM_OK;
}

int gslam_spmv_bench(gslam_graph *g, int prec, int reps, int n_copies, float *ms) {
    if (!g || !ms || reps <= 0 || n_copies <= 0) BAD("bad argument");
    if (prec == 1) {
        int rc = gslam_layout_ensure_fp32(&g->L, g->st);
        if (rc != GSLAM_OK) return rc;
        if (!g->L.val32_fresh) {
            launch_val_to_f32(g->st, 9 * g->L.n_slots, g->L.val, g->L.val32);
            g->L.val32_fresh = true;
        }
    }
    DevLayout &L = g->L;
    const size_t nv = 9 * (size_t)L.n_slots;
    const size_t esz = prec == 1 ? sizeof(float) : sizeof(double);
    const size_t ny = 4 * 32 * (size_t)L.n_slices;
    /* n_copies value arrays back to back (the matrix repeated) and one result per copy:
     * with n_copies large enough the stream exceeds L2 and every launch reads HBM */
    char *vals = nullptr, *ys = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    float t = 0.f;
    int rc = GSLAM_OK;
    if (cudaMalloc(&vals, nv * esz * n_copies) != cudaSuccess || cudaMalloc(&ys, ny * esz * n_copies) != cudaSuccess) {
        g_last_error = "spmv bench: cudaMalloc failed";
        rc = GSLAM_ERR_CUDA;
    }
    if (rc == GSLAM_OK) {
        const void *src = prec == 1 ? (const void *)L.val32 : (const void *)L.val;
        for (int c = 0; c < n_copies; c++)
            cudaMemcpyAsync(vals + c * nv * esz, src, nv * esz, cudaMemcpyDeviceToDevice, g->st);
        auto launch = [&]() {
            if (prec == 1)
                launch_spmv_multi32(g->st, n_copies, g->n_poses, L.n_slices, L.slice_ptr, L.row_len, L.col,
                                    (const float *)vals, (int64_t)nv, L.f[3], (float *)ys, (int64_t)ny);
            else
                launch_spmv_multi64(g->st, n_copies, g->n_poses, L.n_slices, L.slice_ptr, L.row_len, L.col,
                                    (const double *)vals, (int64_t)nv, L.p4a, (double *)ys, (int64_t)ny);
        };
        launch(); /* warm-up */
        cudaError_t e = cudaEventCreate(&a);
        if (e == cudaSuccess) e = cudaEventCreate(&b);
        if (e == cudaSuccess) e = cudaEventRecord(a, g->st);
        for (int i = 0; i < reps && e == cudaSuccess; i++) launch();
        if (e == cudaSuccess) e = cudaEventRecord(b, g->st);
        if (e == cudaSuccess) e = cudaEventSynchronize(b);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&t, a, b);
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e != cudaSuccess) {
            g_last_error = std::string("spmv bench: ") + cudaGetErrorString(e);
            rc = GSLAM_ERR_CUDA;
        }
        /* self-check: copy 0's result against the single-matrix SpMV kernel (same
         * summation order, so equal bit for bit) */
        if (rc == GSLAM_OK) {
            if (prec == 1) launch_spmv32(g->st, g->n_poses, L.n_slices, L.slice_ptr, L.row_len, L.col, L.val32,
                                         L.f[3], L.f[5]);
            else launch_spmv64(g->st, g->n_poses, L.n_slices, L.slice_ptr, L.row_len, L.col, L.val, L.p4a, L.q4);
            std::vector<char> y0(ny * esz), y1(ny * esz);
            cudaMemcpyAsync(y0.data(), ys, ny * esz, cudaMemcpyDeviceToHost, g->st);
            cudaMemcpyAsync(y1.data(), prec == 1 ? (const void *)L.f[5] : (const void *)L.q4, ny * esz,
                            cudaMemcpyDeviceToHost, g->st);
            if (cudaStreamSynchronize(g->st) != cudaSuccess) { g_last_error = "spmv bench: check failed"; rc = GSLAM_ERR_CUDA; }
            else {
                /* components 0..2 of the real rows (padding is never written) */
                bool same = true;
                for (int r = 0; r < g->n_poses && same; r++)
                    same = memcmp(y0.data() + 4 * r * esz, y1.data() + 4 * r * esz, 3 * esz) == 0;
                if (!same) {
                    g_last_error = "spmv bench: the many-matrix kernel disagrees with the single-matrix one";
                    rc = GSLAM_ERR_CUDA;
                }
            }
        }
    }
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    if (vals) cudaFree(vals);
    if (ys) cudaFree(ys);
    if (rc == GSLAM_OK) *ms = t / reps / n_copies;
    return rc;
}

int gslam_spmv_bytes(gslam_graph *g, int prec, int64_t *bytes) {
    if (!g || !bytes) BAD("null argument");
    const int64_t sv = prec == 1 ? 4 : 8;
    /* values + one column index per block + x read once + y written once (3 values/row) */
    *bytes = g->S.nnzb * (9 * sv + 4) + 2 * 3 * (int64_t)g->n_poses * sv;
    return GSLAM_OK;
}

int gslam_landmark_map(gslam_graph *g, uint32_t *n_landmarks, uint32_t *ids, double *ms) {
    if (!g || !n_landmarks) BAD("null argument");
    if (g->factors != GSLAM_FACTORS_REFERENCE) BAD("the landmark map belongs to reference-factor graphs");
    const int n = (int)g->lm_ids.size();
    *n_landmarks = (uint32_t)n;
    if (!ids && !ms) return GSLAM_OK;
    if (ids)
        for (int i = 0; i < n; i++) ids[i] = g->lm_ids[i];
    if (ms) {
        launch_landmark_map(g->st, n, g->d_lm_ptr, g->d_lm_members, g->d_z_step, g->d_z_rb, g->d_poses, g->d_lm_ms);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(ms, g->d_lm_ms, 2 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, g->st));
        CK(cudaStreamSynchronize(g->st));
    }
    return GSLAM_OK;
}

int gslam_cost(gslam_graph *g, double *cost, double *edge_costs) {
    if (!g || !cost) BAD("null argument");
    if (g->factors != GSLAM_FACTORS_REFERENCE) BAD("the round cost belongs to reference-factor graphs");
    DevMem &m = g->mem;
    if (!g->d_cost) {
        CK(dalloc(m, &g->d_edge_cost, std::max<size_t>((size_t)g->n_edges, 1)));
        CK(dalloc(m, &g->d_cost_blocks, (size_t)edge_cost_blocks(g->n_edges)));
        CK(dalloc(m, &g->d_cost, 1));
    }
    launch_edge_costs(g->st, g->n_obs_edges, g->n_poses, g->d_pj, g->d_pk, g->d_z_step, g->d_z_rb,
                      g->d_controls, g->delta, g->lambda, g->mns, g->d_poses, g->d_edge_cost,
                      g->d_cost_blocks, g->d_cost);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(g->h_diff, g->d_cost, sizeof(double), cudaMemcpyDeviceToHost, g->st));
    if (edge_costs)
        CK(cudaMemcpyAsync(edge_costs, g->d_edge_cost, (size_t)g->n_edges * sizeof(double),
                           cudaMemcpyDeviceToHost, g->st));
    CK(cudaStreamSynchronize(g->st));
    *cost = *g->h_diff;
    return GSLAM_OK;
}
