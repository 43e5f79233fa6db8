/*
 * batch_api.cu — the batch entry points of the handle API (include/gslam.h):
 * gslam_create_se2_batch, gslam_batch_round, gslam_batch_layout, and the batched
 * solves behind gslam_solve / gslam_round on a batch handle.
 *
 * No counterpart in the reference, which solves one graph per process and sweeps
 * lambda with a shell loop (README.md:137-160). A batch is one block-diagonal graph:
 * every graph's poses padded to whole 32-row slices, its own lambda and anchor, its own
 * PCG scalars inside one persistent launch of batch.cu's solver.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "gslam.h"
#include "gslam_api_internal.h"
#include "gslam_internal.h"
#include "kernels.cuh"
#include "pcg_common.cuh"

/* batches of SE(2) graphs (one block-diagonal graph, batch.cu's solver)     */
/* ------------------------------------------------------------------------ */

static int batch_partition(gslam_graph *g) {
    BatchState &B = *g->batch;
    const gslam_structure &S = g->S;
    DevMem &m = g->mem;
    int n_sm = 0;
    CK(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, g->device));
    B.block = g->o.threads_per_cta ? g->o.threads_per_cta : 512;
    const int cps = g->o.ctas_per_sm ? g->o.ctas_per_sm : 2; /* two 64-register CTAs per SM by default */
    const int warps = B.block / 32;
    /* slices per CTA: room to balance by slot count, at least one per warp */
    int grid_guess = cps * n_sm;
    B.max_slices = std::max(warps, 2 * ((S.n_slices + grid_guess - 1) / grid_guess));
    B.smem_bytes = 2 * sizeof(double) * (size_t)B.max_slices;
    const int maxg = pcg_batch_max_grid(B.block, B.smem_bytes, g->device);
    if (maxg <= 0) {
        gslam_set_last_error("batched solver cannot be made co-resident at this block size");
        return GSLAM_ERR_NO_DEVICE;
    }
    const int grid = std::max(1, std::min(maxg, grid_guess));
    B.max_slices = std::max(B.max_slices, (S.n_slices + grid - 1) / grid);
    B.smem_bytes = 2 * sizeof(double) * (size_t)B.max_slices;
    /* contiguous ranges of at most max_slices slices minimising the largest slot count */
    const int cap = B.max_slices;
    auto fill = [&](int64_t bound, std::vector<int> *out) {
        int used = 1, nsl = 0;
        int64_t cur = 0;
        if (out) (*out)[0] = 0;
        for (int sl = 0; sl < S.n_slices; sl++) {
            const int64_t w = S.slice_ptr[sl + 1] - S.slice_ptr[sl];
            if (nsl > 0 && (cur + w > bound || nsl == cap)) {
                if (out && used <= grid) (*out)[used] = sl;
                used++;
                cur = 0;
                nsl = 0;
            }
            cur += w;
            nsl++;
        }
        if (out)
            for (int i = std::min(used, grid); i <= grid; i++) (*out)[i] = S.n_slices;
        return used;
    };
    int64_t lo = 0, hi = S.n_slots;
    for (int sl = 0; sl < S.n_slices; sl++) lo = std::max(lo, S.slice_ptr[sl + 1] - S.slice_ptr[sl]);
    while (lo < hi) {
        const int64_t mid = lo + (hi - lo) / 2;
        if (fill(mid, nullptr) <= grid) hi = mid;
        else lo = mid + 1;
    }
    std::vector<int> cs(grid + 1);
    fill(lo, &cs);
    if (cs[grid] != S.n_slices) { gslam_set_last_error("batch partition failed"); return GSLAM_ERR_TOO_LARGE; }
    B.grid = grid;
    /* graph of each slice; graphs of each CTA; CTAs of each graph */
    const int G = B.n_graphs;
    std::vector<int> slice_graph(S.n_slices, 0);
    for (int q = 0; q < G; q++)
        for (int sl = B.pose_off[q] / 32; sl < B.pose_off[q + 1] / 32; sl++) slice_graph[sl] = q;
    std::vector<int> g0(grid, 0), g1(grid, -1), gc0(G, -1), gnc(G, 0), poff(G, 0);
    for (int c = 0; c < grid; c++) {
        if (cs[c + 1] <= cs[c]) continue;
        g0[c] = slice_graph[cs[c]];
        g1[c] = slice_graph[cs[c + 1] - 1];
        if (g1[c] - g0[c] + 1 > pcg_batch_lg_max()) {
            gslam_set_last_error("too many small graphs per CTA for the batched solver");
            return GSLAM_ERR_TOO_LARGE;
        }
        for (int q = g0[c]; q <= g1[c]; q++) {
            if (gc0[q] < 0) gc0[q] = c;
            gnc[q]++;
        }
    }
    int total = 0;
    for (int q = 0; q < G; q++) { poff[q] = total; total += gnc[q]; }
    B.total_parts = total;
    CK(dupload(m, g->st, &B.d_cta_slice, cs));
    CK(dupload(m, g->st, &B.d_slice_graph, slice_graph));
    CK(dupload(m, g->st, &B.d_cta_g0, g0));
    CK(dupload(m, g->st, &B.d_cta_g1, g1));
    CK(dupload(m, g->st, &B.d_graph_cta0, gc0));
    CK(dupload(m, g->st, &B.d_graph_ncta, gnc));
    CK(dupload(m, g->st, &B.d_part_off, poff));
    CK(dalloc(m, &B.d_partials, 4 * (size_t)std::max(total, 1)));
    return GSLAM_OK;
}

int gslam_create_se2_batch(const gslam_se2_graph *graphs, uint32_t n_graphs, const gslam_opts *opts,
                           gslam_graph **out) {
    if (!graphs || !out || n_graphs == 0) BAD("null argument or empty batch");
    *out = nullptr;
    int64_t total = 0, n_edges = 0;
    for (uint32_t q = 0; q < n_graphs; q++) {
        const gslam_se2_graph &in = graphs[q];
        if (in.n_poses == 0 || !in.poses) BAD("a graph of the batch has no poses");
        if (in.n_edges && (!in.edge_i || !in.edge_j || !in.meas || !in.log_w)) BAD("missing edge arrays");
        for (uint32_t e = 0; e < in.n_edges; e++)
            if (in.edge_i[e] >= in.n_poses || in.edge_j[e] >= in.n_poses) BAD("edge pose out of range");
        if (!(in.lambda > 0.0)) BAD("lambda must be positive");
        total += ((int64_t)in.n_poses + 31) / 32 * 32;
        n_edges += in.n_edges;
    }
    if (total > 0x3fffffff || n_edges > 0x7fffffff) { gslam_set_last_error("batch too large"); return GSLAM_ERR_TOO_LARGE; }
    gslam_graph *g = new gslam_graph();
    int rc = common_setup(g, opts);
    if (rc != GSLAM_OK) { gslam_destroy(g); return rc; }
    auto fail = [&](int code) { gslam_destroy(g); return code; };
    g->batch = new BatchState();
    BatchState &B = *g->batch;
    B.n_graphs = (int)n_graphs;
    g->factors = GSLAM_FACTORS_SE2;
    g->n_poses = (int)total;
    g->lambda = 1.0;        /* each graph's lambda is folded into its information weights */
    g->anchor = 0.0;
    g->n_obs_edges = 0;
    g->n_edges = n_edges;
    B.pose_off.assign(n_graphs + 1, 0);
    B.n_real.assign(n_graphs, 0);
    std::vector<unsigned> t1, t2;
    std::vector<double> meas, info, poses(3 * (size_t)total, 0.0), anchor_vals;
    std::vector<int> diag_rows, segments, anchor_rows;
    t1.reserve(n_edges); t2.reserve(n_edges);
    meas.reserve(3 * n_edges); info.reserve(3 * n_edges);
    for (uint32_t q = 0; q < n_graphs; q++) {
        const gslam_se2_graph &in = graphs[q];
        const int off = B.pose_off[q];
        const int padded = (int)((in.n_poses + 31) / 32 * 32);
        B.pose_off[q + 1] = off + padded;
        B.n_real[q] = (int)in.n_poses;
        B.max_chunks = std::max(B.max_chunks, batch_max_chunks(padded));
        segments.push_back(off);
        for (uint32_t e = 0; e < in.n_edges; e++) {
            t1.push_back((unsigned)off + in.edge_i[e]);
            t2.push_back((unsigned)off + in.edge_j[e]);
            for (int k = 0; k < 3; k++) {
                meas.push_back(in.meas[3 * (size_t)e + k]);
                info.push_back(std::exp(in.log_w[3 * (size_t)e + k]) * in.lambda);
            }
        }
        memcpy(poses.data() + 3 * (size_t)off, in.poses, 3 * (size_t)in.n_poses * sizeof(double));
        anchor_rows.push_back(off);
        anchor_vals.push_back(in.anchor);
        diag_rows.push_back(off);
        for (int r = off + (int)in.n_poses; r < off + padded; r++) {
            diag_rows.push_back(r);
            anchor_rows.push_back(r);
            anchor_vals.push_back(1.0);
        }
    }
    DevMem &m = g->mem;
    if (dupload(m, g->st, &g->d_poses, poses) != cudaSuccess || dupload(m, g->st, &g->d_ei, t1) != cudaSuccess ||
        dupload(m, g->st, &g->d_ej, t2) != cudaSuccess || dupload(m, g->st, &g->d_meas, meas) != cudaSuccess ||
        dupload(m, g->st, &g->d_info, info) != cudaSuccess) {
        gslam_set_last_error("upload failed");
        return fail(GSLAM_ERR_CUDA);
    }
    rc = finish_setup(g, t1, t2, &diag_rows, &segments);
    if (rc != GSLAM_OK) return fail(rc);
    std::vector<int64_t> slots(anchor_rows.size());
    for (size_t a = 0; a < anchor_rows.size(); a++) slots[a] = g->S.diag_slot[g->S.iperm[anchor_rows[a]]];
    B.n_anchor = (int)slots.size();
    if (dupload(m, g->st, &B.d_anchor_slots, slots) != cudaSuccess ||
        dupload(m, g->st, &B.d_anchor_vals, anchor_vals) != cudaSuccess ||
        dupload(m, g->st, &B.d_pose_off, B.pose_off) != cudaSuccess ||
        dupload(m, g->st, &B.d_n_real, B.n_real) != cudaSuccess ||
        dalloc(m, &B.d_gdiff, (size_t)n_graphs) != cudaSuccess || dalloc(m, &B.d_res, (size_t)n_graphs) != cudaSuccess ||
        dalloc(m, &B.d_chunk_part, (size_t)n_graphs * B.max_chunks) != cudaSuccess ||
        dalloc(m, &B.d_active, 1) != cudaSuccess ||
        cudaMallocHost(&B.h_res, n_graphs * sizeof(PcgResult)) != cudaSuccess ||
        cudaMallocHost(&B.h_gdiff, n_graphs * sizeof(double)) != cudaSuccess) {
        gslam_set_last_error("batch buffers");
        return fail(GSLAM_ERR_CUDA);
    }
    rc = batch_partition(g);
    if (rc != GSLAM_OK) return fail(rc);
    if (cudaStreamSynchronize(g->st) != cudaSuccess) { gslam_set_last_error("setup failed"); return fail(GSLAM_ERR_CUDA); }
    *out = g;
    return GSLAM_OK;
}

static int batch_solve_mixed(gslam_graph *g, gslam_solve_stats *per_graph, gslam_solve_stats *total);

int batch_solve(gslam_graph *g, gslam_solve_stats *per_graph, gslam_solve_stats *total, const int *d_skip) {
    if (g->o.precision == GSLAM_PREC_MIXED) return batch_solve_mixed(g, per_graph, total);
    BatchState &B = *g->batch;
    DevLayout *L = &g->L;
    cudaStream_t st = g->st;
    launch_diag_inv(st, L->n_rows, L->diag_slot, L->val, L->dinv);
    CK(cudaGetLastError());
    PcgParams P;
    memset(&P, 0, sizeof P);
    P.n_rows = L->n_rows;
    P.n_slices = L->n_slices;
    P.slice_ptr = L->slice_ptr;
    P.row_len = L->row_len;
    P.col = L->col;
    P.val = L->val;
    P.dinv = L->dinv;
    P.b4 = L->b4;
    P.x4 = L->x4; P.r4 = L->r4; P.z4 = L->z4; P.p4a = L->p4a; P.p4b = L->p4b; P.q4 = L->q4;
    P.tol_rel = g->o.tol;
    P.max_iter = g->o.max_iter;
    P.gs = L->gs;
    P.res = L->res;
    const double ms = g->o.barrier_timeout_ms > 0 ? g->o.barrier_timeout_ms : 2000.0;
    P.spin_limit = (long long)(ms * (double)L->clock_khz);
    P.absent_cta = g->o.test_absent_cta;
    if (2.0 * (double)std::max(g->o.max_iter, 0) * B.grid + 8.0 * B.grid >= 4294967295.0) {
        gslam_set_last_error("max_iter too large for the solver's 32-bit barrier counter");
        return GSLAM_ERR_TOO_LARGE;
    }
    BatchParams BP;
    memset(&BP, 0, sizeof BP);
    BP.n_graphs = B.n_graphs;
    BP.cta_slice = B.d_cta_slice;
    BP.slice_graph = B.d_slice_graph;
    BP.cta_g0 = B.d_cta_g0;
    BP.cta_g1 = B.d_cta_g1;
    BP.graph_cta0 = B.d_graph_cta0;
    BP.graph_ncta = B.d_graph_ncta;
    BP.part_off = B.d_part_off;
    BP.total_parts = B.total_parts;
    BP.partials = B.d_partials;
    BP.res = B.d_res;
    BP.active = B.d_active;
    BP.skip = d_skip;
    CK(cudaMemsetAsync(L->gs, 0, sizeof(GridSync), st));
    CK(cudaMemsetAsync(L->res, 0, sizeof(PcgResult), st));
    CK(cudaMemsetAsync(B.d_res, 0, B.n_graphs * sizeof(PcgResult), st));
    CK(cudaMemcpyAsync(B.d_active, &B.n_graphs, sizeof(int), cudaMemcpyHostToDevice, st));
    CK(record_event(L->ev0, st));
    CK(launch_pcg_batch(st, P, BP, B.grid, B.block, B.smem_bytes, false));
    CK(record_event(L->ev1, st));
    CK(cudaMemcpyAsync(g->h_res, L->res, sizeof(PcgResult), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(B.h_res, B.d_res, B.n_graphs * sizeof(PcgResult), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    float solve_ms = 0.f;
    solve_ms = elapsed_ms(L->ev0, L->ev1);
    gslam_solve_stats agg;
    memset(&agg, 0, sizeof agg);
    agg.solve_ms = solve_ms;
    for (int q = 0; q < B.n_graphs; q++) {
        const PcgResult &r = B.h_res[q];
        const double rel = r.bnorm > 0 ? r.rnorm / r.bnorm : 0.0;
        if (per_graph) {
            memset(&per_graph[q], 0, sizeof per_graph[q]);
            per_graph[q].iterations = r.iterations;
            per_graph[q].reason = r.reason;
            per_graph[q].rel_residual = rel;
            per_graph[q].solve_ms = solve_ms;
        }
        agg.iterations = std::max(agg.iterations, r.iterations);
        agg.rel_residual = std::max(agg.rel_residual, rel);
        if (r.reason != GSLAM_STOP_TOL) agg.reason = r.reason;
    }
    if (total) *total = agg;
    if (g->h_res->timeout) {
        gslam_set_last_error("solver barrier wait timed out");
        return GSLAM_ERR_DEVICE_TIMEOUT;
    }
    return GSLAM_OK;
}

/*
 * Mixed-precision batch: iterative refinement driven from the host, every graph at
 * once. Per step: the FP32 right-hand side (the FP64 residual, 0 for graphs already
 * done), one launch of the batched PCG in FP32 (FP32 values and vectors, FP64 D^-1 and
 * dot products, per-graph scalars, inner tolerance inner_tol, each graph capped by what
 * is left of its max_iter), x += d in FP64, and the FP64 residual b - A x with per-graph
 * norms. A graph stops at tol, at max_iter inner iterations, or when a whole inner pass
 * (not one cut short by what is left of max_iter) did not halve the graph's residual
 * (stagnation); the graphs that stagnate are solved again in FP64 and those results are
 * reported.
 */
static int batch_solve_mixed(gslam_graph *g, gslam_solve_stats *per_graph, gslam_solve_stats *total) {
    BatchState &B = *g->batch;
    DevLayout *L = &g->L;
    cudaStream_t st = g->st;
    DevMem &m = g->mem;
    const int G = B.n_graphs;
    int rc = gslam_layout_ensure_fp32(L, st);
    if (rc != GSLAM_OK) return rc;
    if (!L->val32_fresh) {
        launch_val_to_f32(st, 9 * L->n_slots, L->val, L->val32);
        L->val32_fresh = true;
    }
    if (!B.d_bf4) {
        CK(dalloc(m, &B.d_bf4, 4 * 32 * (size_t)L->n_slices));
        CK(dalloc(m, &B.d_gactive, (size_t)G));
        CK(dalloc(m, &B.d_gcap, (size_t)G));
        CK(dalloc(m, &B.d_gres, (size_t)G));
        CK(cudaMallocHost(&B.h_gres, G * sizeof(double)));
    }
    launch_diag_inv(st, L->n_rows, L->diag_slot, L->val, L->dinv);
    /* x = 0; r = b - A 0 = b with per-graph ||b|| */
    CK(cudaMemsetAsync(L->x4, 0, 4 * 32 * (size_t)L->n_slices * sizeof(double), st));
    CK(cudaMemsetAsync(L->q4, 0, 4 * 32 * (size_t)L->n_slices * sizeof(double), st));
    launch_batch_resid(st, G, B.d_pose_off, L->b4, L->q4, L->r4, B.d_gres, B.d_chunk_part, B.max_chunks);
    CK(cudaMemcpyAsync(B.h_gres, B.d_gres, G * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    std::vector<double> bnorm(G), rel(G, 1.0);
    std::vector<int> its(G, 0), refs(G, 0), reason(G, GSLAM_STOP_MAXIT), active(G, 1), cap(G, 0);
    bool stagnated = false;
    for (int q = 0; q < G; q++) {
        bnorm[q] = std::sqrt(B.h_gres[q]);
        if (bnorm[q] == 0.0) { active[q] = 0; reason[q] = GSLAM_STOP_TOL; rel[q] = 0.0; }
    }
    PcgParams P;
    memset(&P, 0, sizeof P);
    P.n_rows = L->n_rows;
    P.n_slices = L->n_slices;
    P.slice_ptr = L->slice_ptr;
    P.row_len = L->row_len;
    P.col = L->col;
    P.val32 = L->val32;
    P.dinv = L->dinv;
    P.xf4 = L->f[0]; P.rf4 = L->f[1]; P.zf4 = L->f[2]; P.pfa4 = L->f[3]; P.pfb4 = L->f[4]; P.qf4 = L->f[5];
    P.tol_rel = g->o.inner_tol;
    P.gs = L->gs;
    P.res = L->res;
    const double ms_lim = g->o.barrier_timeout_ms > 0 ? g->o.barrier_timeout_ms : 2000.0;
    P.spin_limit = (long long)(ms_lim * (double)L->clock_khz);
    P.absent_cta = g->o.test_absent_cta;
    BatchParams BP;
    memset(&BP, 0, sizeof BP);
    BP.n_graphs = G;
    BP.cta_slice = B.d_cta_slice;
    BP.slice_graph = B.d_slice_graph;
    BP.cta_g0 = B.d_cta_g0;
    BP.cta_g1 = B.d_cta_g1;
    BP.graph_cta0 = B.d_graph_cta0;
    BP.graph_ncta = B.d_graph_ncta;
    BP.part_off = B.d_part_off;
    BP.total_parts = B.total_parts;
    BP.partials = B.d_partials;
    BP.res = B.d_res;
    BP.active = B.d_active;
    BP.bf4 = B.d_bf4;
    BP.cap = B.d_gcap;
    CK(record_event(L->ev0, st));
    for (int step = 0; step < std::max(g->o.max_refine, 1); step++) {
        /* each graph's inner pass is capped by what is left of its own budget */
        int n_active = 0, cap_max = 0;
        for (int q = 0; q < G; q++) {
            if (!active[q]) { cap[q] = 0; continue; }
            cap[q] = std::min(g->o.inner_max_iter, g->o.max_iter - its[q]);
            if (cap[q] <= 0) { active[q] = 0; reason[q] = GSLAM_STOP_MAXIT; continue; }
            n_active++;
            cap_max = std::max(cap_max, cap[q]);
        }
        if (n_active == 0) break;
        P.max_iter = cap_max;
        CK(cudaMemcpyAsync(B.d_gactive, active.data(), G * sizeof(int), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(B.d_gcap, cap.data(), G * sizeof(int), cudaMemcpyHostToDevice, st));
        launch_batch_rhs32(st, L->n_rows, B.d_slice_graph, B.d_gactive, L->r4, B.d_bf4);
        CK(cudaMemsetAsync(L->gs, 0, sizeof(GridSync), st));
        CK(cudaMemsetAsync(L->res, 0, sizeof(PcgResult), st));
        CK(cudaMemsetAsync(B.d_res, 0, G * sizeof(PcgResult), st));
        CK(cudaMemcpyAsync(B.d_active, &G, sizeof(int), cudaMemcpyHostToDevice, st));
        CK(launch_pcg_batch(st, P, BP, B.grid, B.block, B.smem_bytes, true));
        launch_batch_add_x(st, L->n_rows, L->f[0], L->x4);
        launch_spmv64(st, L->n_rows, L->n_slices, L->slice_ptr, L->row_len, L->col, L->val, L->x4, L->q4);
        launch_batch_resid(st, G, B.d_pose_off, L->b4, L->q4, L->r4, B.d_gres, B.d_chunk_part, B.max_chunks);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(g->h_res, L->res, sizeof(PcgResult), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(B.h_res, B.d_res, G * sizeof(PcgResult), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(B.h_gres, B.d_gres, G * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (g->h_res->timeout) {
            gslam_set_last_error("solver barrier wait timed out");
            return GSLAM_ERR_DEVICE_TIMEOUT;
        }
        for (int q = 0; q < G; q++) {
            if (!active[q]) continue;
            its[q] += B.h_res[q].iterations;
            refs[q]++;
            const double prev = rel[q];
            rel[q] = std::sqrt(B.h_gres[q]) / bnorm[q];
            if (rel[q] < g->o.tol) { active[q] = 0; reason[q] = GSLAM_STOP_TOL; }
            else if (its[q] >= g->o.max_iter || refs[q] >= g->o.max_refine) { active[q] = 0; reason[q] = GSLAM_STOP_MAXIT; }
            else if (rel[q] > 0.5 * prev && !(B.h_res[q].reason == GSLAM_STOP_MAXIT && cap[q] < g->o.inner_max_iter)) {
                /* a whole inner pass (to its tolerance or its inner_max_iter) did not halve the
                 * FP64 residual: FP32 cannot resolve this graph. A pass cut short by what was
                 * left of the graph's max_iter is not this. */
                active[q] = 0;
                reason[q] = GSLAM_STOP_STAGNATION;
                stagnated = true;
            }
        }
    }
    CK(record_event(L->ev1, st));
    CK(cudaEventSynchronize(L->ev1));
    float solve_ms = 0.f;
    solve_ms = elapsed_ms(L->ev0, L->ev1);
    if (stagnated) {
        /* the FP32 inner solves cannot resolve these graphs: solve just them again in FP64
         * (from x = 0, the reference's start); every other graph keeps its mixed solution */
        std::vector<int> skip(G);
        for (int q = 0; q < G; q++) skip[q] = reason[q] == GSLAM_STOP_STAGNATION ? 0 : 1;
        if (!B.d_skip) CK(dalloc(m, &B.d_skip, (size_t)G));
        CK(cudaMemcpyAsync(B.d_skip, skip.data(), G * sizeof(int), cudaMemcpyHostToDevice, st));
        std::vector<gslam_solve_stats> s64(G);
        gslam_solve_stats tot64;
        gslam_opts keep = g->o;
        g->o.precision = GSLAM_PREC_FP64;
        rc = batch_solve(g, s64.data(), &tot64, B.d_skip);
        g->o = keep;
        if (rc != GSLAM_OK) return rc;
        for (int q = 0; q < G; q++)
            if (!skip[q]) {
                its[q] += s64[q].iterations;
                refs[q] = -refs[q];
                reason[q] = s64[q].reason;
                rel[q] = s64[q].rel_residual;
            }
        solve_ms += (float)tot64.solve_ms;
    }
    gslam_solve_stats agg;
    memset(&agg, 0, sizeof agg);
    agg.solve_ms = solve_ms;
    for (int q = 0; q < G; q++) {
        if (per_graph) {
            memset(&per_graph[q], 0, sizeof per_graph[q]);
            per_graph[q].iterations = its[q];
            per_graph[q].refinements = refs[q];
            per_graph[q].reason = reason[q];
            per_graph[q].rel_residual = rel[q];
            per_graph[q].solve_ms = solve_ms;
        }
        agg.iterations = std::max(agg.iterations, its[q]);
        agg.refinements = std::max(agg.refinements, refs[q]);
        agg.rel_residual = std::max(agg.rel_residual, rel[q]);
        if (reason[q] != GSLAM_STOP_TOL) agg.reason = reason[q];
    }
    if (total) *total = agg;
    return GSLAM_OK;
}

int gslam_batch_round(gslam_graph *g, gslam_solve_stats *per_graph) {
    if (!g || !g->batch) BAD("not a batch");
    BatchState &B = *g->batch;
    if (!g->ev_round0) {
        CK(cudaEventCreate(&g->ev_round0));
        CK(cudaEventCreate(&g->ev_round1));
    }
    CK(record_event(g->ev_round0, g->st));
    int rc = gslam_linearise(g);
    if (rc != GSLAM_OK) return rc;
    rc = gslam_assemble(g);
    if (rc != GSLAM_OK) return rc;
    rc = batch_solve(g, per_graph, nullptr);
    if (rc != GSLAM_OK) return rc;
    launch_pose_update(g->st, g->n_poses, g->L.iperm, g->L.x4, g->d_poses, g->d_dx, g->o.angle_wrap,
                       g->d_block_sums, g->n_upd_blocks, g->d_diff);
    launch_batch_diff(g->st, B.n_graphs, B.d_pose_off, B.d_n_real, g->d_dx, B.d_gdiff, B.d_chunk_part, B.max_chunks);
    CK(cudaGetLastError());
    CK(record_event(g->ev_round1, g->st));
    CK(cudaMemcpyAsync(B.h_gdiff, B.d_gdiff, B.n_graphs * sizeof(double), cudaMemcpyDeviceToHost, g->st));
    CK(cudaStreamSynchronize(g->st));
    float ms = 0.f;
    ms = elapsed_ms(g->ev_round0, g->ev_round1);
    if (per_graph)
        for (int q = 0; q < B.n_graphs; q++) {
            per_graph[q].diff = B.h_gdiff[q];
            per_graph[q].round_ms = ms;
        }
    return GSLAM_OK;
}

int gslam_batch_layout(gslam_graph *g, uint32_t *n_graphs, uint32_t *pose_offset) {
    if (!g || !g->batch || !n_graphs) BAD("not a batch");
    *n_graphs = (uint32_t)g->batch->n_graphs;
    if (pose_offset)
        for (int q = 0; q <= g->batch->n_graphs; q++) pose_offset[q] = (uint32_t)g->batch->pose_off[q];
    return GSLAM_OK;
}

