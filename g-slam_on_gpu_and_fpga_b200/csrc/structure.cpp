/*
 * structure.cpp — one-time symbolic work for a pose graph (host, C++).
 *
 * Replaces, once per graph instead of once per round:
 *   - make_edges' landmark ordering (reference src/cpu_pcg_fp64/GSLAM.c:222-318),
 *     here O(n_z) with a first-appearance table instead of O(max_id * n_z);
 *   - the symbolic half of build_csr_from_edges (MatrixOps.c:173-221), here by
 *     sorting 64-bit block keys instead of a dim x dim byte marker (which the
 *     reference indexes in 32-bit arithmetic, wrapping for dim > 65,535);
 *   - the per-entry slot search of the numeric half (MatrixOps.c:233-272), here
 *     precomputed as per-block contribution lists in edge order, so the device
 *     assembly is a gather that adds in exactly the reference's order.
 */
#include <algorithm>
#include <cstring>
#include <numeric>

#include "gslam_internal.h"
#include "gslam.h"

void gslam_obs_pairs(int64_t n_z, const unsigned *z_lm, std::vector<unsigned> *pj,
                     std::vector<unsigned> *pk) {
    pj->clear();
    pk->clear();
    if (n_z <= 0) return;
    /* landmark ids in order of first appearance; members in z-list order */
    std::vector<std::pair<unsigned, int64_t>> keyed(n_z);
    for (int64_t i = 0; i < n_z; i++) keyed[i] = {z_lm[i], i};
    std::vector<std::pair<unsigned, int64_t>> byid = keyed;
    std::stable_sort(byid.begin(), byid.end(),
                     [](const std::pair<unsigned, int64_t> &a, const std::pair<unsigned, int64_t> &b) {
                         return a.first < b.first;
                     });
    /* groups by id (members ascending in z order); first appearance = first member */
    struct group { int64_t begin, end; };
    std::vector<group> groups;
    for (int64_t i = 0; i < n_z;) {
        int64_t j = i;
        while (j < n_z && byid[j].first == byid[i].first) j++;
        groups.push_back({i, j});
        i = j;
    }
    std::sort(groups.begin(), groups.end(), [&](const group &a, const group &b) {
        return byid[a.begin].second < byid[b.begin].second;
    });
    int64_t total = 0;
    for (const group &g : groups) {
        int64_t k = g.end - g.begin;
        total += k * (k - 1) / 2;
    }
    pj->reserve(total);
    pk->reserve(total);
    for (const group &g : groups)
        for (int64_t a = g.begin; a < g.end; a++)
            for (int64_t b = a + 1; b < g.end; b++) {
                pj->push_back((unsigned)byid[a].second);
                pk->push_back((unsigned)byid[b].second);
            }
}

/*
 * Layout of a block pattern: `keys` are the sorted unique block keys I * N + J
 * (block (0,0) included). Fills everything but the contribution lists.
 */
int gslam_layout_from_blocks(int n_rows, const std::vector<uint64_t> &keys, bool bare_anchor,
                             int sell_window, gslam_structure *s,
                             std::vector<int64_t> *key_slot_out, const std::vector<int> *segments) {
    const uint64_t nb = (uint64_t)n_rows;
    s->n_rows = n_rows;
    s->bare_anchor = bare_anchor;
    s->nnzb = (int64_t)keys.size();
    std::vector<int64_t> rstart(n_rows + 1, 0);
    for (uint64_t k : keys) rstart[k / nb + 1]++;
    for (int i = 0; i < n_rows; i++) rstart[i + 1] += rstart[i];

    /* ---- row permutation: a locality order, then sort by block count inside windows ---- */
    s->perm.resize(n_rows);
    std::iota(s->perm.begin(), s->perm.end(), 0);
    {
        /* one graph: Cuthill-McKee order of the block pattern (the code works per row
         * range, each range's rows staying in it): breadth-first from a lowest-degree row
         * of each component, neighbours taken by
         * ascending degree, so a CTA's contiguous rows are a compact region of the graph
         * and loop closures to rows visited much earlier fall inside it instead of into
         * another CTA's halo. Each row's blocks stay in ascending original column order
         * (the per-row sums are unchanged); only which rows share a slice and a CTA
         * changes. */
        /* batches keep their rows' order (measured: the mixed batch ran 2 % slower in
         * this order, the FP64 batch 1 % faster) */
        std::vector<int> segs = segments ? std::vector<int>{} : std::vector<int>{ 0, n_rows };
        std::vector<int> deg(n_rows), nbr, by_deg;
        std::vector<char> seen(n_rows, 0);
        for (int i = 0; i < n_rows; i++) deg[i] = (int)(rstart[i + 1] - rstart[i]);
        for (size_t q = 0; q + 1 < segs.size(); q++) {
            const int a = segs[q], b = segs[q + 1];
            if (b - a <= 2 * GSLAM_SLICE) continue;
            by_deg.resize(b - a);
            std::iota(by_deg.begin(), by_deg.end(), a);
            std::stable_sort(by_deg.begin(), by_deg.end(), [&](int x, int y) { return deg[x] < deg[y]; });
            int out = a;
            for (int start : by_deg) {
                if (seen[start]) continue;
                seen[start] = 1;
                int head = out;
                s->perm[out++] = start;
                while (head < out) {
                    const int r = s->perm[head++];
                    nbr.clear();
                    for (int64_t k = rstart[r]; k < rstart[r + 1]; k++) {
                        const int c = (int)(keys[k] % nb);
                        if (c >= a && c < b && !seen[c]) { seen[c] = 1; nbr.push_back(c); }
                    }
                    std::stable_sort(nbr.begin(), nbr.end(), [&](int x, int y) { return deg[x] < deg[y]; });
                    for (int c : nbr) s->perm[out++] = c;
                }
            }
        }
    }
    if (sell_window > 1) {
        /* windows restart at every segment start (a batch keeps each graph's rows
         * in its own, slice-aligned range) */
        std::vector<int> seg = segments ? *segments : std::vector<int>{ 0 };
        seg.push_back(n_rows);
        for (size_t q = 0; q + 1 < seg.size(); q++) {
            for (int w0 = seg[q]; w0 < seg[q + 1]; w0 += sell_window) {
                int w1 = std::min(seg[q + 1], w0 + sell_window);
                std::stable_sort(s->perm.begin() + w0, s->perm.begin() + w1, [&](int a, int b) {
                    return (rstart[a + 1] - rstart[a]) > (rstart[b + 1] - rstart[b]);
                });
            }
        }
    }
    s->iperm.assign(n_rows, 0);
    for (int i = 0; i < n_rows; i++) s->iperm[s->perm[i]] = i;

    /* ---- slices ---- */
    s->n_slices = (n_rows + GSLAM_SLICE - 1) / GSLAM_SLICE;
    s->slice_ptr.assign(s->n_slices + 1, 0);
    s->slice_width.assign(s->n_slices, 0);
    s->row_len.assign((size_t)s->n_slices * GSLAM_SLICE, 0);
    s->max_width = 0;
    for (int nr = 0; nr < n_rows; nr++) {
        int old = s->perm[nr];
        int len = (int)(rstart[old + 1] - rstart[old]);
        s->row_len[nr] = len;
        int sl = nr / GSLAM_SLICE;
        s->slice_width[sl] = std::max(s->slice_width[sl], len);
    }
    for (int sl = 0; sl < s->n_slices; sl++) {
        s->slice_ptr[sl + 1] = s->slice_ptr[sl] + (int64_t)GSLAM_SLICE * s->slice_width[sl];
        s->max_width = std::max(s->max_width, s->slice_width[sl]);
    }
    s->n_slots = s->slice_ptr[s->n_slices];
    s->chunk_slice.assign(s->n_slots / GSLAM_SLICE, 0);
    for (int sl = 0; sl < s->n_slices; sl++)
        for (int64_t c = s->slice_ptr[sl] / GSLAM_SLICE; c < s->slice_ptr[sl + 1] / GSLAM_SLICE; c++)
            s->chunk_slice[c] = sl;
    s->col.assign(s->n_slots, -1);
    s->diag_slot.assign(n_rows, -1);

    /* slot of key index k (row-local position j) */
    std::vector<int64_t> key_slot(keys.size());
    for (int old = 0; old < n_rows; old++) {
        int nr = s->iperm[old];
        int sl = nr / GSLAM_SLICE, lane = nr % GSLAM_SLICE;
        for (int64_t k = rstart[old]; k < rstart[old + 1]; k++) {
            int64_t j = k - rstart[old];
            int64_t slot = s->slice_ptr[sl] + j * GSLAM_SLICE + lane;
            key_slot[k] = slot;
            int colold = (int)(keys[k] % nb);
            s->col[slot] = s->iperm[colold];
            if (colold == old) s->diag_slot[nr] = (int)slot;
        }
    }
    s->anchor_slot = key_slot[0];

    /* ---- scalar CSR of the reference ---- */
    const int64_t dim = 3 * (int64_t)n_rows;
    s->csr_row_ptr.assign(dim + 1, 0);
    int64_t p = 0;
    for (int I = 0; I < n_rows; I++) {
        for (int r = 0; r < 3; r++) {
            if (I == 0 && s->bare_anchor) p += 1;
            else p += 3 * (rstart[I + 1] - rstart[I]);
            if (p > INT32_MAX) return GSLAM_ERR_TOO_LARGE;
            s->csr_row_ptr[3 * I + r + 1] = (int)p;
        }
    }
    s->csr_col.assign(p, 0);
    s->slot_csr.assign(s->n_slots, -1);
    for (int I = 0; I < n_rows; I++) {
        for (int r = 0; r < 3; r++) {
            int64_t q = s->csr_row_ptr[3 * I + r];
            if (I == 0 && s->bare_anchor) { s->csr_col[q] = r; continue; }
            for (int64_t k = rstart[I]; k < rstart[I + 1]; k++) {
                int J = (int)(keys[k] % nb);
                for (int c = 0; c < 3; c++) s->csr_col[q++] = 3 * J + c;
            }
        }
        for (int64_t k = rstart[I]; k < rstart[I + 1]; k++)
            s->slot_csr[key_slot[k]] = (I == 0 && s->bare_anchor)
                                           ? -2
                                           : s->csr_row_ptr[3 * I] + 3 * (k - rstart[I]);
    }
    if (key_slot_out) key_slot_out->swap(key_slot);
    return GSLAM_OK;
}

int gslam_build_structure(int n_rows, int64_t n_edges, const unsigned *t1, const unsigned *t2,
                          int sell_window, gslam_structure *s) {
    return gslam_build_structure_ex(n_rows, n_edges, t1, t2, sell_window, nullptr, nullptr, s);
}

int gslam_build_structure_ex(int n_rows, int64_t n_edges, const unsigned *t1, const unsigned *t2,
                             int sell_window, const std::vector<int> *diag_rows,
                             const std::vector<int> *segments, gslam_structure *s) {
    if (n_rows <= 0) return GSLAM_ERR_BAD_INPUT;
    for (int64_t e = 0; e < n_edges; e++)
        if (t1[e] >= (unsigned)n_rows || t2[e] >= (unsigned)n_rows) return GSLAM_ERR_BAD_INPUT;
    const uint64_t nb = (uint64_t)n_rows;
    s->n_edges = n_edges;

    /* ---- unique blocks, row-major, columns ascending ---- */
    std::vector<uint64_t> keys;
    keys.reserve(4 * (size_t)n_edges + 1);
    for (int64_t e = 0; e < n_edges; e++) {
        uint64_t a = t1[e], b = t2[e];
        keys.push_back(a * nb + a);
        keys.push_back(a * nb + b);
        keys.push_back(b * nb + a);
        keys.push_back(b * nb + b);
    }
    bool bare = true;
    for (int64_t e = 0; e < n_edges && bare; e++)
        if (t1[e] == 0 || t2[e] == 0) bare = false;
    keys.push_back(0); /* block (0,0) always exists internally: it carries the anchor */
    if (diag_rows)
        for (int r : *diag_rows) {
            if (r < 0 || r >= n_rows) return GSLAM_ERR_BAD_INPUT;
            keys.push_back((uint64_t)r * nb + (uint64_t)r);
        }
    std::sort(keys.begin(), keys.end());
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    std::vector<int64_t> key_slot;
    int rc = gslam_layout_from_blocks(n_rows, keys, bare, sell_window, s, &key_slot, segments);
    if (rc != GSLAM_OK) return rc;
    std::vector<int64_t> rstart(n_rows + 1, 0);
    for (uint64_t k : keys) rstart[k / nb + 1]++;
    for (int i = 0; i < n_rows; i++) rstart[i + 1] += rstart[i];

    auto slot_of = [&](uint64_t I, uint64_t J) -> int64_t {
        uint64_t key = I * nb + J;
        auto it = std::lower_bound(keys.begin() + rstart[I], keys.begin() + rstart[I + 1], key);
        return key_slot[it - keys.begin()];
    };

    /* ---- assembly contribution lists, edge order, sub-block order UL UR BL BR ---- */
    s->ctr_ptr.assign(s->n_slots + 1, 0);
    std::vector<int64_t> e_slot(4 * (size_t)n_edges);
    for (int64_t e = 0; e < n_edges; e++) {
        uint64_t a = t1[e], b = t2[e];
        e_slot[4 * e + 0] = slot_of(a, a);
        e_slot[4 * e + 1] = slot_of(a, b);
        e_slot[4 * e + 2] = slot_of(b, a);
        e_slot[4 * e + 3] = slot_of(b, b);
        for (int q = 0; q < 4; q++) s->ctr_ptr[e_slot[4 * e + q] + 1]++;
    }
    for (int64_t i = 0; i < s->n_slots; i++) s->ctr_ptr[i + 1] += s->ctr_ptr[i];
    s->ctr.assign(4 * (size_t)n_edges, 0);
    {
        std::vector<int64_t> fill(s->ctr_ptr.begin(), s->ctr_ptr.end() - 1);
        for (int64_t e = 0; e < n_edges; e++)
            for (int q = 0; q < 4; q++) s->ctr[fill[e_slot[4 * e + q]]++] = 4 * e + q;
    }
    /* ---- right-hand-side lists per new row ---- */
    s->xi_ptr.assign(n_rows + 1, 0);
    for (int64_t e = 0; e < n_edges; e++) {
        s->xi_ptr[s->iperm[t1[e]] + 1]++;
        s->xi_ptr[s->iperm[t2[e]] + 1]++;
    }
    for (int i = 0; i < n_rows; i++) s->xi_ptr[i + 1] += s->xi_ptr[i];
    s->xi_ctr.assign(2 * (size_t)n_edges, 0);
    {
        std::vector<int64_t> fill(s->xi_ptr.begin(), s->xi_ptr.end() - 1);
        for (int64_t e = 0; e < n_edges; e++) {
            s->xi_ctr[fill[s->iperm[t1[e]]]++] = 2 * e;
            s->xi_ctr[fill[s->iperm[t2[e]]]++] = 2 * e + 1;
        }
    }

    return GSLAM_OK;
}

/* Landmarks in order of first appearance in the z list, each with its z indices in
 * z-list order: the grouping of make_edges' landmark_keys_zlist (GSLAM.c:246-261). */
void gslam_landmark_groups(int64_t n_z, const unsigned *z_lm, std::vector<unsigned> *ids,
                           std::vector<int64_t> *ptr, std::vector<unsigned> *members) {
    ids->clear();
    ptr->assign(1, 0);
    members->clear();
    std::vector<std::pair<unsigned, int64_t>> byid(n_z);
    for (int64_t i = 0; i < n_z; i++) byid[i] = {z_lm[i], i};
    std::stable_sort(byid.begin(), byid.end(),
                     [](const std::pair<unsigned, int64_t> &a, const std::pair<unsigned, int64_t> &b) {
                         return a.first < b.first;
                     });
    struct group { int64_t begin, end; };
    std::vector<group> groups;
    for (int64_t i = 0; i < n_z;) {
        int64_t j = i;
        while (j < n_z && byid[j].first == byid[i].first) j++;
        groups.push_back({i, j});
        i = j;
    }
    std::sort(groups.begin(), groups.end(), [&](const group &a, const group &b) {
        return byid[a.begin].second < byid[b.begin].second;
    });
    for (const group &gr : groups) {
        ids->push_back(byid[gr.begin].first);
        for (int64_t a = gr.begin; a < gr.end; a++) members->push_back((unsigned)byid[a].second);
        ptr->push_back((int64_t)members->size());
    }
}

/* ------------------------------------------------------------------------ */
/* host-only C ABI utilities                                                 */
/* ------------------------------------------------------------------------ */

extern "C" int gslam_obs_edge_order(uint32_t n_obs, const uint32_t *obs_landmark, uint32_t *pj,
                                    uint32_t *pk, int64_t cap, int64_t *n_pairs) {
    if ((n_obs && !obs_landmark) || !n_pairs) return GSLAM_ERR_BAD_INPUT;
    std::vector<unsigned> a, b;
    gslam_obs_pairs(n_obs, obs_landmark, &a, &b);
    *n_pairs = (int64_t)a.size();
    if (cap > 0 && pj && pk) {
        const int64_t n = std::min<int64_t>(cap, (int64_t)a.size());
        for (int64_t i = 0; i < n; i++) { pj[i] = a[i]; pk[i] = b[i]; }
    }
    return GSLAM_OK;
}

extern "C" int gslam_csr_pattern(uint32_t n_poses, int64_t n_edges, const uint32_t *t1,
                                 const uint32_t *t2, int *row_ptr, int *col_idx, int64_t *nnz) {
    if (n_poses == 0 || !nnz || (n_edges && (!t1 || !t2))) return GSLAM_ERR_BAD_INPUT;
    gslam_structure s;
    int rc = gslam_build_structure((int)n_poses, n_edges, t1, t2, 0, &s);
    if (rc != GSLAM_OK) return rc;
    *nnz = (int64_t)s.csr_col.size();
    if (row_ptr) memcpy(row_ptr, s.csr_row_ptr.data(), s.csr_row_ptr.size() * sizeof(int));
    if (col_idx) memcpy(col_idx, s.csr_col.data(), s.csr_col.size() * sizeof(int));
    return GSLAM_OK;
}

extern "C" int gslam_layout_plan(uint32_t n_poses, int64_t n_edges, const uint32_t *t1,
                                 const uint32_t *t2, int sell_window, uint32_t n_segments,
                                 const int32_t *segment_starts, uint32_t n_diag_rows,
                                 const int32_t *diag_rows, gslam_layout_info *info, int32_t *perm,
                                 int64_t *slice_ptr, int32_t *col, int64_t *ctr_ptr, int64_t *ctr,
                                 int64_t *xi_ptr, int64_t *xi_ctr, int64_t *slot_csr) {
    if (n_poses == 0 || n_poses > 0x3fffffffu || !info || n_edges < 0 || (n_edges && (!t1 || !t2)) ||
        (n_segments && !segment_starts) || (n_diag_rows && !diag_rows))
        return GSLAM_ERR_BAD_INPUT;
    std::vector<int> segs, diag;
    if (n_segments) {
        /* ascending starts inside the rows, the first at row 0 (a batch's graph ranges) */
        for (uint32_t q = 0; q < n_segments; q++) {
            const int32_t a = segment_starts[q];
            if (a < 0 || a >= (int32_t)n_poses || (q == 0 ? a != 0 : a <= segment_starts[q - 1]))
                return GSLAM_ERR_BAD_INPUT;
            segs.push_back(a);
        }
    }
    diag.assign(diag_rows, diag_rows + n_diag_rows);
    gslam_structure s;
    /* the window the graph constructors use (common_setup in api.cu) */
    const int window = sell_window <= 0 ? 1024 : sell_window;
    int rc = gslam_build_structure_ex((int)n_poses, n_edges, t1, t2, window, n_diag_rows ? &diag : nullptr,
                                      n_segments ? &segs : nullptr, &s);
    if (rc != GSLAM_OK) return rc;
    info->n_rows = s.n_rows;
    info->n_slices = s.n_slices;
    info->n_slots = s.n_slots;
    info->nnzb = s.nnzb;
    info->csr_nnz = (int64_t)s.csr_col.size();
    info->anchor_slot = s.anchor_slot;
    info->max_width = s.max_width;
    info->bare_anchor = s.bare_anchor ? 1 : 0;
    auto out = [](auto *dst, const auto &v) {
        if (dst) std::copy(v.begin(), v.end(), dst);
    };
    out(perm, s.perm);
    out(slice_ptr, s.slice_ptr);
    out(col, s.col);
    out(ctr_ptr, s.ctr_ptr);
    out(ctr, s.ctr);
    out(xi_ptr, s.xi_ptr);
    out(xi_ctr, s.xi_ctr);
    out(slot_csr, s.slot_csr);
    return GSLAM_OK;
}
