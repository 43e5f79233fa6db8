/*
 * gslam_internal.h — data layout shared by the host structure builder and the
 * CUDA kernels of libgslam.
 *
 * Matrix layout ("sliced 3x3-block ELL"): the N block rows of Omega are
 * renumbered (new = iperm[old]) by sorting them by block count inside windows
 * of `sell_window` rows, then cut into slices of 32 consecutive new rows. Slice
 * s owns slots [slice_ptr[s], slice_ptr[s+1]); slot (s, j, lane) holds the j-th
 * block (in ascending ORIGINAL column order, the order the reference sums a row
 * in) of new row 32 s + lane. Values are stored entry-major inside a slice so a
 * warp reading entry e of position j touches 32 consecutive values:
 *     val[9 * slice_ptr[s] + (j * 9 + e) * 32 + lane]
 * Columns are stored per slot as new row indices: col[slice_ptr[s] + j * 32 + lane].
 * Rows shorter than their slice's width leave padded slots that are never read.
 *
 * Vectors are indexed by new row and padded to 4 components (32 bytes, one
 * sector) so a column gather is a single aligned sector: v[4 * row + c].
 */
#ifndef GSLAM_INTERNAL_H
#define GSLAM_INTERNAL_H

#include <stdint.h>
#include <vector>

#define GSLAM_SLICE 32

struct gslam_structure {
    int n_rows = 0;          /* N block rows (poses) */
    int n_slices = 0;
    int64_t n_slots = 0;     /* slice_ptr[n_slices] (multiple of 32) */
    int64_t nnzb = 0;        /* real blocks */
    int64_t n_edges = 0;
    int max_width = 0;
    std::vector<int> perm;        /* new row -> old row */
    std::vector<int> iperm;       /* old row -> new row */
    std::vector<int64_t> slice_ptr;   /* [n_slices + 1], in slots */
    std::vector<int> slice_width;     /* [n_slices] */
    std::vector<int> row_len;         /* [32 * n_slices] by new row, 0 for padding rows */
    std::vector<int> col;             /* [n_slots] new column row, -1 for padding */
    std::vector<int> diag_slot;       /* [n_rows] by new row: slot of the diagonal block, -1 if none */
    std::vector<int> chunk_slice;     /* [n_slots / 32]: slice of each group of 32 slots */
    /* assembly: per slot, contributions e*4 + sub (sub 0..3 = UL, UR, BL, BR) in edge order */
    std::vector<int64_t> ctr_ptr;     /* [n_slots + 1] */
    std::vector<int64_t> ctr;         /* [4 * n_edges] */
    /* right-hand side: per new row, contributions e*2 + w (w 0 = upper, 1 = bottom) */
    std::vector<int64_t> xi_ptr;      /* [n_rows + 1] */
    std::vector<int64_t> xi_ctr;      /* [2 * n_edges] */
    int64_t anchor_slot = -1;         /* slot of block (0,0) (gets the 1e6 anchor) */
    /* scalar CSR of the reference (MatrixOps.c:197-221) */
    bool bare_anchor = false;         /* no block touches pose 0: rows 0..2 hold only (d,d) */
    std::vector<int> csr_row_ptr;     /* [3N + 1] */
    std::vector<int> csr_col;         /* [nnz] */
    std::vector<int64_t> slot_csr;    /* [n_slots] CSR position of entry (r=0,c=0) of the slot, -1 padding */
};

/* Layout of a sorted unique block-key pattern (keys I * N + J, (0,0) included). */
int gslam_layout_from_blocks(int n_rows, const std::vector<uint64_t> &keys, bool bare_anchor,
                             int sell_window, gslam_structure *s,
                             std::vector<int64_t> *key_slot_out,
                             const std::vector<int> *segments = nullptr);

/* Builds the structure from the edge list (t1[e], t2[e]) in array order. */
int gslam_build_structure(int n_rows, int64_t n_edges, const unsigned *t1, const unsigned *t2,
                          int sell_window, gslam_structure *s);
/* Same, with extra diagonal blocks (rows that have no edge, e.g. a batch's padding
 * poses) and segment starts at which the row-sorting windows restart. */
int gslam_build_structure_ex(int n_rows, int64_t n_edges, const unsigned *t1, const unsigned *t2,
                             int sell_window, const std::vector<int> *diag_rows,
                             const std::vector<int> *segments, gslam_structure *s);

/* Landmark groups of the z list (first-appearance order, members in z order). */
void gslam_landmark_groups(int64_t n_z, const unsigned *z_lm, std::vector<unsigned> *ids,
                           std::vector<int64_t> *ptr, std::vector<unsigned> *members);

/* Reference edge order for observation edges (GSLAM.c:222-318): pairs of z-list indices. */
void gslam_obs_pairs(int64_t n_z, const unsigned *z_lm, std::vector<unsigned> *pj,
                     std::vector<unsigned> *pk);

#endif
