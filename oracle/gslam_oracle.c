/*
 * gslam_oracle.c — CPU restatement of the reference's per-Gauss-Newton path.
 *
 * TEST INFRASTRUCTURE ONLY. Nothing in the product links, loads or calls this
 * file; only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use
 * it, as the checker. It restates, in plain C and in the reference's exact
 * floating-point operation order, the path of isaacyhe/G-SLAM_on_GPU_and_FPGA
 * src/cpu_pcg_fp64:
 *   read_data            GSLAM.c:415-493
 *   make_edges (order)   GSLAM.c:222-318
 *   ObsEdge_create       ObsEdge.c:10-212      (or_edges.inc)
 *   MotionEdge_create    MotionEdge.c:9-193    (or_edges.inc)
 *   build_csr_from_edges MatrixOps.c:173-273
 *   pcg_solve_sparse     MatrixOps.c:281-391
 *   GN loop / diff       GSLAM.c:55-139
 *   dense GJ inverse     MatrixOps.c:29-91 (+ add_edge GSLAM.c:320-371)
 * Two deliberate differences, neither of which changes a result for N <= 21,845:
 *   - the CSR structure is found by sorting 64-bit block keys instead of the
 *     reference's dim x dim byte marker, which is indexed in 32-bit arithmetic
 *     and wraps for dim > 65,535 (MatrixOps.c:177-204), and needs dim^2 bytes;
 *   - the per-entry slot is found by binary search instead of a linear scan of
 *     the row (columns are unique and ascending, so the slot is the same).
 * Pinning: tests/test_oracle_pin.py compares this file bit for bit with the
 * reference sources compiled from their own tree (oracle/Makefile -> oracle/_ref).
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "crmath.h"
#include "gslam_oracle.h"

/* ---- linearisation, glibc flavour (bit-identical to the reference) ---- */
#define OR_FN(n) n##_glibc
#define OR_SINCOS(x, s, c) do { double _a = (x); *(s) = sin(_a); *(c) = cos(_a); } while (0)
#define OR_SQ(x) pow((x), 2.0)
#include "or_edges.inc"
#undef OR_FN
#undef OR_SINCOS
#undef OR_SQ

/* ---- linearisation, correctly rounded flavour (bit-identical to the CUDA kernels) ---- */
#define OR_FN(n) n##_cr
#define OR_SINCOS(x, s, c) cr_sincos((x), (s), (c))
#define OR_SQ(x) ((x) * (x))
#include "or_edges.inc"
#undef OR_FN
#undef OR_SINCOS
#undef OR_SQ

void or_cr_sincos(double x, double *s, double *c) { cr_sincos(x, s, c); }

/* ------------------------------------------------------------------------ */
/* read_data (GSLAM.c:415-493)                                               */
/* ------------------------------------------------------------------------ */

/*
 * Counts (caps == 0) or fills the u / x / z records of a reference log.
 * Lines are split on single spaces like strtok(line, " "); a first token other
 * than u, x, z sets delta from the second token (the reference's `else` branch).
 * Empty lines are skipped (the reference would dereference a NULL token).
 */
int or_read_log(const char *path, double *delta,
                unsigned *n_u, unsigned *u_step, double *u_nu_om, unsigned cap_u,
                unsigned *n_x, unsigned *x_step, double *x_pose, unsigned cap_x,
                unsigned *n_z, unsigned *z_step, unsigned *z_lm, double *z_rb, unsigned cap_z) {
    FILE *f = fopen(path, "r");
    if (!f) return -1;
    char line[1024];
    unsigned nu = 0, nx = 0, nz = 0;
    while (fgets(line, sizeof line, f)) {
        char *save = NULL;
        char *tok = strtok_r(line, " ", &save);
        if (!tok) continue;
        if (strcmp(tok, "u") == 0) {
            char *a = strtok_r(NULL, " ", &save), *b = strtok_r(NULL, " ", &save),
                 *c = strtok_r(NULL, " ", &save);
            if (!a || !b || !c) { fclose(f); return -2; }
            if (nu < cap_u) {
                u_step[nu] = (unsigned)atoi(a);
                u_nu_om[2 * nu] = atof(b);
                u_nu_om[2 * nu + 1] = atof(c);
            }
            nu++;
        } else if (strcmp(tok, "x") == 0) {
            char *a = strtok_r(NULL, " ", &save), *b = strtok_r(NULL, " ", &save),
                 *c = strtok_r(NULL, " ", &save), *d = strtok_r(NULL, " ", &save);
            if (!a || !b || !c || !d) { fclose(f); return -2; }
            if (nx < cap_x) {
                x_step[nx] = (unsigned)atoi(a);
                x_pose[3 * nx] = atof(b);
                x_pose[3 * nx + 1] = atof(c);
                x_pose[3 * nx + 2] = atof(d);
            }
            nx++;
        } else if (strcmp(tok, "z") == 0) {
            char *a = strtok_r(NULL, " ", &save), *b = strtok_r(NULL, " ", &save),
                 *c = strtok_r(NULL, " ", &save), *d = strtok_r(NULL, " ", &save);
            if (!a || !b || !c || !d) { fclose(f); return -2; }
            if (nz < cap_z) {
                z_step[nz] = (unsigned)atoi(a);
                z_lm[nz] = (unsigned)atoi(b);
                z_rb[2 * nz] = atof(c);
                z_rb[2 * nz + 1] = atof(d);
            }
            nz++;
        } else {
            char *a = strtok_r(NULL, " ", &save);
            if (a && delta) *delta = atof(a);
        }
    }
    fclose(f);
    *n_u = nu; *n_x = nx; *n_z = nz;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* make_edges ordering (GSLAM.c:222-318)                                     */
/* ------------------------------------------------------------------------ */

/*
 * Observation-edge order of the reference: landmarks in order of first
 * appearance in the z list; for a landmark observed k times (z-list order
 * o_0..o_{k-1}) the pairs (o_j, o_k) for j < k, j outer, k inner.
 * Writes up to `cap` pairs of z-list indices; returns the total count.
 */
long or_obs_edge_pairs(unsigned n_z, const unsigned *z_lm, unsigned *pj, unsigned *pk, long cap) {
    if (n_z == 0) return 0;
    unsigned max_id = 0;
    for (unsigned i = 0; i < n_z; i++) if (z_lm[i] > max_id) max_id = z_lm[i];
    unsigned *count = calloc((size_t)max_id + 1, sizeof(unsigned));
    unsigned *first = malloc(((size_t)max_id + 1) * sizeof(unsigned));
    unsigned *order = malloc((size_t)n_z * sizeof(unsigned)); /* distinct ids, first-appearance */
    unsigned n_lm = 0;
    for (unsigned i = 0; i < n_z; i++) {
        unsigned id = z_lm[i];
        if (count[id] == 0) order[n_lm++] = id;
        count[id]++;
    }
    /* offsets of each landmark's group in landmark order */
    unsigned pos = 0;
    for (unsigned l = 0; l < n_lm; l++) { first[order[l]] = pos; pos += count[order[l]]; }
    unsigned *grouped = malloc((size_t)n_z * sizeof(unsigned));
    unsigned *fill = calloc((size_t)max_id + 1, sizeof(unsigned));
    for (unsigned i = 0; i < n_z; i++) {
        unsigned id = z_lm[i];
        grouped[first[id] + fill[id]++] = i;
    }
    long e = 0;
    for (unsigned l = 0; l < n_lm; l++) {
        unsigned id = order[l], base = first[id], k = count[id];
        for (unsigned a = 0; a < k; a++)
            for (unsigned b = a + 1; b < k; b++) {
                if (e < cap) { pj[e] = grouped[base + a]; pk[e] = grouped[base + b]; }
                e++;
            }
    }
    free(count); free(first); free(order); free(grouped); free(fill);
    return e;
}

/* ------------------------------------------------------------------------ */
/* all edges of one round, in the reference's array order (GSLAM.c:62-72)    */
/* ------------------------------------------------------------------------ */

int or_linearise(int use_cr, unsigned n_poses, const double *poses, const double *u_nu_om,
                 double delta, double lambda, const double *mns,
                 const unsigned *z_step, const double *z_rb,
                 long n_obs_edges, const unsigned *pj, const unsigned *pk,
                 unsigned *t1, unsigned *t2, double *blocks) {
    for (long e = 0; e < n_obs_edges; e++) {
        unsigned a = pj[e], b = pk[e];
        unsigned s1 = z_step[a], s2 = z_step[b];
        if (s1 >= n_poses || s2 >= n_poses) return -1;
        t1[e] = s1; t2[e] = s2;
        if (use_cr)
            or_obs_edge_cr(poses + 3 * (size_t)s1, poses + 3 * (size_t)s2, z_rb + 2 * (size_t)a,
                           z_rb + 2 * (size_t)b, blocks + 42 * (size_t)e, NULL, NULL);
        else
            or_obs_edge_glibc(poses + 3 * (size_t)s1, poses + 3 * (size_t)s2, z_rb + 2 * (size_t)a,
                              z_rb + 2 * (size_t)b, blocks + 42 * (size_t)e, NULL, NULL);
    }
    for (unsigned i = 0; i + 1 < n_poses; i++) {
        long e = n_obs_edges + i;
        t1[e] = i; t2[e] = i + 1;
        double nu = u_nu_om[2 * (size_t)(i + 1)], om = u_nu_om[2 * (size_t)(i + 1) + 1];
        if (use_cr)
            or_motion_edge_cr(poses + 3 * (size_t)i, poses + 3 * (size_t)(i + 1), nu, om, delta,
                              lambda, mns, blocks + 42 * (size_t)e, NULL);
        else
            or_motion_edge_glibc(poses + 3 * (size_t)i, poses + 3 * (size_t)(i + 1), nu, om, delta,
                                 lambda, mns, blocks + 42 * (size_t)e, NULL);
    }
    return 0;
}

/*
 * Round cost at `poses` (GSLAM.c:74-87, with the dimensions that code meant and reset
 * every round): per edge in the reference's array order, observation edges
 * hat_e^T Omega hat_e (2x2) and motion edges lambda d^T Omega d (3x3); the total is
 * `cost += c` from 0.0 in that order. edge_cost (may be NULL) receives the terms.
 */
int or_round_cost(int use_cr, unsigned n_poses, const double *poses, const double *u_nu_om,
                  double delta, double lambda, const double *mns, const unsigned *z_step,
                  const double *z_rb, long n_obs_edges, const unsigned *pj, const unsigned *pk,
                  double *edge_cost, double *total) {
    double out[42], acc = 0.0, c;
    for (long e = 0; e < n_obs_edges; e++) {
        unsigned a = pj[e], b = pk[e];
        unsigned s1 = z_step[a], s2 = z_step[b];
        if (s1 >= n_poses || s2 >= n_poses) return -1;
        if (use_cr)
            or_obs_edge_cr(poses + 3 * (size_t)s1, poses + 3 * (size_t)s2, z_rb + 2 * (size_t)a,
                           z_rb + 2 * (size_t)b, out, NULL, &c);
        else
            or_obs_edge_glibc(poses + 3 * (size_t)s1, poses + 3 * (size_t)s2, z_rb + 2 * (size_t)a,
                              z_rb + 2 * (size_t)b, out, NULL, &c);
        if (edge_cost) edge_cost[e] = c;
        acc += c;
    }
    for (unsigned i = 0; i + 1 < n_poses; i++) {
        double nu = u_nu_om[2 * (size_t)(i + 1)], om = u_nu_om[2 * (size_t)(i + 1) + 1];
        if (use_cr)
            or_motion_edge_cr(poses + 3 * (size_t)i, poses + 3 * (size_t)(i + 1), nu, om, delta,
                              lambda, mns, out, &c);
        else
            or_motion_edge_glibc(poses + 3 * (size_t)i, poses + 3 * (size_t)(i + 1), nu, om, delta,
                                 lambda, mns, out, &c);
        if (edge_cost) edge_cost[n_obs_edges + i] = c;
        acc += c;
    }
    *total = acc;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* build_csr_from_edges (MatrixOps.c:173-273), scalable structure            */
/* ------------------------------------------------------------------------ */

static int cmp_u64(const void *a, const void *b) {
    uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
    return (x > y) - (x < y);
}

/* Sorted unique block keys (I * nb + J) of the matrix; returns the count. */
static long block_keys(unsigned nb, long n_edges, const unsigned *t1, const unsigned *t2,
                       uint64_t **keys_out) {
    uint64_t *k = malloc(sizeof(uint64_t) * (4 * (size_t)n_edges + 1));
    long n = 0;
    for (long e = 0; e < n_edges; e++) {
        uint64_t a = t1[e], b = t2[e];
        k[n++] = a * nb + a; k[n++] = a * nb + b; k[n++] = b * nb + a; k[n++] = b * nb + b;
    }
    qsort(k, (size_t)n, sizeof(uint64_t), cmp_u64);
    long u = 0;
    for (long i = 0; i < n; i++) if (u == 0 || k[i] != k[u - 1]) k[u++] = k[i];
    *keys_out = k;
    return u;
}

/* Scalar nnz of the reference CSR (blocks x 9, or the bare anchor diagonal). */
long or_csr_nnz(unsigned dim, long n_edges, const unsigned *t1, const unsigned *t2) {
    unsigned nb = dim / 3;
    uint64_t *k;
    long nkb = block_keys(nb, n_edges, t1, t2, &k);
    int has00 = (nkb > 0 && k[0] == 0);
    free(k);
    return 9 * nkb + (has00 ? 0 : 3);
}

/*
 * Fills row_ptr[dim+1], col_idx[nnz], values[nnz] and xi[dim] exactly as
 * build_csr_from_edges does: values start at +0.0, the 1e6 anchor is added to
 * (0,0), (1,1), (2,2) first, then every edge in array order adds UL, UR, BL, BR
 * entry by entry (r outer, c inner), and xi gets xi_upper / xi_bottom per row.
 */
int or_csr_build_anchor(unsigned dim, long n_edges, const unsigned *t1, const unsigned *t2,
                        const double *blocks, double anchor, int *row_ptr, int *col_idx,
                        double *values, double *xi);

int or_csr_build(unsigned dim, long n_edges, const unsigned *t1, const unsigned *t2,
                 const double *blocks, int *row_ptr, int *col_idx, double *values, double *xi) {
    return or_csr_build_anchor(dim, n_edges, t1, t2, blocks, 1000000.0, row_ptr, col_idx, values, xi);
}

/* Same, with the anchor weight as a parameter (the reference fixes 1e6, MatrixOps.c:227). */
int or_csr_build_anchor(unsigned dim, long n_edges, const unsigned *t1, const unsigned *t2,
                        const double *blocks, double anchor, int *row_ptr, int *col_idx,
                        double *values, double *xi) {
    unsigned nb = dim / 3;
    for (long e = 0; e < n_edges; e++)
        if (t1[e] >= nb || t2[e] >= nb) return -1;
    uint64_t *k;
    long nkb = block_keys(nb, n_edges, t1, t2, &k);
    int has00 = (nkb > 0 && k[0] == 0);
    /* per block row, its blocks are contiguous in k; scalar row 3I+r lists 3J..3J+2 */
    long *brow = calloc((size_t)nb + 1, sizeof(long));
    for (long i = 0; i < nkb; i++) brow[k[i] / nb + 1]++;
    for (unsigned i = 0; i < nb; i++) brow[i + 1] += brow[i];
    long p = 0;
    row_ptr[0] = 0;
    for (unsigned I = 0; I < nb; I++) {
        for (int r = 0; r < 3; r++) {
            if (I == 0 && !has00) {           /* bare anchor entry (d, d) */
                col_idx[p++] = r;
            } else {
                for (long b = brow[I]; b < brow[I + 1]; b++) {
                    unsigned J = (unsigned)(k[b] % nb);
                    for (int c = 0; c < 3; c++) col_idx[p++] = (int)(3 * J + c);
                }
            }
            row_ptr[3 * I + r + 1] = (int)p;
        }
    }
    for (long i = 0; i < p; i++) values[i] = 0.0;
    for (unsigned i = 0; i < dim; i++) xi[i] = 0.0;
    free(brow);
    free(k);
#define OR_SLOT(row, col)                                                        \
    ({ int _lo = row_ptr[(row)], _hi = row_ptr[(row) + 1] - 1, _f = -1;         \
       while (_lo <= _hi) { int _m = (_lo + _hi) / 2;                            \
           if (col_idx[_m] == (int)(col)) { _f = _m; break; }                    \
           if (col_idx[_m] < (int)(col)) _lo = _m + 1; else _hi = _m - 1; }       \
       _f; })
    for (int d = 0; d < 3; d++) values[OR_SLOT(d, d)] += anchor;
    for (long e = 0; e < n_edges; e++) {
        unsigned f1 = t1[e] * 3, f2 = t2[e] * 3;
        const double *B = blocks + 42 * (size_t)e;
        for (int r = 0; r < 3; r++) {
            for (int c = 0; c < 3; c++) {
                values[OR_SLOT(f1 + r, f1 + c)] += B[r * 3 + c];
                values[OR_SLOT(f1 + r, f2 + c)] += B[9 + r * 3 + c];
                values[OR_SLOT(f2 + r, f1 + c)] += B[18 + r * 3 + c];
                values[OR_SLOT(f2 + r, f2 + c)] += B[27 + r * 3 + c];
            }
            xi[f1 + r] += B[36 + r];
            xi[f2 + r] += B[39 + r];
        }
    }
#undef OR_SLOT
    return 0;
}

/* ------------------------------------------------------------------------ */
/* pcg_solve_sparse (MatrixOps.c:281-391) with tolerance / iteration knobs   */
/* ------------------------------------------------------------------------ */

/* Cofactor inverse of the 3x3 diagonal blocks, det == 0 -> 1e-30 (MatrixOps.c:287-315). */
void or_diag_inv(unsigned dim, const int *row_ptr, const int *col_idx, const double *values,
                 double *diag_inv) {
    unsigned nbk = dim / 3;
    for (unsigned blk = 0; blk < nbk; blk++) {
        unsigned base = blk * 3;
        double a[9] = { 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0 };
        for (int r = 0; r < 3; r++)
            for (int p = row_ptr[base + r]; p < row_ptr[base + r + 1]; p++) {
                int c = col_idx[p] - (int)base;
                if (c >= 0 && c < 3) a[r * 3 + c] = values[p];
            }
        double det = a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
                     a[2] * (a[3] * a[7] - a[4] * a[6]);
        if (det == 0.0) det = 1e-30;
        double *v = diag_inv + 9 * (size_t)blk;
        v[0] = (a[4] * a[8] - a[5] * a[7]) / det;
        v[1] = (a[2] * a[7] - a[1] * a[8]) / det;
        v[2] = (a[1] * a[5] - a[2] * a[4]) / det;
        v[3] = (a[5] * a[6] - a[3] * a[8]) / det;
        v[4] = (a[0] * a[8] - a[2] * a[6]) / det;
        v[5] = (a[2] * a[3] - a[0] * a[5]) / det;
        v[6] = (a[3] * a[7] - a[4] * a[6]) / det;
        v[7] = (a[1] * a[6] - a[0] * a[7]) / det;
        v[8] = (a[0] * a[4] - a[1] * a[3]) / det;
    }
}

/* Row-sequential SpMV, q[i] = 0.0 + sum_j a_ij p_j in column order (MatrixOps.c:349-353). */
void or_spmv(unsigned dim, const int *row_ptr, const int *col_idx, const double *values,
             const double *p, double *q) {
    for (unsigned i = 0; i < dim; i++) {
        double acc = 0.0;
        for (int j = row_ptr[i]; j < row_ptr[i + 1]; j++) acc += values[j] * p[col_idx[j]];
        q[i] = acc;
    }
}

/*
 * The reference's PCG: x = 0, r = b, z = D^-1 r, p = z, tol = tol_rel * ||b||;
 * per iteration q = A p, alpha = rz / pq (stop if pq == 0), x += alpha p,
 * r -= alpha q, stop if ||r|| < tol, z = D^-1 r, beta = rz'/rz, p = z + beta p.
 * The reference fixes tol_rel = 1e-6 and max_iter = 500.
 */
int or_pcg(unsigned dim, const int *row_ptr, const int *col_idx, const double *values,
           const double *b, double *x, double tol_rel, int max_iter, int *iters_out,
           double *rnorm_out) {
    unsigned nbk = dim / 3;
    double *dinv = malloc(sizeof(double) * 9 * (size_t)(nbk ? nbk : 1));
    or_diag_inv(dim, row_ptr, col_idx, values, dinv);
    double *r = calloc(dim, sizeof(double)), *z = calloc(dim, sizeof(double));
    double *p = calloc(dim, sizeof(double)), *q = calloc(dim, sizeof(double));
    for (unsigned i = 0; i < dim; i++) { x[i] = 0.0; r[i] = b[i]; }
    for (unsigned blk = 0; blk < nbk; blk++) {
        unsigned base = blk * 3;
        const double *v = dinv + 9 * (size_t)blk;
        for (int rr = 0; rr < 3; rr++) {
            z[base + rr] = 0.0;
            for (int c = 0; c < 3; c++) z[base + rr] += v[rr * 3 + c] * r[base + c];
        }
    }
    for (unsigned i = 0; i < dim; i++) p[i] = z[i];
    double rz_old = 0.0;
    for (unsigned i = 0; i < dim; i++) rz_old += r[i] * z[i];
    double b_norm = 0.0;
    for (unsigned i = 0; i < dim; i++) b_norm += b[i] * b[i];
    b_norm = sqrt(b_norm);
    double tol = tol_rel * b_norm;
    int k;
    double r_norm = b_norm * b_norm;
    for (k = 0; k < max_iter; k++) {
        or_spmv(dim, row_ptr, col_idx, values, p, q);
        double pq = 0.0;
        for (unsigned i = 0; i < dim; i++) pq += p[i] * q[i];
        if (pq == 0.0) break;
        double alpha = rz_old / pq;
        r_norm = 0.0;
        for (unsigned i = 0; i < dim; i++) {
            x[i] += alpha * p[i];
            r[i] -= alpha * q[i];
            r_norm += r[i] * r[i];
        }
        if (sqrt(r_norm) < tol) { k++; break; }
        for (unsigned blk = 0; blk < nbk; blk++) {
            unsigned base = blk * 3;
            const double *v = dinv + 9 * (size_t)blk;
            for (int rr = 0; rr < 3; rr++) {
                z[base + rr] = 0.0;
                for (int c = 0; c < 3; c++) z[base + rr] += v[rr * 3 + c] * r[base + c];
            }
        }
        double rz_new = 0.0;
        for (unsigned i = 0; i < dim; i++) rz_new += r[i] * z[i];
        double beta = rz_new / rz_old;
        for (unsigned i = 0; i < dim; i++) p[i] = z[i] + beta * p[i];
        rz_old = rz_new;
    }
    if (iters_out) *iters_out = k;
    if (rnorm_out) *rnorm_out = sqrt(r_norm);
    free(dinv); free(r); free(z); free(p); free(q);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* GN loop (GSLAM.c:55-139), use_diff = 1 semantics                           */
/* ------------------------------------------------------------------------ */

/*
 * Runs up to `rounds` Gauss-Newton rounds in place on poses[3 * n_poses].
 * diffs[n] receives ||dx|| / sqrt(dim) of round n + 1. The stop rules are the
 * reference's: diff < 0.01, or 20 rounds without a new best diff.
 * Returns the number of rounds executed, or < 0 on bad input.
 */
int or_run(int use_cr, unsigned n_poses, double *poses, const double *u_nu_om, double delta,
           double lambda, unsigned n_z, const unsigned *z_step, const unsigned *z_lm,
           const double *z_rb, unsigned rounds, double tol_rel, int max_iter, double *diffs,
           int *pcg_iters) {
    const double mns[4] = { 0.19, 0.001, 0.13, 0.2 };
    unsigned dim = 3 * n_poses;
    long n_obs = or_obs_edge_pairs(n_z, z_lm, NULL, NULL, 0);
    unsigned *pj = malloc(sizeof(unsigned) * (size_t)(n_obs + 1));
    unsigned *pk = malloc(sizeof(unsigned) * (size_t)(n_obs + 1));
    or_obs_edge_pairs(n_z, z_lm, pj, pk, n_obs);
    long n_edges = n_obs + (n_poses ? n_poses - 1 : 0);
    unsigned *t1 = malloc(sizeof(unsigned) * (size_t)(n_edges + 1));
    unsigned *t2 = malloc(sizeof(unsigned) * (size_t)(n_edges + 1));
    double *blocks = malloc(sizeof(double) * 42 * (size_t)(n_edges + 1));
    double *xi = malloc(sizeof(double) * dim), *dx = malloc(sizeof(double) * dim);
    int *row_ptr = malloc(sizeof(int) * (dim + 1));
    int *col_idx = NULL;
    double *values = NULL;
    double best = 1e30;
    unsigned no_improve = 0;
    int done = 0, rc = 0;
    for (unsigned n = 1; n <= rounds; n++) {
        if (or_linearise(use_cr, n_poses, poses, u_nu_om, delta, lambda, mns, z_step, z_rb, n_obs,
                         pj, pk, t1, t2, blocks) != 0) { rc = -1; break; }
        if (!col_idx) {
            long nnz = or_csr_nnz(dim, n_edges, t1, t2);
            col_idx = malloc(sizeof(int) * (size_t)nnz);
            values = malloc(sizeof(double) * (size_t)nnz);
        }
        or_csr_build(dim, n_edges, t1, t2, blocks, row_ptr, col_idx, values, xi);
        int it = 0;
        or_pcg(dim, row_ptr, col_idx, values, xi, dx, tol_rel, max_iter, &it, NULL);
        if (pcg_iters) pcg_iters[n - 1] = it;
        for (unsigned i = 0; i < n_poses; i++) {
            poses[3 * i] = poses[3 * i] + dx[3 * i];
            poses[3 * i + 1] = poses[3 * i + 1] + dx[3 * i + 1];
            poses[3 * i + 2] = poses[3 * i + 2] + dx[3 * i + 2];
        }
        double diff = (use_cr ? or_norm_cr(dx, dim) : or_norm_glibc(dx, dim)) / sqrt((double)dim);
        if (diffs) diffs[n - 1] = diff;
        done = (int)n;
        if (diff < 0.01) break;
        if (diff < best) { best = diff; no_improve = 0; }
        else if (++no_improve >= 20) break;
    }
    free(pj); free(pk); free(t1); free(t2); free(blocks); free(xi); free(dx);
    free(row_ptr); free(col_idx); free(values);
    return rc < 0 ? rc : done;
}

/* ------------------------------------------------------------------------ */
/* dense Gauss-Jordan inverse (MatrixOps.c:29-91), heap workspace             */
/* ------------------------------------------------------------------------ */

int or_landmark_map(int use_cr, unsigned n_groups, const long *group_ptr, const unsigned *members,
                    const unsigned *z_step, const double *z_rb, const double *poses, double *ms) {
    if (use_cr) landmark_map_cr(n_groups, group_ptr, members, z_step, z_rb, poses, ms);
    else landmark_map_glibc(n_groups, group_ptr, members, z_step, z_rb, poses, ms);
    return 0;
}

int or_gj_inverse(unsigned n, const double *a, double *res) {
    double *t = malloc(sizeof(double) * (size_t)n * n);
    if (!t) return -1;
    for (size_t r = 0; r < n; r++)
        for (size_t c = 0; c < n; c++) {
            t[r * n + c] = a[r * n + c];
            res[r * n + c] = (r == c) ? 1.0 : 0.0;
        }
    for (size_t i = 0; i < n; i++) {
        if (t[i * n + i] == 0.0) {
            for (size_t k = 0; k < (size_t)n * n; k++) res[k] = 0.0;
            free(t);
            return 1;
        }
        for (size_t j = 0; j < n; j++) {
            if (j == i) continue;
            double ratio = t[j * n + i] / t[i * n + i];
            for (size_t k = 0; k < n; k++) {
                t[j * n + k] = t[j * n + k] - ratio * t[i * n + k];
                res[j * n + k] = res[j * n + k] - ratio * res[i * n + k];
            }
        }
    }
    for (size_t i = 0; i < n; i++)
        for (size_t j = 0; j < n; j++) res[i * n + j] = res[i * n + j] / t[i * n + i];
    free(t);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* SE(2) between-factor (no reference counterpart: the configs' pose graphs) */
/* ------------------------------------------------------------------------ */

static double or_wrap(double t) {
    const double pi = 3.141592653589793, two_pi = 6.283185307179586;
    if (t > pi || t <= -pi) {
        t = fmod(t + pi, two_pi);
        if (t < 0.0) t = t + two_pi;
        t = t - pi;
    }
    return t;
}

/*
 * e = [R(th_i)^T (t_j - t_i) - z_t ; wrap(th_j - th_i - z_th)], L = diag(info) * lambda;
 * UL = Ji^T L Ji, UR = Ji^T L Jj, BL = Jj^T L Ji, BR = Jj^T L Jj, xi_u = -Ji^T L e,
 * xi_b = -Jj^T L e; sums over k = 0, 1, 2 from 0.0 with separate multiply and add.
 */
void or_se2_edge(const double *xi, const double *xj, const double *z, const double *info,
                 double lambda, double *out, double *e_out) {
    double s, c;
    cr_sincos(xi[2], &s, &c);
    const double dx = xj[0] - xi[0], dy = xj[1] - xi[1];
    double e[3];
    e[0] = (c * dx + s * dy) - z[0];
    e[1] = (c * dy - s * dx) - z[1];
    e[2] = or_wrap((xj[2] - xi[2]) - z[2]);
    if (e_out) { e_out[0] = e[0]; e_out[1] = e[1]; e_out[2] = e[2]; }
    const double Ji[9] = { -c, -s, c * dy - s * dx, s, -c, -(c * dx) - s * dy, 0.0, 0.0, -1.0 };
    const double Jj[9] = { c, s, 0.0, -s, c, 0.0, 0.0, 0.0, 1.0 };
    double L[3], LJi[9], LJj[9], Le[3];
    for (int k = 0; k < 3; k++) L[k] = info[k] * lambda;
    for (int k = 0; k < 3; k++) {
        for (int cc = 0; cc < 3; cc++) {
            LJi[3 * k + cc] = L[k] * Ji[3 * k + cc];
            LJj[3 * k + cc] = L[k] * Jj[3 * k + cc];
        }
        Le[k] = L[k] * e[k];
    }
    for (int r = 0; r < 3; r++) {
        for (int cc = 0; cc < 3; cc++) {
            double ul = 0.0, ur = 0.0, bl = 0.0, br = 0.0;
            for (int k = 0; k < 3; k++) {
                ul = ul + Ji[3 * k + r] * LJi[3 * k + cc];
                ur = ur + Ji[3 * k + r] * LJj[3 * k + cc];
                bl = bl + Jj[3 * k + r] * LJi[3 * k + cc];
                br = br + Jj[3 * k + r] * LJj[3 * k + cc];
            }
            out[3 * r + cc] = ul;
            out[9 + 3 * r + cc] = ur;
            out[18 + 3 * r + cc] = bl;
            out[27 + 3 * r + cc] = br;
        }
        double xu = 0.0, xb = 0.0;
        for (int k = 0; k < 3; k++) {
            xu = xu + Ji[3 * k + r] * Le[k];
            xb = xb + Jj[3 * k + r] * Le[k];
        }
        out[36 + r] = -xu;
        out[39 + r] = -xb;
    }
}

int or_se2_linearise(long n_edges, const unsigned *ei, const unsigned *ej, const double *poses,
                     const double *meas, const double *info, double lambda, double *blocks,
                     double *errs) {
    for (long e = 0; e < n_edges; e++)
        or_se2_edge(poses + 3 * (size_t)ei[e], poses + 3 * (size_t)ej[e], meas + 3 * (size_t)e,
                    info + 3 * (size_t)e, lambda, blocks + 42 * (size_t)e,
                    errs ? errs + 3 * (size_t)e : NULL);
    return 0;
}
