/*
 * gslam_oracle.h — C restatement of the reference path (test infrastructure only).
 * See gslam_oracle.c for the reference file:line each function follows.
 */
#ifndef GSLAM_ORACLE_H
#define GSLAM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

void or_cr_sincos(double x, double *s, double *c);

int or_read_log(const char *path, double *delta,
                unsigned *n_u, unsigned *u_step, double *u_nu_om, unsigned cap_u,
                unsigned *n_x, unsigned *x_step, double *x_pose, unsigned cap_x,
                unsigned *n_z, unsigned *z_step, unsigned *z_lm, double *z_rb, unsigned cap_z);

long or_obs_edge_pairs(unsigned n_z, const unsigned *z_lm, unsigned *pj, unsigned *pk, long cap);

void or_obs_edge_glibc(const double *x1, const double *x2, const double *z1, const double *z2,
                       double *out, double *hat_e_out, double *cost_out);
void or_obs_edge_cr(const double *x1, const double *x2, const double *z1, const double *z2,
                    double *out, double *hat_e_out, double *cost_out);
void or_motion_edge_glibc(const double *x1, const double *x2, double nu, double omega,
                          double delta, double lambda, const double *mns, double *out,
                          double *cost_out);
void or_motion_edge_cr(const double *x1, const double *x2, double nu, double omega,
                       double delta, double lambda, const double *mns, double *out,
                       double *cost_out);
double or_norm_glibc(const double *v, unsigned n);
double or_norm_cr(const double *v, unsigned n);

int or_linearise(int use_cr, unsigned n_poses, const double *poses, const double *u_nu_om,
                 double delta, double lambda, const double *mns,
                 const unsigned *z_step, const double *z_rb,
                 long n_obs_edges, const unsigned *pj, const unsigned *pk,
                 unsigned *t1, unsigned *t2, double *blocks);

int or_round_cost(int use_cr, unsigned n_poses, const double *poses, const double *u_nu_om,
                  double delta, double lambda, const double *mns, const unsigned *z_step,
                  const double *z_rb, long n_obs_edges, const unsigned *pj, const unsigned *pk,
                  double *edge_cost, double *total);

long or_csr_nnz(unsigned dim, long n_edges, const unsigned *t1, const unsigned *t2);
int or_csr_build(unsigned dim, long n_edges, const unsigned *t1, const unsigned *t2,
                 const double *blocks, int *row_ptr, int *col_idx, double *values, double *xi);

void or_diag_inv(unsigned dim, const int *row_ptr, const int *col_idx, const double *values,
                 double *diag_inv);
void or_spmv(unsigned dim, const int *row_ptr, const int *col_idx, const double *values,
             const double *p, double *q);
int or_pcg(unsigned dim, const int *row_ptr, const int *col_idx, const double *values,
           const double *b, double *x, double tol_rel, int max_iter, int *iters_out,
           double *rnorm_out);

int or_run(int use_cr, unsigned n_poses, double *poses, const double *u_nu_om, double delta,
           double lambda, unsigned n_z, const unsigned *z_step, const unsigned *z_lm,
           const double *z_rb, unsigned rounds, double tol_rel, int max_iter, double *diffs,
           int *pcg_iters);

int or_gj_inverse(unsigned n, const double *a, double *res);
int or_landmark_map(int use_cr, unsigned n_groups, const long *group_ptr, const unsigned *members,
                    const unsigned *z_step, const double *z_rb, const double *poses, double *ms);

int or_csr_build_anchor(unsigned dim, long n_edges, const unsigned *t1, const unsigned *t2,
                        const double *blocks, double anchor, int *row_ptr, int *col_idx,
                        double *values, double *xi);
void or_se2_edge(const double *xi, const double *xj, const double *z, const double *info,
                 double lambda, double *out, double *e_out);
int or_se2_linearise(long n_edges, const unsigned *ei, const unsigned *ej, const double *poses,
                     const double *meas, const double *info, double lambda, double *blocks,
                     double *errs);

#ifdef __cplusplus
}
#endif
#endif
