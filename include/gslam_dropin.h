/*
 * gslam_dropin.h — the reference's own solver entry points, served by libgslam.
 *
 * A program written against isaacyhe/G-SLAM_on_GPU_and_FPGA links against
 * libgslam.so instead of its own MatrixOps.c / device_graph.cu and keeps its
 * main loop. The record layouts below are byte-compatible with the reference's
 * structs (src/cpu_pcg_fp64/Z.h:4-8, U.h:4-8, HAT_X.h:4-7, MatrixOps.h:21-27);
 * define GSLAM_DROPIN_HAVE_REFERENCE_TYPES when the reference headers already
 * declared them.
 *
 * Behaviour follows the reference: the functions return void and, like its
 * cuda_check (src/gpu_pcg_fp64/device_graph.cu:99-106), print the error and
 * exit(1) on failure. Setting GSLAM_DROPIN_NOEXIT=1 in the environment records
 * the failure instead (gslam_dropin_status() / gslam_last_error()) and returns.
 */
#ifndef GSLAM_DROPIN_H
#define GSLAM_DROPIN_H

#ifdef __cplusplus
extern "C" {
#endif

#ifndef GSLAM_DROPIN_HAVE_REFERENCE_TYPES
struct Z {
    unsigned int step;
    unsigned int landmark_id;
    double z[2];
};
struct U {
    unsigned int step;
    double nu;
    double omega;
};
struct HAT_X {
    unsigned int step;
    double hat_x[3];
};
typedef struct {
    int *row_ptr;
    int *col_idx;
    double *values;
    int dim;
    int nnz;
} CSRMatrix;
#endif

/*
 * Replaces pcg_solve_sparse (src/cpu_pcg_fp64/MatrixOps.h:37, MatrixOps.c:281-391):
 * solves csr * x = b with block-Jacobi PCG, x zeroed first, ||r|| < 1e-6 ||b|| or
 * 500 iterations, on the GPU. The CSR's 3x3 block pattern is analysed on the
 * first call and reused while row_ptr / col_idx stay the same.
 */
void pcg_solve_sparse(double *x, CSRMatrix *csr, double *b, unsigned int dim);

/* Replaces device_graph_init (src/gpu_pcg_fp64/device_graph.cuh:23-33). */
void device_graph_init(struct Z *zlist, unsigned int n_obs, struct U *us, unsigned int n_poses,
                       unsigned int dim, double delta, double lambda, const double *mns,
                       int *nnz_out);
/* Replaces device_graph_update (device_graph.cuh:47-52): writes Omega (CSR values) and xi. */
void device_graph_update(struct HAT_X *hat_xs, unsigned int n_poses, double *d_csr_vals,
                         double *d_xi);
/* Replace device_graph_get_row_ptr / _col_idx (device_graph.cuh:59-60): device CSR pattern. */
int *device_graph_get_row_ptr(void);
int *device_graph_get_col_idx(void);
/* Replaces device_build_diag_inv (device_graph.cuh:69; a no-op there as here). */
void device_build_diag_inv(int dim);
/* Replaces device_pcg_solve (device_graph.cuh:83-84): solves from d_csr_vals / d_xi into x_h. */
void device_pcg_solve(double *x_h, double *d_csr_vals, double *d_xi, int dim, int nnz,
                      int max_iter);
/* Replaces device_graph_free (device_graph.cuh:91). */
void device_graph_free(void);

/* Status of the last drop-in call (GSLAM_OK or a GSLAM_ERR_* of gslam.h); no reference counterpart. */
int gslam_dropin_status(void);

#ifdef __cplusplus
}
#endif
#endif
