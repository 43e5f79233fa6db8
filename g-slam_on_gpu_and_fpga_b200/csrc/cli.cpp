/*
 * cli.cpp — the GSLAM program: `GSLAM <use_diff> <lambda> <num_rounds> <drawing_mode> <input_file>`
 * with the reference's arguments, stdout lines and POSE_DUMP_FILE format
 * (src/cpu_pcg_fp64/GSLAM.c:13-220, README.md:53-65), running every round on the GPU.
 *
 * use_diff = 1: diff = ||dx|| / sqrt(dim), stop below 0.01 or after 20 rounds
 *               without a new best (GSLAM.c:104-130).
 * use_diff = 0: the cost criterion of GSLAM.c:74-87 and :108-136, diff =
 *               |cost - last_cost| / cost, stop below 1e-8, with the cost that code
 *               meant: computed afresh each round at the round's starting poses
 *               (gslam_cost). The reference CPU program reads a 3-vector out of a
 *               2-element array and never resets its sum; the reference GPU program
 *               (src/gpu_pcg_fp64/GSLAM.cu:165-171) uses the norm criterion instead.
 * Options beyond the reference, in the environment (defaults reproduce it):
 *   GSLAM_TOL (1e-6), GSLAM_MAXIT (500), GSLAM_PREC (fp64 | mixed), GSLAM_WRAP (0),
 *   GSLAM_STATS=1 prints one JSON line of solver statistics per round on stderr.
 * Drawing (matplotlib) is not part of this program; drawing_mode >= 1 writes the
 * pose dump when POSE_DUMP_FILE is set, as the reference CPU program does.
 */
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "gslam.h"

int main(int argc, char *argv[]) {
    if (argc == 6) {
        printf("Diff: %s ", argv[1]);
        printf("Lambda: %s ", argv[2]);
        printf("Rounds: %s ", argv[3]);
        printf("Drawing: %s ", argv[4]);
        printf("Input file: %s\n", argv[5]);
    } else {
        printf("Usage: ");
        printf("%s Diff_0|1 Lambda Number_of_rounds Drawing_0|1|2|3 path/to/input/file\n", argv[0]);
        return 1;
    }
    const unsigned use_diff = (unsigned)atoi(argv[1]);
    const double lambda = atof(argv[2]);
    const unsigned rounds = (unsigned)atoi(argv[3]);
    const unsigned draw = (unsigned)atoi(argv[4]);

    gslam_log *log = nullptr;
    if (gslam_read_log(argv[5], &log) != GSLAM_OK) {
        printf("Error! Cannot open the input file!");
        return 1;
    }
    const unsigned dim = 3 * log->n_u;
    printf("delta: %f ", log->delta);
    printf("size_of_us: %d ", log->n_u);
    printf("size_of_hat_xs: %d ", log->n_x);
    printf("size_of_zlist: %d ", log->n_z);
    printf("dim: %d\n", dim);
    fflush(stdout);
    if (log->n_x != log->n_u || log->n_x == 0) {
        fprintf(stderr, "gslam: the log needs one u and one x record per pose (got %u u, %u x)\n",
                log->n_u, log->n_x);
        return 1;
    }

    gslam_opts o;
    gslam_opts_default(&o);
    if (const char *s = getenv("GSLAM_TOL")) o.tol = atof(s);
    if (const char *s = getenv("GSLAM_MAXIT")) o.max_iter = atoi(s);
    if (const char *s = getenv("GSLAM_PREC"))
        o.precision = (strcmp(s, "mixed") == 0) ? GSLAM_PREC_MIXED
                    : (strcmp(s, "fp64cg") == 0) ? GSLAM_PREC_FP64_CG : GSLAM_PREC_FP64;
    if (const char *s = getenv("GSLAM_WRAP")) o.angle_wrap = atoi(s);
    const bool stats_json = getenv("GSLAM_STATS") && atoi(getenv("GSLAM_STATS"));

    gslam_reference_graph in;
    memset(&in, 0, sizeof in);
    in.n_poses = log->n_x;
    in.poses = log->x;
    in.controls = log->u;
    in.delta = log->delta;
    in.lambda = lambda;
    in.n_obs = log->n_z;
    in.obs_step = log->z_step;
    in.obs_landmark = log->z_lm;
    in.obs = log->z;
    gslam_graph *g = nullptr;
    int rc = gslam_create_reference(&in, &o, &g);
    if (rc != GSLAM_OK) {
        fprintf(stderr, "gslam: %s (%d)\n", gslam_last_error(), rc);
        return 1;
    }
    double best = 1e30, last_cost = 0.0;
    unsigned no_improve = 0;
    for (unsigned n = 1; n <= rounds; n++) {
        double cost = 0.0;
        if (!use_diff) rc = gslam_cost(g, &cost, nullptr);
        gslam_solve_stats st;
        if (rc == GSLAM_OK) rc = gslam_round(g, &st);
        if (rc != GSLAM_OK) {
            fprintf(stderr, "gslam: %s (%d)\n", gslam_last_error(), rc);
            gslam_destroy(g);
            return 1;
        }
        const double diff = use_diff ? st.diff : fabs(cost - last_cost) / cost;
        printf("%d rounds executed: %.17g\n", n, diff);
        if (stats_json)
            fprintf(stderr,
                    "{\"round\": %u, \"pcg_iterations\": %d, \"refinements\": %d, \"reason\": %d, "
                    "\"rel_residual\": %.6e, \"diff\": %.17g, \"update_norm\": %.17g}\n",
                    n, st.iterations, st.refinements, st.reason, st.rel_residual, diff, st.diff);
        if (use_diff) {
            if (diff < 0.01) break;
            if (diff < best) { best = diff; no_improve = 0; }
            else if (++no_improve >= 20) break;
        } else {
            if (diff < 1e-8) break;
            last_cost = cost;
        }
    }
    if (draw >= 1) {
        const char *dump = getenv("POSE_DUMP_FILE");
        if (dump) {
            std::vector<double> poses(3 * (size_t)log->n_x);
            gslam_get_poses(g, poses.data());
            FILE *df = fopen(dump, "w");
            if (df) {
                for (unsigned i = 0; i < log->n_x; i++)
                    fprintf(df, "%u %.17g %.17g %.17g\n", log->x_step[i], poses[3 * i], poses[3 * i + 1],
                            poses[3 * i + 2]);
                fclose(df);
            }
        }
    }
    gslam_destroy(g);
    gslam_free_log(log);
    return 0;
}
