/*
 * logio.cpp — the reference's log format (read_data, src/cpu_pcg_fp64/GSLAM.c:415-493).
 * Tokens are split on single spaces like strtok(line, " "); numbers are parsed
 * with atoi / atof exactly as the reference does, so every value is the same
 * double. Unlike the reference there are no fixed capacities (131,072 poses,
 * 524,288 observations: GSLAM.c:39-41), empty lines are skipped, and a truncated
 * record is an error instead of a NULL dereference.
 */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "gslam.h"
#include "gslam_api_internal.h"

int gslam_read_log(const char *path, gslam_log **out) {
    if (!path || !out) return GSLAM_ERR_BAD_INPUT;
    *out = nullptr;
    FILE *f = fopen(path, "r");
    if (!f) {
        gslam_set_last_error("Error! Cannot open the input file!");
        return GSLAM_ERR_BAD_INPUT;
    }
    std::vector<uint32_t> us, xs, zs, zl;
    std::vector<double> u, x, z;
    double delta = 0.0;
    char line[1024];
    int rc = GSLAM_OK;
    while (fgets(line, sizeof line, f)) {
        char *save = nullptr;
        char *tok = strtok_r(line, " ", &save);
        if (!tok || tok[0] == '\n' || tok[0] == '\r') continue;
        char *t[4] = { nullptr, nullptr, nullptr, nullptr };
        if (strcmp(tok, "u") == 0) {
            for (int i = 0; i < 3; i++) t[i] = strtok_r(nullptr, " ", &save);
            if (!t[0] || !t[1] || !t[2]) { rc = GSLAM_ERR_BAD_INPUT; break; }
            us.push_back((uint32_t)atoi(t[0]));
            u.push_back(atof(t[1]));
            u.push_back(atof(t[2]));
        } else if (strcmp(tok, "x") == 0) {
            for (int i = 0; i < 4; i++) t[i] = strtok_r(nullptr, " ", &save);
            if (!t[0] || !t[1] || !t[2] || !t[3]) { rc = GSLAM_ERR_BAD_INPUT; break; }
            xs.push_back((uint32_t)atoi(t[0]));
            for (int i = 1; i < 4; i++) x.push_back(atof(t[i]));
        } else if (strcmp(tok, "z") == 0) {
            for (int i = 0; i < 4; i++) t[i] = strtok_r(nullptr, " ", &save);
            if (!t[0] || !t[1] || !t[2] || !t[3]) { rc = GSLAM_ERR_BAD_INPUT; break; }
            zs.push_back((uint32_t)atoi(t[0]));
            zl.push_back((uint32_t)atoi(t[1]));
            z.push_back(atof(t[2]));
            z.push_back(atof(t[3]));
        } else {
            char *a = strtok_r(nullptr, " ", &save);
            if (a) delta = atof(a);
        }
    }
    fclose(f);
    if (rc != GSLAM_OK) {
        gslam_set_last_error("truncated record in the input file");
        return rc;
    }
    gslam_log *L = (gslam_log *)calloc(1, sizeof(gslam_log));
    L->delta = delta;
    L->n_u = (uint32_t)us.size();
    L->n_x = (uint32_t)xs.size();
    L->n_z = (uint32_t)zs.size();
    auto dupu = [](const std::vector<uint32_t> &v) {
        uint32_t *p = (uint32_t *)malloc((v.size() ? v.size() : 1) * sizeof(uint32_t));
        if (!v.empty()) memcpy(p, v.data(), v.size() * sizeof(uint32_t));
        return p;
    };
    auto dupd = [](const std::vector<double> &v) {
        double *p = (double *)malloc((v.size() ? v.size() : 1) * sizeof(double));
        if (!v.empty()) memcpy(p, v.data(), v.size() * sizeof(double));
        return p;
    };
    L->u_step = dupu(us); L->u = dupd(u);
    L->x_step = dupu(xs); L->x = dupd(x);
    L->z_step = dupu(zs); L->z_lm = dupu(zl); L->z = dupd(z);
    *out = L;
    return GSLAM_OK;
}

void gslam_free_log(gslam_log *L) {
    if (!L) return;
    free(L->u_step); free(L->u); free(L->x_step); free(L->x);
    free(L->z_step); free(L->z_lm); free(L->z);
    free(L);
}
