/*
 * shim_protocol.c -- the single-step binding a ForestClaw application adds
 * (INTEGRATION.md, section 1), driven from plain C against include/fc2d_b200.h.
 *
 * ForestClaw keeps each patch's q in a host FArrayBox and calls
 * patch_vt->single_step_update once per patch of a level (cb_single_step,
 * src/fclaw2d_update_single_step.c:44-70) with {total_count, iter} in its buffer
 * (:79-84).  This program plays that caller: it holds every patch in its own host
 * array (as the FArrayBoxes do), hands the patches of each level over in reverse
 * order through fc2d_b200_single_step_update_host, and checks that the arrays it gets
 * back are bit for bit what a second solver computes with its data on the device
 * (fc2d_b200_level_update), for two subcycled steps of a two-level radial dam.
 *
 * Exit status 0 on success; the first mismatch is printed.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "fc2d_b200.h"

#define CHECK(call)                                                                     \
    do {                                                                                \
        int rc_ = (call);                                                               \
        if (rc_ != FC2D_B200_OK) {                                                      \
            fprintf(stderr, "%s failed (%d): %s\n", #call, rc_, fc2d_b200_last_error()); \
            return 2;                                                                   \
        }                                                                               \
    } while (0)

static void dam_options(fc2d_b200_options_t* o)
{
    memset(o, 0, sizeof(*o));
    o->mx = 16; o->my = 16; o->mbc = 2; o->meqn = 3; o->maux = 0; o->mwaves = 3;
    o->order[0] = 2; o->order[1] = 2;
    o->mthlim[0] = o->mthlim[1] = o->mthlim[2] = 4;
    o->mthbc[0] = o->mthbc[1] = o->mthbc[2] = o->mthbc[3] = 1;
    o->rp = FC2D_B200_RP_SW_ROE;
    o->minlevel = 2; o->maxlevel = 3; o->subcycle = 1;
    o->flux_correction = 1; o->fluctuation_correction = 1;
    o->refine_threshold = 0.01; o->coarsen_threshold = 0.002;
    o->ax = -1; o->bx = 1; o->ay = -1; o->by = 1; o->mi = 1; o->mj = 1;
    o->app = FC2D_B200_APP_RADIALDAM;
    o->grav = 1.0; o->r0 = 0.3; o->hin = 2.0; o->hout = 1.0;
    o->precision = FC2D_B200_PREC_FP64;
    o->threshold_variable = 1;
    o->max_cfl = 1.0; o->desired_cfl = 0.9; o->nout = 1; o->regrid_interval = 1;
}

int main(void)
{
    fc2d_b200_options_t o;
    dam_options(&o);
    fc2d_b200_solver_t *host_side = NULL, *device_side = NULL;
    CHECK(fc2d_b200_create(&o, &host_side));
    CHECK(fc2d_b200_create(&o, &device_side));
    CHECK(fc2d_b200_initialize(host_side));
    CHECK(fc2d_b200_initialize(device_side));
    int np = 0;
    CHECK(fc2d_b200_num_patches(host_side, &np));
    int *level = malloc(sizeof(int) * np), *block = malloc(sizeof(int) * np);
    int *gx = malloc(sizeof(int) * np), *gy = malloc(sizeof(int) * np);
    CHECK(fc2d_b200_patch_info(host_side, level, block, gx, gy));
    const size_t nq = (size_t)(o.mx + 2 * o.mbc) * (o.my + 2 * o.mbc) * o.meqn;
    double* all = malloc(sizeof(double) * nq * np);
    CHECK(fc2d_b200_get_q(host_side, all));
    /* one host array per patch, like the FArrayBoxes */
    double** fab = malloc(sizeof(double*) * np);
    for (int p = 0; p < np; p++) {
        fab[p] = malloc(sizeof(double) * nq);
        memcpy(fab[p], all + (size_t)p * nq, sizeof(double) * nq);
    }
    int lmin = 99, lmax = -1;
    for (int p = 0; p < np; p++) { if (level[p] < lmin) lmin = level[p]; if (level[p] > lmax) lmax = level[p]; }
    double t = 0.0;
    const double dt = 0.004;
    for (int step = 0; step < 2; step++) {
        for (int l = lmax; l >= lmin; l--) {
            int count = 0;
            for (int p = 0; p < np; p++) count += level[p] == l;
            const double dtl = dt / (double)(1 << (l - lmin));
            int iter = 0;
            double cfl_host = 0.0, cfl_dev = 0.0;
            for (int p = np - 1; p >= 0; p--) {            /* reverse order: the library finds each slot */
                if (level[p] != l) continue;
                double cfl = -1.0;
                CHECK(fc2d_b200_single_step_update_host(host_side, l, gx[p], gy[p], fab[p], NULL, iter, count, t,
                                                        dtl, &cfl));
                if (iter + 1 < count && cfl != 0.0) { fprintf(stderr, "cfl before the launch\n"); return 1; }
                if (iter + 1 == count) cfl_host = cfl;
                iter++;
            }
            CHECK(fc2d_b200_level_update(device_side, l, t, dtl, &cfl_dev));
            if (cfl_host != cfl_dev) { fprintf(stderr, "level %d cfl %.17g vs %.17g\n", l, cfl_host, cfl_dev); return 1; }
        }
        t += dt;
    }
    CHECK(fc2d_b200_get_q(device_side, all));
    for (int p = 0; p < np; p++)
        for (size_t k = 0; k < nq; k++)
            if (fab[p][k] != all[(size_t)p * nq + k]) {
                fprintf(stderr, "patch %d cell %zu: %.17g vs %.17g\n", p, k, fab[p][k], all[(size_t)p * nq + k]);
                return 1;
            }
    printf("shim protocol ok: %d patches, levels %d-%d\n", np, lmin, lmax);
    CHECK(fc2d_b200_destroy(host_side));
    CHECK(fc2d_b200_destroy(device_side));
    return 0;
}
