/*
 * orc_amr.c -- oracle restatement of ForestClaw's forest-level orchestration
 * (test infrastructure; see oracle.h for the parity status).
 *
 *   level stepping + subcycling    src/fclaw2d_advance.c:54-357
 *   single-step level update       src/fclaw2d_update_single_step.c:44-103,
 *                                  src/solvers/fc2d_clawpack4.6/fc2d_clawpack46.cpp:259-444
 *   ghost update (one process)     src/fclaw2d_ghost_fill.c:611-830
 *   face / corner fill callbacks   src/fclaw2d_face_neighbors.c:195-450, src/fclaw2d_corner_neighbors.c:301-535
 *   physical BC                    src/fclaw2d_physical_bc.c:46-76, fc2d_clawpack46.cpp:94-146
 *   time interpolation             src/fclaw2d_timeinterp.c:29-57, clawpatch.cpp:474-526
 *   time sync                      src/fclaw2d_time_sync.c:66-202, clawpatch_conservation.c:207-280
 *   regrid / initial refinement    src/fclaw2d_regrid.c:44-335, src/fclaw2d_initialize.c:150-230
 *   neighbour relations            src/fclaw2d_patch.c:980-1034, src/fclaw2d_regrid.c:337-400
 *
 * The forest itself (p4est's role: leaves, face/corner neighbours, 2:1 face+corner
 * balance) is a brute-force quadtree over a brick of equally oriented blocks; the
 * p4est semantics it restates are listed beside each function.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "orc_amr.h"

#define MAXL 24

/* ------------------------------------------------------------------------- */
/* hashing of (level, gx, gy)                                                  */
/* ------------------------------------------------------------------------- */
static long long hkey(int l, int x, int y) { return ((long long)l << 56) | ((long long)x << 28) | (long long)y; }

static void hash_build(orc_sim* s)
{
    free(s->hkey); free(s->hval);
    s->hcap = 16;
    while (s->hcap < 4 * s->np + 16) s->hcap <<= 1;
    s->hkey = (long long*)malloc(sizeof(long long) * s->hcap);
    s->hval = (int*)malloc(sizeof(int) * s->hcap);
    for (int k = 0; k < s->hcap; k++) s->hkey[k] = -1;
    for (int i = 0; i < s->np; i++) {
        long long k = hkey(s->p[i].level, s->p[i].gx, s->p[i].gy);
        unsigned long long h = (unsigned long long)k * 0x9E3779B97F4A7C15ull;
        int pos = (int)(h >> 40) & (s->hcap - 1);
        while (s->hkey[pos] != -1) pos = (pos + 1) & (s->hcap - 1);
        s->hkey[pos] = k; s->hval[pos] = i;
    }
}

static int lookup(const orc_sim* s, int l, int x, int y)
{
    if (l < 0 || x < 0 || y < 0) return -1;
    if (x >= s->cfg.mi << l || y >= s->cfg.mj << l) return -1;
    long long k = hkey(l, x, y);
    unsigned long long h = (unsigned long long)k * 0x9E3779B97F4A7C15ull;
    int pos = (int)(h >> 40) & (s->hcap - 1);
    while (s->hkey[pos] != -1) {
        if (s->hkey[pos] == k) return s->hval[pos];
        pos = (pos + 1) & (s->hcap - 1);
    }
    return -1;
}

static unsigned long long interleave(unsigned x, unsigned y)
{
    unsigned long long r = 0;
    for (int b = 0; b < 32; b++) {
        r |= (unsigned long long)((x >> b) & 1u) << (2 * b);
        r |= (unsigned long long)((y >> b) & 1u) << (2 * b + 1);
    }
    return r;
}

/* p4est brick tree numbering: Morton order of the block positions. */
static int brick_block(const orc_config* c, int bx, int by)
{
    unsigned long long key = interleave((unsigned)bx, (unsigned)by);
    int rank = 0;
    for (int j = 0; j < c->mj; j++)
        for (int i = 0; i < c->mi; i++)
            if (interleave((unsigned)i, (unsigned)j) < key) rank++;
    return rank;
}

/* ------------------------------------------------------------------------- */
/* patch memory                                                                */
/* ------------------------------------------------------------------------- */
static void patch_alloc(orc_sim* s, orc_patch* P)
{
    const orc_config* c = &s->cfg;
    P->q = (double*)calloc(s->nq, sizeof(double));
    P->qlast = (double*)calloc(s->nq, sizeof(double));
    P->qinterp = c->subcycle ? (double*)calloc(s->nq, sizeof(double)) : NULL;
    P->aux = c->maux > 0 ? (double*)calloc(s->naux, sizeof(double)) : NULL;
    P->area = c->problem == ORC_PROB_SPHERE
                  ? (double*)calloc((size_t)(c->mx + 2 * c->mbc + 2) * (c->my + 2 * c->mbc + 2), sizeof(double))
                  : NULL;
    const int mx = c->mx, my = c->my, meqn = c->meqn;
    size_t n = 0;
    n += 2 * (size_t)my * meqn * 2 + 2 * (size_t)mx * meqn * 2;   /* fp fm gp gm */
    n += 2 * 2 * (size_t)my * meqn + 2 * 2 * (size_t)mx * meqn;   /* ef */
    n += 2 * (size_t)(my + mx) * 2;                                 /* el, area */
    double* m = (double*)calloc(n, sizeof(double));
    orc_regs* r = &P->regs;
    r->mem = m;
    for (int k = 0; k < 2; k++) { r->fp[k] = m; m += my * meqn; r->fm[k] = m; m += my * meqn; }
    for (int k = 0; k < 2; k++) { r->gp[k] = m; m += mx * meqn; r->gm[k] = m; m += mx * meqn; }
    r->ef[0] = m; m += 2 * my * meqn; r->ef[1] = m; m += 2 * my * meqn;
    r->ef[2] = m; m += 2 * mx * meqn; r->ef[3] = m; m += 2 * mx * meqn;
    r->el[0] = m; m += my; r->el[1] = m; m += my; r->el[2] = m; m += mx; r->el[3] = m; m += mx;
    r->area[0] = m; m += my; r->area[1] = m; m += my; r->area[2] = m; m += mx; r->area[3] = m; m += mx;
}

static void patch_free(orc_patch* P)
{
    free(P->q); free(P->qlast); free(P->qinterp); free(P->aux); free(P->regs.mem); free(P->area); free(P->qsave);
    P->q = P->qlast = P->qinterp = P->aux = P->area = P->qsave = NULL; P->regs.mem = NULL;
}

/* clawpatch_define (fclaw2d_clawpatch.cpp:192-...) geometry + time_sync_setup
 * (fclaw2d_clawpatch_utils.f:259-314, non-manifold branch). */
static void patch_geometry(orc_sim* s, orc_patch* P)
{
    const orc_config* c = &s->cfg;
    int l = P->level;
    int bx = P->gx >> l, by = P->gy >> l;
    int ix = P->gx - (bx << l), iy = P->gy - (by << l);
    double w = 1.0 / (double)(1 << l);
    double xl = ix * w, yl = iy * w, xu = (ix + 1) * w, yu = (iy + 1) * w;
    double xlo, ylo, xup, yup;
    const int sphere = c->problem == ORC_PROB_SPHERE;   /* six blocks [0,1]^2, gx = block 2^l + ix */
    if ((c->mi == 1 && c->mj == 1) || sphere) { xlo = xl; ylo = yl; xup = xu; yup = yu; }
    else {
        xlo = (double)(bx + xl) / c->mi; xup = (double)(bx + xu) / c->mi;
        ylo = (double)(by + yl) / c->mj; yup = (double)(by + yu) / c->mj;
    }
    P->block = sphere ? bx : brick_block(c, bx, by);
    P->xlower = c->ax + (c->bx - c->ax) * xlo;
    double xupper = c->ax + (c->bx - c->ax) * xup;
    P->ylower = c->ay + (c->by - c->ay) * ylo;
    double yupper = c->ay + (c->by - c->ay) * yup;
    P->dx = (xupper - P->xlower) / c->mx;
    P->dy = (yupper - P->ylower) / c->my;
    double dxdy = P->dx * P->dy;
    for (int j = 0; j < c->my; j++) {
        P->regs.area[0][j] = dxdy; P->regs.area[1][j] = dxdy;
        P->regs.el[0][j] = P->dy; P->regs.el[1][j] = P->dy;
    }
    for (int i = 0; i < c->mx; i++) {
        P->regs.area[2][i] = dxdy; P->regs.area[3][i] = dxdy;
        P->regs.el[2][i] = P->dx; P->regs.el[3][i] = P->dx;
    }
    unsigned sh = (unsigned)(MAXL - l);
    P->morton = interleave((unsigned)ix << sh, (unsigned)iy << sh);
}

static int cmp_p4est(const void* a, const void* b)
{
    const orc_patch* A = (const orc_patch*)a;
    const orc_patch* B = (const orc_patch*)b;
    if (A->block != B->block) return A->block < B->block ? -1 : 1;
    if (A->morton != B->morton) return A->morton < B->morton ? -1 : 1;
    return 0;
}

/* ------------------------------------------------------------------------- */
/* neighbour relations (p4est face/corner neighbour semantics on a balanced   */
/* forest; fclaw2d_regrid.c:337-400, fclaw2d_patch.c:980-1034)                */
/* ------------------------------------------------------------------------- */
static const int FDX[4] = {-1, 1, 0, 0}, FDY[4] = {0, 0, -1, 1};

static void set_neighbors(orc_sim* s)
{
    for (int ip = 0; ip < s->np; ip++) {
        orc_patch* P = &s->p[ip];
        int l = P->level;
        P->has_fine_nbr = 0; P->on_cf = 0;
        for (int f = 0; f < 4; f++) {
            int nx, ny;
            P->face_nbr[f][0] = P->face_nbr[f][1] = -1;
            P->phys[f] = orc_step(s, l, P->gx, P->gy, FDX[f], FDY[f], &nx, &ny) != 1;
            if (P->phys[f]) { P->face_type[f] = NB_BOUNDARY; continue; }
            int k = lookup(s, l, nx, ny);
            if (k >= 0) { P->face_type[f] = NB_SAME; P->face_nbr[f][0] = k; continue; }
            k = lookup(s, l - 1, nx >> 1, ny >> 1);
            if (k >= 0) { P->face_type[f] = NB_DOUBLE; P->face_nbr[f][0] = k; P->on_cf = 1; continue; }
            /* the two half-size leaves: our children along face f, one step across it */
            int c0x, c0y, c1x, c1y;
            {
                int ax = 2 * P->gx + (f == 1), ay = 2 * P->gy + (f == 3);
                int bx2 = ax + (f >= 2), by2 = ay + (f < 2);
                orc_step(s, l + 1, ax, ay, FDX[f], FDY[f], &c0x, &c0y);
                orc_step(s, l + 1, bx2, by2, FDX[f], FDY[f], &c1x, &c1y);
            }
            int a = lookup(s, l + 1, c0x, c0y), b = lookup(s, l + 1, c1x, c1y);
            if (a < 0 || b < 0) { fprintf(stderr, "oracle: unbalanced forest at face\n"); abort(); }
            P->face_type[f] = NB_HALF; P->face_nbr[f][0] = a; P->face_nbr[f][1] = b;
            P->has_fine_nbr = 1; P->on_cf = 1;
        }
        for (int c = 0; c < 4; c++) {
            int f0 = (c & 1) ? 1 : 0, f1 = (c & 2) ? 3 : 2;
            P->has_corner[c] = 0; P->corner_nbr[c] = -1; P->corner_type[c] = NB_BOUNDARY;
            P->bcc[c] = 0;
            if (P->phys[f0] || P->phys[f1]) continue;
            int dx = (c & 1) ? 1 : -1, dy = (c & 2) ? 1 : -1;
            int nx, ny;
            if (orc_step(s, l, P->gx, P->gy, dx, dy, &nx, &ny) < 0) {
                /* cube corner: three blocks meet, no corner neighbour (corner_neighbors.c case 4) */
                P->bcc[c] = 3;
                continue;
            }
            int k = lookup(s, l, nx, ny);
            if (k >= 0) { P->has_corner[c] = 1; P->corner_type[c] = NB_SAME; P->corner_nbr[c] = k; continue; }
            {
                int fx, fy;
                orc_step(s, l + 1, 2 * P->gx + (dx > 0), 2 * P->gy + (dy > 0), dx, dy, &fx, &fy);
                k = lookup(s, l + 1, fx, fy);
            }
            if (k >= 0) {
                P->has_corner[c] = 1; P->corner_type[c] = NB_HALF; P->corner_nbr[c] = k;
                P->has_fine_nbr = 1; P->on_cf = 1; continue;
            }
            k = lookup(s, l - 1, nx >> 1, ny >> 1);
            int cx = P->gx + (c & 1), cy = P->gy + (c >> 1);
            if (k >= 0 && (cx % 2) == 0 && (cy % 2) == 0) {
                P->has_corner[c] = 1; P->corner_type[c] = NB_DOUBLE; P->corner_nbr[c] = k; P->on_cf = 1;
            }
        }
    }
}

/* Rebuild the derived tables after the patch array changed. */
static void forest_finalize(orc_sim* s)
{
    qsort(s->p, (size_t)s->np, sizeof(orc_patch), cmp_p4est);
    hash_build(s);
    set_neighbors(s);
    free(s->lev_list);
    s->lev_list = (int*)malloc(sizeof(int) * (s->np + 1));
    int n = 0;
    s->minlevel_present = 99; s->maxlevel_present = -1;
    for (int l = 0; l < 31; l++) {
        s->lev_start[l] = n;
        for (int i = 0; i < s->np; i++)
            if (s->p[i].level == l) {
                s->lev_list[n++] = i;
                if (l < s->minlevel_present) s->minlevel_present = l;
                if (l > s->maxlevel_present) s->maxlevel_present = l;
            }
    }
    s->lev_start[31] = n;
}

#define FOR_LEVEL(s, l, idx) for (int _k = (l) >= 0 && (l) < 31 ? (s)->lev_start[l] : 0, \
    _e = (l) >= 0 && (l) < 31 ? (s)->lev_start[(l) + 1] : 0, idx; _k < _e && ((idx = (s)->lev_list[_k]), 1); _k++)

/* ------------------------------------------------------------------------- */
/* ghost update                                                                */
/* ------------------------------------------------------------------------- */
static double* tsdata(orc_patch* P, int time_interp) { return time_interp ? P->qinterp : P->q; }

static void copy2ghost(orc_sim* s, int level, int time_interp)
{
    FOR_LEVEL(s, level, ip) {
        orc_patch* P = &s->p[ip];
        for (int f = 0; f < 4; f++)
            if (P->face_type[f] == NB_SAME) {
                orc_patch* N = &s->p[P->face_nbr[f][0]];
                orc_copy_face(s, tsdata(P, time_interp), tsdata(N, time_interp), P, N, f);
            }
    }
    FOR_LEVEL(s, level, ip) {
        orc_patch* P = &s->p[ip];
        for (int c = 0; c < 4; c++)
            if (P->has_corner[c] && P->corner_type[c] == NB_SAME) {
                orc_patch* N = &s->p[P->corner_nbr[c]];
                orc_copy_corner(s, tsdata(P, time_interp), tsdata(N, time_interp), P, N, c);
            }
    }
}

static void average2ghost(orc_sim* s, int level, int time_interp)
{
    FOR_LEVEL(s, level, ip) {
        orc_patch* P = &s->p[ip];
        if (!P->on_cf) continue;
        for (int f = 0; f < 4; f++)
            if (P->face_type[f] == NB_HALF)
                for (int ig = 0; ig < 2; ig++) {
                    orc_patch* F = &s->p[P->face_nbr[f][ig]];
                    orc_average_face(s, tsdata(P, time_interp), F->q, P, F, f);
                }
    }
    FOR_LEVEL(s, level, ip) {
        orc_patch* P = &s->p[ip];
        if (!P->on_cf) continue;
        for (int c = 0; c < 4; c++)
            if (P->has_corner[c] && P->corner_type[c] == NB_HALF) {
                orc_patch* F = &s->p[P->corner_nbr[c]];
                orc_average_corner(s, tsdata(P, time_interp), F->q, P, F, c);
            }
    }
}

static void interpolate2ghost(orc_sim* s, int level, int time_interp)
{
    FOR_LEVEL(s, level, ip) {
        orc_patch* P = &s->p[ip];
        if (!P->on_cf) continue;
        for (int f = 0; f < 4; f++)
            if (P->face_type[f] == NB_HALF)
                for (int ig = 0; ig < 2; ig++) {
                    orc_patch* F = &s->p[P->face_nbr[f][ig]];
                    orc_interpolate_face(s, tsdata(P, time_interp), F->q, P, F, f);
                }
    }
    FOR_LEVEL(s, level, ip) {
        orc_patch* P = &s->p[ip];
        if (!P->on_cf) continue;
        for (int c = 0; c < 4; c++)
            if (P->has_corner[c] && P->corner_type[c] == NB_HALF) {
                orc_patch* F = &s->p[P->corner_nbr[c]];
                orc_interpolate_corner(s, tsdata(P, time_interp), F->q, P, F, c);
            }
    }
}

static void setphysical(orc_sim* s, int level, int time_interp)
{
    FOR_LEVEL(s, level, ip) {
        orc_patch* P = &s->p[ip];
        int mthbc[4], any = 0;
        for (int f = 0; f < 4; f++) { mthbc[f] = P->phys[f] ? s->cfg.mthbc[f] : -1; any |= P->phys[f]; }
        if (!any) continue;
        orc_bc2(s->cfg.mx, s->cfg.my, s->cfg.mbc, s->cfg.meqn, tsdata(P, time_interp), mthbc,
                s->cfg.problem == ORC_PROB_SHOCKBUBBLE ? s->inflow : NULL);
    }
}

/* fclaw2d_ghost_update_async with one process (every patch is interior to the
 * partition): the step-2 and final-physical stages, in order. */
static void ghost_update(orc_sim* s, int minlevel, int maxlevel, int time_interp)
{
    int mincoarse = minlevel, maxcoarse = maxlevel - 1;
    /* average_fine2coarse_ghost */
    for (int l = maxcoarse; l >= mincoarse; l--) average2ghost(s, l, 0);
    if (time_interp) average2ghost(s, mincoarse - 1, 1);
    /* copy_samelevel */
    for (int l = maxlevel; l >= minlevel; l--) copy2ghost(s, l, 0);
    if (time_interp) copy2ghost(s, minlevel - 1, 1);
    /* fill_physical_ghost(mincoarse, maxcoarse) */
    for (int l = maxcoarse; l >= mincoarse; l--) setphysical(s, l, 0);
    if (time_interp) setphysical(s, mincoarse - 1, 1);
    /* interpolate_coarse2fine_ghost */
    for (int l = maxcoarse; l >= mincoarse; l--) interpolate2ghost(s, l, 0);
    if (time_interp) interpolate2ghost(s, mincoarse - 1, 1);
    /* fill_physical_ghost(minfine, maxfine) */
    int minfine = mincoarse + 1, maxfine = maxlevel;
    for (int l = maxfine; l >= minfine; l--) setphysical(s, l, 0);
    if (time_interp) setphysical(s, minfine - 1, 1);
    /* fill_physical_ghost(minlevel, maxlevel), BOUNDARY_ALL */
    for (int l = maxlevel; l >= minlevel; l--) setphysical(s, l, 0);
    if (time_interp) setphysical(s, minlevel - 1, 1);
}

void orc_ghost_update_all(orc_sim* s, double t)
{
    (void)t;
    ghost_update(s, s->minlevel_present, s->maxlevel_present, 0);
}

/* ------------------------------------------------------------------------- */
/* time sync                                                                   */
/* ------------------------------------------------------------------------- */
enum { RESET_F2C = 1, RESET_SAMESIZE = 2, RESET_PHYS = 3 };

static void time_sync_reset(orc_sim* s, int coarse_level, int mode)
{
    int fine_level = coarse_level + 1;
    int nlev = (mode == RESET_F2C) ? 2 : 1;
    for (int pass = 0; pass < nlev; pass++) {
        int lev = coarse_level + pass;
        FOR_LEVEL(s, lev, ip) {
            orc_patch* P = &s->p[ip];
            for (int k = 0; k < 4; k++) {
                int reset = 0;
                if (mode == RESET_F2C)
                    reset = (P->face_type[k] == NB_HALF && P->level == coarse_level) ||
                            (P->face_type[k] == NB_DOUBLE && P->level == fine_level);
                else if (mode == RESET_SAMESIZE)
                    reset = (P->face_type[k] == NB_SAME && P->level == coarse_level);
                else
                    reset = (P->face_type[k] == NB_BOUNDARY);
                if (reset) orc_regs_reset_face(s, P, k);
            }
        }
    }
}

static void time_sync(orc_sim* s, int minlevel, int maxlevel)
{
    (void)maxlevel;
    const int maxl = s->cfg.maxlevel;
    for (int level = maxl; level >= minlevel; level--) {
        FOR_LEVEL(s, level, ip) {
            orc_patch* P = &s->p[ip];
            for (int f = 0; f < 4; f++)
                if (P->face_type[f] == NB_SAME)
                    orc_time_sync_samesize(s, P, &s->p[P->face_nbr[f][0]], f);
        }
        time_sync_reset(s, level, RESET_SAMESIZE);
        if (level < maxl) {
            FOR_LEVEL(s, level, ip) {
                orc_patch* P = &s->p[ip];
                for (int f = 0; f < 4; f++)
                    if (P->face_type[f] == NB_HALF)
                        for (int ig = 0; ig < 2; ig++)
                            orc_time_sync_f2c(s, P, &s->p[P->face_nbr[f][ig]], f);
            }
            time_sync_reset(s, level, RESET_F2C);
        }
    }
    for (int level = maxl; level >= minlevel; level--) time_sync_reset(s, level, RESET_PHYS);
}

/* ------------------------------------------------------------------------- */
/* level update                                                                */
/* ------------------------------------------------------------------------- */
static double update_level(orc_sim* s, int level, double t, double dt)
{
    const orc_config* c = &s->cfg;
    orc_rpn2_t rpn2; orc_rpt2_t rpt2;
    orc_rp_select(c->rp, &rpn2, &rpt2);
    const int n0 = s->lev_start[level], n1 = s->lev_start[level + 1];
    double maxcfl = 0.0;
    const size_t wsz = orc_ws_size(c->mx, c->my, c->mbc, c->meqn, c->maux, c->mwaves);
#pragma omp parallel num_threads(s->nthreads) reduction(max : maxcfl)
    {
        double* work = (double*)calloc(wsz, sizeof(double));
        double* fl = (double*)calloc(4 * s->nq, sizeof(double));
        double *fm = fl, *fp = fl + s->nq, *gm = fl + 2 * s->nq, *gp = fl + 3 * s->nq;
#pragma omp for schedule(static)
        for (int k = n0; k < n1; k++) {
            orc_patch* P = &s->p[s->lev_list[k]];
            orc_b4step2(s, P, t, dt);
            memcpy(P->qlast, P->q, s->nq * sizeof(double));
            if (c->time_sync && c->flux_correction) orc_store_flux(s, P, dt);
            double cfl = orc_step2(c, rpn2, rpt2, work, P->q, P->aux, P->dx, P->dy, dt, fm, fp, gm, gp, P->bcc);
            if (c->time_sync && c->fluctuation_correction)
                orc_accumulate_waves(s, P, dt, P->dx, P->dy, fp, fm, gp, gm);
            if (c->src_kind == 1) {
                /* src2 (clawpack46_update, fc2d_clawpack46.cpp:436-441): linear damping of field 1 */
                const size_t ncell = (size_t)s->nx * s->ny;
                for (size_t k = 0; k < ncell; k++) P->q[k] = P->q[k] - dt * c->src_rate * P->q[k];
            }
            if (cfl > maxcfl) maxcfl = cfl;
        }
        free(work); free(fl);
    }
    s->cell_updates += (double)(n1 - n0) * c->mx * c->my;
    return maxcfl;
}

static void timeinterp_level_data(orc_sim* s, int level, double alpha)
{
    FOR_LEVEL(s, level, ip) {
        orc_patch* P = &s->p[ip];
        if (P->has_fine_nbr) orc_timeinterp(s, P->q, P->qlast, P->qinterp, alpha);
    }
}

/* ------------------------------------------------------------------------- */
/* fclaw2d_advance_all_levels                                                  */
/* ------------------------------------------------------------------------- */
typedef struct { int last_step, step_inc, total_steps; double current_time, dt_step; } tsc_t;

static double advance_level(orc_sim* s, tsc_t* ts, int level, int curr_fine_step, double maxcfl)
{
    double cfl = update_level(s, level, ts[level].current_time, ts[level].dt_step);
    maxcfl = fmax(maxcfl, cfl);
    ts[level].last_step += ts[level].step_inc;
    ts[level].current_time += ts[level].dt_step;
    if (level > s->minlevel_present) {
        int last_coarse_step = ts[level - 1].last_step;
        if (last_coarse_step == curr_fine_step) {
            double c2 = advance_level(s, ts, level - 1, last_coarse_step, maxcfl);
            maxcfl = fmax(maxcfl, c2);
            if (s->cfg.subcycle) {
                int coarse_inc = ts[level - 1].step_inc;
                int new_curr_step = ts[level].last_step;
                double alpha = ((double)(new_curr_step % coarse_inc)) / coarse_inc;
                timeinterp_level_data(s, level - 1, alpha);
            }
        }
    }
    return maxcfl;
}

double orc_advance(orc_sim* s, double t, double dt)
{
    const orc_config* c = &s->cfg;
    tsc_t ts[32];
    memset(ts, 0, sizeof(ts));
    for (int l = c->minlevel; l <= c->maxlevel; l++) { ts[l].last_step = 0; ts[l].current_time = t; }
    if (c->subcycle) {
        double dt_level = dt;
        int steps_inc = 1 << (s->maxlevel_present - c->minlevel);
        int total = 1;
        for (int l = c->minlevel; l <= c->maxlevel; l++) {
            ts[l].dt_step = dt_level; ts[l].total_steps = total; ts[l].step_inc = steps_inc;
            dt_level /= 2; steps_inc /= 2; total *= 2;
        }
    } else {
        int rf = 1 << (c->maxlevel - c->minlevel);
        for (int l = c->minlevel; l <= c->maxlevel; l++) {
            ts[l].step_inc = 1; ts[l].dt_step = dt / rf; ts[l].total_steps = rf;
        }
    }
    const int minlevel = s->minlevel_present, maxlevel = s->maxlevel_present;
    double maxcfl = 0;
    int nfine = ts[maxlevel].total_steps;
    for (int nf = 0; nf < nfine; nf++) {
        double cfl = advance_level(s, ts, maxlevel, nf, maxcfl);
        maxcfl = fmax(cfl, maxcfl);
        if (ts[maxlevel].last_step < ts[maxlevel].total_steps) {
            if (c->subcycle) {
                int ti = maxlevel - 1;
                while (ts[maxlevel].last_step % ts[ti].step_inc == 0) ti--;
                ghost_update(s, ti + 1, maxlevel, 1);
                if (c->time_sync) time_sync(s, ti + 1, maxlevel);
            } else {
                ghost_update(s, minlevel, maxlevel, 0);
                if (c->time_sync) time_sync(s, minlevel, maxlevel);
            }
        }
    }
    ghost_update(s, minlevel, maxlevel, 0);
    if (c->time_sync) time_sync(s, minlevel, maxlevel);
    s->t_curr = t + dt;
    return maxcfl;
}

/* ------------------------------------------------------------------------- */
/* forest adaptation (p4est_wrap adapt: refine marked, coarsen fully-marked   */
/* families, 2:1 face+corner balance) and repopulation                        */
/* ------------------------------------------------------------------------- */
typedef struct { int level, gx, gy; } leaf_t;

static int leaf_find(const leaf_t* L, int n, int l, int x, int y)
{
    for (int i = 0; i < n; i++) if (L[i].level == l && L[i].gx == x && L[i].gy == y) return i;
    return -1;
}

/* Hash set over a leaf list. */
typedef struct { int cap; long long* key; } lset_t;
static void lset_init(lset_t* h, const leaf_t* L, int n)
{
    h->cap = 16; while (h->cap < 4 * n + 16) h->cap <<= 1;
    h->key = (long long*)malloc(sizeof(long long) * h->cap);
    for (int k = 0; k < h->cap; k++) h->key[k] = -1;
    for (int i = 0; i < n; i++) {
        long long k = hkey(L[i].level, L[i].gx, L[i].gy);
        unsigned long long hh = (unsigned long long)k * 0x9E3779B97F4A7C15ull;
        int pos = (int)(hh >> 40) & (h->cap - 1);
        while (h->key[pos] != -1 && h->key[pos] != k) pos = (pos + 1) & (h->cap - 1);
        h->key[pos] = k;
    }
}
static int lset_has(const lset_t* h, int l, int x, int y)
{
    if (l < 0 || x < 0 || y < 0) return 0;
    long long k = hkey(l, x, y);
    unsigned long long hh = (unsigned long long)k * 0x9E3779B97F4A7C15ull;
    int pos = (int)(hh >> 40) & (h->cap - 1);
    while (h->key[pos] != -1) { if (h->key[pos] == k) return 1; pos = (pos + 1) & (h->cap - 1); }
    return 0;
}

/* 2:1 balance across faces and corners: refine any leaf that is coarser by two
 * or more levels than a leaf touching it.  Returns the new leaf count. */
static int balance(const orc_sim* s, leaf_t** Lp, int n)
{
    leaf_t* L = *Lp;
    for (;;) {
        lset_t h; lset_init(&h, L, n);
        char* ref = (char*)calloc((size_t)n, 1);
        int any = 0;
        for (int i = 0; i < n; i++) {
            int l = L[i].level;
            for (int dy = -1; dy <= 1; dy++)
                for (int dx = -1; dx <= 1; dx++) {
                    if (!dx && !dy) continue;
                    int x, y;
                    if (orc_step(s, l, L[i].gx, L[i].gy, dx, dy, &x, &y) != 1) continue;
                    for (int k = l - 2; k >= 0; k--) {
                        if (lset_has(&h, k, x >> (l - k), y >> (l - k))) {
                            int j = leaf_find(L, n, k, x >> (l - k), y >> (l - k));
                            if (!ref[j]) { ref[j] = 1; any = 1; }
                            break;
                        }
                    }
                }
        }
        free(h.key);
        if (!any) { free(ref); break; }
        int nn = 0;
        for (int i = 0; i < n; i++) nn += ref[i] ? 4 : 1;
        leaf_t* M = (leaf_t*)malloc(sizeof(leaf_t) * nn);
        int m = 0;
        for (int i = 0; i < n; i++) {
            if (!ref[i]) { M[m++] = L[i]; continue; }
            for (int c = 0; c < 4; c++) {
                M[m].level = L[i].level + 1; M[m].gx = 2 * L[i].gx + (c & 1); M[m].gy = 2 * L[i].gy + (c >> 1); m++;
            }
        }
        free(ref); free(L); L = M; n = nn;
    }
    *Lp = L;
    return n;
}

/* Build the new forest from marks and repopulate patch data.
 * mark: +1 refine, -1 coarsen (whole family), 0 keep.  Returns 1 if changed. */
static int adapt(orc_sim* s, const int* mark, int domain_init)
{
    const int np = s->np;
    leaf_t* L = (leaf_t*)malloc(sizeof(leaf_t) * (4 * np + 4));
    int n = 0, changed = 0;
    char* done = (char*)calloc((size_t)np, 1);
    for (int i = 0; i < np; i++) {
        if (done[i]) continue;
        orc_patch* P = &s->p[i];
        if (mark[i] > 0) {
            for (int c = 0; c < 4; c++) {
                L[n].level = P->level + 1; L[n].gx = 2 * P->gx + (c & 1); L[n].gy = 2 * P->gy + (c >> 1); n++;
            }
            changed = 1; done[i] = 1;
        } else if (mark[i] < 0) {
            /* family: all four siblings must be leaves marked for coarsening */
            int px = P->gx >> 1, py = P->gy >> 1, l = P->level;
            int sib[4], ok = 1;
            for (int c = 0; c < 4; c++) {
                sib[c] = lookup(s, l, 2 * px + (c & 1), 2 * py + (c >> 1));
                if (sib[c] < 0 || mark[sib[c]] >= 0) ok = 0;
            }
            if (ok) {
                L[n].level = l - 1; L[n].gx = px; L[n].gy = py; n++;
                for (int c = 0; c < 4; c++) done[sib[c]] = 1;
                changed = 1;
            } else {
                L[n].level = l; L[n].gx = P->gx; L[n].gy = P->gy; n++; done[i] = 1;
            }
        } else {
            L[n].level = P->level; L[n].gx = P->gx; L[n].gy = P->gy; n++; done[i] = 1;
        }
    }
    free(done);
    n = balance(s, &L, n);
    /* did anything change with respect to the old forest? */
    if (!changed) {
        int same = (n == np);
        for (int i = 0; same && i < n; i++) if (lookup(s, L[i].level, L[i].gx, L[i].gy) < 0) same = 0;
        if (same) { free(L); return 0; }
    }
    orc_patch* NP = (orc_patch*)calloc((size_t)n, sizeof(orc_patch));
    char* kept = (char*)calloc((size_t)np, 1);
    for (int i = 0; i < n; i++) {
        orc_patch* Q = &NP[i];
        Q->level = L[i].level; Q->gx = L[i].gx; Q->gy = L[i].gy;
        int old = lookup(s, Q->level, Q->gx, Q->gy);
        if (old >= 0) {                                   /* FCLAW2D_PATCH_SAMESIZE: keep data */
            orc_patch* O = &s->p[old];
            *Q = *O;
            kept[old] = 1;
            continue;
        }
        patch_alloc(s, Q);
        patch_geometry(s, Q);
        const int sphere = s->cfg.problem == ORC_PROB_SPHERE;
        int parent = lookup(s, Q->level - 1, Q->gx >> 1, Q->gy >> 1);
        if (parent >= 0) {                                /* HALFSIZE: new fine patch */
            if (sphere) orc_sphere_area(s, Q, 0);         /* fclaw2d_metric_patch_build */
            orc_setaux(s, Q);
            if (domain_init) orc_qinit(s, Q);
            else orc_interpolate2fine(s, s->p[parent].q, Q->q, (Q->gx & 1) + 2 * (Q->gy & 1),
                                      s->p[parent].area, Q->area);
            continue;
        }
        int ch[4], all = 1;
        for (int c = 0; c < 4; c++) {
            ch[c] = lookup(s, Q->level + 1, 2 * Q->gx + (c & 1), 2 * Q->gy + (c >> 1));
            if (ch[c] < 0) all = 0;
        }
        if (all) {                                        /* DOUBLESIZE: new coarse patch */
            if (sphere) {                                 /* fclaw2d_metric_patch_build_from_fine */
                for (int c = 0; c < 4; c++) orc_sphere_area_from_fine(s, Q, &s->p[ch[c]], c);
                orc_sphere_area(s, Q, 1);
            }
            orc_setaux(s, Q);
            if (domain_init) orc_qinit(s, Q);
            else for (int c = 0; c < 4; c++) orc_average2coarse(s, Q->q, s->p[ch[c]].q, c, Q->area, s->p[ch[c]].area);
            continue;
        }
        fprintf(stderr, "oracle: adapt produced a patch more than one level from the old forest\n");
        abort();
    }
    for (int i = 0; i < np; i++) if (!kept[i]) patch_free(&s->p[i]);
    free(kept); free(L); free(s->p);
    s->p = NP; s->np = n;
    forest_finalize(s);
    return 1;
}

/* Refinement smoothing of fclaw2d_domain_adapt (src/fclaw2d_convenience.c:507-645).
 * The tags set target levels (fclaw2d_patch_mark_refine / _mark_coarsen,
 * src/forestclaw2d.c:1400-1450: level + 1 / level - 1); each patch then takes the
 * largest target level among itself and its face and corner neighbours of level
 * >= smooth_level, looking further only while that maximum does not exceed its
 * own level, and is marked to refine or coarsen by the sign of the difference. */
static void smooth_marks(const orc_sim* s, int* mark)
{
    const int np = s->np, smooth_level = s->cfg.smooth_level;
    int* tl = (int*)malloc(sizeof(int) * (size_t)(np > 0 ? np : 1));
    for (int i = 0; i < np; i++) tl[i] = s->p[i].level + mark[i];
    for (int i = 0; i < np; i++) {
        const orc_patch* P = &s->p[i];
        const int level = P->level;
        int mt = tl[i];
        for (int f = 0; mt <= level && f < 4; f++) {
            const int t = P->face_type[f];
            if (t == NB_BOUNDARY) continue;
            const int nn = (t == NB_HALF) ? 2 : 1;
            for (int k = 0; k < nn; k++) {
                const int nb = P->face_nbr[f][k];
                if (s->p[nb].level >= smooth_level && tl[nb] > mt) mt = tl[nb];
            }
        }
        for (int cn = 0; mt <= level && cn < 4; cn++) {
            if (!P->has_corner[cn]) continue;
            const int nb = P->corner_nbr[cn];
            if (s->p[nb].level >= smooth_level && tl[nb] > mt) mt = tl[nb];
        }
        mark[i] = (mt < level) ? -1 : (mt > level) ? 1 : 0;
    }
    free(tl);
}

static int regrid_impl(orc_sim* s, int domain_init)
{
    const orc_config* c = &s->cfg;
    int* mark = (int*)calloc((size_t)s->np, sizeof(int));
    /* families first (cb_regrid_tag4coarsening), then refinement (cb_fclaw2d_regrid_tag4refinement) */
    for (int i = 0; i < s->np; i++) {
        orc_patch* P = &s->p[i];
        if (P->level <= c->minlevel || (P->gx & 1) || (P->gy & 1)) continue;
        const orc_patch* fam[4];
        int ok = 1;
        for (int k = 0; k < 4; k++) {
            int j = lookup(s, P->level, P->gx + (k & 1), P->gy + (k >> 1));
            if (j < 0) { ok = 0; break; }
            fam[k] = &s->p[j];
        }
        if (!ok) continue;
        if (orc_tag_coarsen(s, fam, domain_init))
            for (int k = 0; k < 4; k++) mark[lookup(s, P->level, P->gx + (k & 1), P->gy + (k >> 1))] = -1;
    }
    for (int i = 0; i < s->np; i++)
        if (s->p[i].level < c->maxlevel && orc_tag_refine(s, &s->p[i], domain_init)) mark[i] = 1;
    if (c->smooth_refine) smooth_marks(s, mark);
    int changed = adapt(s, mark, domain_init);
    free(mark);
    return changed;
}

int orc_regrid(orc_sim* s)
{
    int changed = regrid_impl(s, 0);
    if (changed) ghost_update(s, s->minlevel_present, s->maxlevel_present, 0);
    return changed;
}

/* ------------------------------------------------------------------------- */
/* save / restore a step, and the run loop                                     */
/* ------------------------------------------------------------------------- */
void orc_save_step(orc_sim* s)
{
    for (int i = 0; i < s->np; i++) {
        orc_patch* P = &s->p[i];
        if (!P->qsave) P->qsave = (double*)malloc(sizeof(double) * s->nq);
        memcpy(P->qsave, P->q, sizeof(double) * s->nq);
    }
}

void orc_restore_step(orc_sim* s)
{
    for (int i = 0; i < s->np; i++)
        if (s->p[i].qsave) memcpy(s->p[i].q, s->p[i].qsave, sizeof(double) * s->nq);
}

/* outstyle_1 (src/fclaw2d_run.c:113-265) with reduce_cfl (one process: the global
 * maximum is the local one) and advance_one_step off. */
int orc_run(orc_sim* s, orc_run_stats* st)
{
    const orc_config* c = &s->cfg;
    memset(st, 0, sizeof(*st));
    const double final_time = c->tfinal;
    const int nout = c->nout > 0 ? c->nout : 1;
    double dt_minlevel = c->initial_dt;
    const double t0 = 0;
    const double dt_outer = (final_time - t0) / ((double)nout);
    double t_curr = t0;
    int n_inner = 0;
    for (int n = 0; n < nout; n++) {
        const double tstart = t_curr;
        const double tend = tstart + dt_outer;
        while (t_curr < tend) {
            if (!c->use_fixed_dt) orc_save_step(s);
            double dt_step = dt_minlevel;
            const double tol = 1e-2 * dt_step;
            int took_small_step = 0;
            if (!c->use_fixed_dt) {
                const double small_step = tend - (t_curr + dt_step);
                if (small_step < tol) {
                    dt_step = tend - t_curr;
                    if (small_step < 0) took_small_step = 1;
                }
            }
            const double maxcfl_step = orc_advance(s, t_curr, dt_step);
            st->count_amr_advance++;
            if (maxcfl_step > c->max_cfl) {
                if (!c->use_fixed_dt) {
                    orc_restore_step(s);
                    dt_minlevel = dt_minlevel * c->desired_cfl / maxcfl_step;
                    st->rejected++;
                    continue;
                }
            }
            n_inner++;
            t_curr += dt_step;
            if (!c->use_fixed_dt) {
                const double dt_new = dt_minlevel * c->desired_cfl / maxcfl_step;
                if (!took_small_step) dt_minlevel = dt_new;
            }
            if (c->regrid_interval > 0 && n_inner % c->regrid_interval == 0) {
                if (orc_regrid(s)) st->count_amr_new_domain++;
                st->count_amr_regrid++;
            }
        }
    }
    st->steps = n_inner;
    st->global_num_patches = s->np;
    st->t_final = t_curr;
    return 0;
}

/* ------------------------------------------------------------------------- */
/* API                                                                         */
/* ------------------------------------------------------------------------- */
orc_sim* orc_create(const orc_config* cfg)
{
    orc_sim* s = (orc_sim*)calloc(1, sizeof(orc_sim));
    s->cfg = *cfg;
    if (s->cfg.mi <= 0) s->cfg.mi = 1;
    if (s->cfg.mj <= 0) s->cfg.mj = 1;
    if (s->cfg.problem == ORC_PROB_SPHERE) { s->cfg.mi = 6; s->cfg.mj = 1; }
    s->nx = cfg->mx + 2 * cfg->mbc;
    s->ny = cfg->my + 2 * cfg->mbc;
    s->nq = (size_t)s->nx * s->ny * cfg->meqn;
    s->naux = (size_t)s->nx * s->ny * (cfg->maux > 0 ? cfg->maux : 0);
    s->dummy = (double*)calloc((size_t)(cfg->mx + 4 * cfg->mbc) * (cfg->my + 4 * cfg->mbc) * cfg->meqn, sizeof(double));
    if (cfg->problem == ORC_PROB_SHOCKBUBBLE) {
        double ps[3];
        orc_euler_postshock(cfg->gamma, cfg->mach, ps);
        s->inflow[0] = ps[0]; s->inflow[1] = ps[0] * ps[1]; s->inflow[2] = 0.0; s->inflow[3] = ps[2];
    }
#ifdef _OPENMP
    s->nthreads = cfg->nthreads > 0 ? cfg->nthreads : omp_get_max_threads();
#else
    s->nthreads = 1;
#endif
    return s;
}

void orc_destroy(orc_sim* s)
{
    if (!s) return;
    for (int i = 0; i < s->np; i++) patch_free(&s->p[i]);
    free(s->p); free(s->lev_list); free(s->hkey); free(s->hval); free(s->dummy);
    free(s);
}

int orc_initialize(orc_sim* s)
{
    const orc_config* c = &s->cfg;
    int l = c->minlevel;
    int nxl = c->mi << l, nyl = c->mj << l;
    s->np = nxl * nyl;
    s->p = (orc_patch*)calloc((size_t)s->np, sizeof(orc_patch));
    int k = 0;
    for (int y = 0; y < nyl; y++)
        for (int x = 0; x < nxl; x++) {
            orc_patch* P = &s->p[k++];
            P->level = l; P->gx = x; P->gy = y;
            patch_alloc(s, P);
            patch_geometry(s, P);
        }
    forest_finalize(s);
    for (int i = 0; i < s->np; i++) {
        if (c->problem == ORC_PROB_SPHERE) orc_sphere_area(s, &s->p[i], 0);
        orc_setaux(s, &s->p[i]);
        orc_qinit(s, &s->p[i]);
    }
    if (c->minlevel < c->maxlevel)
        for (int lev = c->minlevel; lev <= c->maxlevel; lev++)
            if (!regrid_impl(s, 1)) break;
    s->t_curr = 0;
    return s->np;
}

int orc_num_patches(const orc_sim* s) { return s->np; }

void orc_patch_info(const orc_sim* s, int* level, int* block, int* ix, int* iy)
{
    int n = 0;
    for (int l = 0; l < 31; l++)
        for (int k = s->lev_start[l]; k < s->lev_start[l + 1]; k++) {
            const orc_patch* P = &s->p[s->lev_list[k]];
            level[n] = P->level; block[n] = P->block; ix[n] = P->gx; iy[n] = P->gy; n++;
        }
}

void orc_get_q(const orc_sim* s, double* out)
{
    int n = 0;
    for (int l = 0; l < 31; l++)
        for (int k = s->lev_start[l]; k < s->lev_start[l + 1]; k++)
            memcpy(out + (size_t)(n++) * s->nq, s->p[s->lev_list[k]].q, s->nq * sizeof(double));
}

void orc_set_q(orc_sim* s, const double* in)
{
    int n = 0;
    for (int l = 0; l < 31; l++)
        for (int k = s->lev_start[l]; k < s->lev_start[l + 1]; k++)
            memcpy(s->p[s->lev_list[k]].q, in + (size_t)(n++) * s->nq, s->nq * sizeof(double));
}

void orc_get_aux(const orc_sim* s, double* out)
{
    int n = 0;
    for (int l = 0; l < 31; l++)
        for (int k = s->lev_start[l]; k < s->lev_start[l + 1]; k++) {
            if (s->naux) memcpy(out + (size_t)n * s->naux, s->p[s->lev_list[k]].aux, s->naux * sizeof(double));
            n++;
        }
}

int orc_registers_size(const orc_sim* s)
{
    const int mx = s->cfg.mx, my = s->cfg.my, meqn = s->cfg.meqn;
    return 4 * my * meqn + 4 * mx * meqn + 4 * my * meqn + 4 * mx * meqn;
}

/* Per patch: fp0 fp1 fm0 fm1 (my*meqn each), gp0 gp1 gm0 gm1 (mx*meqn), ef0..ef3. */
void orc_get_registers(const orc_sim* s, double* out)
{
    const int mx = s->cfg.mx, my = s->cfg.my, meqn = s->cfg.meqn;
    int n = 0;
    size_t sz = (size_t)orc_registers_size(s);
    for (int l = 0; l < 31; l++)
        for (int k = s->lev_start[l]; k < s->lev_start[l + 1]; k++) {
            const orc_regs* r = &s->p[s->lev_list[k]].regs;
            double* o = out + (size_t)(n++) * sz;
            for (int a = 0; a < 2; a++) { memcpy(o, r->fp[a], sizeof(double) * my * meqn); o += my * meqn; }
            for (int a = 0; a < 2; a++) { memcpy(o, r->fm[a], sizeof(double) * my * meqn); o += my * meqn; }
            for (int a = 0; a < 2; a++) { memcpy(o, r->gp[a], sizeof(double) * mx * meqn); o += mx * meqn; }
            for (int a = 0; a < 2; a++) { memcpy(o, r->gm[a], sizeof(double) * mx * meqn); o += mx * meqn; }
            memcpy(o, r->ef[0], sizeof(double) * 2 * my * meqn); o += 2 * my * meqn;
            memcpy(o, r->ef[1], sizeof(double) * 2 * my * meqn); o += 2 * my * meqn;
            memcpy(o, r->ef[2], sizeof(double) * 2 * mx * meqn); o += 2 * mx * meqn;
            memcpy(o, r->ef[3], sizeof(double) * 2 * mx * meqn); o += 2 * mx * meqn;
        }
}

/* fclaw2d_clawpatch46_fort_conservation_check (diagnostics.f:13-55): Kahan sum of
 * q*dx*dy over interior cells, patches in level-major order. */
void orc_mass(const orc_sim* s, double* out)
{
    const orc_config* c = &s->cfg;
    const int mx = c->mx, my = c->my, mbc = c->mbc, meqn = c->meqn, nx = s->nx, ny = s->ny;
    for (int m = 1; m <= meqn; m++) {
        double sum = 0, comp = 0;
        for (int l = 0; l < 31; l++)
            for (int k = s->lev_start[l]; k < s->lev_start[l + 1]; k++) {
                const orc_patch* P = &s->p[s->lev_list[k]];
                double area = P->dx * P->dy;
                for (int j = 1; j <= my; j++)
                    for (int i = 1; i <= mx; i++) {
                        /* manifold: area(i,j) (diagnostics.f:40-42) */
                        if (P->area) area = P->area[ORC_AIDX(i, j, mbc, mx + 2 * mbc + 2)];
                        double y = P->q[QIDX(i, j, m, mbc, nx, ny)] * area - comp;
                        double t = sum + y;
                        comp = (t - sum) - y;
                        sum = t;
                    }
            }
        out[m - 1] = sum;
    }
}

double orc_cell_updates(const orc_sim* s) { return s->cell_updates; }
