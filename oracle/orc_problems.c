/*
 * orc_problems.c -- oracle copies of the app callbacks (qinit, setaux, b4step2,
 * tagging) for the benchmark problems (test infrastructure).
 *
 *   swirl:      applications/clawpack/advection/2d/swirl/user_4.6/qinit.f, b4step2.f:25-36, psi.f:9
 *   radial dam: applications/clawpack/shallow/2d/radialdam/user_4.6/qinit.f (cell-centre variant
 *               of the disc test; cellave2 sub-cell quadrature is not used)
 *   tagging:    fort_4.6/fclaw2d_clawpatch46_tag4refinement.f, _tag4coarsening.f with the
 *               gradient criterion of fort_user/fclaw2d_clawpatch_gradient_exceeds_th.f90
 *               scaled by dx (refine where |grad h| dx exceeds the threshold)
 *   bathymetry: tsunami problem, b = -1 + 0.5 exp(-50 |x - c|^2), eta = sum of Gaussian bumps
 *   sphere:     cubed sphere (applications/clawpack/advection/2d/sphere): metric and aux in
 *               orc_sphere.c; q = background + exp(-(theta1/w)^2) + exp(-(theta2/w)^2) at the mapped
 *               cell centres; minmax tagging (fort_user/fclaw2d_clawpatch_minmax_exceeds_th.f90)
 */
#include <math.h>
#include <string.h>
#include "orc_amr.h"

static double swirl_psi(double x, double y, double pi)
{
    double sx = sin(pi * x), sy = sin(pi * y);
    return ((sx * sx) * (sy * sy)) / pi;
}

/* angle between unit vectors */
static double sphere_angle(const double* x, const double* c)
{
    double cx = x[1] * c[2] - x[2] * c[1], cy = x[2] * c[0] - x[0] * c[2], cz = x[0] * c[1] - x[1] * c[0];
    return atan2(sqrt(cx * cx + cy * cy + cz * cz), x[0] * c[0] + x[1] * c[1] + x[2] * c[2]);
}

/* range of field 1 over the padded patch (minmax criterion) */
static void patch_minmax(const orc_sim* s, const orc_patch* P, double* lo, double* hi)
{
    const orc_config* c = &s->cfg;
    const int mbc = c->mbc, nx = s->nx, ny = s->ny;
    for (int j = 1 - mbc; j <= c->my + mbc; j++)
        for (int i = 1 - mbc; i <= c->mx + mbc; i++) {
            double v = P->q[QIDX(i, j, 1, mbc, nx, ny)];
            *lo = fmin(*lo, v);
            *hi = fmax(*hi, v);
        }
}

void orc_setaux(const orc_sim* s, orc_patch* P)
{
    const orc_config* c = &s->cfg;
    const int mx = c->mx, my = c->my, mbc = c->mbc, nx = s->nx, ny = s->ny;
    if (c->problem == ORC_PROB_SPHERE) { orc_sphere_setaux(s, P); return; }
    if (c->problem == ORC_PROB_TSUNAMI) {
        double cx = c->pdata[0], cy = c->pdata[1];
        for (int j = 1 - mbc; j <= my + mbc; j++)
            for (int i = 1 - mbc; i <= mx + mbc; i++) {
                double xc = P->xlower + (i - 0.5) * P->dx, yc = P->ylower + (j - 0.5) * P->dy;
                double r2 = (xc - cx) * (xc - cx) + (yc - cy) * (yc - cy);
                P->aux[QIDX(i, j, 1, mbc, nx, ny)] = -1.0 + 0.5 * exp(-50.0 * r2);
            }
    }
}

void orc_qinit(const orc_sim* s, orc_patch* P)
{
    const orc_config* c = &s->cfg;
    const int mx = c->mx, my = c->my, mbc = c->mbc, meqn = c->meqn, nx = s->nx, ny = s->ny;
    if (c->problem == ORC_PROB_SPHERE) {
        double w = c->pdata[10], bg = c->pdata[11];
        for (int j = 1 - mbc; j <= my + mbc; j++)
            for (int i = 1 - mbc; i <= mx + mbc; i++) {
                double x[3];
                orc_cs_map(P->block, P->xlower + (i - 0.5) * P->dx, P->ylower + (j - 0.5) * P->dy, &x[0], &x[1], &x[2]);
                double t1 = sphere_angle(x, &c->pdata[4]) / w, t2 = sphere_angle(x, &c->pdata[7]) / w;
                P->q[QIDX(i, j, 1, mbc, nx, ny)] = bg + exp(-(t1 * t1)) + exp(-(t2 * t2));
            }
        return;
    }
    if (c->problem == ORC_PROB_SWIRL) {
        for (int m = 1; m <= meqn; m++)
            for (int i = 1 - mbc; i <= mx + mbc; i++) {
                double xc = P->xlower + (i - 0.5) * P->dx;
                for (int j = 1 - mbc; j <= my + mbc; j++)
                    P->q[QIDX(i, j, m, mbc, nx, ny)] = (xc < 0.5) ? 1.0 : 0.0;
            }
    } else if (c->problem == ORC_PROB_RADIALDAM || c->problem == ORC_PROB_UNIFORM_SW) {
        for (int i = 1 - mbc; i <= mx + mbc; i++) {
            double xc = P->xlower + (i - 0.5) * P->dx;
            for (int j = 1 - mbc; j <= my + mbc; j++) {
                double yc = P->ylower + (j - 0.5) * P->dy;
                double r2 = (xc - c->x0) * (xc - c->x0) + (yc - c->y0) * (yc - c->y0);
                double win = (r2 - c->r0 * c->r0 < 0.0) ? 1.0 : 0.0;
                P->q[QIDX(i, j, 1, mbc, nx, ny)] = c->hin * win + c->hout * (1.0 - win);
                P->q[QIDX(i, j, 2, mbc, nx, ny)] = 0.0;
                P->q[QIDX(i, j, 3, mbc, nx, ny)] = 0.0;
            }
        }
    } else if (c->problem == ORC_PROB_SHOCKBUBBLE) {
        /* shockbubble/user_4.6/qinit.f:24-62: bubble (by cell centre) of density rhob
         * at pressure 1, ambient (1, 0, 0, 1/(gamma-1)), post-shock state where the
         * cell's lower edge is left of x = 0.2 */
        const double gamma1 = c->gamma - 1.0;
        for (int i = 1 - mbc; i <= mx + mbc; i++) {
            const double xclow = P->xlower + (i - 1) * P->dx;
            const double xc = P->xlower + (i - 0.5) * P->dx;
            for (int j = 1 - mbc; j <= my + mbc; j++) {
                const double yc = P->ylower + (j - 0.5) * P->dy;
                const double r2 = (xc - c->x0) * (xc - c->x0) + (yc - c->y0) * (yc - c->y0);
                const double win = (r2 - c->r0 * c->r0 < 0.0) ? 1.0 : 0.0;
                double q[4];
                q[0] = win * c->rhob + (1.0 - win) * 1.0;
                q[1] = 0.0;
                q[2] = 0.0;
                q[3] = 1.0 / gamma1;
                if (xclow < 0.2) { q[0] = s->inflow[0]; q[1] = s->inflow[1]; q[2] = 0.0; q[3] = s->inflow[3]; }
                for (int m = 1; m <= meqn; m++) P->q[QIDX(i, j, m, mbc, nx, ny)] = q[m - 1];
            }
        }
    } else if (c->problem == ORC_PROB_TSUNAMI) {
        int nb = (int)c->pdata[2];
        for (int j = 1 - mbc; j <= my + mbc; j++)
            for (int i = 1 - mbc; i <= mx + mbc; i++) {
                double xc = P->xlower + (i - 0.5) * P->dx, yc = P->ylower + (j - 0.5) * P->dy;
                double eta = 0.0;
                for (int k = 0; k < nb; k++) {
                    double A = c->pdata[3 + 4 * k], w = c->pdata[4 + 4 * k];
                    double bx = c->pdata[5 + 4 * k], by = c->pdata[6 + 4 * k];
                    double r2 = (xc - bx) * (xc - bx) + (yc - by) * (yc - by);
                    eta = eta + A * exp(-r2 / (w * w));
                }
                double b = P->aux[QIDX(i, j, 1, mbc, nx, ny)];
                P->q[QIDX(i, j, 1, mbc, nx, ny)] = eta - b;
                P->q[QIDX(i, j, 2, mbc, nx, ny)] = 0.0;
                P->q[QIDX(i, j, 3, mbc, nx, ny)] = 0.0;
            }
    }
}

/* swirl b4step2.f:25-36: edge velocities from stream-function differences at t + dt/2. */
void orc_b4step2(const orc_sim* s, orc_patch* P, double t, double dt)
{
    const orc_config* c = &s->cfg;
    if (c->problem != ORC_PROB_SWIRL || c->tperiod == 0.0) return;
    const int mx = c->mx, my = c->my, mbc = c->mbc, nx = s->nx, ny = s->ny;
    const double pi = 4.0 * atan(1.0), pi2 = 2.0 * pi;
    double vt = cos(pi2 * (t + dt / 2.0) / c->tperiod);
    double vty = vt / P->dy, vtx = vt / P->dx;
    for (int j = 1 - mbc; j <= my + mbc; j++) {
        double yll = P->ylower + (j - 1) * P->dy;
        for (int i = 1 - mbc; i <= mx + mbc; i++) {
            double xll = P->xlower + (i - 1) * P->dx;
            double pij = swirl_psi(xll, yll, pi);
            P->aux[QIDX(i, j, 1, mbc, nx, ny)] = vty * (swirl_psi(xll, yll + P->dy, pi) - pij);
            P->aux[QIDX(i, j, 2, mbc, nx, ny)] = -(vtx * (swirl_psi(xll + P->dx, yll, pi) - pij));
        }
    }
}

/* gradient criterion (gradient_exceeds_th.f90, unmapped branch) scaled by dx. */
static int grad_exceeds(const orc_sim* s, const orc_patch* P, const double* q, int i, int j, double thr)
{
    const int mbc = s->cfg.mbc, nx = s->nx, ny = s->ny;
    double dx2 = 2 * P->dx, dy2 = 2 * P->dy;
    double dqx = (q[QIDX(i + 1, j, 1, mbc, nx, ny)] - q[QIDX(i - 1, j, 1, mbc, nx, ny)]) / dx2;
    double dqy = (q[QIDX(i, j + 1, 1, mbc, nx, ny)] - q[QIDX(i, j - 1, 1, mbc, nx, ny)]) / dy2;
    double ds = sqrt(dqx * dqx + dqy * dqy + 0.0 * 0.0);
    return ds * P->dx > thr;
}

int orc_tag_refine(const orc_sim* s, const orc_patch* P, int init_flag)
{
    (void)init_flag;
    const orc_config* c = &s->cfg;
    if (c->problem == ORC_PROB_SPHERE) {
        int mbc = c->mbc;
        double lo = P->q[QIDX(1, 1, 1, mbc, s->nx, s->ny)], hi = lo;
        patch_minmax(s, P, &lo, &hi);
        return hi - lo > c->refine_threshold;
    }
    for (int j = 1; j <= c->my; j++)
        for (int i = 1; i <= c->mx; i++)
            if (grad_exceeds(s, P, P->q, i, j, c->refine_threshold)) return 1;
    return 0;
}

int orc_tag_coarsen(const orc_sim* s, const orc_patch* const* fam, int init_flag)
{
    const orc_config* c = &s->cfg;
    if (init_flag) return 0;
    if (c->problem == ORC_PROB_SPHERE) {
        /* running range over the whole family (tag4coarsening.f:35-58) */
        int mbc = c->mbc;
        double lo = fam[0]->q[QIDX(1, 1, 1, mbc, s->nx, s->ny)], hi = lo;
        for (int k = 0; k < 4; k++) patch_minmax(s, fam[k], &lo, &hi);
        return !(hi - lo > c->coarsen_threshold);
    }
    for (int k = 0; k < 4; k++)
        for (int i = 1; i <= c->mx; i++)
            for (int j = 1; j <= c->my; j++)
                if (grad_exceeds(s, fam[k], fam[k]->q, i, j, c->coarsen_threshold)) return 0;
    return 1;
}
