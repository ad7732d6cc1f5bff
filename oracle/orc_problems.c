/*
 * orc_problems.c -- oracle copies of the app callbacks (qinit, setaux, b4step2,
 * tagging) for the benchmark problems (test infrastructure).
 *
 *   swirl:      applications/clawpack/advection/2d/swirl/user_4.6/qinit.f, b4step2.f:25-36, psi.f:9
 *   radial dam: applications/clawpack/shallow/2d/radialdam/user_4.6/qinit.f: the disc of fdisc.f
 *               either by the cell-centre test (qinit_sharp = 1) or by the reference's cell
 *               average, src/fortran_source2d/cellave2.f (sub-cell polygon area with Brent's zeroin)
 *   tagging:    fort_4.6/fclaw2d_clawpatch46_tag4refinement.f, _tag4coarsening.f with the
 *               criteria of fort_user/fclaw2d_clawpatch_{value,difference,minmax,gradient}_exceeds_th.f90
 *               (tag_criteria), or each problem's built-in one: the gradient criterion scaled by
 *               dx (refine where |grad h| dx exceeds the threshold)
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

/* ---- cellave2 (src/fortran_source2d/cellave2.f) --------------------------------- */
typedef struct { double x0, y0, r0, xc0, yc0, xc1, yc1; } disc_t;

/* fdisc (applications/clawpack/shallow/2d/radialdam/fdisc.f:1-27, unmapped branch) */
static double fdisc(const disc_t* D, double x, double y)
{
    double r2 = (x - D->x0) * (x - D->x0) + (y - D->y0) * (y - D->y0);
    return r2 - D->r0 * D->r0;
}

/* fss (cellave2.f:104-117): fdisc at fraction s of the way between two corners */
static double fss(const disc_t* D, double s)
{
    double x = D->xc0 + s * (D->xc1 - D->xc0);
    double y = D->yc0 + s * (D->yc1 - D->yc0);
    return fdisc(D, x, y);
}

/* zeroin (cellave2.f:120-250): R. Brent's root finder (Algorithms for Minimization
 * without Derivatives, 1973, procedure zero) in the netlib form the reference
 * carries, including its step of -xm (not -tol1) when a tiny step goes left. */
static double zeroin(const disc_t* D, double ax, double bx, double tol)
{
    double eps = 1.0, tol1, a, b, c, d, e, fa, fb, fc, xm, p, q, r, s;
    do { eps = eps / 2.0; tol1 = 1.0 + eps; } while (tol1 > 1.0);
    a = ax; b = bx;
    fa = fss(D, a); fb = fss(D, b);
    for (;;) {
        /* label 20: begin step */
        c = a; fc = fa; d = b - a; e = d;
        for (;;) {
            /* label 30 */
            if (!(fabs(fc) >= fabs(fb))) { a = b; b = c; c = a; fa = fb; fb = fc; fc = fa; }
            /* label 40: convergence test */
            tol1 = 2.0 * eps * fabs(b) + 0.5 * tol;
            xm = 0.5 * (c - b);
            if (fabs(xm) <= tol1 || fb == 0.0) return b;
            if (fabs(e) < tol1 || fabs(fa) <= fabs(fb)) {
                d = xm; e = d;                                   /* label 70: bisection */
            } else {
                if (a == c) {                                    /* linear interpolation */
                    s = fb / fa; p = 2.0 * xm * s; q = 1.0 - s;
                } else {                                         /* label 50: inverse quadratic */
                    q = fa / fc; r = fb / fc; s = fb / fa;
                    p = s * (2.0 * xm * q * (q - r) - (b - a) * (r - 1.0));
                    q = (q - 1.0) * (r - 1.0) * (s - 1.0);
                }
                if (p > 0.0) q = -q;                             /* label 60 */
                p = fabs(p);
                if ((2.0 * p) >= (3.0 * xm * q - fabs(tol1 * q)) || p >= fabs(0.5 * e * q)) {
                    d = xm; e = d;                               /* label 70 */
                } else {
                    e = d; d = p / q;
                }
            }
            /* label 80: complete step */
            a = b; fa = fb;
            if (fabs(d) > tol1) b = b + d;
            if (fabs(d) <= tol1) {
                if (xm >= 0) b = b + tol1;
                else b = b - xm;
            }
            fb = fss(D, b);
            if ((fb * (fc / fabs(fc))) > 0.0) break;             /* go to 20 */
        }
    }
}

/* cellave2 (cellave2.f:2-100): fraction of the cell [xlow, xlow+dx] x [ylow, ylow+dy]
 * on the negative side of fdisc, as the area of the polygon of the inside corners
 * and the edge crossings. */
static double cellave2(disc_t* D, double xlow, double ylow, double dx, double dy)
{
    double xx[5], yy[5], x[10], y[10];
    int fl[5], alll = 1, allr = 1, iv = 0;
    xx[0] = xlow; xx[1] = xlow; xx[2] = xlow + dx; xx[3] = xlow + dx; xx[4] = xx[0];
    yy[0] = ylow; yy[1] = ylow + dy; yy[2] = ylow + dy; yy[3] = ylow; yy[4] = yy[0];
    for (int i = 0; i < 4; i++) {
        fl[i] = fdisc(D, xx[i], yy[i]) < 0.0;
        alll = alll && fl[i];
        allr = allr && !fl[i];
    }
    fl[4] = fl[0];
    if (alll) return 1.0;
    if (allr) return 0.0;
    for (int i = 0; i < 4; i++) {
        if (fl[i]) { x[iv] = xx[i]; y[iv] = yy[i]; iv++; }
        if (fl[i] != fl[i + 1]) {
            D->xc0 = xx[i]; D->yc0 = yy[i]; D->xc1 = xx[i + 1]; D->yc1 = yy[i + 1];
            double ss = zeroin(D, 0.0, 1.0, 1.0e-14);
            x[iv] = xx[i] + ss * (xx[i + 1] - xx[i]);
            y[iv] = yy[i] + ss * (yy[i + 1] - yy[i]);
            iv++;
        }
    }
    if (iv == 0) return 0.0;
    x[iv] = x[0]; y[iv] = y[0];
    double area = 0.0;
    for (int i = 0; i < iv; i++) area = area + 0.5 * (y[i] + y[i + 1]) * (x[i + 1] - x[i]);
    return area / (dx * dy);
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
        disc_t D = {c->x0, c->y0, c->r0, 0, 0, 0, 0};
        for (int i = 1 - mbc; i <= mx + mbc; i++) {
            double xc = P->xlower + (i - 0.5) * P->dx;
            double xlow = P->xlower + (i - 1.0) * P->dx;
            for (int j = 1 - mbc; j <= my + mbc; j++) {
                double yc = P->ylower + (j - 0.5) * P->dy;
                double win;
                if (c->qinit_sharp) {
                    double r2 = (xc - c->x0) * (xc - c->x0) + (yc - c->y0) * (yc - c->y0);
                    win = (r2 - c->r0 * c->r0 < 0.0) ? 1.0 : 0.0;
                } else {
                    double ylow = P->ylower + (j - 1.0) * P->dy;
                    win = cellave2(&D, xlow, ylow, P->dx, P->dy);
                }
                P->q[QIDX(i, j, 1, mbc, nx, ny)] = c->hin * win + c->hout * (1.0 - win);
                P->q[QIDX(i, j, 2, mbc, nx, ny)] = 0.0;
                P->q[QIDX(i, j, 3, mbc, nx, ny)] = 0.0;
            }
        }
    } else if (c->problem == ORC_PROB_ROTATION || c->problem == ORC_PROB_ACOUSTICS) {
        /* a disc of radius r0 at (x0, y0) by the cell centre: q = 1 inside (rotation), or
         * pressure hin inside and hout outside with the fluid at rest (acoustics) */
        for (int i = 1 - mbc; i <= mx + mbc; i++) {
            const double xc = P->xlower + (i - 0.5) * P->dx;
            for (int j = 1 - mbc; j <= my + mbc; j++) {
                const double yc = P->ylower + (j - 0.5) * P->dy;
                const double r2 = (xc - c->x0) * (xc - c->x0) + (yc - c->y0) * (yc - c->y0);
                const int in = r2 < c->r0 * c->r0;
                if (c->problem == ORC_PROB_ROTATION) P->q[QIDX(i, j, 1, mbc, nx, ny)] = in ? 1.0 : 0.0;
                else {
                    P->q[QIDX(i, j, 1, mbc, nx, ny)] = in ? c->hin : c->hout;
                    for (int m = 2; m <= meqn; m++) P->q[QIDX(i, j, m, mbc, nx, ny)] = 0.0;
                }
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

/* Test app of the application-solver interface (ORC_PROB_ROTATION): the stream function
 * psi = omega ((x - 1/2)^2 + (y - 1/2)^2) / 2 and the factor vt = 1 - (t + dt/2)/2, applied
 * the way applications/cudaclaw/advection/2d/swirl/user_cuda/b4step2.cu:22-45 applies its
 * own (differences over dy and dx, then times vt); omega = pdata[26]. */
static double rot_psi(double x, double y, double omega)
{
    return omega * ((x - 0.5) * (x - 0.5) + (y - 0.5) * (y - 0.5)) / 2.0;
}

static void rotation_b4step2(const orc_sim* s, orc_patch* P, double t, double dt)
{
    const orc_config* c = &s->cfg;
    const int mx = c->mx, my = c->my, mbc = c->mbc, nx = s->nx, ny = s->ny;
    const double omega = c->pdata[26];
    const double vt = 1.0 - (t + dt / 2.0) / 2.0;
    for (int j = 1 - mbc; j <= my + mbc; j++)
        for (int i = 1 - mbc; i <= mx + mbc; i++) {
            const double xll = P->xlower + (i - 1) * P->dx, yll = P->ylower + (j - 1) * P->dy;
            const double p1 = rot_psi(xll, yll + P->dy, omega), p2 = rot_psi(xll, yll, omega),
                         p3 = rot_psi(xll + P->dx, yll, omega);
            double a0 = (p1 - p2) / P->dy, a1 = -(p3 - p2) / P->dx;
            a0 = a0 * vt;
            a1 = a1 * vt;
            P->aux[QIDX(i, j, 1, mbc, nx, ny)] = a0;
            P->aux[QIDX(i, j, 2, mbc, nx, ny)] = a1;
        }
}

/* swirl b4step2.f:25-36: edge velocities from stream-function differences at t + dt/2. */
void orc_b4step2(const orc_sim* s, orc_patch* P, double t, double dt)
{
    const orc_config* c = &s->cfg;
    if (c->problem == ORC_PROB_ROTATION) { rotation_b4step2(s, P, t, dt); return; }
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

/* fclaw2d_clawpatch_tag_criteria (fort_user/fclaw2d_clawpatch_tag_criteria.c) for cell (i, j):
 * 1 exceeds, 0 does not, -1 inconclusive (ghost cell of a stencil criterion).
 * value_exceeds_th.f90, difference_exceeds_th.f90, minmax_exceeds_th.f90,
 * gradient_exceeds_th.f90 (unmapped branch); ORC_TAG_GRADIENT_DX multiplies the
 * gradient by dx. */
static int exceeds_th(const orc_sim* s, int crit, const orc_patch* P, const double* q, int i, int j, int mq,
                      const double* qmin, const double* qmax, double thr, int is_ghost)
{
    const int mbc = s->cfg.mbc, nx = s->nx, ny = s->ny;
#define QQ(ii, jj) q[QIDX((ii), (jj), mq, mbc, nx, ny)]
    switch (crit) {
    case ORC_TAG_VALUE:
        return QQ(i, j) > thr;
    case ORC_TAG_MINMAX:
        return qmax[mq - 1] - qmin[mq - 1] > thr;
    case ORC_TAG_DIFFERENCE: {
        if (is_ghost) return -1;
        double dqx = fabs(QQ(i + 1, j) - QQ(i - 1, j));
        double dqy = fabs(QQ(i, j + 1) - QQ(i, j - 1));
        return fmax(dqx, dqy) > thr;
    }
    default: {   /* gradient */
        if (is_ghost) return -1;
        double dx2 = 2 * P->dx, dy2 = 2 * P->dy;
        double dqx = (QQ(i + 1, j) - QQ(i - 1, j)) / dx2;
        double dqy = (QQ(i, j + 1) - QQ(i, j - 1)) / dy2;
        double ds = sqrt(dqx * dqx + dqy * dqy + 0.0 * 0.0);
        if (crit == ORC_TAG_GRADIENT_DX) ds = ds * P->dx;
        return ds > thr;
    }
    }
#undef QQ
}

static int is_ghost46(int i, int j, int mx, int my) { return i < 1 || j < 1 || i > mx || j > my; }

/* fclaw2d_clawpatch46_fort_tag4refinement (fort_4.6/fclaw2d_clawpatch46_tag4refinement.f:11-75):
 * running min/max over the padded patch, j outer, first exceeding cell tags. */
static int tag4refinement46(const orc_sim* s, const orc_patch* P, int crit, double thr)
{
    const orc_config* c = &s->cfg;
    const int mx = c->mx, my = c->my, mbc = c->mbc, meqn = c->meqn, nx = s->nx, ny = s->ny;
    const int mq = c->threshold_variable > 0 ? c->threshold_variable : 1;
    double qmin[16], qmax[16];
    for (int m = 1; m <= meqn; m++) { qmin[m - 1] = P->q[QIDX(1, 1, m, mbc, nx, ny)]; qmax[m - 1] = qmin[m - 1]; }
    for (int j = 1 - mbc; j <= my + mbc; j++)
        for (int i = 1 - mbc; i <= mx + mbc; i++) {
            for (int m = 1; m <= meqn; m++) {
                double v = P->q[QIDX(i, j, m, mbc, nx, ny)];
                qmin[m - 1] = fmin(qmin[m - 1], v);
                qmax[m - 1] = fmax(qmax[m - 1], v);
            }
            if (exceeds_th(s, crit, P, P->q, i, j, mq, qmin, qmax, thr, is_ghost46(i, j, mx, my)) > 0) return 1;
        }
    return 0;
}

/* fclaw2d_clawpatch46_fort_tag4coarsening (fort_4.6/fclaw2d_clawpatch46_tag4coarsening.f:11-60)
 * and test_refine (:80-130): min/max carried across the four siblings, i outer;
 * the family coarsens unless some cell exceeds the threshold. */
static int tag4coarsening46(const orc_sim* s, const orc_patch* const* fam, int crit, double thr)
{
    const orc_config* c = &s->cfg;
    const int mx = c->mx, my = c->my, mbc = c->mbc, meqn = c->meqn, nx = s->nx, ny = s->ny;
    const int mq = c->threshold_variable > 0 ? c->threshold_variable : 1;
    double qmin[16], qmax[16];
    for (int m = 1; m <= meqn; m++) { qmin[m - 1] = fam[0]->q[QIDX(1, 1, m, mbc, nx, ny)]; qmax[m - 1] = qmin[m - 1]; }
    for (int k = 0; k < 4; k++)
        for (int i = 1 - mbc; i <= mx + mbc; i++)
            for (int j = 1 - mbc; j <= my + mbc; j++) {
                for (int m = 1; m <= meqn; m++) {
                    double v = fam[k]->q[QIDX(i, j, m, mbc, nx, ny)];
                    qmin[m - 1] = fmin(v, qmin[m - 1]);
                    qmax[m - 1] = fmax(v, qmax[m - 1]);
                }
                if (exceeds_th(s, crit, fam[k], fam[k]->q, i, j, mq, qmin, qmax, thr, is_ghost46(i, j, mx, my)) > 0)
                    return 0;
            }
    return 1;
}

int orc_tag_refine(const orc_sim* s, const orc_patch* P, int init_flag)
{
    (void)init_flag;
    const orc_config* c = &s->cfg;
    /* clawpatch_tag4refinement (fclaw2d_clawpatch.cpp:800-850): a negative threshold always refines */
    if (c->tag_criteria != ORC_TAG_APP) {
        if (c->refine_threshold < 0) return 1;
        return tag4refinement46(s, P, c->tag_criteria, c->refine_threshold);
    }
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
    /* clawpatch_tag4coarsening (fclaw2d_clawpatch.cpp:853-910): coarsen only with a positive threshold */
    if (c->tag_criteria != ORC_TAG_APP) {
        if (!(c->coarsen_threshold > 0)) return 0;
        return tag4coarsening46(s, fam, c->tag_criteria, c->coarsen_threshold);
    }
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
