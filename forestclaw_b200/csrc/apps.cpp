// apps.cpp -- host-side app callbacks of the built-in problems.
//
//   swirl:      applications/clawpack/advection/2d/swirl/user_4.6/qinit.f, b4step2.f:25-36, psi.f:9.
//               The time-independent part of b4step2, psi(x,y+dy)-psi(x,y) and
//               psi(x+dx,y)-psi(x,y), is stored as aux; the fused update kernel
//               scales it by cos(2 pi (t+dt/2)/T)/dy and -cos(...)/dx each step.
//   radial dam: applications/clawpack/shallow/2d/radialdam/user_4.6/qinit.f: the disc of
//               fdisc.f by the cell-centre test, or (qinit_cellave) by the cell averages of
//               src/fortran_source2d/cellave2.f: the area of the polygon of the cell's inside
//               corners and its edge crossings, found by Brent's zeroin.
//   tsunami:    bathymetry b = -1 + 0.5 exp(-50|x-c|^2) in aux(:,:,1), surface eta = sum of bumps.
//   shock-bubble: applications/clawpack/euler/2d/shockbubble/user_4.6/qinit.f:24-62 (bubble by
//               cell centre), inflow of user_4.6/bc2.f:53-60, post-shock state from the
//               Rankine-Hugoniot relations of setprob.f:59-62 for the pressure ratio of a
//               Mach-M shock, 1 + 2 gamma (M^2 - 1) / (gamma + 1).
//   sphere:     advection on the cubed sphere (applications/clawpack/advection/2d/sphere):
//               solid-body rotation psi = omega (axis . x) (the reference's psi.f rotates about
//               the y axis), q = background + two Gaussians exp(-(theta/w)^2) of the angle
//               theta to their centres, evaluated at the mapped cell centres.  The metric and
//               aux (capacity, edge velocities) are computed on the device (k_metric.cu).
//               pdata: axis[0..2], omega[3], centre 1 [4..6], centre 2 [7..9], width [10],
//               background [11].
//   tagging:    fort_4.6/fclaw2d_clawpatch46_tag4refinement.f / _tag4coarsening.f with the
//               criteria of fort_user/fclaw2d_clawpatch_{value,difference,minmax,gradient}_exceeds_th.f90;
//               the apps' built-in choice is the gradient times dx, or minmax for the sphere.
#include "apps.hpp"
#include <cmath>
#include "fcb_sphere.h"

namespace fcb {

static inline size_t qi(const Dims& d, int i, int j, int m)
{
    return (size_t)(i + d.mbc - 1) + (size_t)(j + d.mbc - 1) * d.nx() + (size_t)(m - 1) * d.nxy();
}

static double swirl_psi(double x, double y, double pi)
{
    const double sx = std::sin(pi * x), sy = std::sin(pi * y);
    return ((sx * sx) * (sy * sy)) / pi;
}

void app_sphere_flow(const fc2d_b200_options_t& o, double axis[3], double* omega)
{
    const double a = o.pdata[0], b = o.pdata[1], c = o.pdata[2];
    const double n = std::sqrt(a * a + b * b + c * c);
    axis[0] = a / n; axis[1] = b / n; axis[2] = c / n;
    *omega = o.pdata[3];
}

// angle between the unit vectors x and c
static double sphere_angle(const double* x, const double* c)
{
    const double cx = x[1] * c[2] - x[2] * c[1], cy = x[2] * c[0] - x[0] * c[2], cz = x[0] * c[1] - x[1] * c[0];
    return std::atan2(std::sqrt(cx * cx + cy * cy + cz * cz), x[0] * c[0] + x[1] * c[1] + x[2] * c[2]);
}

// ---- cellave2 (src/fortran_source2d/cellave2.f) ----------------------------------
namespace {
struct Disc {
    double x0, y0, r0;
    double xc0 = 0, yc0 = 0, xc1 = 0, yc1 = 0;   // the edge being searched
    // fdisc.f (unmapped): negative inside the disc
    double f(double x, double y) const { return ((x - x0) * (x - x0) + (y - y0) * (y - y0)) - r0 * r0; }
    // fss: f at fraction s along the current edge
    double fs(double s) const { return f(xc0 + s * (xc1 - xc0), yc0 + s * (yc1 - yc0)); }
};

// Brent's root finder (R. Brent, Algorithms for Minimization without Derivatives, 1973,
// procedure zero) in the netlib form of cellave2.f:120-250, whose short step to the
// left is -xm rather than -tol1.
double brent_zero(const Disc& D, double ax, double bx, double tol)
{
    double eps = 1.0, tol1;
    do { eps = eps / 2.0; tol1 = 1.0 + eps; } while (tol1 > 1.0);
    double a = ax, b = bx, fa = D.fs(a), fb = D.fs(b);
    double c, fc, d, e, xm, p, q, r, sv;
    for (;;) {
        c = a; fc = fa; d = b - a; e = d;
        for (;;) {
            if (!(std::fabs(fc) >= std::fabs(fb))) { a = b; b = c; c = a; fa = fb; fb = fc; fc = fa; }
            tol1 = 2.0 * eps * std::fabs(b) + 0.5 * tol;
            xm = 0.5 * (c - b);
            if (std::fabs(xm) <= tol1 || fb == 0.0) return b;
            bool bisect = std::fabs(e) < tol1 || std::fabs(fa) <= std::fabs(fb);
            if (!bisect) {
                if (a == c) { sv = fb / fa; p = 2.0 * xm * sv; q = 1.0 - sv; }
                else {
                    q = fa / fc; r = fb / fc; sv = fb / fa;
                    p = sv * (2.0 * xm * q * (q - r) - (b - a) * (r - 1.0));
                    q = (q - 1.0) * (r - 1.0) * (sv - 1.0);
                }
                if (p > 0.0) q = -q;
                p = std::fabs(p);
                if ((2.0 * p) >= (3.0 * xm * q - std::fabs(tol1 * q)) || p >= std::fabs(0.5 * e * q)) bisect = true;
                else { e = d; d = p / q; }
            }
            if (bisect) { d = xm; e = d; }
            a = b; fa = fb;
            if (std::fabs(d) > tol1) b = b + d;
            if (std::fabs(d) <= tol1) b = (xm >= 0) ? b + tol1 : b - xm;
            fb = D.fs(b);
            if ((fb * (fc / std::fabs(fc))) > 0.0) break;
        }
    }
}

// Fraction of the cell [xlow, xlow + dx] x [ylow, ylow + dy] inside the disc.
double disc_fraction(Disc& D, double xlow, double ylow, double dx, double dy)
{
    const double xx[5] = {xlow, xlow, xlow + dx, xlow + dx, xlow};
    const double yy[5] = {ylow, ylow + dy, ylow + dy, ylow, ylow};
    bool fl[5], all_in = true, all_out = true;
    for (int i = 0; i < 4; i++) {
        fl[i] = D.f(xx[i], yy[i]) < 0.0;
        all_in = all_in && fl[i];
        all_out = all_out && !fl[i];
    }
    fl[4] = fl[0];
    if (all_in) return 1.0;
    if (all_out) return 0.0;
    double x[10], y[10];
    int n = 0;
    for (int i = 0; i < 4; i++) {
        if (fl[i]) { x[n] = xx[i]; y[n] = yy[i]; n++; }
        if (fl[i] != fl[i + 1]) {
            D.xc0 = xx[i]; D.yc0 = yy[i]; D.xc1 = xx[i + 1]; D.yc1 = yy[i + 1];
            const double ss = brent_zero(D, 0.0, 1.0, 1.0e-14);
            x[n] = xx[i] + ss * (xx[i + 1] - xx[i]);
            y[n] = yy[i] + ss * (yy[i + 1] - yy[i]);
            n++;
        }
    }
    if (n == 0) return 0.0;
    x[n] = x[0]; y[n] = y[0];
    double area = 0.0;
    for (int i = 0; i < n; i++) area = area + 0.5 * (y[i] + y[i + 1]) * (x[i + 1] - x[i]);
    return area / (dx * dy);
}
}  // namespace

void app_setaux(const fc2d_b200_options_t& o, const Dims& d, const PatchInfo& P, double* aux)
{
    const int mx = d.mx, my = d.my, mbc = d.mbc;
    if (o.app == FC2D_B200_APP_SWIRL) {
        const double pi = 4.0 * std::atan(1.0);
        for (int j = 1 - mbc; j <= my + mbc; j++) {
            const double yll = P.ylower + (j - 1) * P.dy;
            for (int i = 1 - mbc; i <= mx + mbc; i++) {
                const double xll = P.xlower + (i - 1) * P.dx;
                const double pij = swirl_psi(xll, yll, pi);
                aux[qi(d, i, j, 1)] = swirl_psi(xll, yll + P.dy, pi) - pij;
                aux[qi(d, i, j, 2)] = swirl_psi(xll + P.dx, yll, pi) - pij;
            }
        }
    } else if (o.app == FC2D_B200_APP_TSUNAMI) {
        const double cx = o.pdata[0], cy = o.pdata[1];
        for (int j = 1 - mbc; j <= my + mbc; j++)
            for (int i = 1 - mbc; i <= mx + mbc; i++) {
                const double xc = P.xlower + (i - 0.5) * P.dx, yc = P.ylower + (j - 0.5) * P.dy;
                const double r2 = (xc - cx) * (xc - cx) + (yc - cy) * (yc - cy);
                aux[qi(d, i, j, 1)] = -1.0 + 0.5 * std::exp(-50.0 * r2);
            }
    }
}

void app_qinit(const fc2d_b200_options_t& o, const Dims& d, const PatchInfo& P, const double* aux, double* q)
{
    const int mx = d.mx, my = d.my, mbc = d.mbc, meqn = d.meqn;
    if (o.app == FC2D_B200_APP_SPHERE) {
        const double w = o.pdata[10], bg = o.pdata[11];
        for (int j = 1 - mbc; j <= my + mbc; j++)
            for (int i = 1 - mbc; i <= mx + mbc; i++) {
                double x[3];
                cs_map(P.block, P.xlower + (i - 0.5) * P.dx, P.ylower + (j - 0.5) * P.dy, &x[0], &x[1], &x[2]);
                const double t1 = sphere_angle(x, &o.pdata[4]) / w, t2 = sphere_angle(x, &o.pdata[7]) / w;
                q[qi(d, i, j, 1)] = bg + std::exp(-(t1 * t1)) + std::exp(-(t2 * t2));
            }
        return;
    }
    if (o.app == FC2D_B200_APP_SWIRL) {
        for (int m = 1; m <= meqn; m++)
            for (int i = 1 - mbc; i <= mx + mbc; i++) {
                const double xc = P.xlower + (i - 0.5) * P.dx;
                for (int j = 1 - mbc; j <= my + mbc; j++) q[qi(d, i, j, m)] = (xc < 0.5) ? 1.0 : 0.0;
            }
    } else if (o.app == FC2D_B200_APP_RADIALDAM) {
        Disc D{o.x0, o.y0, o.r0};
        for (int i = 1 - mbc; i <= mx + mbc; i++) {
            const double xc = P.xlower + (i - 0.5) * P.dx;
            const double xlow = P.xlower + (i - 1.0) * P.dx;
            for (int j = 1 - mbc; j <= my + mbc; j++) {
                const double yc = P.ylower + (j - 0.5) * P.dy;
                double win;
                if (o.qinit_cellave) {
                    win = disc_fraction(D, xlow, P.ylower + (j - 1.0) * P.dy, P.dx, P.dy);
                } else {
                    const double r2 = (xc - o.x0) * (xc - o.x0) + (yc - o.y0) * (yc - o.y0);
                    win = (r2 - o.r0 * o.r0 < 0.0) ? 1.0 : 0.0;
                }
                q[qi(d, i, j, 1)] = o.hin * win + o.hout * (1.0 - win);
                q[qi(d, i, j, 2)] = 0.0;
                q[qi(d, i, j, 3)] = 0.0;
            }
        }
    } else if (o.app == FC2D_B200_APP_SHOCKBUBBLE) {
        double qinf[4];
        app_inflow_state(o, qinf);
        const double gamma1 = o.gamma - 1.0;
        for (int i = 1 - mbc; i <= mx + mbc; i++) {
            const double xclow = P.xlower + (i - 1) * P.dx;
            const double xc = P.xlower + (i - 0.5) * P.dx;
            for (int j = 1 - mbc; j <= my + mbc; j++) {
                const double yc = P.ylower + (j - 0.5) * P.dy;
                const double r2 = (xc - o.x0) * (xc - o.x0) + (yc - o.y0) * (yc - o.y0);
                const double win = (r2 - o.r0 * o.r0 < 0.0) ? 1.0 : 0.0;
                double v[4];
                v[0] = win * o.rhob + (1.0 - win) * 1.0;
                v[1] = 0.0;
                v[2] = 0.0;
                v[3] = 1.0 / gamma1;
                if (xclow < 0.2) { v[0] = qinf[0]; v[1] = qinf[1]; v[2] = 0.0; v[3] = qinf[3]; }
                for (int m = 1; m <= meqn; m++) q[qi(d, i, j, m)] = v[m - 1];
            }
        }
    } else if (o.app == FC2D_B200_APP_TSUNAMI) {
        const int nb = (int)o.pdata[2];
        for (int j = 1 - mbc; j <= my + mbc; j++)
            for (int i = 1 - mbc; i <= mx + mbc; i++) {
                const double xc = P.xlower + (i - 0.5) * P.dx, yc = P.ylower + (j - 0.5) * P.dy;
                double eta = 0.0;
                for (int k = 0; k < nb; k++) {
                    const double A = o.pdata[3 + 4 * k], w = o.pdata[4 + 4 * k];
                    const double bx = o.pdata[5 + 4 * k], by = o.pdata[6 + 4 * k];
                    const double r2 = (xc - bx) * (xc - bx) + (yc - by) * (yc - by);
                    eta = eta + A * std::exp(-r2 / (w * w));
                }
                q[qi(d, i, j, 1)] = eta - aux[qi(d, i, j, 1)];
                q[qi(d, i, j, 2)] = 0.0;
                q[qi(d, i, j, 3)] = 0.0;
            }
    }
}

bool app_inflow_state(const fc2d_b200_options_t& o, double* q)
{
    if (o.app != FC2D_B200_APP_SHOCKBUBBLE) return false;
    const double gam = o.gamma, gamma1 = gam - 1.0, mach = o.mach;
    const double pinf = 1.0 + 2.0 * gam * (mach * mach - 1.0) / (gam + 1.0);
    const double rinf = (gamma1 + (gam + 1.0) * pinf) / ((gam + 1.0) + gamma1 * pinf);
    const double vinf = (1.0 / std::sqrt(gam)) * (pinf - 1.0) / std::sqrt(0.5 * ((gam + 1.0) / gam) * pinf + 0.5 * gamma1 / gam);
    const double einf = 0.5 * rinf * vinf * vinf + pinf / gamma1;
    q[0] = rinf; q[1] = rinf * vinf; q[2] = 0.0; q[3] = einf;
    return true;
}

int tag_criterion(const fc2d_b200_options_t& o)
{
    if (o.refinement_criteria != FC2D_B200_TAG_APP) return o.refinement_criteria;
    return o.app == FC2D_B200_APP_SPHERE ? FC2D_B200_TAG_MINMAX : FC2D_B200_TAG_GRADIENT_DX;
}

// Criterion value of cell (i, j) compared with a threshold by the caller; for the
// stencil criteria only interior cells count.
static double tag_value(int crit, const Dims& d, const PatchInfo& P, const double* q, int i, int j, int mq)
{
    if (crit == FC2D_B200_TAG_VALUE) return q[qi(d, i, j, mq)];
    if (crit == FC2D_B200_TAG_DIFFERENCE) {
        const double dqx = std::fabs(q[qi(d, i + 1, j, mq)] - q[qi(d, i - 1, j, mq)]);
        const double dqy = std::fabs(q[qi(d, i, j + 1, mq)] - q[qi(d, i, j - 1, mq)]);
        return std::fmax(dqx, dqy);
    }
    const double dx2 = 2 * P.dx, dy2 = 2 * P.dy;
    const double dqx = (q[qi(d, i + 1, j, mq)] - q[qi(d, i - 1, j, mq)]) / dx2;
    const double dqy = (q[qi(d, i, j + 1, mq)] - q[qi(d, i, j - 1, mq)]) / dy2;
    const double ds = std::sqrt(dqx * dqx + dqy * dqy + 0.0 * 0.0);
    return crit == FC2D_B200_TAG_GRADIENT_DX ? ds * P.dx : ds;
}

int app_tag_refine(const fc2d_b200_options_t& o, const Dims& d, const PatchInfo& P, const double* q)
{
    // clawpatch_tag4refinement (fclaw2d_clawpatch.cpp:800-850): a negative threshold always refines
    if (o.refine_threshold < 0) return 1;
    const int crit = tag_criterion(o), mq = o.threshold_variable > 0 ? o.threshold_variable : 1;
    if (crit == FC2D_B200_TAG_MINMAX) {
        double lo = q[qi(d, 1, 1, mq)], hi = lo;
        for (int j = 1 - d.mbc; j <= d.my + d.mbc; j++)
            for (int i = 1 - d.mbc; i <= d.mx + d.mbc; i++) {
                lo = std::fmin(lo, q[qi(d, i, j, mq)]);
                hi = std::fmax(hi, q[qi(d, i, j, mq)]);
            }
        return hi - lo > o.refine_threshold ? 1 : 0;
    }
    const int g = (crit == FC2D_B200_TAG_VALUE) ? d.mbc : 0;   // value tests the ghost cells too
    for (int j = 1 - g; j <= d.my + g; j++)
        for (int i = 1 - g; i <= d.mx + g; i++)
            if (tag_value(crit, d, P, q, i, j, mq) > o.refine_threshold) return 1;
    return 0;
}

}  // namespace fcb
