// apps.cpp -- host-side app callbacks of the built-in problems.
//
//   swirl:      applications/clawpack/advection/2d/swirl/user_4.6/qinit.f, b4step2.f:25-36, psi.f:9.
//               The time-independent part of b4step2, psi(x,y+dy)-psi(x,y) and
//               psi(x+dx,y)-psi(x,y), is stored as aux; the fused update kernel
//               scales it by cos(2 pi (t+dt/2)/T)/dy and -cos(...)/dx each step.
//   radial dam: applications/clawpack/shallow/2d/radialdam/user_4.6/qinit.f with the
//               disc test at the cell centre.
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
//               gradient criterion (fort_user/fclaw2d_clawpatch_gradient_exceeds_th.f90) times dx;
//               the sphere uses the minmax criterion (fclaw2d_clawpatch_minmax_exceeds_th.f90).
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
        for (int i = 1 - mbc; i <= mx + mbc; i++) {
            const double xc = P.xlower + (i - 0.5) * P.dx;
            for (int j = 1 - mbc; j <= my + mbc; j++) {
                const double yc = P.ylower + (j - 0.5) * P.dy;
                const double r2 = (xc - o.x0) * (xc - o.x0) + (yc - o.y0) * (yc - o.y0);
                const double win = (r2 - o.r0 * o.r0 < 0.0) ? 1.0 : 0.0;
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

static bool grad_exceeds(const Dims& d, const PatchInfo& P, const double* q, int i, int j, double thr)
{
    const double dx2 = 2 * P.dx, dy2 = 2 * P.dy;
    const double dqx = (q[qi(d, i + 1, j, 1)] - q[qi(d, i - 1, j, 1)]) / dx2;
    const double dqy = (q[qi(d, i, j + 1, 1)] - q[qi(d, i, j - 1, 1)]) / dy2;
    const double ds = std::sqrt(dqx * dqx + dqy * dqy + 0.0 * 0.0);
    return ds * P.dx > thr;
}

int app_tag_refine(const fc2d_b200_options_t& o, const Dims& d, const PatchInfo& P, const double* q)
{
    if (o.app == FC2D_B200_APP_SPHERE) {
        // minmax: range of field 1 over the padded patch
        double lo = q[qi(d, 1, 1, 1)], hi = lo;
        for (int j = 1 - d.mbc; j <= d.my + d.mbc; j++)
            for (int i = 1 - d.mbc; i <= d.mx + d.mbc; i++) {
                lo = std::fmin(lo, q[qi(d, i, j, 1)]);
                hi = std::fmax(hi, q[qi(d, i, j, 1)]);
            }
        return hi - lo > o.refine_threshold ? 1 : 0;
    }
    for (int j = 1; j <= d.my; j++)
        for (int i = 1; i <= d.mx; i++)
            if (grad_exceeds(d, P, q, i, j, o.refine_threshold)) return 1;
    return 0;
}

int app_coarsen_ok(const fc2d_b200_options_t& o, const Dims& d, const PatchInfo& P, const double* q)
{
    for (int i = 1; i <= d.mx; i++)
        for (int j = 1; j <= d.my; j++)
            if (grad_exceeds(d, P, q, i, j, o.coarsen_threshold)) return 0;
    return 1;
}

}  // namespace fcb
