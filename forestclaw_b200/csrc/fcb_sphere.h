// fcb_sphere.h -- the cubed-sphere mapping and the solid-body-rotation stream
// function, callable from host (g++) and device (nvcc) code.
//
// Every function uses only + - * / and sqrt (correctly rounded on both sides) in
// one fixed order, so a unit built without FMA contraction gives the same bits on
// the host and on the device.  tan is evaluated as sin/cos from their Taylor
// series (x^25, x^24), accurate to a few ulp for |x| < 1.45, which covers the
// mapped coordinates of every node a patch with mx >= 8 and mbc = 2 touches.
//
// Mapping: src/mappings/cubedsphere/mapc2m_cubedsphere.f (blocks 0..5 = faces of the
// cube, the gnomonic map x = z tan(xi), y = z tan(eta), z = R / sqrt(1 + tan^2 xi +
// tan^2 eta) with xi, eta = pi/2 (xc - 1/2), (yc - 1/2), then a per-block permutation
// and sign of the coordinates).  R = 1.
#pragma once
#ifdef __CUDACC__
#define FCB_HD __host__ __device__ __forceinline__
#else
#include <cmath>
#define FCB_HD inline
#endif

namespace fcb {

constexpr double FCB_PI = 3.14159265358979311600e+00;   // the double nearest pi (= 4 atan 1)

FCB_HD double fcb_tan(double x)
{
    const double x2 = x * x;
    // sin x = x (1 - x^2/(2.3) (1 - x^2/(4.5) (1 - ...)))
    double s = 1.0 - x2 / (24.0 * 25.0);
    s = 1.0 - (x2 / (22.0 * 23.0)) * s;
    s = 1.0 - (x2 / (20.0 * 21.0)) * s;
    s = 1.0 - (x2 / (18.0 * 19.0)) * s;
    s = 1.0 - (x2 / (16.0 * 17.0)) * s;
    s = 1.0 - (x2 / (14.0 * 15.0)) * s;
    s = 1.0 - (x2 / (12.0 * 13.0)) * s;
    s = 1.0 - (x2 / (10.0 * 11.0)) * s;
    s = 1.0 - (x2 / (8.0 * 9.0)) * s;
    s = 1.0 - (x2 / (6.0 * 7.0)) * s;
    s = 1.0 - (x2 / (4.0 * 5.0)) * s;
    s = 1.0 - (x2 / (2.0 * 3.0)) * s;
    s = x * s;
    // cos x = 1 - x^2/(1.2) (1 - x^2/(3.4) (1 - ...))
    double c = 1.0 - x2 / (23.0 * 24.0);
    c = 1.0 - (x2 / (21.0 * 22.0)) * c;
    c = 1.0 - (x2 / (19.0 * 20.0)) * c;
    c = 1.0 - (x2 / (17.0 * 18.0)) * c;
    c = 1.0 - (x2 / (15.0 * 16.0)) * c;
    c = 1.0 - (x2 / (13.0 * 14.0)) * c;
    c = 1.0 - (x2 / (11.0 * 12.0)) * c;
    c = 1.0 - (x2 / (9.0 * 10.0)) * c;
    c = 1.0 - (x2 / (7.0 * 8.0)) * c;
    c = 1.0 - (x2 / (5.0 * 6.0)) * c;
    c = 1.0 - (x2 / (3.0 * 4.0)) * c;
    c = 1.0 - (x2 / (1.0 * 2.0)) * c;
    return s / c;
}

// mapc2m_cubedsphere + csphere_basic: block coordinates (xc, yc) -> point on the unit sphere.
FCB_HD void cs_map(int block, double xc, double yc, double* xp, double* yp, double* zp)
{
    const double txi = fcb_tan(0.5 * FCB_PI * (xc - 0.5));
    const double teta = fcb_tan(0.5 * FCB_PI * (yc - 0.5));
    const double z = 1.0 / sqrt(txi * txi + teta * teta + 1.0);
    const double a = z * txi, b = z * teta;   // csphere_basic's (xp, yp, zp) = (a, b, z)
    if (block == 0) { *yp = a; *xp = b; *zp = -z; }
    else if (block == 1) { *zp = a; *xp = b; *yp = z; }
    else if (block == 2) { *zp = a; *yp = b; *xp = -z; }
    else if (block == 3) { *xp = a; *yp = b; *zp = z; }
    else if (block == 4) { *xp = a; *zp = b; *yp = -z; }
    else { *yp = a; *zp = b; *xp = z; }
}

// Stream function of solid-body rotation about the unit axis (ax, ay, az) with
// angular speed w: psi = w (axis . x) (the reference's sphere/psi.f uses the y axis).
FCB_HD double cs_psi(const double* axis, double w, double x, double y, double z)
{
    return w * (axis[0] * x + axis[1] * y + axis[2] * z);
}

// The bilinear-quad area of four mapped points (fclaw2d_metric_default_fort.f90:278-332):
// |T_xi x T_eta| at the quad's centre.  p[corner][xyz], corners (0,0),(1,0),(0,1),(1,1).
FCB_HD double cs_quad_area(const double p[4][3])
{
    double txi[3], teta[3];
    for (int m = 0; m < 3; m++) {
        const double a00 = p[0][m];
        const double a01 = p[1][m] - p[0][m];
        const double a10 = p[2][m] - p[0][m];
        const double a11 = ((p[3][m] - p[1][m]) - p[2][m]) + a00;
        txi[m] = a01 + a11 * 0.5;
        teta[m] = a10 + a11 * 0.5;
    }
    const double w0 = txi[1] * teta[2] - txi[2] * teta[1];
    const double w1 = -txi[0] * teta[2] + txi[2] * teta[0];
    const double w2 = txi[0] * teta[1] - txi[1] * teta[0];
    return sqrt(w0 * w0 + w1 * w1 + w2 * w2);
}

}  // namespace fcb
