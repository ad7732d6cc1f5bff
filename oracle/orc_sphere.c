/*
 * orc_sphere.c -- the oracle's cubed-sphere domain (test infrastructure; the
 * product never links it).
 *
 *   mapping     src/mappings/cubedsphere/mapc2m_cubedsphere.f (block permutations, gnomonic
 *               map x = z tan xi, y = z tan eta, z = 1/sqrt(1 + tan^2 xi + tan^2 eta))
 *   area        src/patches/metric/fortran_source2d/fclaw2d_metric_default_fort.f90:110-176
 *               (sum over 2^(maxlevel-level) sub-quads per direction, ii outer, jj inner,
 *               of the bilinear-quad area, get_area_approx/norm_cross :278-332); from fine
 *               :690-755 (cells 0..mx+1 from the children in igrid order) plus the ghost
 *               cells from scratch (compute_area_ghost, is_area_interior :259-266)
 *   aux         applications/clawpack/advection/2d/all/user46_setaux_manifold.f
 *   transforms  src/forestclaw2d.c:609-980 (transform_face, transform_face2): a cell of one
 *               patch in another patch's index space across a block face; children of a
 *               coarse cell in the coarse patch's (x, y) order
 *
 * The connectivity (p4est_connectivity_new_cubed) is not in the reference tree;
 * it is derived from the mapping: block faces whose mapped edges coincide are
 * joined, and the map between the two blocks' coordinates is the plane isometry
 * taking depth beyond one face to depth inside the other.  tan is sin/cos from
 * their Taylor series (to x^25, x^24) so the oracle and the device metric agree
 * bit for bit.
 */
#include <math.h>
#include <stdlib.h>
#include "orc_amr.h"

static const double PI_D = 3.14159265358979311600e+00;

double orc_tan(double x)
{
    const double x2 = x * x;
    double s = 1.0 - x2 / (24.0 * 25.0);
    double c = 1.0 - x2 / (23.0 * 24.0);
    for (int k = 22; k >= 2; k -= 2) s = 1.0 - (x2 / ((double)k * (double)(k + 1))) * s;
    for (int k = 21; k >= 1; k -= 2) c = 1.0 - (x2 / ((double)k * (double)(k + 1))) * c;
    return (x * s) / c;
}

void orc_cs_map(int block, double xc, double yc, double* xp, double* yp, double* zp)
{
    double txi = orc_tan(0.5 * PI_D * (xc - 0.5));
    double teta = orc_tan(0.5 * PI_D * (yc - 0.5));
    double z = 1.0 / sqrt(txi * txi + teta * teta + 1.0);
    double a = z * txi, b = z * teta;
    switch (block) {
    case 0: *yp = a; *xp = b; *zp = -z; break;
    case 1: *zp = a; *xp = b; *yp = z; break;
    case 2: *zp = a; *yp = b; *xp = -z; break;
    case 3: *xp = a; *yp = b; *zp = z; break;
    case 4: *xp = a; *zp = b; *yp = -z; break;
    default: *yp = a; *zp = b; *xp = z; break;
    }
}

static double quad_area(double q[2][2][3])
{
    double txi[3], teta[3];
    for (int m = 0; m < 3; m++) {
        double a00 = q[0][0][m];
        double a01 = q[1][0][m] - q[0][0][m];
        double a10 = q[0][1][m] - q[0][0][m];
        double a11 = q[1][1][m] - q[1][0][m] - q[0][1][m] + a00;
        txi[m] = a01 + a11 * 0.5;
        teta[m] = a10 + a11 * 0.5;
    }
    double w1 = txi[1] * teta[2] - txi[2] * teta[1];
    double w2 = -txi[0] * teta[2] + txi[2] * teta[0];
    double w3 = txi[0] * teta[1] - txi[1] * teta[0];
    return sqrt(w1 * w1 + w2 * w2 + w3 * w3);
}

/* ---------------- connectivity ---------------- */
typedef struct { int nb, nf, flip; int M[2][2]; int c[2]; } cs_face_t;
static cs_face_t CS[6][4];
static int cs_ready = 0;

static void edge_point(int b, int f, double t, double* p)
{
    double x = (f == 0) ? 0.0 : (f == 1) ? 1.0 : t;
    double y = (f == 2) ? 0.0 : (f == 3) ? 1.0 : t;
    orc_cs_map(b, x, y, &p[0], &p[1], &p[2]);
}

static int near3(const double* a, const double* b)
{
    return fabs(a[0] - b[0]) + fabs(a[1] - b[1]) + fabs(a[2] - b[2]) < 1e-9;
}

/* point (x, y) of block b, beyond face f, in the coordinates of the joined block */
static void face_map(int f, const cs_face_t* F, double x, double y, double* x2, double* y2)
{
    double depth, t;
    if (f == 0) { depth = -x; t = y; }
    else if (f == 1) { depth = x - 1.0; t = y; }
    else if (f == 2) { depth = -y; t = x; }
    else { depth = y - 1.0; t = x; }
    double u = F->flip ? 1.0 - t : t;
    if (F->nf == 0) { *x2 = depth; *y2 = u; }
    else if (F->nf == 1) { *x2 = 1.0 - depth; *y2 = u; }
    else if (F->nf == 2) { *x2 = u; *y2 = depth; }
    else { *x2 = u; *y2 = 1.0 - depth; }
}

static void cs_init(void)
{
    if (cs_ready) return;
    for (int b = 0; b < 6; b++)
        for (int f = 0; f < 4; f++) {
            cs_face_t* F = &CS[b][f];
            double p1[3], p3[3];
            edge_point(b, f, 0.25, p1);
            edge_point(b, f, 0.75, p3);
            F->nb = -1;
            for (int b2 = 0; b2 < 6 && F->nb < 0; b2++) {
                if (b2 == b) continue;
                for (int f2 = 0; f2 < 4; f2++) {
                    double q1[3], q3[3];
                    edge_point(b2, f2, 0.25, q1);
                    edge_point(b2, f2, 0.75, q3);
                    if (near3(p1, q1) && near3(p3, q3)) { F->nb = b2; F->nf = f2; F->flip = 0; break; }
                    if (near3(p1, q3) && near3(p3, q1)) { F->nb = b2; F->nf = f2; F->flip = 1; break; }
                }
            }
            if (F->nb < 0) abort();
            double x0, y0, x1, y1, x2, y2;
            face_map(f, F, 0.0, 0.0, &x0, &y0);
            face_map(f, F, 1.0, 0.0, &x1, &y1);
            face_map(f, F, 0.0, 1.0, &x2, &y2);
            F->c[0] = (int)lround(x0); F->c[1] = (int)lround(y0);
            F->M[0][0] = (int)lround(x1 - x0); F->M[1][0] = (int)lround(y1 - y0);
            F->M[0][1] = (int)lround(x2 - x0); F->M[1][1] = (int)lround(y2 - y0);
        }
    cs_ready = 1;
}

int orc_cs_nb(int b, int f) { cs_init(); return CS[b][f].nb; }

/* cell (X, Y) of block b at n cells per side, in the block joined at face f */
static void cs_xform(int b, int f, long n, long X, long Y, long* X2, long* Y2)
{
    const cs_face_t* F = &CS[b][f];
    /* cell centre (X + 1/2)/n through x' = M x + c, back to an index */
    *X2 = (F->M[0][0] * (2 * X + 1) + F->M[0][1] * (2 * Y + 1) + 2 * n * F->c[0] - 1) / 2;
    *Y2 = (F->M[1][0] * (2 * X + 1) + F->M[1][1] * (2 * Y + 1) + 2 * n * F->c[1] - 1) / 2;
}

static int face_between(int a, int b)
{
    for (int f = 0; f < 4; f++) if (CS[a][f].nb == b) return f;
    return -1;
}

int orc_step(const orc_sim* s, int l, int x, int y, int dx, int dy, int* ox, int* oy)
{
    const orc_config* c = &s->cfg;
    if (c->problem != ORC_PROB_SPHERE) {
        *ox = x + dx; *oy = y + dy;
        return (*ox >= 0 && *oy >= 0 && *ox < (c->mi << l) && *oy < (c->mj << l)) ? 1 : 0;
    }
    cs_init();
    long n = 1L << l;
    int b = (int)(x / n);
    long ix = x - b * n + dx, iy = (long)y + dy;
    int outx = ix < 0 || ix >= n, outy = iy < 0 || iy >= n;
    if (!outx && !outy) { *ox = (int)(b * n + ix); *oy = (int)iy; return 1; }
    if (outx && outy) return -1;      /* across a cube corner: no diagonal neighbour */
    int f = outx ? (ix < 0 ? 0 : 1) : (iy < 0 ? 2 : 3);
    long X2, Y2;
    cs_xform(b, f, n, ix, iy, &X2, &Y2);
    *ox = (int)(CS[b][f].nb * n + X2); *oy = (int)Y2;
    return 1;
}

/* block and cell origin of a patch at its own level */
static void origin(const orc_sim* s, const orc_patch* P, int* b, long* X0, long* Y0)
{
    const orc_config* c = &s->cfg;
    if (c->problem != ORC_PROB_SPHERE) { *b = 0; *X0 = (long)P->gx * c->mx; *Y0 = (long)P->gy * c->my; return; }
    long n = 1L << P->level;
    *b = (int)(P->gx / n);
    *X0 = (P->gx - *b * n) * c->mx;
    *Y0 = (long)P->gy * c->my;
}

static void to_block(int b, int b2, long n, long X, long Y, long* X2, long* Y2)
{
    if (b == b2) { *X2 = X; *Y2 = Y; return; }
    cs_init();
    int f = face_between(b, b2);
    if (f < 0) abort();
    cs_xform(b, f, n, X, Y, X2, Y2);
}

void orc_xf_same(const orc_sim* s, const orc_patch* P, const orc_patch* N, int i, int j, int* i2, int* j2)
{
    int b, bn; long X0, Y0, XN, YN, X2, Y2;
    origin(s, P, &b, &X0, &Y0);
    origin(s, N, &bn, &XN, &YN);
    to_block(b, bn, (long)s->cfg.mx << P->level, X0 + i - 1, Y0 + j - 1, &X2, &Y2);
    *i2 = (int)(X2 - XN + 1); *j2 = (int)(Y2 - YN + 1);
}

void orc_xf_half(const orc_sim* s, const orc_patch* C, const orc_patch* F, int ic, int jc, int* i2, int* j2)
{
    int b, bf; long X0, Y0, XF, YF;
    origin(s, C, &b, &X0, &Y0);
    origin(s, F, &bf, &XF, &YF);
    for (int m = 0; m < 4; m++) {
        long X2, Y2;
        to_block(b, bf, (long)s->cfg.mx << (C->level + 1), 2 * (X0 + ic - 1) + (m & 1), 2 * (Y0 + jc - 1) + (m >> 1),
                 &X2, &Y2);
        i2[m] = (int)(X2 - XF + 1); j2[m] = (int)(Y2 - YF + 1);
    }
}

/* ---------------- metric ---------------- */
#define AIDX(i, j, mbc, ax) ((size_t)((j) + (mbc)) * (size_t)(ax) + (size_t)((i) + (mbc)))

static double area_cell(const orc_patch* P, int i, int j, int rfactor)
{
    double dxf = P->dx / rfactor, dyf = P->dy / rfactor;
    double xe = P->xlower + (i - 1) * P->dx, ye = P->ylower + (j - 1) * P->dy;
    double sum = 0.0;
    for (int ii = 0; ii < rfactor; ii++)
        for (int jj = 0; jj < rfactor; jj++) {
            double q[2][2][3];
            for (int a = 0; a < 2; a++)
                for (int c = 0; c < 2; c++)
                    orc_cs_map(P->block, xe + (ii + a) * dxf, ye + (jj + c) * dyf, &q[a][c][0], &q[a][c][1], &q[a][c][2]);
            sum = sum + quad_area(q);
        }
    return sum;
}

void orc_sphere_area(const orc_sim* s, orc_patch* P, int ghost_only)
{
    const orc_config* c = &s->cfg;
    const int mx = c->mx, my = c->my, mbc = c->mbc, ax = mx + 2 * mbc + 2;
    const int rfactor = 1 << (c->maxlevel - P->level);
    for (int j = -mbc; j <= my + mbc + 1; j++)
        for (int i = -mbc; i <= mx + mbc + 1; i++) {
            if (ghost_only && i >= 0 && i <= mx + 1 && j >= 0 && j <= my + 1) continue;
            P->area[AIDX(i, j, mbc, ax)] = area_cell(P, i, j, rfactor);
        }
}

void orc_sphere_area_from_fine(const orc_sim* s, orc_patch* C, const orc_patch* F, int igrid)
{
    const orc_config* c = &s->cfg;
    const int mx = c->mx, my = c->my, mbc = c->mbc, ax = mx + 2 * mbc + 2;
    int ig = igrid % 2, jg = (igrid - ig) / 2;
    int ic_add = ig * mx / 2, jc_add = jg * mx / 2;
    for (int j = 0; j <= my / 2 + 1; j++)
        for (int i = 0; i <= mx / 2 + 1; i++) {
            double sum = 0;
            for (int jj = 1; jj <= 2; jj++)
                for (int ii = 1; ii <= 2; ii++)
                    sum = sum + F->area[AIDX((i - 1) * 2 + ii, (j - 1) * 2 + jj, mbc, ax)];
            C->area[AIDX(i + ic_add, j + jc_add, mbc, ax)] = sum;
        }
}

void orc_sphere_setaux(const orc_sim* s, orc_patch* P)
{
    const orc_config* c = &s->cfg;
    const int mx = c->mx, my = c->my, mbc = c->mbc, nx = s->nx, ny = s->ny, ax = mx + 2 * mbc + 2;
    double axis[3], omega;
    orc_sphere_flow(c, axis, &omega);
    double dxdy = P->dx * P->dy;
    for (int i = 1 - mbc; i <= mx + mbc; i++)
        for (int j = 1 - mbc; j <= my + mbc; j++)
            P->aux[QIDX(i, j, 1, mbc, nx, ny)] = P->area[AIDX(i, j, mbc, ax)] / dxdy;
    /* psi at node (i, j) = the lower-left corner of cell (i, j) */
#define PSI_NODE(ii, jj, out) do { double x_, y_, z_; \
        orc_cs_map(P->block, P->xlower + ((ii) - 1) * P->dx, P->ylower + ((jj) - 1) * P->dy, &x_, &y_, &z_); \
        out = omega * (axis[0] * x_ + axis[1] * y_ + axis[2] * z_); } while (0)
    for (int i = 1 - mbc; i <= mx + mbc; i++)
        for (int j = 1 - mbc; j <= my + mbc; j++) {
            double p1, p2;
            PSI_NODE(i, j + 1, p1);
            PSI_NODE(i, j, p2);
            P->aux[QIDX(i, j, 2, mbc, nx, ny)] = (p1 - p2) / P->dy;
        }
    for (int j = 1 - mbc; j <= my + mbc; j++)
        for (int i = 1 - mbc; i <= mx + mbc; i++) {
            double p1, p2;
            PSI_NODE(i + 1, j, p1);
            PSI_NODE(i, j, p2);
            P->aux[QIDX(i, j, 3, mbc, nx, ny)] = -((p1 - p2) / P->dx);
        }
#undef PSI_NODE
}

void orc_sphere_flow(const orc_config* c, double* axis, double* omega)
{
    double n = sqrt(c->pdata[0] * c->pdata[0] + c->pdata[1] * c->pdata[1] + c->pdata[2] * c->pdata[2]);
    axis[0] = c->pdata[0] / n; axis[1] = c->pdata[1] / n; axis[2] = c->pdata[2] / n;
    *omega = c->pdata[3];
}
