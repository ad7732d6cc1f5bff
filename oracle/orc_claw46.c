/*
 * orc_claw46.c -- oracle restatement of the clawpack 4.6 patch update (test infrastructure).
 *
 * Follows, step for step and in Fortran evaluation order:
 *   src/solvers/fc2d_clawpack4.6/fortran_source/clawpack46_step2_wrap.f:1-127  (q update :107-125)
 *   src/solvers/fc2d_clawpack4.6/fortran_source/clawpack46_step2.f:5-237       (sweeps)
 *   src/solvers/fc2d_clawpack4.6/fortran_source/clawpack46_step2.f:242-310     (fix_corners)
 *   src/solvers/fc2d_clawpack4.6/fortran_source/clawpack46_flux2.f:4-228
 *   src/solvers/fc2d_clawpack4.6/fortran_source/clawpack46_flux2fw.f:4-243
 *   src/solvers/fc2d_clawpack4.6/fortran_source/clawpack46_inlinelimiter.f:4-118
 *   src/solvers/fc2d_clawpack4.6/fortran_source/clawpack46_bc2_default.f:1-213
 *   src/solvers/fc2d_clawpack4.6/fortran_source/clawpack46_time_sync.f:37-226
 * and the app Riemann solvers cited beside each function.
 * Compiled with -ffp-contract=off; see oracle.h for the parity status.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "orc_internal.h"

/* ------------------------------------------------------------------------- */
/* Limiter: clawpack46_inlinelimiter.f:59-104                                  */
/* ------------------------------------------------------------------------- */
static double dmax1(double a, double b) { return a > b ? a : b; }
static double dmin1(double a, double b) { return a < b ? a : b; }

double orc_limiter_phi(int mthlim, double r)
{
    double c, th;
    switch (mthlim) {
    case 1: return dmax1(0.0, dmin1(1.0, r));                                   /* minmod  :293 */
    case 2: return dmax1(dmax1(0.0, dmin1(1.0, 2.0 * r)), dmin1(2.0, r));       /* superbee:300 */
    case 3: return (r + fabs(r)) / (1.0 + fabs(r));                             /* van Leer:307 */
    case 4:                                                                     /* MC      :314-315 */
        c = (1.0 + r) / 2.0;
        return dmax1(0.0, dmin1(dmin1(c, 2.0), 2.0 * r));
    case 5: return r;                                                           /* Beam-Warming :322 */
    case 6:                                                                     /* gen. minmod :329-330 */
        th = (double)1.3f;   /* single-precision literal assigned to a double */
        return dmax1(0.0, dmin1(dmin1(th * r, (1 + r) / 2.0), th));
    default: return 1.0;
    }
}

/* clawpack46_inlinelimiter.f:267-343.  wave is (1-mbc:maxm+mbc, meqn, mwaves). */
static void inlinelimiter(int maxm, int meqn, int mwaves, int mbc, int mx,
                          double* wave, const double* s, const int* mthlim)
{
    const int L = maxm + 2 * mbc;
    for (int mw = 1; mw <= mwaves; mw++) {
        if (mthlim[mw - 1] == 0) continue;
        double dotr = 0.0, dotl;
        for (int i = 0; i <= mx + 1; i++) {
            double wnorm2 = 0.0;
            dotl = dotr;
            dotr = 0.0;
            for (int m = 1; m <= meqn; m++) {
                double w = wave[I1(i) + (m - 1) * L + (mw - 1) * L * meqn];
                double wn = wave[I1(i + 1) + (m - 1) * L + (mw - 1) * L * meqn];
                wnorm2 = wnorm2 + w * w;
                dotr = dotr + w * wn;
            }
            if (i == 0) continue;
            if (wnorm2 == 0.0) continue;
            double r = (s[I1(i) + (mw - 1) * L] > 0.0) ? dotl / wnorm2 : dotr / wnorm2;
            double wl = orc_limiter_phi(mthlim[mw - 1], r);
            for (int m = 1; m <= meqn; m++)
                wave[I1(i) + (m - 1) * L + (mw - 1) * L * meqn] =
                    wl * wave[I1(i) + (m - 1) * L + (mw - 1) * L * meqn];
        }
    }
}

/* ------------------------------------------------------------------------- */
/* Riemann solvers                                                             */
/* ------------------------------------------------------------------------- */

/* applications/clawpack/advection/2d/all/clawpack46_rpn2adv.f (whole file). */
static void rpn2_adv(orc_rpctx* ctx, int ixy, int maxm, int meqn, int mwaves, int maux, int mbc, int mx,
                     const double* ql, const double* qr, const double* auxl, const double* auxr,
                     double* wave, double* s, double* amdq, double* apdq)
{
    (void)ctx; (void)maux; (void)auxr;
    const int L = maxm + 2 * mbc;
    const int iface = ixy;
    for (int i = 2 - mbc; i <= mx + mbc; i++) {
        for (int mq = 1; mq <= meqn; mq++) {
            double delta = ql[I1(i) + (mq - 1) * L] - qr[I1(i - 1) + (mq - 1) * L];
            for (int mw = 1; mw <= mwaves; mw++)
                wave[I1(i) + (mq - 1) * L + (mw - 1) * L * meqn] = delta;
        }
        for (int mw = 1; mw <= mwaves; mw++)
            s[I1(i) + (mw - 1) * L] = auxl[I1(i) + (iface - 1) * L];
        for (int mq = 1; mq <= meqn; mq++) {
            double am = 0.0, ap = 0.0;
            for (int mw = 1; mw <= mwaves; mw++) {
                double sw = s[I1(i) + (mw - 1) * L];
                double w = wave[I1(i) + (mq - 1) * L + (mw - 1) * L * meqn];
                am = am + dmin1(sw, 0.0) * w;
                ap = ap + dmax1(sw, 0.0) * w;
            }
            amdq[I1(i) + (mq - 1) * L] = am;
            apdq[I1(i) + (mq - 1) * L] = ap;
        }
    }
}

/* applications/clawpack/advection/2d/all/clawpack46_rpt2adv.f (whole file). */
static void rpt2_adv(orc_rpctx* ctx, int ixy, int maxm, int meqn, int mwaves, int maux, int mbc, int mx,
                     const double* ql, const double* qr, const double* aux1, const double* aux2,
                     const double* aux3, int imp, const double* asdq, double* bmasdq, double* bpasdq)
{
    (void)ctx; (void)mwaves; (void)maux; (void)ql; (void)qr; (void)aux1;
    const int L = maxm + 2 * mbc;
    const int kv = 3 - ixy;
    for (int i = 2 - mbc; i <= mx + mbc; i++) {
        int i1 = i - 2 + imp;
        for (int mq = 1; mq <= meqn; mq++) {
            bmasdq[I1(i) + (mq - 1) * L] = dmin1(aux2[I1(i1) + (kv - 1) * L], 0.0) * asdq[I1(i) + (mq - 1) * L];
            bpasdq[I1(i) + (mq - 1) * L] = dmax1(aux3[I1(i1) + (kv - 1) * L], 0.0) * asdq[I1(i) + (mq - 1) * L];
        }
    }
}

/* applications/clawpack/advection/2d/all/clawpack46_rpn2adv_manifold.f: speed aux(i, 1 + ixy). */
static void rpn2_adv_manifold(orc_rpctx* ctx, int ixy, int maxm, int meqn, int mwaves, int maux, int mbc, int mx,
                              const double* ql, const double* qr, const double* auxl, const double* auxr,
                              double* wave, double* s, double* amdq, double* apdq)
{
    (void)ctx; (void)maux; (void)auxr; (void)mwaves;
    const int L = maxm + 2 * mbc;
    for (int i = 2 - mbc; i <= mx + mbc; i++) {
        for (int m = 1; m <= meqn; m++)
            wave[I1(i) + (m - 1) * L] = ql[I1(i) + (m - 1) * L] - qr[I1(i - 1) + (m - 1) * L];
        s[I1(i)] = auxl[I1(i) + ixy * L];
        for (int m = 1; m <= meqn; m++) {
            amdq[I1(i) + (m - 1) * L] = dmin1(s[I1(i)], 0.0) * wave[I1(i) + (m - 1) * L];
            apdq[I1(i) + (m - 1) * L] = dmax1(s[I1(i)], 0.0) * wave[I1(i) + (m - 1) * L];
        }
    }
}

/* applications/clawpack/advection/2d/all/clawpack46_rpt2adv_manifold.f: aux(i1, iface + 1), iface = 3 - ixy. */
static void rpt2_adv_manifold(orc_rpctx* ctx, int ixy, int maxm, int meqn, int mwaves, int maux, int mbc, int mx,
                              const double* ql, const double* qr, const double* aux1, const double* aux2,
                              const double* aux3, int imp, const double* asdq, double* bmasdq, double* bpasdq)
{
    (void)ctx; (void)mwaves; (void)maux; (void)ql; (void)qr; (void)aux1;
    const int L = maxm + 2 * mbc;
    const int iface = 3 - ixy;
    for (int i = 2 - mbc; i <= mx + mbc; i++) {
        int i1 = i - 2 + imp;
        for (int m = 1; m <= meqn; m++) {
            bmasdq[I1(i) + (m - 1) * L] = dmin1(aux2[I1(i1) + iface * L], 0.0) * asdq[I1(i) + (m - 1) * L];
            bpasdq[I1(i) + (m - 1) * L] = dmax1(aux3[I1(i1) + iface * L], 0.0) * asdq[I1(i) + (m - 1) * L];
        }
    }
}

/* applications/clawpack/shallow/2d/rp/clawpack46_rpn2.f:1-247 (Roe + Harten-Hyman fix).
 * The Roe averages are kept in ctx (the Fortran common block /comroe/). */
static void rpn2_sw_roe(orc_rpctx* ctx, int ixy, int maxm, int meqn, int mwaves, int maux, int mbc, int mx,
                        const double* ql, const double* qr, const double* auxl, const double* auxr,
                        double* wave, double* s, double* amdq, double* apdq)
{
    (void)maux; (void)auxl; (void)auxr;
    const int L = maxm + 2 * mbc;
    const double grav = ctx->grav;
    const int mu = (ixy == 1) ? 2 : 3;
    const int mv = (ixy == 1) ? 3 : 2;
#define QL(i, m) ql[I1(i) + ((m) - 1) * L]
#define QR(i, m) qr[I1(i) + ((m) - 1) * L]
#define WAVE(i, m, mw) wave[I1(i) + ((m) - 1) * L + ((mw) - 1) * L * meqn]
#define S(i, mw) s[I1(i) + ((mw) - 1) * L]
    /* :91-99 */
    for (int i = 2 - mbc; i <= mx + mbc; i++) {
        ctx->h[I1(i)] = (QR(i - 1, 1) + QL(i, 1)) / 2.0;
        double hsqrtl = sqrt(QR(i - 1, 1));
        double hsqrtr = sqrt(QL(i, 1));
        double hsq2 = hsqrtl + hsqrtr;
        ctx->u[I1(i)] = (QR(i - 1, mu) / hsqrtl + QL(i, mu) / hsqrtr) / hsq2;
        ctx->v[I1(i)] = (QR(i - 1, mv) / hsqrtl + QL(i, mv) / hsqrtr) / hsq2;
        ctx->a[I1(i)] = sqrt(grav * ctx->h[I1(i)]);
    }
    /* :105-129 */
    for (int i = 2 - mbc; i <= mx + mbc; i++) {
        double u = ctx->u[I1(i)], v = ctx->v[I1(i)], a = ctx->a[I1(i)];
        double d1 = QL(i, 1) - QR(i - 1, 1);
        double d2 = QL(i, mu) - QR(i - 1, mu);
        double d3 = QL(i, mv) - QR(i - 1, mv);
        double a1 = ((u + a) * d1 - d2) / (2.0 * a);
        double a2 = -(v * d1) + d3;
        double a3 = (-((u - a) * d1) + d2) / (2.0 * a);
        WAVE(i, 1, 1) = a1;
        WAVE(i, mu, 1) = a1 * (u - a);
        WAVE(i, mv, 1) = a1 * v;
        S(i, 1) = u - a;
        WAVE(i, 1, 2) = 0.0;
        WAVE(i, mu, 2) = 0.0;
        WAVE(i, mv, 2) = a2;
        S(i, 2) = u;
        WAVE(i, 1, 3) = a3;
        WAVE(i, mu, 3) = a3 * (u + a);
        WAVE(i, mv, 3) = a3 * v;
        S(i, 3) = u + a;
    }
    /* entropy fix, :170-229 */
    for (int i = 2 - mbc; i <= mx + mbc; i++) {
        double* am = &amdq[I1(i)];
        double him1 = QR(i - 1, 1);
        double s0 = QR(i - 1, mu) / him1 - sqrt(grav * him1);
        if (s0 > 0.0 && S(i, 1) > 0.0) {
            for (int m = 1; m <= 3; m++) am[(m - 1) * L] = 0.0;
            continue;
        }
        double h1 = QR(i - 1, 1) + WAVE(i, 1, 1);
        double hu1 = QR(i - 1, mu) + WAVE(i, mu, 1);
        double s1 = hu1 / h1 - sqrt(grav * h1);
        double sfract;
        if (s0 < 0.0 && s1 > 0.0) sfract = s0 * ((s1 - S(i, 1)) / (s1 - s0));
        else if (S(i, 1) < 0.0) sfract = S(i, 1);
        else sfract = 0.0;
        for (int m = 1; m <= 3; m++) am[(m - 1) * L] = sfract * WAVE(i, m, 1);
        if (S(i, 2) > 0.0) continue;
        for (int m = 1; m <= 3; m++) am[(m - 1) * L] = am[(m - 1) * L] + S(i, 2) * WAVE(i, m, 2);
        double hi = QL(i, 1);
        double s03 = QL(i, mu) / hi + sqrt(grav * hi);
        double h3 = QL(i, 1) - WAVE(i, 1, 3);
        double hu3 = QL(i, mu) - WAVE(i, mu, 3);
        double s3 = hu3 / h3 + sqrt(grav * h3);
        if (s3 < 0.0 && s03 > 0.0) sfract = s3 * ((s03 - S(i, 3)) / (s03 - s3));
        else if (S(i, 3) < 0.0) sfract = S(i, 3);
        else continue;
        for (int m = 1; m <= 3; m++) am[(m - 1) * L] = am[(m - 1) * L] + sfract * WAVE(i, m, 3);
    }
    /* :234-242 */
    for (int m = 1; m <= 3; m++)
        for (int i = 2 - mbc; i <= mx + mbc; i++) {
            double df = 0.0;
            for (int mw = 1; mw <= mwaves; mw++) df = df + S(i, mw) * WAVE(i, m, mw);
            apdq[I1(i) + (m - 1) * L] = df - amdq[I1(i) + (m - 1) * L];
        }
#undef QL
#undef QR
#undef WAVE
#undef S
}

/* applications/clawpack/shallow/2d/rp/clawpack46_rpt2.f:248-321, reading the Roe
 * averages left in ctx by rpn2_sw_roe (common /comroe/). */
static void rpt2_sw_roe(orc_rpctx* ctx, int ixy, int maxm, int meqn, int mwaves, int maux, int mbc, int mx,
                        const double* ql, const double* qr, const double* aux1, const double* aux2,
                        const double* aux3, int imp, const double* asdq, double* bmasdq, double* bpasdq)
{
    (void)maux; (void)ql; (void)qr; (void)aux1; (void)aux2; (void)aux3; (void)imp;
    const int L = maxm + 2 * mbc;
    const int mu = (ixy == 1) ? 2 : 3;
    const int mv = (ixy == 1) ? 3 : 2;
    for (int i = 2 - mbc; i <= mx + mbc; i++) {
        double u = ctx->u[I1(i)], v = ctx->v[I1(i)], a = ctx->a[I1(i)];
        double q1 = asdq[I1(i)], qmu = asdq[I1(i) + (mu - 1) * L], qmv = asdq[I1(i) + (mv - 1) * L];
        double a1 = ((v + a) * q1 - qmv) / (2.0 * a);
        double a2 = qmu - u * q1;
        double a3 = (-((v - a) * q1) + qmv) / (2.0 * a);
        double wb[3][3];   /* wb[m-1][mw-1] */
        double sb[3];
        wb[0][0] = a1; wb[mu - 1][0] = a1 * u; wb[mv - 1][0] = a1 * (v - a); sb[0] = v - a;
        wb[0][1] = 0.0; wb[mu - 1][1] = a2; wb[mv - 1][1] = 0.0; sb[1] = v;
        wb[0][2] = a3; wb[mu - 1][2] = a3 * u; wb[mv - 1][2] = a3 * (v + a); sb[2] = v + a;
        for (int m = 1; m <= meqn; m++) {
            double bm = 0.0, bp = 0.0;
            for (int mw = 1; mw <= mwaves; mw++) {
                bm = bm + dmin1(sb[mw - 1], 0.0) * wb[m - 1][mw - 1];
                bp = bp + dmax1(sb[mw - 1], 0.0) * wb[m - 1][mw - 1];
            }
            bmasdq[I1(i) + (m - 1) * L] = bm;
            bpasdq[I1(i) + (m - 1) * L] = bp;
        }
    }
}

/* An application's own device solver restated in the 1-D array form: the radial
 * acoustics pair of applications/cudaclaw/acoustics/2d/radial/user_cuda/rpn2acoustics.cu:30-68
 * (waves -alpha1 z / alpha1 and alpha2 z / alpha2 with speeds -c, c) and
 * rpt2acoustics.cu:88-118, with c = sqrt(bulk/rho), z = c rho (setprob_cuda, :10-27).
 * The left state of interface i is qr(i-1), the right one ql(i). */
static void acoustics_cz(const orc_rpctx* ctx, double* c, double* z)
{
    const double rho = ctx->cfg->pdata[24], bulk = ctx->cfg->pdata[25];
    *c = sqrt(bulk / rho);
    *z = *c * rho;
}

static void rpn2_acoustics(orc_rpctx* ctx, int ixy, int maxm, int meqn, int mwaves, int maux, int mbc, int mx,
                           const double* ql, const double* qr, const double* auxl, const double* auxr,
                           double* wave, double* s, double* amdq, double* apdq)
{
    (void)mwaves; (void)maux; (void)auxl; (void)auxr;
    const int L = maxm + 2 * mbc;
    const int mu = ixy, mv = 3 - ixy;                 /* 0-based: 1 + idir, 2 - idir */
    double c, z;
    acoustics_cz(ctx, &c, &z);
    for (int i = 2 - mbc; i <= mx + mbc; i++) {
        double qlv[3], qrv[3], w0[3], w1[3];
        for (int m = 0; m < 3; m++) { qlv[m] = qr[I1(i - 1) + m * L]; qrv[m] = ql[I1(i) + m * L]; }
        const double s0 = -c, s1 = c;
        const double d0 = qrv[0] - qlv[0], d1 = qrv[mu] - qlv[mu];
        const double alpha1 = (-d0 + z * d1) / (2.0 * z);
        const double alpha2 = (d0 + z * d1) / (2.0 * z);
        w0[0] = -alpha1 * z; w0[mu] = alpha1; w0[mv] = 0;
        w1[0] = alpha2 * z;  w1[mu] = alpha2; w1[mv] = 0;
        s[I1(i)] = s0; s[I1(i) + L] = s1;
        for (int m = 0; m < meqn; m++) {
            wave[I1(i) + m * L] = w0[m];
            wave[I1(i) + m * L + L * meqn] = w1[m];
            amdq[I1(i) + m * L] = s0 * w0[m];
            apdq[I1(i) + m * L] = s1 * w1[m];
        }
    }
}

static void rpt2_acoustics(orc_rpctx* ctx, int ixy, int maxm, int meqn, int mwaves, int maux, int mbc, int mx,
                           const double* ql, const double* qr, const double* aux1, const double* aux2,
                           const double* aux3, int imp, const double* asdq, double* bmasdq, double* bpasdq)
{
    (void)mwaves; (void)maux; (void)ql; (void)qr; (void)aux1; (void)aux2; (void)aux3; (void)imp; (void)meqn;
    const int L = maxm + 2 * mbc;
    const int mu = ixy, mv = 3 - ixy;
    double c, z;
    acoustics_cz(ctx, &c, &z);
    for (int i = 2 - mbc; i <= mx + mbc; i++) {
        const double d0 = asdq[I1(i)], d1 = asdq[I1(i) + mv * L];
        const double alpha1 = (-d0 + z * d1) / (2.0 * z);
        const double alpha2 = (d0 + z * d1) / (2.0 * z);
        bmasdq[I1(i)] = c * alpha1 * z; bmasdq[I1(i) + mu * L] = 0; bmasdq[I1(i) + mv * L] = -c * alpha1;
        bpasdq[I1(i)] = c * alpha2 * z; bpasdq[I1(i) + mu * L] = 0; bpasdq[I1(i) + mv * L] = c * alpha2;
    }
}

void orc_rp_select(int rp, orc_rpn2_t* rpn2, orc_rpt2_t* rpt2)
{
    switch (rp) {
    case ORC_RP_ADVECTION: *rpn2 = rpn2_adv; *rpt2 = rpt2_adv; break;
    case ORC_RP_SW_ROE:    *rpn2 = rpn2_sw_roe; *rpt2 = rpt2_sw_roe; break;
    case ORC_RP_SW_FWAVE:  *rpn2 = orc_rpn2_fwave; *rpt2 = orc_rpt2_fwave; break;
    case ORC_RP_EULER_EXACT: *rpn2 = orc_rpn2_euler; *rpt2 = orc_rpt2_euler; break;
    case ORC_RP_ADVECTION_MANIFOLD: *rpn2 = rpn2_adv_manifold; *rpt2 = rpt2_adv_manifold; break;
    case ORC_RP_ACOUSTICS: *rpn2 = rpn2_acoustics; *rpt2 = rpt2_acoustics; break;
    default: *rpn2 = NULL; *rpt2 = NULL; break;
    }
}

/* ------------------------------------------------------------------------- */
/* flux2: clawpack46_flux2.f:4-228                                            */
/* ------------------------------------------------------------------------- */
static void flux2(orc_rpctx* ctx, orc_rpn2_t rpn2, orc_rpt2_t rpt2,
                  int ixy, int maxm, int meqn, int maux, int mbc, int mx,
                  const double* q1d, double* dtdx1d, const double* aux1, const double* aux2,
                  const double* aux3, double* faddm, double* faddp, double* gaddm, double* gaddp,
                  double* cfl1d, double* wave, double* s, double* amdq, double* apdq,
                  double* cqxx, double* bmasdq, double* bpasdq,
                  int mwaves, const int* method, const int* mthlim)
{
    const int L = maxm + 2 * mbc;
    int limit = 0;
    for (int mw = 1; mw <= mwaves; mw++) if (mthlim[mw - 1] > 0) limit = 1;
    /* :101-110 */
    for (int jside = 1; jside <= 2; jside++)
        for (int m = 1; m <= meqn; m++)
            for (int i = 1 - mbc; i <= mx + mbc; i++) {
                faddm[I1(i) + (m - 1) * L] = 0.0;
                faddp[I1(i) + (m - 1) * L] = 0.0;
                gaddm[I1(i) + (m - 1) * L + (jside - 1) * L * meqn] = 0.0;
                gaddp[I1(i) + (m - 1) * L + (jside - 1) * L * meqn] = 0.0;
            }
    /* :116 */
    rpn2(ctx, ixy, maxm, meqn, mwaves, maux, mbc, mx, q1d, q1d, aux2, aux2, wave, s, amdq, apdq);
    /* :121-126 */
    for (int i = 2 - mbc; i <= mx + mbc - 1; i++)
        for (int m = 1; m <= meqn; m++) {
            faddp[I1(i) + (m - 1) * L] = faddp[I1(i) + (m - 1) * L] - apdq[I1(i) + (m - 1) * L];
            faddm[I1(i) + (m - 1) * L] = faddm[I1(i) + (m - 1) * L] + amdq[I1(i) + (m - 1) * L];
        }
    /* :129-137 */
    double cfl = 0.0;
    for (int mw = 1; mw <= mwaves; mw++)
        for (int i = 1; i <= mx + 1; i++) {
            double sv = s[I1(i) + (mw - 1) * L];
            cfl = dmax1(dmax1(cfl, dtdx1d[I1(i)] * sv), -(dtdx1d[I1(i - 1)] * sv));
        }
    *cfl1d = cfl;
    /* :139-170 */
    if (method[1] == 2) {
        if (limit) inlinelimiter(maxm, meqn, mwaves, mbc, mx, wave, s, mthlim);
        for (int i = 2 - mbc; i <= mx + mbc; i++) {
            double dtdxave = 0.5 * (dtdx1d[I1(i - 1)] + dtdx1d[I1(i)]);
            for (int m = 1; m <= meqn; m++) {
                double c = 0.0;
                for (int mw = 1; mw <= mwaves; mw++) {
                    double sa = fabs(s[I1(i) + (mw - 1) * L]);
                    c = c + sa * (1.0 - sa * dtdxave) * wave[I1(i) + (m - 1) * L + (mw - 1) * L * meqn];
                }
                cqxx[I1(i) + (m - 1) * L] = c;
                faddm[I1(i) + (m - 1) * L] = faddm[I1(i) + (m - 1) * L] + 0.5 * c;
                faddp[I1(i) + (m - 1) * L] = faddp[I1(i) + (m - 1) * L] + 0.5 * c;
            }
        }
    }
    /* :172-225 */
    if (method[2] > 0) {
        if (method[1] > 1 && method[2] == 2) {
            for (int i = 2 - mbc; i <= mx + mbc - 1; i++)
                for (int m = 1; m <= meqn; m++) {
                    amdq[I1(i) + (m - 1) * L] = amdq[I1(i) + (m - 1) * L] + cqxx[I1(i) + (m - 1) * L];
                    apdq[I1(i) + (m - 1) * L] = apdq[I1(i) + (m - 1) * L] - cqxx[I1(i) + (m - 1) * L];
                }
        }
        rpt2(ctx, ixy, maxm, meqn, mwaves, maux, mbc, mx, q1d, q1d, aux1, aux2, aux3, 1, amdq, bmasdq, bpasdq);
        for (int m = 1; m <= meqn; m++)
            for (int i = 2 - mbc; i <= mx + mbc; i++) {
                double g = 0.5 * dtdx1d[I1(i - 1)] * bmasdq[I1(i) + (m - 1) * L];
                gaddm[I1(i - 1) + (m - 1) * L] = gaddm[I1(i - 1) + (m - 1) * L] - g;
                gaddp[I1(i - 1) + (m - 1) * L] = gaddp[I1(i - 1) + (m - 1) * L] - g;
                g = 0.5 * dtdx1d[I1(i - 1)] * bpasdq[I1(i) + (m - 1) * L];
                gaddm[I1(i - 1) + (m - 1) * L + L * meqn] = gaddm[I1(i - 1) + (m - 1) * L + L * meqn] - g;
                gaddp[I1(i - 1) + (m - 1) * L + L * meqn] = gaddp[I1(i - 1) + (m - 1) * L + L * meqn] - g;
            }
        rpt2(ctx, ixy, maxm, meqn, mwaves, maux, mbc, mx, q1d, q1d, aux1, aux2, aux3, 2, apdq, bmasdq, bpasdq);
        for (int m = 1; m <= meqn; m++)
            for (int i = 2 - mbc; i <= mx + mbc; i++) {
                double g = 0.5 * dtdx1d[I1(i)] * bmasdq[I1(i) + (m - 1) * L];
                gaddm[I1(i) + (m - 1) * L] = gaddm[I1(i) + (m - 1) * L] - g;
                gaddp[I1(i) + (m - 1) * L] = gaddp[I1(i) + (m - 1) * L] - g;
                g = 0.5 * dtdx1d[I1(i)] * bpasdq[I1(i) + (m - 1) * L];
                gaddm[I1(i) + (m - 1) * L + L * meqn] = gaddm[I1(i) + (m - 1) * L + L * meqn] - g;
                gaddp[I1(i) + (m - 1) * L + L * meqn] = gaddp[I1(i) + (m - 1) * L + L * meqn] - g;
            }
    }
}

/* ------------------------------------------------------------------------- */
/* flux2fw: clawpack46_flux2fw.f:4-243 (f-wave variant)                       */
/* ------------------------------------------------------------------------- */
static void flux2fw(orc_rpctx* ctx, orc_rpn2_t rpn2, orc_rpt2_t rpt2,
                    int ixy, int maxm, int meqn, int maux, int mbc, int mx,
                    const double* q1d, double* dtdx1d, const double* aux1, const double* aux2,
                    const double* aux3, double* faddm, double* faddp, double* gaddm, double* gaddp,
                    double* cfl1d, double* fwave, double* s, double* amdq, double* apdq,
                    double* cqxx, double* bmasdq, double* bpasdq,
                    int mwaves, const int* method, const int* mthlim)
{
    const int L = maxm + 2 * mbc;
    int limit = 0;
    for (int mw = 1; mw <= mwaves; mw++) if (mthlim[mw - 1] > 0) limit = 1;
    for (int jside = 1; jside <= 2; jside++)
        for (int m = 1; m <= meqn; m++)
            for (int i = 1 - mbc; i <= mx + mbc; i++) {
                faddm[I1(i) + (m - 1) * L] = 0.0;
                faddp[I1(i) + (m - 1) * L] = 0.0;
                gaddm[I1(i) + (m - 1) * L + (jside - 1) * L * meqn] = 0.0;
                gaddp[I1(i) + (m - 1) * L + (jside - 1) * L * meqn] = 0.0;
            }
    rpn2(ctx, ixy, maxm, meqn, mwaves, maux, mbc, mx, q1d, q1d, aux2, aux2, fwave, s, amdq, apdq);
    for (int i = 1; i <= mx + 1; i++)
        for (int m = 1; m <= meqn; m++) {
            faddp[I1(i) + (m - 1) * L] = faddp[I1(i) + (m - 1) * L] - apdq[I1(i) + (m - 1) * L];
            faddm[I1(i) + (m - 1) * L] = faddm[I1(i) + (m - 1) * L] + amdq[I1(i) + (m - 1) * L];
        }
    double cfl = 0.0;
    for (int mw = 1; mw <= mwaves; mw++)
        for (int i = 1; i <= mx + 1; i++) {
            double sv = s[I1(i) + (mw - 1) * L];
            cfl = dmax1(dmax1(cfl, dtdx1d[I1(i)] * sv), -(dtdx1d[I1(i - 1)] * sv));
        }
    *cfl1d = cfl;
    if (method[1] != 1) {
        if (limit) inlinelimiter(maxm, meqn, mwaves, mbc, mx, fwave, s, mthlim);
        for (int i = 1; i <= mx + 1; i++) {
            double dtdxave = 0.5 * (dtdx1d[I1(i - 1)] + dtdx1d[I1(i)]);
            for (int m = 1; m <= meqn; m++) {
                double c = 0.0;
                for (int mw = 1; mw <= mwaves; mw++) {
                    double sv = s[I1(i) + (mw - 1) * L];
                    c = c + copysign(1.0, sv) * (1.0 - fabs(sv) * dtdxave) *
                                fwave[I1(i) + (m - 1) * L + (mw - 1) * L * meqn];
                }
                cqxx[I1(i) + (m - 1) * L] = c;
                faddm[I1(i) + (m - 1) * L] = faddm[I1(i) + (m - 1) * L] + 0.5 * c;
                faddp[I1(i) + (m - 1) * L] = faddp[I1(i) + (m - 1) * L] + 0.5 * c;
            }
        }
    }
    if (method[2] == 0) return;
    if (method[1] > 1 && method[2] == 2) {
        for (int i = 1; i <= mx + 1; i++)
            for (int m = 1; m <= meqn; m++) {
                amdq[I1(i) + (m - 1) * L] = amdq[I1(i) + (m - 1) * L] + cqxx[I1(i) + (m - 1) * L];
                apdq[I1(i) + (m - 1) * L] = apdq[I1(i) + (m - 1) * L] - cqxx[I1(i) + (m - 1) * L];
            }
    }
    rpt2(ctx, ixy, maxm, meqn, mwaves, maux, mbc, mx, q1d, q1d, aux1, aux2, aux3, 1, amdq, bmasdq, bpasdq);
    for (int m = 1; m <= meqn; m++)
        for (int i = 1; i <= mx + 1; i++) {
            double g = 0.5 * dtdx1d[I1(i - 1)] * bmasdq[I1(i) + (m - 1) * L];
            gaddm[I1(i - 1) + (m - 1) * L] = gaddm[I1(i - 1) + (m - 1) * L] - g;
            gaddp[I1(i - 1) + (m - 1) * L] = gaddp[I1(i - 1) + (m - 1) * L] - g;
            g = 0.5 * dtdx1d[I1(i - 1)] * bpasdq[I1(i) + (m - 1) * L];
            gaddm[I1(i - 1) + (m - 1) * L + L * meqn] = gaddm[I1(i - 1) + (m - 1) * L + L * meqn] - g;
            gaddp[I1(i - 1) + (m - 1) * L + L * meqn] = gaddp[I1(i - 1) + (m - 1) * L + L * meqn] - g;
        }
    rpt2(ctx, ixy, maxm, meqn, mwaves, maux, mbc, mx, q1d, q1d, aux1, aux2, aux3, 2, apdq, bmasdq, bpasdq);
    for (int m = 1; m <= meqn; m++)
        for (int i = 1; i <= mx + 1; i++) {
            double g = 0.5 * dtdx1d[I1(i - 1)] * bmasdq[I1(i) + (m - 1) * L];
            gaddm[I1(i) + (m - 1) * L] = gaddm[I1(i) + (m - 1) * L] - g;
            gaddp[I1(i) + (m - 1) * L] = gaddp[I1(i) + (m - 1) * L] - g;
            g = 0.5 * dtdx1d[I1(i - 1)] * bpasdq[I1(i) + (m - 1) * L];
            gaddm[I1(i) + (m - 1) * L + L * meqn] = gaddm[I1(i) + (m - 1) * L + L * meqn] - g;
            gaddp[I1(i) + (m - 1) * L + L * meqn] = gaddp[I1(i) + (m - 1) * L + L * meqn] - g;
        }
}

/* ------------------------------------------------------------------------- */
/* fix_corners: clawpack46_step2.f:242-310 (cubed-sphere 3-patch block corners) */
/* ------------------------------------------------------------------------- */
static void fix_corners(int mx, int my, int mbc, int meqn, double* q, int sweep_dir, const int* bcc)
{
    const int nx = mx + 2 * mbc, ny = my + 2 * mbc;
    double ihat[4] = {0.5, mx + 0.5, 0.5, mx + 0.5};
    double jhat[4] = {0.5, 0.5, my + 0.5, my + 0.5};
    for (int k = 0; k <= 3; k++) {
        if (bcc[k] != 3) continue;
        int use_b = (sweep_dir == 0 && (k == 0 || k == 3)) || (sweep_dir == 1 && (k == 1 || k == 2));
        for (int ibc = 1; ibc <= mbc; ibc++)
            for (int jbc = 1; jbc <= mbc; jbc++) {
                int i1 = (k == 0 || k == 2) ? 1 - ibc : mx + ibc;
                int j1 = (k == 0 || k == 1) ? 1 - jbc : my + jbc;
                int idata, jdata;
                if (use_b) {
                    idata = j1 + (int)(ihat[k] - jhat[k]);
                    jdata = -i1 + (int)(ihat[k] + jhat[k]);
                } else {
                    idata = -j1 + (int)(ihat[k] + jhat[k]);
                    jdata = i1 - (int)(ihat[k] - jhat[k]);
                }
                for (int m = 1; m <= meqn; m++)
                    q[QIDX(i1, j1, m, mbc, nx, ny)] = q[QIDX(idata, jdata, m, mbc, nx, ny)];
            }
    }
}

/* ------------------------------------------------------------------------- */
/* step2 + step2_wrap update                                                  */
/* ------------------------------------------------------------------------- */
size_t orc_ws_size(int mx, int my, int mbc, int meqn, int maux, int mwaves)
{
    int maxm = mx > my ? mx : my;
    size_t L = (size_t)(maxm + 2 * mbc);
    size_t n = 0;
    n += L * meqn * 2;                 /* faddm, faddp */
    n += L * meqn * 2 * 2;             /* gaddm, gaddp */
    n += L * meqn;                     /* q1d */
    n += L * 2;                        /* dtdx1d, dtdy1d */
    n += L * (maux > 0 ? maux : 1) * 3;/* aux1..3 */
    n += L * meqn * mwaves + L * mwaves; /* wave, s */
    n += L * meqn * 5;                 /* amdq apdq cqxx bmasdq bpasdq */
    n += L * 5;                        /* comroe */
    return n;
}

double orc_step2(const orc_config* cfg, orc_rpn2_t rpn2, orc_rpt2_t rpt2, double* work,
                 double* qold, const double* aux, double dx, double dy, double dt,
                 double* fm, double* fp, double* gm, double* gp, const int* block_corner_count)
{
    const int mx = cfg->mx, my = cfg->my, mbc = cfg->mbc, meqn = cfg->meqn, maux = cfg->maux;
    const int mwaves = cfg->mwaves, mcapa = cfg->mcapa;
    const int maxm = mx > my ? mx : my;
    const int L = maxm + 2 * mbc;
    const int nx = mx + 2 * mbc, ny = my + 2 * mbc;
    const int mauxw = maux > 0 ? maux : 1;
    int method[7] = {0, cfg->order[0], cfg->order[1], 0, 0, 0, 0};

    double* faddm = work;
    double* faddp = faddm + L * meqn;
    double* gaddm = faddp + L * meqn;
    double* gaddp = gaddm + 2 * L * meqn;
    double* q1d = gaddp + 2 * L * meqn;
    double* dtdx1d = q1d + L * meqn;
    double* dtdy1d = dtdx1d + L;
    double* aux1 = dtdy1d + L;
    double* aux2 = aux1 + L * mauxw;
    double* aux3 = aux2 + L * mauxw;
    double* wave = aux3 + L * mauxw;
    double* s = wave + L * meqn * mwaves;
    double* amdq = s + L * mwaves;
    double* apdq = amdq + L * meqn;
    double* cqxx = apdq + L * meqn;
    double* bmasdq = cqxx + L * meqn;
    double* bpasdq = bmasdq + L * meqn;
    orc_rpctx ctx;
    ctx.grav = cfg->grav;
    ctx.dry_tolerance = cfg->pdata[31] > 0 ? cfg->pdata[31] : 1e-3;
    ctx.u = bpasdq + L * meqn;
    ctx.v = ctx.u + L;
    ctx.a = ctx.v + L;
    ctx.h = ctx.a + L;
    ctx.e = ctx.h + L;
    ctx.gamma = cfg->gamma;
    ctx.newton_tol = cfg->newton_tol;
    ctx.cfg = cfg;

    double cflgrid = 0.0;
    const double dtdx = dt / dx, dtdy = dt / dy;
    /* step2.f:82-91 */
    for (size_t k = 0; k < (size_t)nx * ny * meqn; k++) { fm[k] = 0.0; fp[k] = 0.0; gm[k] = 0.0; gp[k] = 0.0; }
    if (mcapa == 0)
        for (int i = 1 - mbc; i <= maxm + mbc; i++) { dtdx1d[I1(i)] = dtdx; dtdy1d[I1(i)] = dtdy; }

    void (*fluxfn)(orc_rpctx*, orc_rpn2_t, orc_rpt2_t, int, int, int, int, int, int, const double*, double*,
                   const double*, const double*, const double*, double*, double*, double*, double*,
                   double*, double*, double*, double*, double*, double*, double*, double*, int,
                   const int*, const int*) = cfg->use_fwaves ? flux2fw : flux2;

    fix_corners(mx, my, mbc, meqn, qold, 0, block_corner_count);
    /* x-sweeps, step2.f:113-167 */
    for (int j = 2 - mbc; j <= my + mbc - 1; j++) {
        for (int m = 1; m <= meqn; m++)
            for (int i = 1 - mbc; i <= mx + mbc; i++) q1d[I1(i) + (m - 1) * L] = qold[QIDX(i, j, m, mbc, nx, ny)];
        if (mcapa > 0)
            for (int i = 1 - mbc; i <= mx + mbc; i++) dtdx1d[I1(i)] = dtdx / aux[QIDX(i, j, mcapa, mbc, nx, ny)];
        if (maux > 0)
            for (int ma = 1; ma <= maux; ma++)
                for (int i = 1 - mbc; i <= mx + mbc; i++) {
                    aux1[I1(i) + (ma - 1) * L] = aux[QIDX(i, j - 1, ma, mbc, nx, ny)];
                    aux2[I1(i) + (ma - 1) * L] = aux[QIDX(i, j, ma, mbc, nx, ny)];
                    aux3[I1(i) + (ma - 1) * L] = aux[QIDX(i, j + 1, ma, mbc, nx, ny)];
                }
        double cfl1d;
        fluxfn(&ctx, rpn2, rpt2, 1, maxm, meqn, maux, mbc, mx, q1d, dtdx1d, aux1, aux2, aux3,
               faddm, faddp, gaddm, gaddp, &cfl1d, wave, s, amdq, apdq, cqxx, bmasdq, bpasdq,
               mwaves, method, cfg->mthlim);
        cflgrid = dmax1(cflgrid, cfl1d);
        for (int m = 1; m <= meqn; m++)
            for (int i = 2 - mbc; i <= mx + mbc; i++) {
                size_t c = QIDX(i, j, m, mbc, nx, ny), cu = QIDX(i, j + 1, m, mbc, nx, ny);
                fm[c] = fm[c] + faddm[I1(i) + (m - 1) * L];
                fp[c] = fp[c] + faddp[I1(i) + (m - 1) * L];
                gm[c] = gm[c] + gaddm[I1(i) + (m - 1) * L];
                gp[c] = gp[c] + gaddp[I1(i) + (m - 1) * L];
                gm[cu] = gm[cu] + gaddm[I1(i) + (m - 1) * L + L * meqn];
                gp[cu] = gp[cu] + gaddp[I1(i) + (m - 1) * L + L * meqn];
            }
    }
    fix_corners(mx, my, mbc, meqn, qold, 1, block_corner_count);
    /* y-sweeps, step2.f:182-236 */
    for (int i = 2 - mbc; i <= mx + mbc - 1; i++) {
        for (int m = 1; m <= meqn; m++)
            for (int j = 1 - mbc; j <= my + mbc; j++) q1d[I1(j) + (m - 1) * L] = qold[QIDX(i, j, m, mbc, nx, ny)];
        if (mcapa > 0)
            for (int j = 1 - mbc; j <= my + mbc; j++) dtdy1d[I1(j)] = dtdy / aux[QIDX(i, j, mcapa, mbc, nx, ny)];
        if (maux > 0)
            for (int ma = 1; ma <= maux; ma++)
                for (int j = 1 - mbc; j <= my + mbc; j++) {
                    aux1[I1(j) + (ma - 1) * L] = aux[QIDX(i - 1, j, ma, mbc, nx, ny)];
                    aux2[I1(j) + (ma - 1) * L] = aux[QIDX(i, j, ma, mbc, nx, ny)];
                    aux3[I1(j) + (ma - 1) * L] = aux[QIDX(i + 1, j, ma, mbc, nx, ny)];
                }
        double cfl1d;
        fluxfn(&ctx, rpn2, rpt2, 2, maxm, meqn, maux, mbc, my, q1d, dtdy1d, aux1, aux2, aux3,
               faddm, faddp, gaddm, gaddp, &cfl1d, wave, s, amdq, apdq, cqxx, bmasdq, bpasdq,
               mwaves, method, cfg->mthlim);
        cflgrid = dmax1(cflgrid, cfl1d);
        for (int m = 1; m <= meqn; m++)
            for (int j = 2 - mbc; j <= my + mbc; j++) {
                size_t c = QIDX(i, j, m, mbc, nx, ny), cr = QIDX(i + 1, j, m, mbc, nx, ny);
                gm[c] = gm[c] + faddm[I1(j) + (m - 1) * L];
                gp[c] = gp[c] + faddp[I1(j) + (m - 1) * L];
                fm[c] = fm[c] + gaddm[I1(j) + (m - 1) * L];
                fp[c] = fp[c] + gaddp[I1(j) + (m - 1) * L];
                fm[cr] = fm[cr] + gaddm[I1(j) + (m - 1) * L + L * meqn];
                fp[cr] = fp[cr] + gaddp[I1(j) + (m - 1) * L + L * meqn];
            }
    }
    /* step2_wrap.f:107-125 */
    for (int m = 1; m <= meqn; m++)
        for (int i = 1 - mbc; i <= mx + mbc - 1; i++)
            for (int j = 1 - mbc; j <= my + mbc - 1; j++) {
                size_t c = QIDX(i, j, m, mbc, nx, ny);
                size_t cr = QIDX(i + 1, j, m, mbc, nx, ny), cu = QIDX(i, j + 1, m, mbc, nx, ny);
                if (mcapa == 0)
                    qold[c] = qold[c] - dtdx * (fm[cr] - fp[c]) - dtdy * (gm[cu] - gp[c]);
                else
                    qold[c] = qold[c] - (dtdx * (fm[cr] - fp[c]) + dtdy * (gm[cu] - gp[c])) /
                                            aux[QIDX(i, j, mcapa, mbc, nx, ny)];
            }
    return cflgrid;
}

double orc_patch_step2(const orc_config* cfg, double* q, const double* aux,
                       double dx, double dy, double dt,
                       double* fm, double* fp, double* gm, double* gp)
{
    orc_rpn2_t rpn2; orc_rpt2_t rpt2;
    orc_rp_select(cfg->rp, &rpn2, &rpt2);
    double* work = (double*)calloc(orc_ws_size(cfg->mx, cfg->my, cfg->mbc, cfg->meqn, cfg->maux, cfg->mwaves), sizeof(double));
    int bcc[4] = {0, 0, 0, 0};
    double cfl = orc_step2(cfg, rpn2, rpt2, work, q, aux, dx, dy, dt, fm, fp, gm, gp, bcc);
    free(work);
    return cfl;
}

/* ------------------------------------------------------------------------- */
/* bc2 default: clawpack46_bc2_default.f:1-213 (mthbc<0 means "not a physical side").
 * mthbc = 0 (user) with an inflow state: the shock-bubble inflow of
 * applications/clawpack/euler/2d/shockbubble/user_4.6/bc2.f:53-60 on that side. */
/* ------------------------------------------------------------------------- */
void orc_bc2(int mx, int my, int mbc, int meqn, double* q, const int* mthbc, const double* inflow)
{
    const int nx = mx + 2 * mbc, ny = my + 2 * mbc;
#define Q(i, j, m) q[QIDX(i, j, m, mbc, nx, ny)]
    if (mthbc[0] == 0 && inflow) {
        for (int ibc = 1; ibc <= mbc; ibc++)
            for (int j = 1 - mbc; j <= my + mbc; j++)
                for (int m = 1; m <= meqn; m++) Q(1 - ibc, j, m) = inflow[m - 1];
    }
    if (mthbc[0] == 1) {
        for (int m = 1; m <= meqn; m++) for (int ibc = 1; ibc <= mbc; ibc++)
            for (int j = 1 - mbc; j <= my + mbc; j++) Q(1 - ibc, j, m) = Q(1, j, m);
    } else if (mthbc[0] == 3) {
        for (int m = 1; m <= meqn; m++) for (int ibc = 1; ibc <= mbc; ibc++)
            for (int j = 1 - mbc; j <= my + mbc; j++) Q(1 - ibc, j, m) = Q(ibc, j, m);
        for (int ibc = 1; ibc <= mbc; ibc++)
            for (int j = 1 - mbc; j <= my + mbc; j++) Q(1 - ibc, j, 2) = -Q(ibc, j, 2);
    }
    if (mthbc[1] == 1) {
        for (int m = 1; m <= meqn; m++) for (int ibc = 1; ibc <= mbc; ibc++)
            for (int j = 1 - mbc; j <= my + mbc; j++) Q(mx + ibc, j, m) = Q(mx, j, m);
    } else if (mthbc[1] == 3) {
        for (int m = 1; m <= meqn; m++) for (int ibc = 1; ibc <= mbc; ibc++)
            for (int j = 1 - mbc; j <= my + mbc; j++) Q(mx + ibc, j, m) = Q(mx + 1 - ibc, j, m);
        for (int ibc = 1; ibc <= mbc; ibc++)
            for (int j = 1 - mbc; j <= my + mbc; j++) Q(mx + ibc, j, 2) = -Q(mx + 1 - ibc, j, 2);
    }
    if (mthbc[2] == 1) {
        for (int m = 1; m <= meqn; m++) for (int jbc = 1; jbc <= mbc; jbc++)
            for (int i = 1 - mbc; i <= mx + mbc; i++) Q(i, 1 - jbc, m) = Q(i, 1, m);
    } else if (mthbc[2] == 3) {
        for (int m = 1; m <= meqn; m++) for (int jbc = 1; jbc <= mbc; jbc++)
            for (int i = 1 - mbc; i <= mx + mbc; i++) Q(i, 1 - jbc, m) = Q(i, jbc, m);
        for (int jbc = 1; jbc <= mbc; jbc++)
            for (int i = 1 - mbc; i <= mx + mbc; i++) Q(i, 1 - jbc, 3) = -Q(i, jbc, 3);
    }
    if (mthbc[3] == 1) {
        for (int m = 1; m <= meqn; m++) for (int jbc = 1; jbc <= mbc; jbc++)
            for (int i = 1 - mbc; i <= mx + mbc; i++) Q(i, my + jbc, m) = Q(i, my, m);
    } else if (mthbc[3] == 3) {
        for (int m = 1; m <= meqn; m++) for (int jbc = 1; jbc <= mbc; jbc++)
            for (int i = 1 - mbc; i <= mx + mbc; i++) Q(i, my + jbc, m) = Q(i, my + 1 - jbc, m);
        for (int jbc = 1; jbc <= mbc; jbc++)
            for (int i = 1 - mbc; i <= mx + mbc; i++) Q(i, my + jbc, 3) = -Q(i, my + 1 - jbc, 3);
    }
#undef Q
}
