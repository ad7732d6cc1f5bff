/*
 * orc_euler.c -- 2D Euler equations for the CPU oracle (test infrastructure).
 *
 * Normal solver: exact Riemann solver (Newton iteration on p*, Toro, "Riemann
 * Solvers and Numerical Methods for Fluid Dynamics", ch. 4: pressure functions
 * 4.6-4.7, PVRS start 4.47, sampling 4.5).  It has no counterpart in the
 * reference; it is the FP64 definition the B200 kernels are checked against.
 *   amdq = F(q0) - F(qL), apdq = F(qR) - F(q0), q0 = Godunov state at x/t = 0;
 *   waves  w1 = q*L - qL, w2 = q*R - q*L, w3 = qR - q*R;
 *   speeds s1 = left shock speed (or rarefaction head uL - aL), s2 = u*,
 *          s3 = right shock speed (or rarefaction head uR + aR).
 * Interfaces without a pressure or normal-velocity jump take p* = p, u* = u
 * without iterating (0 Newton iterations; the values equal the first Newton step's).
 * The Roe averages of applications/clawpack/euler/2d/rp/clawpack46_rpn2_euler4.f:83-100
 * are formed as well, for the transverse solver clawpack46_rpt2_euler4.f:56-94
 * (restated below).
 *
 * Powers use the exp/log below (Cody-Waite reduction by ln 2, atanh series for
 * log, Taylor series for exp), written with + - * / only, so a device
 * implementation with the same operation order gives the same bits.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>
#include "orc_internal.h"

static const double LN2_HI = 6.93147180369123816490e-01;   /* ln 2 with the low 32 bits cleared */
static const double LN2_LO = 1.90821492927058770002e-10;   /* ln 2 - LN2_HI */
static const double INV_LN2 = 1.44269504088896338700e+00;
static const double SQRT2 = 1.41421356237309514547e+00;

/* log x for normal x > 0: x = m 2^e, m in [1/sqrt2, sqrt2), log m = 2 atanh(s),
 * s = (m-1)/(m+1), series to s^23. */
double orc_log(double x)
{
    uint64_t b;
    memcpy(&b, &x, 8);
    int e = (int)((b >> 52) & 0x7ff) - 1023;
    b = (b & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL;
    double m;
    memcpy(&m, &b, 8);
    if (m > SQRT2) { m = m * 0.5; e = e + 1; }
    const double s = (m - 1.0) / (m + 1.0);
    const double s2 = s * s;
    double p = 1.0 / 23.0;
    p = p * s2 + 1.0 / 21.0;
    p = p * s2 + 1.0 / 19.0;
    p = p * s2 + 1.0 / 17.0;
    p = p * s2 + 1.0 / 15.0;
    p = p * s2 + 1.0 / 13.0;
    p = p * s2 + 1.0 / 11.0;
    p = p * s2 + 1.0 / 9.0;
    p = p * s2 + 1.0 / 7.0;
    p = p * s2 + 1.0 / 5.0;
    p = p * s2 + 1.0 / 3.0;
    p = p * s2 + 1.0;
    const double lm = 2.0 * s * p;
    const double de = (double)e;
    return de * LN2_HI + (de * LN2_LO + lm);
}

/* exp y for |y| < 700: y = k ln2 + r, |r| <= ln2/2, Taylor series to r^17. */
double orc_exp(double y)
{
    const double kd = floor(y * INV_LN2 + 0.5);
    const double r = (y - kd * LN2_HI) - kd * LN2_LO;
    double p = 1.0 + r / 17.0;
    p = 1.0 + (r / 16.0) * p;
    p = 1.0 + (r / 15.0) * p;
    p = 1.0 + (r / 14.0) * p;
    p = 1.0 + (r / 13.0) * p;
    p = 1.0 + (r / 12.0) * p;
    p = 1.0 + (r / 11.0) * p;
    p = 1.0 + (r / 10.0) * p;
    p = 1.0 + (r / 9.0) * p;
    p = 1.0 + (r / 8.0) * p;
    p = 1.0 + (r / 7.0) * p;
    p = 1.0 + (r / 6.0) * p;
    p = 1.0 + (r / 5.0) * p;
    p = 1.0 + (r / 4.0) * p;
    p = 1.0 + (r / 3.0) * p;
    p = 1.0 + (r / 2.0) * p;
    p = 1.0 + r * p;
    const int k = (int)kd;
    const uint64_t sb = (uint64_t)(k + 1023) << 52;
    double scale;
    memcpy(&scale, &sb, 8);
    return p * scale;
}

double orc_pow(double x, double a) { return orc_exp(a * orc_log(x)); }

/* Newton-iteration histogram (bins 0..31, last bin = 31 or more). */
static long g_newton_hist[32];
void orc_newton_hist(long* out, int reset)
{
    for (int k = 0; k < 32; k++) out[k] = g_newton_hist[k];
    if (reset) memset(g_newton_hist, 0, sizeof(g_newton_hist));
}

typedef struct { double gam, g1, g2, g3, g4, g5, g6, g7, gm1; } eos_t;

static eos_t eos_make(double gam)
{
    eos_t e;
    e.gam = gam;
    e.g1 = (gam - 1.0) / (2.0 * gam);
    e.g2 = (gam + 1.0) / (2.0 * gam);
    e.g3 = 2.0 * gam / (gam - 1.0);
    e.g4 = 2.0 / (gam - 1.0);
    e.g5 = 2.0 / (gam + 1.0);
    e.g6 = (gam - 1.0) / (gam + 1.0);
    e.g7 = (gam - 1.0) / 2.0;
    e.gm1 = gam - 1.0;
    return e;
}

/* Toro 4.6-4.7 and their derivatives. */
static void prefun(const eos_t* E, double p, double rk, double pk, double ak, double* f, double* fd)
{
    if (p <= pk) {
        const double prat = p / pk;
        const double z = orc_exp(E->g1 * orc_log(prat));
        *f = E->g4 * ak * (z - 1.0);
        *fd = (z / prat) / (rk * ak);
    } else {
        const double bk = E->g6 * pk;
        const double qrt = sqrt((E->g5 / rk) / (bk + p));
        *f = (p - pk) * qrt;
        *fd = (1.0 - 0.5 * (p - pk) / (bk + p)) * qrt;
    }
}

/* Exact solver for primitive states (rho, u, p) left/right.  seed <= 0: PVRS.
 * out: p*, u*, rho*L, rho*R, a*L, a*R.  Returns the Newton iteration count. */
int orc_euler_star(double gam, const double* wl, const double* wr, double seed, double tol, double* out)
{
    const eos_t E = eos_make(gam);
    const double rl = wl[0], ul = wl[1], pl = wl[2], rr = wr[0], ur = wr[1], pr = wr[2];
    const double al = sqrt(gam * pl / rl), ar = sqrt(gam * pr / rr);
    const double du = ur - ul;
    const double tolpre = 1.0e-6;
    double p;
    if (seed > 0.0 && seed < INFINITY) p = seed;
    else {
        const double ppv = 0.5 * (pl + pr) - 0.125 * du * (rl + rr) * (al + ar);
        p = ppv > tolpre ? ppv : tolpre;
    }
    double fl = 0.0, fr = 0.0, fdl, fdr;
    int it = 0;
    if (pl == pr && ul == ur) {
        /* no pressure or normal-velocity jump: p* = p, u* = u exactly (what the
         * first Newton step returns bit for bit); no iteration is needed */
        p = pl;
    } else {
        /* Newton from the seed; where it does not converge (or leaves the finite
         * numbers), once more from the PVRS estimate: Newton stays the judge */
        const int seeded = seed > 0.0 && seed < INFINITY;
        int ok = 0;
        for (int pass = 0; pass < (seeded ? 2 : 1) && !ok; pass++) {
            if (pass == 1) {
                const double ppv = 0.5 * (pl + pr) - 0.125 * du * (rl + rr) * (al + ar);
                p = ppv > tolpre ? ppv : tolpre;
            }
            for (int k = 1; k <= 64; k++) {
                prefun(&E, p, rl, pl, al, &fl, &fdl);
                prefun(&E, p, rr, pr, ar, &fr, &fdr);
                double pn = p - (fl + fr + du) / (fdl + fdr);
                if (pn < 0.0) pn = tolpre;
                const double change = 2.0 * fabs(pn - p) / (pn + p);
                p = pn;
                it++;
                if (change <= tol) { ok = 1; break; }
            }
            ok = ok && isfinite(p);
        }
        if (it > 64) it = 64;
    }
    const double us = 0.5 * (ul + ur) + 0.5 * (fr - fl);
    out[0] = p;
    out[1] = us;
    /* star densities and sound speeds (p* = pK: the rarefaction formulas give
     * rhoK, aK exactly, since log 1 = 0 and exp 0 = 1 in orc_log / orc_exp) */
    if (p > pl) { const double q = p / pl; out[2] = rl * ((q + E.g6) / (E.g6 * q + 1.0)); out[4] = sqrt(gam * p / out[2]); }
    else if (p == pl) { out[2] = rl; out[4] = al; }
    else { const double lq = orc_log(p / pl); out[2] = rl * orc_exp(lq / gam); out[4] = al * orc_exp(E.g1 * lq); }
    if (p > pr) { const double q = p / pr; out[3] = rr * ((q + E.g6) / (E.g6 * q + 1.0)); out[5] = sqrt(gam * p / out[3]); }
    else if (p == pr) { out[3] = rr; out[5] = ar; }
    else { const double lq = orc_log(p / pr); out[3] = rr * orc_exp(lq / gam); out[5] = ar * orc_exp(E.g1 * lq); }
    return it;
}

/* Normal flux of a primitive state with its total energy. */
static void eflux(double r, double u, double v, double p, double en, double* f)
{
    f[0] = r * u;
    f[1] = r * u * u + p;
    f[2] = r * u * v;
    f[3] = u * (en + p);
}

/* One interface: qL, qR conserved (rho, m_normal, m_tangential, E); waves/speeds/
 * fluctuations in the same component order.  Returns the Newton iteration count. */
int orc_euler_interface(double gam, double tol, const double* ql, const double* qr, double seed,
                        double wave[3][4], double s[3], double* amdq, double* apdq)
{
    const eos_t E = eos_make(gam);
    const double rl = ql[0], ul = ql[1] / rl, vl = ql[2] / rl;
    const double pl = E.gm1 * (ql[3] - 0.5 * (ql[1] * ql[1] + ql[2] * ql[2]) / rl);
    const double rr = qr[0], ur = qr[1] / rr, vr = qr[2] / rr;
    const double pr = E.gm1 * (qr[3] - 0.5 * (qr[1] * qr[1] + qr[2] * qr[2]) / rr);
    const double al = sqrt(gam * pl / rl), ar = sqrt(gam * pr / rr);
    const double wl[3] = {rl, ul, pl}, wr[3] = {rr, ur, pr};
    double st[6];
    const int it = orc_euler_star(gam, wl, wr, seed, tol, st);
    const double ps = st[0], us = st[1], rsl = st[2], rsr = st[3], asl = st[4], asr = st[5];
    /* wave speeds */
    const double shl = ul - al, shr = ur + ar;
    double sl, sr;
    if (ps > pl) sl = ul - al * sqrt(E.g2 * (ps / pl) + E.g1); else sl = shl;
    if (ps > pr) sr = ur + ar * sqrt(E.g2 * (ps / pr) + E.g1); else sr = shr;
    s[0] = sl; s[1] = us; s[2] = sr;
    /* star states and waves */
    const double esl = ps / E.gm1 + 0.5 * rsl * (us * us + vl * vl);
    const double esr = ps / E.gm1 + 0.5 * rsr * (us * us + vr * vr);
    const double qsl[4] = {rsl, rsl * us, rsl * vl, esl};
    const double qsr[4] = {rsr, rsr * us, rsr * vr, esr};
    for (int m = 0; m < 4; m++) {
        wave[0][m] = qsl[m] - ql[m];
        wave[1][m] = qsr[m] - qsl[m];
        wave[2][m] = qr[m] - qsr[m];
    }
    /* Godunov state at x/t = 0 (Toro 4.5) */
    double r0, u0, v0, p0, e0;
    int which;   /* 0: left state, 1: left star, 2: left fan, 3: right star, 4: right state, 5: right fan */
    if (0.0 <= us) {
        v0 = vl;
        if (ps > pl) which = (0.0 <= sl) ? 0 : 1;
        else if (0.0 <= shl) which = 0;
        else which = (0.0 > us - asl) ? 1 : 2;
    } else {
        v0 = vr;
        if (ps > pr) which = (0.0 >= sr) ? 4 : 3;
        else if (0.0 >= shr) which = 4;
        else which = (0.0 < us + asr) ? 3 : 5;
    }
    if (which == 0) { r0 = rl; u0 = ul; p0 = pl; e0 = ql[3]; }
    else if (which == 4) { r0 = rr; u0 = ur; p0 = pr; e0 = qr[3]; }
    else if (which == 1) { r0 = rsl; u0 = us; p0 = ps; e0 = esl; }
    else if (which == 3) { r0 = rsr; u0 = us; p0 = ps; e0 = esr; }
    else if (which == 2) {
        const double c = E.g5 + (E.g6 / al) * ul;
        const double lc = orc_log(c);
        r0 = rl * orc_exp(E.g4 * lc);
        u0 = E.g5 * (al + E.g7 * ul);
        p0 = pl * orc_exp(E.g3 * lc);
        e0 = p0 / E.gm1 + 0.5 * r0 * (u0 * u0 + v0 * v0);
    } else {
        const double c = E.g5 - (E.g6 / ar) * ur;
        const double lc = orc_log(c);
        r0 = rr * orc_exp(E.g4 * lc);
        u0 = E.g5 * (-ar + E.g7 * ur);
        p0 = pr * orc_exp(E.g3 * lc);
        e0 = p0 / E.gm1 + 0.5 * r0 * (u0 * u0 + v0 * v0);
    }
    double f0[4], fl[4], fr[4];
    eflux(r0, u0, v0, p0, e0, f0);
    eflux(rl, ul, vl, pl, ql[3], fl);
    eflux(rr, ur, vr, pr, qr[3], fr);
    for (int m = 0; m < 4; m++) { amdq[m] = f0[m] - fl[m]; apdq[m] = fr[m] - f0[m]; }
    return it;
}

/* Roe averages of the interface between qlo (cell i-1) and qhi (cell i), states in
 * (rho, rho u, rho v, E) order, mu / mv the normal and tangential momentum (0-based):
 * clawpack46_rpn2_euler4.f:84-99 with gamma1 = gamma - 1. */
static void roe_averages(double gamma1, int mu, int mv, const double* qlo, const double* qhi, double* u_out,
                         double* v_out, double* enth_out, double* a_out, double* g1a2_out)
{
    const double rhsqrtl = sqrt(qlo[0]);
    const double rhsqrtr = sqrt(qhi[0]);
    const double pl = gamma1 * (qlo[3] - 0.5 * (qlo[1] * qlo[1] + qlo[2] * qlo[2]) / qlo[0]);
    const double pr = gamma1 * (qhi[3] - 0.5 * (qhi[1] * qhi[1] + qhi[2] * qhi[2]) / qhi[0]);
    const double rhsq2 = rhsqrtl + rhsqrtr;
    const double u = (qlo[mu] / rhsqrtl + qhi[mu] / rhsqrtr) / rhsq2;
    const double v = (qlo[mv] / rhsqrtl + qhi[mv] / rhsqrtr) / rhsq2;
    const double enth = ((qlo[3] + pl) / rhsqrtl + (qhi[3] + pr) / rhsqrtr) / rhsq2;
    const double u2v2 = u * u + v * v;
    const double a2 = gamma1 * (enth - 0.5 * u2v2);
    *u_out = u;
    *v_out = v;
    *enth_out = enth;
    *a_out = sqrt(a2);
    *g1a2_out = gamma1 / a2;
}

/* rpn2 for the oracle's flux2: exact normal solve + Roe averages for rpt2
 * (clawpack46_rpn2_euler4.f:83-100 with gamma1 = gamma - 1). */
void orc_rpn2_euler(orc_rpctx* ctx, int ixy, int maxm, int meqn, int mwaves, int maux, int mbc, int mx,
                    const double* ql, const double* qr, const double* auxl, const double* auxr,
                    double* wave, double* s, double* amdq, double* apdq)
{
    (void)maux; (void)auxl; (void)auxr; (void)mwaves;
    const int L = maxm + 2 * mbc;
    const double gam = ctx->gamma, gamma1 = gam - 1.0;
    const int mu = (ixy == 1) ? 2 : 3;
    const int mv = (ixy == 1) ? 3 : 2;
#define QL(i, m) ql[I1(i) + ((m) - 1) * L]
#define QR(i, m) qr[I1(i) + ((m) - 1) * L]
    for (int i = 2 - mbc; i <= mx + mbc; i++) {
        /* Roe averages, clawpack46_rpn2_euler4.f:84-99 */
        const double qlo[4] = {QR(i - 1, 1), QR(i - 1, 2), QR(i - 1, 3), QR(i - 1, 4)};
        const double qhi[4] = {QL(i, 1), QL(i, 2), QL(i, 3), QL(i, 4)};
        roe_averages(gamma1, mu - 1, mv - 1, qlo, qhi, &ctx->u[I1(i)], &ctx->v[I1(i)], &ctx->h[I1(i)],
                     &ctx->a[I1(i)], &ctx->e[I1(i)]);
        /* exact normal solve in (rho, m_normal, m_tangential, E) order */
        const double qa[4] = {QR(i - 1, 1), QR(i - 1, mu), QR(i - 1, mv), QR(i - 1, 4)};
        const double qb[4] = {QL(i, 1), QL(i, mu), QL(i, mv), QL(i, 4)};
        double w[3][4], sp[3], am[4], ap[4];
        const int it = orc_euler_interface(gam, ctx->newton_tol, qa, qb, 0.0, w, sp, am, ap);
        {
            const int bin = it < 31 ? it : 31;
#pragma omp atomic
            g_newton_hist[bin]++;
        }
        const int comp[4] = {1, mu, mv, 4};
        for (int mw = 1; mw <= 3; mw++) {
            s[I1(i) + (mw - 1) * L] = sp[mw - 1];
            for (int k = 0; k < 4; k++) wave[I1(i) + (comp[k] - 1) * L + (mw - 1) * L * meqn] = w[mw - 1][k];
        }
        for (int k = 0; k < 4; k++) {
            amdq[I1(i) + (comp[k] - 1) * L] = am[k];
            apdq[I1(i) + (comp[k] - 1) * L] = ap[k];
        }
    }
#undef QL
#undef QR
}

/* applications/clawpack/euler/2d/rp/clawpack46_rpt2_euler4.f:56-94 */
void orc_rpt2_euler(orc_rpctx* ctx, int ixy, int maxm, int meqn, int mwaves, int maux, int mbc, int mx,
                    const double* ql, const double* qr, const double* aux1, const double* aux2,
                    const double* aux3, int imp, const double* asdq, double* bmasdq, double* bpasdq)
{
    (void)maux; (void)ql; (void)qr; (void)aux1; (void)aux2; (void)aux3; (void)imp; (void)mwaves;
    const int L = maxm + 2 * mbc;
    const int mu = (ixy == 1) ? 2 : 3;
    const int mv = (ixy == 1) ? 3 : 2;
#define AS(i, m) asdq[I1(i) + ((m) - 1) * L]
    for (int i = 2 - mbc; i <= mx + mbc; i++) {
        const double u = ctx->u[I1(i)], v = ctx->v[I1(i)], enth = ctx->h[I1(i)], a = ctx->a[I1(i)];
        const double g1a2 = ctx->e[I1(i)];
        const double u2v2 = u * u + v * v;
        const double euv = enth - u2v2;
        const double a3 = g1a2 * (euv * AS(i, 1) + u * AS(i, mu) + v * AS(i, mv) - AS(i, 4));
        const double a2 = AS(i, mu) - u * AS(i, 1);
        const double a4 = (AS(i, mv) + (a - v) * AS(i, 1) - a * a3) / (2.0 * a);
        const double a1 = AS(i, 1) - a3 - a4;
        double wb[4][3], sb[3];
        wb[0][0] = a1; wb[mu - 1][0] = a1 * u; wb[mv - 1][0] = a1 * (v - a); wb[3][0] = a1 * (enth - v * a); sb[0] = v - a;
        wb[0][1] = a3; wb[mu - 1][1] = a3 * u + a2; wb[mv - 1][1] = a3 * v; wb[3][1] = a3 * 0.5 * u2v2 + a2 * u; sb[1] = v;
        wb[0][2] = a4; wb[mu - 1][2] = a4 * u; wb[mv - 1][2] = a4 * (v + a); wb[3][2] = a4 * (enth + v * a); sb[2] = v + a;
        for (int m = 1; m <= meqn; m++) {
            double bm = 0.0, bp = 0.0;
            for (int mw = 1; mw <= 3; mw++) {
                bm = bm + (sb[mw - 1] < 0.0 ? sb[mw - 1] : 0.0) * wb[m - 1][mw - 1];
                bp = bp + (sb[mw - 1] > 0.0 ? sb[mw - 1] : 0.0) * wb[m - 1][mw - 1];
            }
            bmasdq[I1(i) + (m - 1) * L] = bm;
            bpasdq[I1(i) + (m - 1) * L] = bp;
        }
    }
#undef AS
}

/* The transverse split of one interface (test entry): the Roe averages of the
 * interface between qlo (cell i-1) and qhi (cell i) as rpn2 forms them, then
 * orc_rpt2_euler on a one-interface strip.  ixy = 1 (x) or 2 (y); states, asdq,
 * bm, bp in (rho, rho u, rho v, E) order. */
void orc_euler_rpt2_point(double gam, int ixy, const double* qlo, const double* qhi, const double* asdq, double* bm,
                          double* bp)
{
    enum { mbc = 1, mx = 0, maxm = 0, L = 2 };      /* the strip's loop visits i = 1 only */
    const int mu = (ixy == 1) ? 2 : 3, mv = (ixy == 1) ? 3 : 2;
    double u[L], v[L], h[L], a[L], e[L], as[4 * L], bms[4 * L], bps[4 * L];
    orc_rpctx ctx;
    memset(&ctx, 0, sizeof(ctx));
    ctx.u = u; ctx.v = v; ctx.h = h; ctx.a = a; ctx.e = e; ctx.gamma = gam;
    roe_averages(gam - 1.0, mu - 1, mv - 1, qlo, qhi, &u[I1(1)], &v[I1(1)], &h[I1(1)], &a[I1(1)], &e[I1(1)]);
    for (int m = 0; m < 4; m++) as[I1(1) + m * L] = asdq[m];
    orc_rpt2_euler(&ctx, ixy, maxm, 4, 3, 0, mbc, mx, NULL, NULL, NULL, NULL, NULL, 1, as, bms, bps);
    for (int m = 0; m < 4; m++) { bm[m] = bms[I1(1) + m * L]; bp[m] = bps[I1(1) + m * L]; }
}

/* Euler flux of one cell in direction idir (0: x, 1: y), the rpn2_cons of the
 * time-sync flux store. */
void orc_euler_cons_flux(double gam, int idir, const double* q, double* flux)
{
    const int mu = (idir == 0) ? 1 : 2, mv = (idir == 0) ? 2 : 1;
    const double r = q[0], un = q[mu] / r;
    const double p = (gam - 1.0) * (q[3] - 0.5 * (q[1] * q[1] + q[2] * q[2]) / r);
    flux[0] = q[mu];
    flux[mu] = q[mu] * un + p;
    flux[mv] = q[mv] * un;
    flux[3] = un * (q[3] + p);
}

/* Post-shock state of a planar shock of Mach number M moving into (rho, p) =
 * (1, 1) at rest: the Rankine-Hugoniot relations used by
 * applications/clawpack/euler/2d/shockbubble/setprob.f:59-62, pressure ratio
 * 1 + 2 gamma (M^2 - 1) / (gamma + 1).  out: rho, u, E. */
void orc_euler_postshock(double gam, double mach, double* out)
{
    const double gamma1 = gam - 1.0;
    const double pinf = 1.0 + 2.0 * gam * (mach * mach - 1.0) / (gam + 1.0);
    const double rinf = (gamma1 + (gam + 1.0) * pinf) / ((gam + 1.0) + gamma1 * pinf);
    const double vinf = (1.0 / sqrt(gam)) * (pinf - 1.0) / sqrt(0.5 * ((gam + 1.0) / gam) * pinf + 0.5 * gamma1 / gam);
    out[0] = rinf;
    out[1] = vinf;
    out[2] = 0.5 * rinf * vinf * vinf + pinf / gamma1;
}
