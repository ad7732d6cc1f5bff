/*
 * orc_rp_fwave.c -- oracle restatement of the shallow-water f-wave solvers with
 * bathymetry (test infrastructure; see oracle.h for the parity status).
 *
 *   rpn2: applications/clawpack/shallow/2d/rp/rpn2_tsunami.f90:3-175 (+ simple_riemann :180-222)
 *   rpt2: applications/clawpack/shallow/2d/rp/rpt2_tsunami.f90:3-170
 * aux(:,1) holds the bathymetry b.  ctx->dry_tolerance is common /common_swe/.
 */
#include <math.h>
#include "orc_internal.h"

void orc_rpn2_fwave(orc_rpctx* ctx, int ixy, int maxm, int meqn, int mwaves, int maux, int mbc, int mx,
                    const double* ql, const double* qr, const double* auxl, const double* auxr,
                    double* fwave, double* s, double* amdq, double* apdq)
{
    (void)maux;
    const int L = maxm + 2 * mbc;
    const double grav = ctx->grav;
    const int mu = (ixy == 1) ? 2 : 3;
    const int mv = (ixy == 1) ? 3 : 2;
    for (int i = 2 - mbc; i <= mx + mbc; i++) {
        double hL = qr[I1(i - 1)], hR = ql[I1(i)];
        double huL = qr[I1(i - 1) + (mu - 1) * L], huR = ql[I1(i) + (mu - 1) * L];
        double bL = auxr[I1(i - 1)], bR = auxl[I1(i)];
        double hvL = qr[I1(i - 1) + (mv - 1) * L], hvR = ql[I1(i) + (mv - 1) * L];
        double uR = huR / hR, vR = hvR / hR;
        double phiR = 0.5 * grav * (hR * hR) + (huR * huR) / hR;
        double uL = huL / hL, vL = hvL / hL;
        double phiL = 0.5 * grav * (hL * hL) + (huL * huL) / hL;
        double uhat = (sqrt(grav * hL) * uL + sqrt(grav * hR) * uR) / (sqrt(grav * hR) + sqrt(grav * hL));
        double chat = sqrt(grav * 0.5 * (hR + hL));
        /* simple_riemann (rpn2_tsunami.f90:180-222) */
        double hbar = 0.5 * (hR + hL);
        double fd1 = (hR * uR) - (hL * uL);
        double fd2 = phiR - phiL + grav * hbar * (bR - bL);
        double fd3 = hR * uR * vR - hL * uL * vL;
        double s1 = fmin(uL - sqrt(grav * hL), uhat - chat);
        double s3 = fmax(uR + sqrt(grav * hR), uhat + chat);
        double s2 = 0.5 * (s1 + s3);
        double b1 = -(fd2 - s3 * fd1) / (s3 - s1);
        double b3 = (fd2 - s1 * fd1) / (s3 - s1);
        double b2 = fd3 - b1 * vL - b3 * vR;
        double fw[3][3];   /* fw[row][wave], rows (h, normal, transverse) */
        fw[0][0] = b1; fw[1][0] = b1 * s1; fw[2][0] = b1 * vL;
        fw[0][1] = 0.0; fw[1][1] = 0.0; fw[2][1] = b2;
        fw[0][2] = b3; fw[1][2] = b3 * s3; fw[2][2] = b3 * vR;
        double sw[3] = {s1, s2, s3};
        for (int mw = 1; mw <= mwaves; mw++) {
            s[I1(i) + (mw - 1) * L] = sw[mw - 1];
            fwave[I1(i) + 0 * L + (mw - 1) * L * meqn] = fw[0][mw - 1];
            fwave[I1(i) + 1 * L + (mw - 1) * L * meqn] = fw[mu - 1][mw - 1];
            fwave[I1(i) + 2 * L + (mw - 1) * L * meqn] = fw[mv - 1][mw - 1];
        }
    }
    for (int i = 2 - mbc; i <= mx + mbc; i++) {
        double szm[3], szp[3];
        for (int mw = 1; mw <= mwaves; mw++) {
            double z = copysign(1.0, s[I1(i) + (mw - 1) * L]);
            szm[mw - 1] = (1 - z) / 2;
            szp[mw - 1] = (1 + z) / 2;
        }
        for (int mq = 1; mq <= meqn; mq++) {
            const double* f = &fwave[I1(i) + (mq - 1) * L];
            double am = szm[0] * f[0];
            am = am + szm[1] * f[L * meqn];
            am = am + szm[2] * f[2 * L * meqn];
            double ap = szp[0] * f[0];
            ap = ap + szp[1] * f[L * meqn];
            ap = ap + szp[2] * f[2 * L * meqn];
            amdq[I1(i) + (mq - 1) * L] = am;
            apdq[I1(i) + (mq - 1) * L] = ap;
        }
    }
}

void orc_rpt2_fwave(orc_rpctx* ctx, int ixy, int maxm, int meqn, int mwaves, int maux, int mbc, int mx,
                    const double* ql, const double* qr, const double* aux1, const double* aux2,
                    const double* aux3, int imp, const double* asdq, double* bmasdq, double* bpasdq)
{
    (void)maux;
    const int L = maxm + 2 * mbc;
    const double g = ctx->grav;
    const double tol = ctx->dry_tolerance;
    const int mu = (ixy == 1) ? 2 : 3;
    const int mv = (ixy == 1) ? 3 : 2;
    for (int i = 2 - mbc; i <= mx + mbc; i++) {
        double hl = qr[I1(i - 1)], hr = ql[I1(i)];
        double hul = qr[I1(i - 1) + (mu - 1) * L], hur = ql[I1(i) + (mu - 1) * L];
        double hvl = qr[I1(i - 1) + (mv - 1) * L], hvr = ql[I1(i) + (mv - 1) * L];
        double ul, vl, ur, vr;
        if (hl < tol) { hl = 0.0; ul = 0.0; vl = 0.0; } else { ul = hul / hl; vl = hvl / hl; }
        if (hr < tol) { hr = 0.0; ur = 0.0; vr = 0.0; } else { ur = hur / hr; vr = hvr / hr; }
        double sv[3] = {0.0, 0.0, 0.0}, beta[3] = {0.0, 0.0, 0.0};
        double r[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};   /* r[m][mw] */
        int skip = (hl <= tol && hr <= tol);
        if (!skip) {
            double eta, topo1, topo3;
            if (imp == 1) { eta = qr[I1(i - 1)] + aux2[I1(i - 1)]; topo1 = aux1[I1(i - 1)]; topo3 = aux3[I1(i - 1)]; }
            else { eta = ql[I1(i)] + aux2[I1(i)]; topo1 = aux1[I1(i)]; topo3 = aux3[I1(i)]; }
            if (eta < fmax(topo1, topo3)) skip = 1;
        }
        if (!skip) {
            double vhat = (vr * sqrt(hr)) / (sqrt(hr) + sqrt(hl)) + (vl * sqrt(hl)) / (sqrt(hr) + sqrt(hl));
            double uhat = (ur * sqrt(hr)) / (sqrt(hr) + sqrt(hl)) + (ul * sqrt(hl)) / (sqrt(hr) + sqrt(hl));
            double hhat = (hr + hl) / 2.0;
            double roe1 = vhat - sqrt(g * hhat);
            double roe3 = vhat + sqrt(g * hhat);
            double s1l = vl - sqrt(g * hl);
            double s3r = vr + sqrt(g * hr);
            double s1 = fmin(roe1, s1l);
            double s3 = fmax(roe3, s3r);
            double s2 = uhat;
            sv[0] = s1; sv[1] = s2; sv[2] = s3;
            double delf1 = asdq[I1(i)], delf2 = asdq[I1(i) + (mu - 1) * L], delf3 = asdq[I1(i) + (mv - 1) * L];
            beta[0] = (s3 * delf1 / (s3 - s1)) - (delf3 / (s3 - s1));
            beta[1] = -(s2 * delf1) + delf2;
            beta[2] = (delf3 / (s3 - s1)) - (s1 * delf1 / (s3 - s1));
            r[0][0] = 1.0; r[mu - 1][0] = s2; r[mv - 1][0] = s1;
            r[0][1] = 0.0; r[mu - 1][1] = 1.0; r[mv - 1][1] = 0.0;
            r[0][2] = 1.0; r[mu - 1][2] = s2; r[mv - 1][2] = s3;
        }
        double szm[3], szp[3];
        for (int mw = 1; mw <= mwaves; mw++) {
            double z = copysign(1.0, sv[mw - 1]);
            szm[mw - 1] = (1 - z) / 2 * sv[mw - 1] * beta[mw - 1];
            szp[mw - 1] = (1 + z) / 2 * sv[mw - 1] * beta[mw - 1];
        }
        for (int mq = 1; mq <= meqn; mq++) {
            double bm = szm[0] * r[mq - 1][0];
            bm = bm + szm[1] * r[mq - 1][1];
            bm = bm + szm[2] * r[mq - 1][2];
            double bp = szp[0] * r[mq - 1][0];
            bp = bp + szp[1] * r[mq - 1][1];
            bp = bp + szp[2] * r[mq - 1][2];
            bmasdq[I1(i) + (mq - 1) * L] = bm;
            bpasdq[I1(i) + (mq - 1) * L] = bp;
        }
    }
}
