/*
 * orc_patch46.c -- oracle restatement of the clawpatch 4.6 ghost-cell, regrid
 * and time-sync kernels (test infrastructure; see oracle.h for parity status).
 *
 * Only the same-orientation index transforms (one block, or a brick of blocks
 * sharing one coordinate orientation) are covered: there every transform of
 * src/forestclaw2d.c:609-1360 reduces to a shift in brick-global cell indices
 * with the canonical child order of transform_face2/transform_corner2.
 *
 *   copy face/corner        fort_4.6/fclaw2d_clawpatch46_copy.f:17-133
 *   average face/corner     fort_4.6/fclaw2d_clawpatch46_average.f:16-272
 *   average2coarse          fort_4.6/fclaw2d_clawpatch46_average.f:282-364
 *   interpolate face/corner fort_4.6/fclaw2d_clawpatch46_interpolate.f:30-314
 *   interpolate2fine        fort_4.6/fclaw2d_clawpatch46_interpolate.f:324-392
 *   compute_slopes          fclaw2d_clawpatch_utils.f:11-66 (mth = 5)
 *   timeinterp              fort_4.6/fclaw2d_clawpatch46_timeinterp.f:11-78
 *   time-sync f2c/samesize  clawpack46_time_sync.f:254-704
 */
#include <math.h>
#include <string.h>
#include "orc_amr.h"

/* fclaw2d_clawpatch_utils.f:45-63 with mth = 5 (AMRClaw slopes). */
static double compute_slopes(double sl, double sr)
{
    double sc = (sl + sr) / 2.0;
    double m = fmin(fmin(2 * fabs(sl), 2 * fabs(sr)), fabs(sc));
    return m * fmax(0.0, copysign(1.0, sl * sr)) * copysign(1.0, sc);
}

/* Index maps between patches (src/forestclaw2d.c:609-980, through
 * fclaw2d_clawpatch_transform.c:81-190): orc_xf_same maps a cell of P to N's
 * index space at the same level; orc_xf_half gives the four children of a
 * coarse cell in the fine patch, in the coarse patch's (x, y) order.  Both go
 * across cubed-sphere block faces (orc_sphere.c); on a brick they are shifts. */

/* ---------------- copy ---------------- */
void orc_copy_face(const orc_sim* s, double* qthis, const double* qnbr, const orc_patch* P, const orc_patch* N, int iface)
{
    const orc_config* c = &s->cfg;
    const int mx = c->mx, my = c->my, mbc = c->mbc, meqn = c->meqn, nx = s->nx, ny = s->ny;
    int ilo, ihi, jlo, jhi;
    if (iface == 0) { ilo = 1 - mbc; ihi = 0; jlo = 1; jhi = my; }
    else if (iface == 1) { ilo = mx + 1; ihi = mx + mbc; jlo = 1; jhi = my; }
    else if (iface == 2) { ilo = 1; ihi = mx; jlo = 1 - mbc; jhi = 0; }
    else { ilo = 1; ihi = mx; jlo = my + 1; jhi = my + mbc; }
    for (int m = 1; m <= meqn; m++)
        for (int j = jlo; j <= jhi; j++)
            for (int i = ilo; i <= ihi; i++) {
                int i2, j2;
                orc_xf_same(s, P, N, i, j, &i2, &j2);
                qthis[QIDX(i, j, m, mbc, nx, ny)] = qnbr[QIDX(i2, j2, m, mbc, nx, ny)];
            }
}

void orc_copy_corner(const orc_sim* s, double* qthis, const double* qnbr, const orc_patch* P, const orc_patch* N, int icorner)
{
    const orc_config* c = &s->cfg;
    const int mx = c->mx, my = c->my, mbc = c->mbc, meqn = c->meqn, nx = s->nx, ny = s->ny;
    for (int m = 1; m <= meqn; m++)
        for (int ibc = 1; ibc <= mbc; ibc++)
            for (int jbc = 1; jbc <= mbc; jbc++) {
                int i1 = (icorner & 1) ? mx + ibc : 1 - ibc;
                int j1 = (icorner & 2) ? my + jbc : 1 - jbc;
                int i2, j2;
                orc_xf_same(s, P, N, i1, j1, &i2, &j2);
                qthis[QIDX(i1, j1, m, mbc, nx, ny)] = qnbr[QIDX(i2, j2, m, mbc, nx, ny)];
            }
}

/* ---------------- average ---------------- */
static int valid_average(int i, int j, int mx, int my) { return 1 <= i && i <= mx && 1 <= j && j <= my; }

/* one coarse ghost cell from its four children (average.f:96-128): the plain mean,
 * or on a manifold sum(q_f a_f) / sum(a_f) with the fine cells' areas */
static void average_cell(const orc_sim* s, double* qc, const double* qf, const orc_patch* F, int ic, int jc,
                         const int* i2, const int* j2, int mq)
{
    const orc_config* c = &s->cfg;
    const int mbc = c->mbc, nx = s->nx, ny = s->ny, ax = c->mx + 2 * mbc + 2;
    if (F->area) {
        double sum = 0, af = 0;
        for (int m = 0; m < 4; m++) {
            double q = qf[QIDX(i2[m], j2[m], mq, mbc, nx, ny)];
            double kf = F->area[ORC_AIDX(i2[m], j2[m], mbc, ax)];
            sum = sum + q * kf;
            af = af + kf;
        }
        qc[QIDX(ic, jc, mq, mbc, nx, ny)] = sum / af;
        return;
    }
    double sum = 0;
    for (int m = 0; m < 4; m++) sum = sum + qf[QIDX(i2[m], j2[m], mq, mbc, nx, ny)];
    qc[QIDX(ic, jc, mq, mbc, nx, ny)] = sum / (double)4;
}

void orc_average_face(const orc_sim* s, double* qc, const double* qf, const orc_patch* C, const orc_patch* F, int iface_coarse)
{
    const orc_config* c = &s->cfg;
    const int mx = c->mx, my = c->my, mbc = c->mbc, meqn = c->meqn;
    const int idir = iface_coarse / 2;
    for (int mq = 1; mq <= meqn; mq++) {
        for (int a = 1; a <= (idir == 0 ? my : mbc); a++)
            for (int b = 1; b <= (idir == 0 ? mbc : mx); b++) {
                int ic, jc;
                if (idir == 0) { jc = a; ic = (iface_coarse == 0) ? 1 - b : mx + b; }
                else { ic = b; jc = (iface_coarse == 2) ? 1 - a : my + a; }
                int i2[4], j2[4], ok = 1;
                orc_xf_half(s, C, F, ic, jc, i2, j2);
                for (int m = 0; m < 4; m++) ok = ok && valid_average(i2[m], j2[m], mx, my);
                if (ok) average_cell(s, qc, qf, F, ic, jc, i2, j2, mq);
            }
    }
}

void orc_average_corner(const orc_sim* s, double* qc, const double* qf, const orc_patch* C, const orc_patch* F, int icorner)
{
    const orc_config* c = &s->cfg;
    const int mx = c->mx, my = c->my, mbc = c->mbc, meqn = c->meqn;
    for (int ibc = 1; ibc <= mbc; ibc++)
        for (int jbc = 1; jbc <= mbc; jbc++) {
            int i1 = (icorner & 1) ? mx + ibc : 1 - ibc;
            int j1 = (icorner & 2) ? my + jbc : 1 - jbc;
            int i2[4], j2[4];
            orc_xf_half(s, C, F, i1, j1, i2, j2);
            for (int mq = 1; mq <= meqn; mq++) average_cell(s, qc, qf, F, i1, j1, i2, j2, mq);
        }
}

/* ---------------- interpolate ---------------- */
static int valid_interp(int i, int j, int mx, int my, int mbc)
{
    return 1 - mbc <= i && i <= mx + mbc && 1 - mbc <= j && j <= my + mbc;
}

/* the four fine cells of coarse cell (ic, jc), at the children's offsets of
 * +-1/4 in the coarse patch's axes (interpolate.f:84-95, 150-170) */
static void interp_cell(const orc_sim* s, const double* qc, double* qf, int ic, int jc, const int* i2, const int* j2, int mq)
{
    const int mbc = s->cfg.mbc, nx = s->nx, ny = s->ny;
    double q0 = qc[QIDX(ic, jc, mq, mbc, nx, ny)];
    double sl = (q0 - qc[QIDX(ic - 1, jc, mq, mbc, nx, ny)]);
    double sr = (qc[QIDX(ic + 1, jc, mq, mbc, nx, ny)] - q0);
    double gradx = compute_slopes(sl, sr);
    sl = (q0 - qc[QIDX(ic, jc - 1, mq, mbc, nx, ny)]);
    sr = (qc[QIDX(ic, jc + 1, mq, mbc, nx, ny)] - q0);
    double grady = compute_slopes(sl, sr);
    for (int m = 0; m < 4; m++) {
        int ii = m & 1, jj = m >> 1;
        double shiftx = (ii - 0.5) / 2.0, shifty = (jj - 0.5) / 2.0;
        qf[QIDX(i2[m], j2[m], mq, mbc, nx, ny)] = q0 + gradx * shiftx + grady * shifty;
    }
}

void orc_interpolate_face(const orc_sim* s, const double* qc, double* qf, const orc_patch* C, const orc_patch* F, int iface_coarse)
{
    const orc_config* c = &s->cfg;
    const int mx = c->mx, my = c->my, mbc = c->mbc, meqn = c->meqn;
    const int idir = iface_coarse / 2;
    for (int mq = 1; mq <= meqn; mq++)
        for (int b = 1; b <= mbc / 2; b++)
            for (int a = 1; a <= mx; a++) {
                int ic, jc;
                if (idir == 0) { ic = (iface_coarse == 0) ? b : mx - b + 1; jc = a; }
                else { jc = (iface_coarse == 2) ? b : my - b + 1; ic = a; }
                int i2[4], j2[4], ok = 1;
                orc_xf_half(s, C, F, ic, jc, i2, j2);
                for (int m = 0; m < 4; m++) ok = ok && valid_interp(i2[m], j2[m], mx, my, mbc);
                if (ok) interp_cell(s, qc, qf, ic, jc, i2, j2, mq);
            }
}

void orc_interpolate_corner(const orc_sim* s, const double* qc, double* qf, const orc_patch* C, const orc_patch* F, int icorner)
{
    const orc_config* c = &s->cfg;
    const int mx = c->mx, my = c->my, mbc = c->mbc, meqn = c->meqn;
    for (int ibc = 1; ibc <= mbc / 2; ibc++)
        for (int jbc = 1; jbc <= mbc / 2; jbc++) {
            int ic = (icorner & 1) ? mx - ibc + 1 : ibc;
            int jc = (icorner & 2) ? my - jbc + 1 : jbc;
            int i2[4], j2[4];
            orc_xf_half(s, C, F, ic, jc, i2, j2);
            for (int mq = 1; mq <= meqn; mq++) interp_cell(s, qc, qf, ic, jc, i2, j2, mq);
        }
}

/* interpolate2fine (regrid): coarse patch -> child igrid (interpolate.f:324-392); on a
 * manifold fixcapaq2 (:409-470) then gives each coarse cell's mass back to its children. */
void orc_interpolate2fine(const orc_sim* s, const double* qcoarse, double* qfine, int igrid,
                          const double* acoarse, const double* afine)
{
    const orc_config* c = &s->cfg;
    const int mx = c->mx, my = c->my, mbc = c->mbc, meqn = c->meqn, nx = s->nx, ny = s->ny;
    const int ax = mx + 2 * mbc + 2;
    int ig = igrid % 2, jg = (igrid - ig) / 2;
    int i1 = 1 - ig, i2 = mx / 2 + (1 - ig), ic_add = ig * mx / 2;
    int j1 = 1 - jg, j2 = my / 2 + (1 - jg), jc_add = jg * my / 2;
    for (int mq = 1; mq <= meqn; mq++)
        for (int j = j1; j <= j2; j++)
            for (int i = i1; i <= i2; i++) {
                int ic = i + ic_add, jc = j + jc_add;
                double q0 = qcoarse[QIDX(ic, jc, mq, mbc, nx, ny)];
                double sl = (q0 - qcoarse[QIDX(ic - 1, jc, mq, mbc, nx, ny)]);
                double sr = (qcoarse[QIDX(ic + 1, jc, mq, mbc, nx, ny)] - q0);
                double gradx = compute_slopes(sl, sr);
                sl = (q0 - qcoarse[QIDX(ic, jc - 1, mq, mbc, nx, ny)]);
                sr = (qcoarse[QIDX(ic, jc + 1, mq, mbc, nx, ny)] - q0);
                double grady = compute_slopes(sl, sr);
                for (int ii = 1; ii <= 2; ii++)
                    for (int jj = 1; jj <= 2; jj++) {
                        double shiftx = (ii - 2 / 2.0 - 0.5) / 2;
                        double shifty = (jj - 2 / 2.0 - 0.5) / 2;
                        qfine[QIDX((i - 1) * 2 + ii, (j - 1) * 2 + jj, mq, mbc, nx, ny)] =
                            q0 + shiftx * gradx + shifty * grady;
                    }
            }
    if (!acoarse) return;
    double r2 = 4;
    for (int m = 1; m <= meqn; m++)
        for (int i = 1; i <= mx / 2; i++)
            for (int j = 1; j <= my / 2; j++) {
                double sum = 0.0;
                for (int ii = 1; ii <= 2; ii++)
                    for (int jj = 1; jj <= 2; jj++) {
                        int ifine = (i - 1) * 2 + ii, jfine = (j - 1) * 2 + jj;
                        sum = sum + afine[ORC_AIDX(ifine, jfine, mbc, ax)] * qfine[QIDX(ifine, jfine, m, mbc, nx, ny)];
                    }
                double kc = acoarse[ORC_AIDX(i + ic_add, j + jc_add, mbc, ax)];
                double qc = qcoarse[QIDX(i + ic_add, j + jc_add, m, mbc, nx, ny)];
                double cons_diff = (qc * kc - sum) / r2;
                for (int ii = 1; ii <= 2; ii++)
                    for (int jj = 1; jj <= 2; jj++) {
                        int ifine = (i - 1) * 2 + ii, jfine = (j - 1) * 2 + jj;
                        qfine[QIDX(ifine, jfine, m, mbc, nx, ny)] =
                            qfine[QIDX(ifine, jfine, m, mbc, nx, ny)] + cons_diff / afine[ORC_AIDX(ifine, jfine, mbc, ax)];
                    }
            }
}

/* average2coarse (regrid): child igrid -> coarse patch interior quarter (average.f:282-364);
 * on a manifold sum(kf qf) / kc with the coarse patch's (new) areas. */
void orc_average2coarse(const orc_sim* s, double* qcoarse, const double* qfine, int igrid,
                        const double* acoarse, const double* afine)
{
    const orc_config* c = &s->cfg;
    const int mx = c->mx, my = c->my, mbc = c->mbc, meqn = c->meqn, nx = s->nx, ny = s->ny;
    const int ax = mx + 2 * mbc + 2;
    int ig = igrid % 2, jg = (igrid - ig) / 2;
    int ic_add = ig * mx / 2, jc_add = jg * mx / 2;
    for (int mq = 1; mq <= meqn; mq++)
        for (int j = 1; j <= my / 2; j++)
            for (int i = 1; i <= mx / 2; i++) {
                double sum = 0;
                for (int jj = 1; jj <= 2; jj++)
                    for (int ii = 1; ii <= 2; ii++) {
                        int fi = (i - 1) * 2 + ii, fj = (j - 1) * 2 + jj;
                        double qf = qfine[QIDX(fi, fj, mq, mbc, nx, ny)];
                        if (acoarse) sum = sum + afine[ORC_AIDX(fi, fj, mbc, ax)] * qf;
                        else sum = sum + qf;
                    }
                if (acoarse) qcoarse[QIDX(i + ic_add, j + jc_add, mq, mbc, nx, ny)] = sum / acoarse[ORC_AIDX(i + ic_add, j + jc_add, mbc, ax)];
                else qcoarse[QIDX(i + ic_add, j + jc_add, mq, mbc, nx, ny)] = sum / 4;
            }
}

/* Brick shifts used by the time-sync corrections below (same orientation; the
 * cubed sphere runs without time sync): transform_face same-block path
 * (forestclaw2d.c:655-662) and transform_face2's canonical first child. */
static void same_shift(const orc_patch* a, const orc_patch* b, int mx, int my, int* si, int* sj)
{
    *si = (a->gx - b->gx) * mx;
    *sj = (a->gy - b->gy) * my;
}

static void half_first(const orc_patch* a, const orc_patch* b, int mx, int my, int i, int j, int* di, int* dj)
{
    *di = 1 + (2 * a->gx - b->gx) * mx + 2 * (i - 1);
    *dj = 1 + (2 * a->gy - b->gy) * my + 2 * (j - 1);
}

/* ---------------- time interpolation ---------------- */
void orc_timeinterp(const orc_sim* s, const double* qcurr, const double* qlast, double* qinterp, double alpha)
{
    const orc_config* c = &s->cfg;
    const int mx = c->mx, my = c->my, mbc = c->mbc, meqn = c->meqn, nx = s->nx, ny = s->ny;
    const int mint = mbc;
#define TI(i, j) { size_t k_ = QIDX(i, j, m, mbc, nx, ny); qinterp[k_] = qlast[k_] + alpha * (qcurr[k_] - qlast[k_]); }
    for (int m = 1; m <= meqn; m++) {
        for (int j = 1; j <= my - mint; j++) for (int i = 1; i <= mint; i++) TI(i, j);
        for (int j = 1; j <= mint; j++) for (int i = mint + 1; i <= mx; i++) TI(i, j);
        for (int j = mint + 1; j <= my; j++) for (int i = mx - mint + 1; i <= mx; i++) TI(i, j);
        for (int j = my - mint + 1; j <= my; j++) for (int i = 1; i <= mx - mint; i++) TI(i, j);
    }
#undef TI
}

/* ---------------- time sync ---------------- */
/* fc46_is_valid_correct / fc46_skip_this_grid, clawpack46_time_sync.f:707-741 */
static int valid_correct(int i, int j, int mx, int my)
{
    int i1 = 1 <= i && i <= mx, j1 = 1 <= j && j <= my;
    return i1 != j1;
}
static int skip_ok(int di, int dj, int mx, int my)
{
    return valid_correct(di, dj, mx, my) && valid_correct(di + 1, dj, mx, my) &&
           valid_correct(di, dj + 1, mx, my) && valid_correct(di + 1, dj + 1, mx, my);
}

/* clawpack46_fort_time_sync_f2c, clawpack46_time_sync.f:254-498 (same orientation: sc = 1). */
void orc_time_sync_f2c(const orc_sim* s, orc_patch* C, const orc_patch* F, int iface_coarse)
{
    const orc_config* c = &s->cfg;
    const int mx = c->mx, my = c->my, mbc = c->mbc, meqn = c->meqn, nx = s->nx, ny = s->ny;
    const int dnx = mx + 4 * mbc, dny = my + 4 * mbc;
    double* dummy = s->dummy;   /* (1-2mbc:mx+2mbc, 1-2mbc:my+2mbc, meqn) */
    memset(dummy, 0, sizeof(double) * (size_t)dnx * dny * meqn);
#define DUM(i, j, m) dummy[QIDX(i, j, m, 2 * mbc, dnx, dny)]
    const orc_regs* rf = &F->regs;
    const orc_regs* rc = &C->regs;
    for (int mq = 1; mq <= meqn; mq++) {
        for (int j = 1; j <= my / 2; j++) {
            int jj1 = 2 * (j - 1) + 1, jj2 = 2 * (j - 1) + 2;
            double fm = rf->fm[0][RJ(jj1, mq, my)] + rf->fm[0][RJ(jj2, mq, my)];
            double ef = rf->ef[0][RJK(jj1, mq, 1, my, meqn)] + rf->ef[0][RJK(jj2, mq, 1, my, meqn)];
            for (int jj = jj1; jj <= jj2; jj++)
                for (int ii = -1; ii <= 0; ii++) { DUM(ii, jj, mq) = fm; DUM(ii - 2, jj, mq) = ef; }
            double fp = rf->fp[1][RJ(jj1, mq, my)] + rf->fp[1][RJ(jj2, mq, my)];
            ef = rf->ef[1][RJK(jj1, mq, 1, my, meqn)] + rf->ef[1][RJK(jj2, mq, 1, my, meqn)];
            for (int jj = jj1; jj <= jj2; jj++)
                for (int ii = 1; ii <= 2; ii++) { DUM(mx + ii, jj, mq) = fp; DUM(mx + ii + 2, jj, mq) = ef; }
        }
        for (int i = 1; i <= mx / 2; i++) {
            int ii1 = 2 * (i - 1) + 1, ii2 = 2 * (i - 1) + 2;
            double gm = rf->gm[0][RJ(ii1, mq, mx)] + rf->gm[0][RJ(ii2, mq, mx)];
            double ef = rf->ef[2][RJK(ii1, mq, 1, mx, meqn)] + rf->ef[2][RJK(ii2, mq, 1, mx, meqn)];
            for (int ii = ii1; ii <= ii2; ii++)
                for (int jj = -1; jj <= 0; jj++) { DUM(ii, jj, mq) = gm; DUM(ii, jj - 2, mq) = ef; }
            double gp = rf->gp[1][RJ(ii1, mq, mx)] + rf->gp[1][RJ(ii2, mq, mx)];
            ef = rf->ef[3][RJK(ii1, mq, 1, mx, meqn)] + rf->ef[3][RJK(ii2, mq, 1, mx, meqn)];
            for (int ii = ii1; ii <= ii2; ii++)
                for (int jj = 1; jj <= 2; jj++) { DUM(ii, my + jj, mq) = gp; DUM(ii, my + jj + 2, mq) = ef; }
        }
    }
    const int sc = 1;
    double* q = C->q;
    for (int mq = 1; mq <= meqn; mq++) {
        if (iface_coarse / 2 == 0) {
            for (int jc = 1; jc <= my; jc++) {
                double deltac = 0, areac = 1;
                int ic, di, dj, di2, dj2;
                if (iface_coarse == 0) {
                    ic = 1;
                    half_first(C, F, mx, my, ic, jc, &di, &dj);
                    areac = rc->area[0][jc - 1];
                    if (skip_ok(di, dj, mx, my)) {
                        double fp = DUM(di, dj, mq);
                        half_first(C, F, mx, my, ic + 1, jc, &di2, &dj2);
                        double ef = sc * DUM(di2, dj2, mq);
                        deltac = (ef - rc->ef[0][RJK(jc, mq, 0, my, meqn)]) - (fp - rc->fp[0][RJ(jc, mq, my)]);
                    }
                } else {
                    ic = mx;
                    half_first(C, F, mx, my, ic, jc, &di, &dj);
                    areac = rc->area[1][jc - 1];
                    if (skip_ok(di, dj, mx, my)) {
                        double fm = DUM(di, dj, mq);
                        half_first(C, F, mx, my, ic - 1, jc, &di2, &dj2);
                        double ef = sc * DUM(di2, dj2, mq);
                        deltac = (rc->ef[1][RJK(jc, mq, 0, my, meqn)] - ef) - (fm - rc->fm[1][RJ(jc, mq, my)]);
                    }
                }
                q[QIDX(ic, jc, mq, mbc, nx, ny)] = q[QIDX(ic, jc, mq, mbc, nx, ny)] + deltac / areac;
            }
        } else {
            for (int ic = 1; ic <= mx; ic++) {
                double deltac = 0, areac = 1;
                int jc, di, dj, di2, dj2;
                if (iface_coarse == 2) {
                    jc = 1;
                    half_first(C, F, mx, my, ic, jc, &di, &dj);
                    areac = rc->area[2][ic - 1];
                    if (skip_ok(di, dj, mx, my)) {
                        double gp = DUM(di, dj, mq);
                        half_first(C, F, mx, my, ic, jc + 1, &di2, &dj2);
                        double ef = sc * DUM(di2, dj2, mq);
                        deltac = (ef - rc->ef[2][RJK(ic, mq, 0, mx, meqn)]) - (gp - rc->gp[0][RJ(ic, mq, mx)]);
                    }
                } else {
                    jc = my;
                    half_first(C, F, mx, my, ic, jc, &di, &dj);
                    areac = rc->area[3][ic - 1];
                    if (skip_ok(di, dj, mx, my)) {
                        double gm = DUM(di, dj, mq);
                        half_first(C, F, mx, my, ic, jc - 1, &di2, &dj2);
                        double ef = sc * DUM(di2, dj2, mq);
                        deltac = (rc->ef[3][RJK(ic, mq, 0, mx, meqn)] - ef) - (gm - rc->gm[1][RJ(ic, mq, mx)]);
                    }
                }
                q[QIDX(ic, jc, mq, mbc, nx, ny)] = q[QIDX(ic, jc, mq, mbc, nx, ny)] + deltac / areac;
            }
        }
    }
#undef DUM
}

/* clawpack46_fort_time_sync_samesize, clawpack46_time_sync.f:528-704 (same orientation: sc = 1). */
void orc_time_sync_samesize(const orc_sim* s, orc_patch* P, const orc_patch* N, int this_iface)
{
    const orc_config* c = &s->cfg;
    const int mx = c->mx, my = c->my, mbc = c->mbc, meqn = c->meqn, nx = s->nx, ny = s->ny;
    double* dummy = s->dummy;   /* (1-mbc:mx+mbc, 1-mbc:my+mbc, meqn) */
    memset(dummy, 0, sizeof(double) * (size_t)nx * ny * meqn);
#define DUM(i, j, m) dummy[QIDX(i, j, m, mbc, nx, ny)]
    const orc_regs* rn = &N->regs;
    const orc_regs* rt = &P->regs;
    for (int mq = 1; mq <= meqn; mq++) {
        for (int j = 1; j <= my; j++) {
            DUM(0, j, mq) = rn->fm[0][RJ(j, mq, my)];
            DUM(-1, j, mq) = rn->ef[0][RJK(j, mq, 1, my, meqn)];
            DUM(mx + 1, j, mq) = rn->fp[1][RJ(j, mq, my)];
            DUM(mx + 2, j, mq) = rn->ef[1][RJK(j, mq, 1, my, meqn)];
        }
        for (int i = 1; i <= mx; i++) {
            DUM(i, 0, mq) = rn->gm[0][RJ(i, mq, mx)];
            DUM(i, -1, mq) = rn->ef[2][RJK(i, mq, 1, mx, meqn)];
            DUM(i, my + 1, mq) = rn->gp[1][RJ(i, mq, mx)];
            DUM(i, my + 2, mq) = rn->ef[3][RJK(i, mq, 1, mx, meqn)];
        }
    }
    int si, sj;
    same_shift(P, N, mx, my, &si, &sj);
    const int sc = 1;
    double* q = P->q;
    for (int mq = 1; mq <= meqn; mq++) {
        if (this_iface / 2 == 0) {
            for (int j = 1; j <= my; j++) {
                double delta, area;
                int i1;
                if (this_iface == 0) {
                    i1 = 1;
                    double fp = DUM(i1 + si, j + sj, mq);
                    double ef = sc * DUM(i1 + 1 + si, j + sj, mq);
                    delta = (ef - rt->ef[0][RJK(j, mq, 0, my, meqn)]) - (fp - rt->fp[0][RJ(j, mq, my)]);
                    area = rt->area[0][j - 1];
                } else {
                    i1 = mx;
                    double fm = DUM(i1 + si, j + sj, mq);
                    double ef = sc * DUM(i1 - 1 + si, j + sj, mq);
                    delta = (rt->ef[1][RJK(j, mq, 0, my, meqn)] - ef) - (fm - rt->fm[1][RJ(j, mq, my)]);
                    area = rt->area[1][j - 1];
                }
                q[QIDX(i1, j, mq, mbc, nx, ny)] = q[QIDX(i1, j, mq, mbc, nx, ny)] + 0.5 * delta / area;
            }
        } else {
            for (int i = 1; i <= mx; i++) {
                double delta, area;
                int j1;
                if (this_iface == 2) {
                    j1 = 1;
                    double gp = DUM(i + si, j1 + sj, mq);
                    double ef = sc * DUM(i + si, j1 + 1 + sj, mq);
                    delta = (ef - rt->ef[2][RJK(i, mq, 0, mx, meqn)]) - (gp - rt->gp[0][RJ(i, mq, mx)]);
                    area = rt->area[2][i - 1];
                } else {
                    j1 = my;
                    double gm = DUM(i + si, j1 + sj, mq);
                    double ef = sc * DUM(i + si, j1 - 1 + sj, mq);
                    delta = (rt->ef[3][RJK(i, mq, 0, mx, meqn)] - ef) - (gm - rt->gm[1][RJ(i, mq, mx)]);
                    area = rt->area[3][i - 1];
                }
                q[QIDX(i, j1, mq, mbc, nx, ny)] = q[QIDX(i, j1, mq, mbc, nx, ny)] + 0.5 * delta / area;
            }
        }
    }
#undef DUM
}

/* clawpack46_time_sync_store_flux, clawpack46_time_sync.f:37-156, with the
 * shallow-water rpn2_cons of applications/clawpack/shallow/2d/radialdam/rpn2cons_update.f. */
static void rpn2_cons_sw(int meqn, int idir, const double* q, double grav, double* flux)
{
    (void)meqn;
    int mu = (idir == 0) ? 2 : 3, mv = (idir == 0) ? 3 : 2;
    double hun = q[mu - 1], hut = q[mv - 1], h = q[0];
    double un = hun / h;
    flux[0] = hun;
    flux[mu - 1] = (hun * hun) / h + 0.5 * grav * (h * h);
    flux[mv - 1] = un * hut;
}

static void rpn2_cons(const orc_config* c, int idir, const double* q, double* flux)
{
    if (c->rp == ORC_RP_EULER_EXACT) orc_euler_cons_flux(c->gamma, idir, q, flux);
    else rpn2_cons_sw(c->meqn, idir, q, c->grav, flux);
}

void orc_store_flux(const orc_sim* s, orc_patch* P, double dt)
{
    const orc_config* c = &s->cfg;
    const int mx = c->mx, my = c->my, mbc = c->mbc, meqn = c->meqn, nx = s->nx, ny = s->ny;
    double qv[8] = {0}, fl[8] = {0};
    orc_regs* r = &P->regs;
    for (int j = 1; j <= my; j++) {
        for (int k = 0; k <= 1; k++) {
            for (int m = 1; m <= meqn; m++) qv[m - 1] = P->q[QIDX(1 - k, j, m, mbc, nx, ny)];
            rpn2_cons(c, 0, qv, fl);
            for (int m = 1; m <= meqn; m++)
                r->ef[0][RJK(j, m, k, my, meqn)] = r->ef[0][RJK(j, m, k, my, meqn)] + dt * r->el[0][j - 1] * fl[m - 1];
        }
        for (int k = 0; k <= 1; k++) {
            for (int m = 1; m <= meqn; m++) qv[m - 1] = P->q[QIDX(mx + k, j, m, mbc, nx, ny)];
            rpn2_cons(c, 0, qv, fl);
            for (int m = 1; m <= meqn; m++)
                r->ef[1][RJK(j, m, k, my, meqn)] = r->ef[1][RJK(j, m, k, my, meqn)] + dt * r->el[1][j - 1] * fl[m - 1];
        }
    }
    for (int i = 1; i <= mx; i++) {
        for (int k = 0; k <= 1; k++) {
            for (int m = 1; m <= meqn; m++) qv[m - 1] = P->q[QIDX(i, 1 - k, m, mbc, nx, ny)];
            rpn2_cons(c, 1, qv, fl);
            for (int m = 1; m <= meqn; m++)
                r->ef[2][RJK(i, m, k, mx, meqn)] = r->ef[2][RJK(i, m, k, mx, meqn)] + dt * r->el[2][i - 1] * fl[m - 1];
        }
        for (int k = 0; k <= 1; k++) {
            for (int m = 1; m <= meqn; m++) qv[m - 1] = P->q[QIDX(i, my + k, m, mbc, nx, ny)];
            rpn2_cons(c, 1, qv, fl);
            for (int m = 1; m <= meqn; m++)
                r->ef[3][RJK(i, m, k, mx, meqn)] = r->ef[3][RJK(i, m, k, mx, meqn)] + dt * r->el[3][i - 1] * fl[m - 1];
        }
    }
}

/* clawpack46_time_sync_accumulate_waves, clawpack46_time_sync.f:163-226 */
void orc_accumulate_waves(const orc_sim* s, orc_patch* P, double dt, double dx, double dy,
                          const double* fp, const double* fm, const double* gp, const double* gm)
{
    const orc_config* c = &s->cfg;
    const int mx = c->mx, my = c->my, mbc = c->mbc, meqn = c->meqn, nx = s->nx, ny = s->ny;
    orc_regs* r = &P->regs;
    for (int j = 1; j <= my; j++)
        for (int m = 1; m <= meqn; m++) {
            r->fp[0][RJ(j, m, my)] = r->fp[0][RJ(j, m, my)] - dt * dy * fp[QIDX(1, j, m, mbc, nx, ny)];
            r->fm[0][RJ(j, m, my)] = r->fm[0][RJ(j, m, my)] + dt * dy * fm[QIDX(1, j, m, mbc, nx, ny)];
            r->fp[1][RJ(j, m, my)] = r->fp[1][RJ(j, m, my)] - dt * dy * fp[QIDX(mx + 1, j, m, mbc, nx, ny)];
            r->fm[1][RJ(j, m, my)] = r->fm[1][RJ(j, m, my)] + dt * dy * fm[QIDX(mx + 1, j, m, mbc, nx, ny)];
        }
    for (int i = 1; i <= mx; i++)
        for (int m = 1; m <= meqn; m++) {
            r->gp[0][RJ(i, m, mx)] = r->gp[0][RJ(i, m, mx)] - dt * dx * gp[QIDX(i, 1, m, mbc, nx, ny)];
            r->gm[0][RJ(i, m, mx)] = r->gm[0][RJ(i, m, mx)] + dt * dx * gm[QIDX(i, 1, m, mbc, nx, ny)];
            r->gp[1][RJ(i, m, mx)] = r->gp[1][RJ(i, m, mx)] - dt * dx * gp[QIDX(i, my + 1, m, mbc, nx, ny)];
            r->gm[1][RJ(i, m, mx)] = r->gm[1][RJ(i, m, mx)] + dt * dx * gm[QIDX(i, my + 1, m, mbc, nx, ny)];
        }
}

/* fclaw2d_clawpatch_time_sync_reset, fclaw2d_clawpatch_conservation.c:207-280 (one face). */
void orc_regs_reset_face(const orc_sim* s, orc_patch* P, int k)
{
    const int mx = s->cfg.mx, my = s->cfg.my, meqn = s->cfg.meqn;
    orc_regs* r = &P->regs;
    if (k / 2 == 0) {
        for (int j = 0; j < meqn * my; j++) {
            r->fm[k][j] = 0; r->fp[k][j] = 0; r->ef[k][j] = 0; r->ef[k][j + meqn * my] = 0;
        }
    } else {
        for (int i = 0; i < meqn * mx; i++) {
            r->gm[k - 2][i] = 0; r->gp[k - 2][i] = 0; r->ef[k][i] = 0; r->ef[k][i + meqn * mx] = 0;
        }
    }
}
