// k_step2.cuh -- fused per-level patch update (clawpack 4.6 step2 + step2_wrap).
//
// One CTA advances one patch.  The padded patch (mx+2mbc)(my+2mbc)meqn is staged
// in shared memory with coalesced loads; every x- and y-interface of the
// reference's sweeps gets a thread; the flux arrays fm/fp/gm/gp of
// clawpack46_step2.f are accumulated in shared memory in exactly the
// reference's order (x-sweeps row by row, then y-sweeps column by column) by
// gathering per-interface results, so no atomics are needed and repeated runs
// are bitwise identical.  The same CTA also performs, from the staged tile,
//   b4step2 (swirl edge velocities),         user_4.6/b4step2.f:25-36
//   save_current_step (q -> qlast),          fclaw2d_clawpatch.cpp (save_current_step)
//   time-sync flux store / wave accumulation clawpack46_time_sync.f:37-226
//   the conservative q update over i,j = 1-mbc..mx+mbc-1 (clawpack46_step2_wrap.f:107-125)
//   and the warp-shuffle CFL maximum.
//
// Index conventions: padded 0-based cell (ic, jc), ic = i + mbc - 1 for the
// Fortran index i.  Interface ic sits between cells ic-1 and ic.
#pragma once
#include <cuda_runtime.h>
#include "fcb_common.h"
#include "riemann.cuh"

namespace fcb {

enum { APP_NONE = 0, APP_SWIRL = 1, APP_RADIALDAM = 2, APP_TSUNAMI = 3 };

template <class RP, int MX, int MY, int MBC, bool FWAVE>
struct Step2Geom {
    static constexpr int NX = MX + 2 * MBC, NY = MY + 2 * MBC, NXY = NX * NY;
    static constexpr int MEQN = RP::MEQN, MWAVES = RP::MWAVES, MAUX = RP::MAUX, NEXTRA = RP::NEXTRA;
    static constexpr int NIX = (NY - 2) * (NX - 1);          // x-sweep interfaces
    static constexpr int NIY = (NX - 2) * (NY - 1);          // y-sweep interfaces
    static constexpr int NI = NIX > NIY ? NIX : NIY;
    // per-interface record of the normal solve: waves, speeds, amdq, apdq, solver extra
    static constexpr int W_WAVE = 0, W_S = MWAVES * MEQN, W_AM = W_S + MWAVES, W_AP = W_AM + MEQN,
                         W_EX = W_AP + MEQN, WSZ = W_EX + NEXTRA;
    // per-interface transverse terms: A1, A2 (from amdq), B1, B2 (from apdq), flags
    static constexpr int TSZ = 4 * MEQN;
    static constexpr int AUXS = MAUX > 0 ? MAUX : 0;
    static constexpr size_t SMEM_DOUBLES = (size_t)MEQN * NXY * 5 + (size_t)AUXS * NXY + (size_t)WSZ * NI +
                                           (size_t)TSZ * NI + 64;
    static constexpr size_t SMEM_BYTES = SMEM_DOUBLES * sizeof(double) + (size_t)NI * 4;
    // conservation registers (fclaw2d_clawpatch_conservation.h:56-77), per patch
    static constexpr int R_FP0 = 0, R_FP1 = MY * MEQN, R_FM0 = 2 * MY * MEQN, R_FM1 = 3 * MY * MEQN;
    static constexpr int R_GP0 = 4 * MY * MEQN, R_GP1 = R_GP0 + MX * MEQN, R_GM0 = R_GP0 + 2 * MX * MEQN,
                         R_GM1 = R_GP0 + 3 * MX * MEQN;
    static constexpr int R_EF0 = R_GP0 + 4 * MX * MEQN, R_EF1 = R_EF0 + 2 * MY * MEQN,
                         R_EF2 = R_EF1 + 2 * MY * MEQN, R_EF3 = R_EF2 + 2 * MX * MEQN,
                         NREG = R_EF3 + 2 * MX * MEQN;
    // interface ranges of flux2 (FWAVE=false) / flux2fw (FWAVE=true) in padded indices
};

// Shallow-water flux function used by the time-sync flux store
// (applications/clawpack/shallow/2d/radialdam/rpn2cons_update.f).
template <typename T>
__device__ __forceinline__ void rpn2_cons_sw(int idir, const T* q, T grav, T* flux)
{
    const int mu = (idir == 0) ? 1 : 2, mv = (idir == 0) ? 2 : 1;
    T hun = q[mu], hut = q[mv], h = q[0];
    T un = hun / h;
    flux[0] = hun;
    flux[mu] = (hun * hun) / h + T(0.5) * grav * (h * h);
    flux[mv] = un * hut;
}

template <class RP, int MX, int MY, int MBC, bool FWAVE, int NT>
__global__ void __launch_bounds__(NT)
step2_f64_kernel(double* __restrict__ q, double* __restrict__ qlast, const double* __restrict__ aux,
                 double* __restrict__ regs, const PatchDesc* __restrict__ desc, int p0, StepParams sp,
                 unsigned long long* __restrict__ cfl_bits)
{
    using G = Step2Geom<RP, MX, MY, MBC, FWAVE>;
    constexpr int NX = G::NX, NY = G::NY, NXY = G::NXY, MEQN = G::MEQN, MWAVES = G::MWAVES;
    constexpr int MAUX = G::MAUX, NEXTRA = G::NEXTRA, NI = G::NI, WSZ = G::WSZ;
    // flux2 / flux2fw interface ranges (padded): Godunov, cqxx, amdq+=cqxx, transverse, CFL
    constexpr int GOD_LO = FWAVE ? MBC : 1, GOD_HI = FWAVE ? MX + MBC : NX - 2;
    constexpr int CQ_LO = FWAVE ? MBC : 1, CQ_HI = FWAVE ? MX + MBC : NX - 1;
    constexpr int AC_LO = FWAVE ? MBC : 1, AC_HI = FWAVE ? MX + MBC : NX - 2;
    constexpr int TR_LO = FWAVE ? MBC : 1, TR_HI = FWAVE ? MX + MBC : NX - 1;
    constexpr int GOD_LOY = FWAVE ? MBC : 1, GOD_HIY = FWAVE ? MY + MBC : NY - 2;
    constexpr int CQ_LOY = FWAVE ? MBC : 1, CQ_HIY = FWAVE ? MY + MBC : NY - 1;
    constexpr int AC_LOY = FWAVE ? MBC : 1, AC_HIY = FWAVE ? MY + MBC : NY - 2;
    constexpr int TR_LOY = FWAVE ? MBC : 1, TR_HIY = FWAVE ? MY + MBC : NY - 1;

    extern __shared__ double smem[];
    double* Qs = smem;                              // [MEQN][NY][NX]
    double* FMs = Qs + MEQN * NXY;
    double* FPs = FMs + MEQN * NXY;
    double* GMs = FPs + MEQN * NXY;
    double* GPs = GMs + MEQN * NXY;
    double* As = GPs + MEQN * NXY;                  // [MAUX][NY][NX]
    double* W = As + G::AUXS * NXY;                 // [WSZ][NI]  (SoA)
    double* Tt = W + (size_t)WSZ * NI;              // [TSZ][NI]
    double* red = Tt + (size_t)G::TSZ * NI;         // 64 doubles for reductions
    unsigned char* tflag = (unsigned char*)(red + 64);   // [NI] presence bits of A/B terms

    const int tid = threadIdx.x;
    const int p = p0 + blockIdx.x;
    const PatchDesc pd = desc[p];
    const double dx = pd.dx, dy = pd.dy;
    const double dt = sp.dt;
    const double dtdx = dt / dx, dtdy = dt / dy;
    double* qg = q + (size_t)p * MEQN * NXY;

    // ---- stage q (and aux) in shared memory --------------------------------
    for (int k = tid; k < MEQN * NXY; k += NT) {
        double v = qg[k];
        Qs[k] = v;
        if (sp.save_last) qlast[(size_t)p * MEQN * NXY + k] = v;
        FMs[k] = 0.0; FPs[k] = 0.0; GMs[k] = 0.0; GPs[k] = 0.0;
    }
    if (MAUX > 0) {
        const double* ag = aux + (size_t)p * G::AUXS * NXY;
        if (sp.app == APP_SWIRL) {
            // b4step2: aux(:,:,1) = vty*(psi(x,y+dy)-psi), aux(:,:,2) = -vtx*(psi(x+dx,y)-psi);
            // the stored aux holds the psi differences.
            const double vty = sp.vt / dy, vtx = sp.vt / dx;
            for (int k = tid; k < NXY; k += NT) {
                As[k] = vty * ag[k];
                As[NXY + k] = -(vtx * ag[NXY + k]);
            }
        } else {
            for (int k = tid; k < G::AUXS * NXY; k += NT) As[k] = ag[k];
        }
    }
    __syncthreads();

    const int mcapa = sp.mcapa;
    auto dtdx1d_x = [&](int ic, int jc) -> double {
        return mcapa > 0 ? dtdx / As[(mcapa - 1) * NXY + jc * NX + ic] : dtdx;
    };
    auto dtdy1d_y = [&](int ic, int jc) -> double {
        return mcapa > 0 ? dtdy / As[(mcapa - 1) * NXY + jc * NX + ic] : dtdy;
    };

    // ---- time-sync flux store (before the update) ----------------------------
    double* rg = regs + (size_t)p * G::NREG;
    if (MEQN >= 3 && sp.store_flux) {
        // faces 0,1: j = 1..my, k = 0,1 ; faces 2,3: i = 1..mx, k = 0,1
        for (int it = tid; it < 2 * 2 * MY + 2 * 2 * MX; it += NT) {
            int face, j, k;
            if (it < 4 * MY) { face = it / (2 * MY); int r = it % (2 * MY); j = r / 2; k = r % 2; }
            else { int r2 = it - 4 * MY; face = 2 + r2 / (2 * MX); int r = r2 % (2 * MX); j = r / 2; k = r % 2; }
            int ic, jc;
            if (face == 0) { ic = MBC - k; jc = MBC + j; }
            else if (face == 1) { ic = MX + MBC - 1 + k; jc = MBC + j; }
            else if (face == 2) { ic = MBC + j; jc = MBC - k; }
            else { ic = MBC + j; jc = MY + MBC - 1 + k; }
            double qv[MEQN >= 3 ? MEQN : 3], fl[MEQN >= 3 ? MEQN : 3];
            for (int m = 0; m < MEQN; m++) qv[m] = Qs[m * NXY + jc * NX + ic];
            rpn2_cons_sw<double>(face / 2, qv, sp.grav, fl);
            const int n = (face < 2) ? MY : MX;
            const double el = (face < 2) ? dy : dx;
            const int base = (face == 0) ? G::R_EF0 : (face == 1) ? G::R_EF1 : (face == 2) ? G::R_EF2 : G::R_EF3;
            for (int m = 0; m < MEQN; m++) {
                double* r = &rg[base + j + m * n + k * n * MEQN];
                *r = *r + dt * el * fl[m];
            }
        }
    }

    double cflmax = 0.0;

    // =================== x-sweeps (clawpack46_step2.f:113-167) ===================
    // X1: normal Riemann problems
    for (int k = tid; k < G::NIX; k += NT) {
        const int jc = 1 + k / (NX - 1), ic = 1 + k % (NX - 1);
        double qL[MEQN], qR[MEQN], aL[MAUX > 0 ? MAUX : 1], aR[MAUX > 0 ? MAUX : 1];
        for (int m = 0; m < MEQN; m++) { qL[m] = Qs[m * NXY + jc * NX + ic - 1]; qR[m] = Qs[m * NXY + jc * NX + ic]; }
        for (int a = 0; a < MAUX; a++) { aL[a] = As[a * NXY + jc * NX + ic - 1]; aR[a] = As[a * NXY + jc * NX + ic]; }
        double wave[MWAVES][MEQN], s[MWAVES], am[MEQN], ap[MEQN], ex[NEXTRA];
        RP::template rpn2<double>(1, qL, qR, aL, aR, wave, s, am, ap, ex, sp.grav);
        for (int mw = 0; mw < MWAVES; mw++) {
            for (int m = 0; m < MEQN; m++) W[(G::W_WAVE + mw * MEQN + m) * NI + k] = wave[mw][m];
            W[(G::W_S + mw) * NI + k] = s[mw];
        }
        for (int m = 0; m < MEQN; m++) { W[(G::W_AM + m) * NI + k] = am[m]; W[(G::W_AP + m) * NI + k] = ap[m]; }
        for (int e = 0; e < NEXTRA; e++) W[(G::W_EX + e) * NI + k] = ex[e];
        if (ic >= MBC && ic <= MX + MBC) {
            const double d1 = dtdx1d_x(ic, jc), d0 = dtdx1d_x(ic - 1, jc);
            for (int mw = 0; mw < MWAVES; mw++)
                cflmax = dmax1(dmax1(cflmax, d1 * s[mw]), -(d0 * s[mw]));
        }
    }
    __syncthreads();
    // X2: limiter, second-order correction, fadd, transverse splitting
    for (int k = tid; k < G::NIX; k += NT) {
        const int jc = 1 + k / (NX - 1), ic = 1 + k % (NX - 1);
        double wave[MWAVES][MEQN], s[MWAVES], am[MEQN], ap[MEQN], ex[NEXTRA], cq[MEQN];
        for (int mw = 0; mw < MWAVES; mw++) {
            for (int m = 0; m < MEQN; m++) wave[mw][m] = W[(G::W_WAVE + mw * MEQN + m) * NI + k];
            s[mw] = W[(G::W_S + mw) * NI + k];
        }
        for (int m = 0; m < MEQN; m++) { am[m] = W[(G::W_AM + m) * NI + k]; ap[m] = W[(G::W_AP + m) * NI + k]; }
        for (int e = 0; e < NEXTRA; e++) ex[e] = W[(G::W_EX + e) * NI + k];
        double faddm[MEQN], faddp[MEQN];
        for (int m = 0; m < MEQN; m++) { faddm[m] = 0.0; faddp[m] = 0.0; }
        if (ic >= GOD_LO && ic <= GOD_HI)
            for (int m = 0; m < MEQN; m++) { faddp[m] = faddp[m] - ap[m]; faddm[m] = faddm[m] + am[m]; }
        const bool second = FWAVE ? (sp.order1 != 1) : (sp.order1 == 2);
        if (second) {
            if (ic >= MBC && ic <= MX + MBC) {
                // inline limiter (clawpack46_inlinelimiter.f:267-343) with unlimited neighbours
                for (int mw = 0; mw < MWAVES; mw++) {
                    const int ml = sp.mthlim[mw];
                    if (ml == 0) continue;
                    double wnorm2 = 0.0, dotl = 0.0, dotr = 0.0;
                    for (int m = 0; m < MEQN; m++) {
                        const double w = wave[mw][m];
                        const double wl = W[(G::W_WAVE + mw * MEQN + m) * NI + k - 1];
                        const double wr = W[(G::W_WAVE + mw * MEQN + m) * NI + k + 1];
                        wnorm2 = wnorm2 + w * w;
                        dotl = dotl + wl * w;
                        dotr = dotr + w * wr;
                    }
                    if (wnorm2 == 0.0) continue;
                    const double r = (s[mw] > 0.0) ? dotl / wnorm2 : dotr / wnorm2;
                    const double wlim = limiter_phi<double>(ml, r);
                    for (int m = 0; m < MEQN; m++) wave[mw][m] = wlim * wave[mw][m];
                }
            }
            if (ic >= CQ_LO && ic <= CQ_HI) {
                const double dtdxave = 0.5 * (dtdx1d_x(ic - 1, jc) + dtdx1d_x(ic, jc));
                for (int m = 0; m < MEQN; m++) {
                    double c = 0.0;
                    for (int mw = 0; mw < MWAVES; mw++) {
                        if (FWAVE) c = c + sgn1(s[mw]) * (1.0 - fabs(s[mw]) * dtdxave) * wave[mw][m];
                        else { const double sa = fabs(s[mw]); c = c + sa * (1.0 - sa * dtdxave) * wave[mw][m]; }
                    }
                    cq[m] = c;
                    faddm[m] = faddm[m] + 0.5 * c;
                    faddp[m] = faddp[m] + 0.5 * c;
                }
            }
        }
        for (int m = 0; m < MEQN; m++) {
            FMs[m * NXY + jc * NX + ic] = 0.0 + faddm[m];
            FPs[m * NXY + jc * NX + ic] = 0.0 + faddp[m];
        }
        unsigned char fl = 0;
        if (sp.order2 > 0 && ic >= TR_LO && ic <= TR_HI) {
            if (sp.order1 > 1 && sp.order2 == 2 && ic >= AC_LO && ic <= AC_HI)
                for (int m = 0; m < MEQN; m++) { am[m] = am[m] + cq[m]; ap[m] = ap[m] - cq[m]; }
            double qL[MEQN], qR[MEQN];
            for (int m = 0; m < MEQN; m++) { qL[m] = Qs[m * NXY + jc * NX + ic - 1]; qR[m] = Qs[m * NXY + jc * NX + ic]; }
            double a1[MAUX > 0 ? MAUX : 1], a2[MAUX > 0 ? MAUX : 1], a3[MAUX > 0 ? MAUX : 1];
            double bm[MEQN], bp[MEQN];
            // amdq: aux of cell i1 = ic-1 on rows jc-1, jc, jc+1
            for (int a = 0; a < MAUX; a++) {
                a1[a] = As[a * NXY + (jc - 1) * NX + ic - 1];
                a2[a] = As[a * NXY + jc * NX + ic - 1];
                a3[a] = As[a * NXY + (jc + 1) * NX + ic - 1];
            }
            RP::template rpt2<double>(1, 1, qL, qR, a1, a2, a3, ex, am, bm, bp, sp.grav, sp.dry_tolerance);
            const double dlo = dtdx1d_x(ic - 1, jc);
            for (int m = 0; m < MEQN; m++) {
                Tt[(0 * MEQN + m) * NI + k] = 0.5 * dlo * bm[m];
                Tt[(1 * MEQN + m) * NI + k] = 0.5 * dlo * bp[m];
            }
            for (int a = 0; a < MAUX; a++) {
                a1[a] = As[a * NXY + (jc - 1) * NX + ic];
                a2[a] = As[a * NXY + jc * NX + ic];
                a3[a] = As[a * NXY + (jc + 1) * NX + ic];
            }
            RP::template rpt2<double>(1, 2, qL, qR, a1, a2, a3, ex, ap, bm, bp, sp.grav, sp.dry_tolerance);
            const double dhi = FWAVE ? dlo : dtdx1d_x(ic, jc);
            for (int m = 0; m < MEQN; m++) {
                Tt[(2 * MEQN + m) * NI + k] = 0.5 * dhi * bm[m];
                Tt[(3 * MEQN + m) * NI + k] = 0.5 * dhi * bp[m];
            }
            fl = 1;
        }
        tflag[k] = fl;
    }
    __syncthreads();
    // X3: gadd -> gm/gp.  gm(ic,jc) = ((0 + G2(row jc-1)) + G1(row jc)), gp identical.
    for (int c = tid; c < NXY; c += NT) {
        const int jc = c / NX, ic = c % NX;
        if (ic < 1 || jc < 1) continue;                  // accumulation range ic >= 1, rows >= 1
        for (int m = 0; m < MEQN; m++) {
            double g = 0.0;
            // row jc-1 (its gadd(:,2)) contributes to gm(ic,jc)
            if (jc - 1 >= 1 && jc - 1 <= NY - 2) {
                const int r = jc - 1;
                double v = 0.0;
                if (ic + 1 <= NX - 1) { const int kk = (r - 1) * (NX - 1) + ic; if (tflag[kk]) v = v - Tt[(1 * MEQN + m) * NI + kk]; }
                { const int kk = (r - 1) * (NX - 1) + ic - 1; if (tflag[kk]) v = v - Tt[(3 * MEQN + m) * NI + kk]; }
                g = g + v;
            }
            if (jc <= NY - 2) {
                const int r = jc;
                double v = 0.0;
                if (ic + 1 <= NX - 1) { const int kk = (r - 1) * (NX - 1) + ic; if (tflag[kk]) v = v - Tt[(0 * MEQN + m) * NI + kk]; }
                { const int kk = (r - 1) * (NX - 1) + ic - 1; if (tflag[kk]) v = v - Tt[(2 * MEQN + m) * NI + kk]; }
                g = g + v;
            }
            GMs[m * NXY + c] = g;
            GPs[m * NXY + c] = g;
        }
    }
    __syncthreads();

    // =================== y-sweeps (clawpack46_step2.f:182-236) ===================
    // interface k -> column ic = 1 + k / (NY-1), interface jc = 1 + k % (NY-1)
    for (int k = tid; k < G::NIY; k += NT) {
        const int ic = 1 + k / (NY - 1), jc = 1 + k % (NY - 1);
        double qL[MEQN], qR[MEQN], aL[MAUX > 0 ? MAUX : 1], aR[MAUX > 0 ? MAUX : 1];
        for (int m = 0; m < MEQN; m++) { qL[m] = Qs[m * NXY + (jc - 1) * NX + ic]; qR[m] = Qs[m * NXY + jc * NX + ic]; }
        for (int a = 0; a < MAUX; a++) { aL[a] = As[a * NXY + (jc - 1) * NX + ic]; aR[a] = As[a * NXY + jc * NX + ic]; }
        double wave[MWAVES][MEQN], s[MWAVES], am[MEQN], ap[MEQN], ex[NEXTRA];
        RP::template rpn2<double>(2, qL, qR, aL, aR, wave, s, am, ap, ex, sp.grav);
        for (int mw = 0; mw < MWAVES; mw++) {
            for (int m = 0; m < MEQN; m++) W[(G::W_WAVE + mw * MEQN + m) * NI + k] = wave[mw][m];
            W[(G::W_S + mw) * NI + k] = s[mw];
        }
        for (int m = 0; m < MEQN; m++) { W[(G::W_AM + m) * NI + k] = am[m]; W[(G::W_AP + m) * NI + k] = ap[m]; }
        for (int e = 0; e < NEXTRA; e++) W[(G::W_EX + e) * NI + k] = ex[e];
        if (jc >= MBC && jc <= MY + MBC) {
            const double d1 = dtdy1d_y(ic, jc), d0 = dtdy1d_y(ic, jc - 1);
            for (int mw = 0; mw < MWAVES; mw++)
                cflmax = dmax1(dmax1(cflmax, d1 * s[mw]), -(d0 * s[mw]));
        }
    }
    __syncthreads();
    for (int k = tid; k < G::NIY; k += NT) {
        const int ic = 1 + k / (NY - 1), jc = 1 + k % (NY - 1);
        double wave[MWAVES][MEQN], s[MWAVES], am[MEQN], ap[MEQN], ex[NEXTRA], cq[MEQN];
        for (int mw = 0; mw < MWAVES; mw++) {
            for (int m = 0; m < MEQN; m++) wave[mw][m] = W[(G::W_WAVE + mw * MEQN + m) * NI + k];
            s[mw] = W[(G::W_S + mw) * NI + k];
        }
        for (int m = 0; m < MEQN; m++) { am[m] = W[(G::W_AM + m) * NI + k]; ap[m] = W[(G::W_AP + m) * NI + k]; }
        for (int e = 0; e < NEXTRA; e++) ex[e] = W[(G::W_EX + e) * NI + k];
        double faddm[MEQN], faddp[MEQN];
        for (int m = 0; m < MEQN; m++) { faddm[m] = 0.0; faddp[m] = 0.0; }
        if (jc >= GOD_LOY && jc <= GOD_HIY)
            for (int m = 0; m < MEQN; m++) { faddp[m] = faddp[m] - ap[m]; faddm[m] = faddm[m] + am[m]; }
        const bool second = FWAVE ? (sp.order1 != 1) : (sp.order1 == 2);
        if (second) {
            if (jc >= MBC && jc <= MY + MBC) {
                for (int mw = 0; mw < MWAVES; mw++) {
                    const int ml = sp.mthlim[mw];
                    if (ml == 0) continue;
                    double wnorm2 = 0.0, dotl = 0.0, dotr = 0.0;
                    for (int m = 0; m < MEQN; m++) {
                        const double w = wave[mw][m];
                        const double wl = W[(G::W_WAVE + mw * MEQN + m) * NI + k - 1];
                        const double wr = W[(G::W_WAVE + mw * MEQN + m) * NI + k + 1];
                        wnorm2 = wnorm2 + w * w;
                        dotl = dotl + wl * w;
                        dotr = dotr + w * wr;
                    }
                    if (wnorm2 == 0.0) continue;
                    const double r = (s[mw] > 0.0) ? dotl / wnorm2 : dotr / wnorm2;
                    const double wlim = limiter_phi<double>(ml, r);
                    for (int m = 0; m < MEQN; m++) wave[mw][m] = wlim * wave[mw][m];
                }
            }
            if (jc >= CQ_LOY && jc <= CQ_HIY) {
                const double dtdxave = 0.5 * (dtdy1d_y(ic, jc - 1) + dtdy1d_y(ic, jc));
                for (int m = 0; m < MEQN; m++) {
                    double c = 0.0;
                    for (int mw = 0; mw < MWAVES; mw++) {
                        if (FWAVE) c = c + sgn1(s[mw]) * (1.0 - fabs(s[mw]) * dtdxave) * wave[mw][m];
                        else { const double sa = fabs(s[mw]); c = c + sa * (1.0 - sa * dtdxave) * wave[mw][m]; }
                    }
                    cq[m] = c;
                    faddm[m] = faddm[m] + 0.5 * c;
                    faddp[m] = faddp[m] + 0.5 * c;
                }
            }
        }
        for (int m = 0; m < MEQN; m++) {
            GMs[m * NXY + jc * NX + ic] = GMs[m * NXY + jc * NX + ic] + faddm[m];
            GPs[m * NXY + jc * NX + ic] = GPs[m * NXY + jc * NX + ic] + faddp[m];
        }
        unsigned char fl = 0;
        if (sp.order2 > 0 && jc >= TR_LOY && jc <= TR_HIY) {
            if (sp.order1 > 1 && sp.order2 == 2 && jc >= AC_LOY && jc <= AC_HIY)
                for (int m = 0; m < MEQN; m++) { am[m] = am[m] + cq[m]; ap[m] = ap[m] - cq[m]; }
            double qL[MEQN], qR[MEQN];
            for (int m = 0; m < MEQN; m++) { qL[m] = Qs[m * NXY + (jc - 1) * NX + ic]; qR[m] = Qs[m * NXY + jc * NX + ic]; }
            double a1[MAUX > 0 ? MAUX : 1], a2[MAUX > 0 ? MAUX : 1], a3[MAUX > 0 ? MAUX : 1];
            double bm[MEQN], bp[MEQN];
            // amdq: aux of sweep cell i1 = jc-1 on columns ic-1, ic, ic+1
            for (int a = 0; a < MAUX; a++) {
                a1[a] = As[a * NXY + (jc - 1) * NX + ic - 1];
                a2[a] = As[a * NXY + (jc - 1) * NX + ic];
                a3[a] = As[a * NXY + (jc - 1) * NX + ic + 1];
            }
            RP::template rpt2<double>(2, 1, qL, qR, a1, a2, a3, ex, am, bm, bp, sp.grav, sp.dry_tolerance);
            const double dlo = dtdy1d_y(ic, jc - 1);
            for (int m = 0; m < MEQN; m++) {
                Tt[(0 * MEQN + m) * NI + k] = 0.5 * dlo * bm[m];
                Tt[(1 * MEQN + m) * NI + k] = 0.5 * dlo * bp[m];
            }
            for (int a = 0; a < MAUX; a++) {
                a1[a] = As[a * NXY + jc * NX + ic - 1];
                a2[a] = As[a * NXY + jc * NX + ic];
                a3[a] = As[a * NXY + jc * NX + ic + 1];
            }
            RP::template rpt2<double>(2, 2, qL, qR, a1, a2, a3, ex, ap, bm, bp, sp.grav, sp.dry_tolerance);
            const double dhi = FWAVE ? dlo : dtdy1d_y(ic, jc);
            for (int m = 0; m < MEQN; m++) {
                Tt[(2 * MEQN + m) * NI + k] = 0.5 * dhi * bm[m];
                Tt[(3 * MEQN + m) * NI + k] = 0.5 * dhi * bp[m];
            }
            fl = 1;
        }
        tflag[k] = fl;
    }
    __syncthreads();
    // Y3: gadd -> fm/fp.  fm(ic,jc) = (fm + G2(col ic-1)) + G1(col ic)
    for (int c = tid; c < NXY; c += NT) {
        const int jc = c / NX, ic = c % NX;
        if (jc < 1) continue;
        for (int m = 0; m < MEQN; m++) {
            double fm = FMs[m * NXY + c], fp = FPs[m * NXY + c];
            if (ic - 1 >= 1 && ic - 1 <= NX - 2) {
                const int col = ic - 1;
                double v = 0.0;
                if (jc + 1 <= NY - 1) { const int kk = (col - 1) * (NY - 1) + jc; if (tflag[kk]) v = v - Tt[(1 * MEQN + m) * NI + kk]; }
                { const int kk = (col - 1) * (NY - 1) + jc - 1; if (tflag[kk]) v = v - Tt[(3 * MEQN + m) * NI + kk]; }
                fm = fm + v; fp = fp + v;
            }
            if (ic >= 1 && ic <= NX - 2) {
                const int col = ic;
                double v = 0.0;
                if (jc + 1 <= NY - 1) { const int kk = (col - 1) * (NY - 1) + jc; if (tflag[kk]) v = v - Tt[(0 * MEQN + m) * NI + kk]; }
                { const int kk = (col - 1) * (NY - 1) + jc - 1; if (tflag[kk]) v = v - Tt[(2 * MEQN + m) * NI + kk]; }
                fm = fm + v; fp = fp + v;
            }
            FMs[m * NXY + c] = fm;
            FPs[m * NXY + c] = fp;
        }
    }
    __syncthreads();

    // ---- time-sync wave accumulation (clawpack46_time_sync.f:163-226) --------
    if (sp.accumulate_waves) {
        const double dtdyv = dt * dy, dtdxv = dt * dx;
        for (int it = tid; it < (MY + MX) * MEQN; it += NT) {
            if (it < MY * MEQN) {
                const int j = it % MY, m = it / MY;
                const int jc = MBC + j;
                const int cl = m * NXY + jc * NX + MBC, cr = m * NXY + jc * NX + MX + MBC;
                double* r;
                r = &rg[G::R_FP0 + j + m * MY]; *r = *r - dtdyv * FPs[cl];
                r = &rg[G::R_FM0 + j + m * MY]; *r = *r + dtdyv * FMs[cl];
                r = &rg[G::R_FP1 + j + m * MY]; *r = *r - dtdyv * FPs[cr];
                r = &rg[G::R_FM1 + j + m * MY]; *r = *r + dtdyv * FMs[cr];
            } else {
                const int i2 = it - MY * MEQN;
                const int i = i2 % MX, m = i2 / MX;
                const int ic = MBC + i;
                const int cb = m * NXY + MBC * NX + ic, ct = m * NXY + (MY + MBC) * NX + ic;
                double* r;
                r = &rg[G::R_GP0 + i + m * MX]; *r = *r - dtdxv * GPs[cb];
                r = &rg[G::R_GM0 + i + m * MX]; *r = *r + dtdxv * GMs[cb];
                r = &rg[G::R_GP1 + i + m * MX]; *r = *r - dtdxv * GPs[ct];
                r = &rg[G::R_GM1 + i + m * MX]; *r = *r + dtdxv * GMs[ct];
            }
        }
    }

    // ---- q update over i,j = 1-mbc..mx+mbc-1 (clawpack46_step2_wrap.f:107-125) ----
    for (int k = tid; k < MEQN * NXY; k += NT) {
        const int m = k / NXY, c = k % NXY;
        const int jc = c / NX, ic = c % NX;
        double v = Qs[k];
        if (ic <= NX - 2 && jc <= NY - 2) {
            const int b = m * NXY;
            if (mcapa == 0)
                v = v - dtdx * (FMs[b + c + 1] - FPs[b + c]) - dtdy * (GMs[b + c + NX] - GPs[b + c]);
            else
                v = v - (dtdx * (FMs[b + c + 1] - FPs[b + c]) + dtdy * (GMs[b + c + NX] - GPs[b + c])) /
                            As[(mcapa - 1) * NXY + c];
        }
        qg[k] = v;
    }

    // ---- CFL maximum: warp shuffles, then one atomic per CTA -----------------
    for (int off = 16; off > 0; off >>= 1) cflmax = dmax1(cflmax, __shfl_xor_sync(0xffffffffu, cflmax, off));
    if ((tid & 31) == 0) red[tid >> 5] = cflmax;
    __syncthreads();
    if (tid < 32) {
        double v = (tid < NT / 32) ? red[tid] : 0.0;
        for (int off = 16; off > 0; off >>= 1) v = dmax1(v, __shfl_xor_sync(0xffffffffu, v, off));
        if (tid == 0) {
            unsigned long long bits = (unsigned long long)__double_as_longlong(v);
            if (v != v) bits = 0x7ff8000000000000ull;   // NaN (e.g. negative depth) wins the max
            atomicMax(cfl_bits, bits);
        }
    }
}

}  // namespace fcb
