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
// TW is the arithmetic type of the waves, speeds, limiter, second-order
// correction and transverse splitting.  TW = double is the FP64 path (built
// without FMA contraction: bitwise equal to the FP64 CPU path).  TW = float is
// the FP32-wave path: the flux arrays fm/fp/gm/gp, the q update, the time-sync
// registers and the CFL reduction stay FP64, and the Godunov split is taken as
// an FP64 remainder, amdq = [f(q_i) - f(q_{i-1})](FP64) - apdq, so that
// amdq + apdq telescopes to FP64 round-off and mass stays conserved to
// FP64 accuracy although the waves are FP32.
//
// Index conventions: padded 0-based cell (ic, jc), ic = i + mbc - 1 for the
// Fortran index i.  Interface ic sits between cells ic-1 and ic.
#pragma once
#include <cuda_runtime.h>
#include <type_traits>
#include "fcb_common.h"
#include "fcb_launch.cuh"
#include "riemann.cuh"
#include "k_mlp.cuh"

namespace fcb {

enum { APP_NONE = 0, APP_SWIRL = 1, APP_RADIALDAM = 2, APP_TSUNAMI = 3, APP_SHOCKBUBBLE = 4 };

// Optional solver hooks.  A solver struct that declares USER_HOOKS = true may also
// declare HAS_B4STEP2 / HAS_SRC2 with the cell-wise b4step2 / src2 of
// include/fc2d_b200_user.cuh, and AUX_BOTH = true to receive in rpt2 the aux of
// both cells beside the interface, cudaclaw's layout (cudaclaw_flux2.cu:682-694):
// aux1/aux2/aux3[imp * maux + m], imp = 0 for the left cell, 1 for the right.
// Solvers whose field 0 is a water depth declare DEPTH = true: a negative depth is
// reported through the status word.
template <class RP, class = void> struct RPDepth { static constexpr bool value = false; };
template <class RP> struct RPDepth<RP, std::void_t<decltype(RP::DEPTH)>> { static constexpr bool value = RP::DEPTH; };

template <class RP, class = void>
struct RPHooks { static constexpr bool B4 = false, SRC = false, AUX_BOTH = false; };
template <class RP>
struct RPHooks<RP, std::void_t<decltype(RP::USER_HOOKS)>> {
    static constexpr bool B4 = RP::HAS_B4STEP2, SRC = RP::HAS_SRC2, AUX_BOTH = RP::AUX_BOTH;
};

template <class RP, int MX, int MY, int MBC, typename TW, int NT = 0>
struct Step2Geom {
    static constexpr bool F32 = std::is_same<TW, float>::value;
    static constexpr int NX = MX + 2 * MBC, NY = MY + 2 * MBC, NXY = NX * NY;
    static constexpr int MEQN = RP::MEQN, MWAVES = RP::MWAVES, MAUX = RP::MAUX, NEXTRA = RP::NEXTRA;
    static constexpr int NIX = (NY - 2) * (NX - 1);          // x-sweep interfaces
    // y-sweep interfaces, numbered with i fastest (k = (jc-1)(NX-2) + ic-1), so the
    // threads of a warp touch consecutive cells of a row of the shared-memory arrays
    static constexpr int NIY = (NX - 2) * (NY - 1);
    static constexpr int NI = NIX > NIY ? NIX : NIY;
    // REG: every interface of a sweep has its own thread, so the normal solve
    // (speeds, fluctuations, Roe averages) stays in registers across the
    // barrier and only the waves, which the limiter reads from the neighbours,
    // go through shared memory.
    static constexpr bool REG = NT >= NI;
    // per-interface record of the normal solve: waves, speeds, amdq, apdq, solver extra
    static constexpr int W_WAVE = 0, W_S = MWAVES * MEQN, W_AM = W_S + MWAVES, W_AP = W_AM + MEQN,
                         W_EX = W_AP + MEQN, WSZ_FULL = W_EX + NEXTRA;
    static constexpr int WSZ = REG ? MWAVES * MEQN : WSZ_FULL;
    // per-interface transverse terms: A1, A2 (from amdq), B1, B2 (from apdq)
    static constexpr int TSZ = 4 * MEQN;
    static constexpr int AUXS = MAUX > 0 ? MAUX : 0;
    static constexpr bool USE_FLX = F32 && RP::CONS_FLUX;   // per-cell FP64 fluxes (remainder / Godunov split)
    static constexpr size_t DOUBLES = (size_t)MEQN * NXY * 5 + (size_t)AUXS * NXY +
                                      (USE_FLX ? (size_t)MEQN * NXY : 0) + 64;
    static constexpr size_t TWS = (size_t)WSZ * NI + (size_t)TSZ * NI + (F32 ? (size_t)MEQN * NXY : 0);
    static constexpr size_t SMEM_BYTES = DOUBLES * 8 + TWS * sizeof(TW) + NI;
    // conservation registers (fclaw2d_clawpatch_conservation.h:56-77), per patch
    static constexpr int R_FP0 = 0, R_FP1 = MY * MEQN, R_FM0 = 2 * MY * MEQN, R_FM1 = 3 * MY * MEQN;
    static constexpr int R_GP0 = 4 * MY * MEQN, R_GP1 = R_GP0 + MX * MEQN, R_GM0 = R_GP0 + 2 * MX * MEQN,
                         R_GM1 = R_GP0 + 3 * MX * MEQN;
    static constexpr int R_EF0 = R_GP0 + 4 * MX * MEQN, R_EF1 = R_EF0 + 2 * MY * MEQN,
                         R_EF2 = R_EF1 + 2 * MY * MEQN, R_EF3 = R_EF2 + 2 * MX * MEQN,
                         NREG = R_EF3 + 2 * MX * MEQN;
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

// Correctly rounded, uncontracted multiply / add.  The FP32-wave unit is built with
// FMA contraction; the second-order correction must not be contracted, or the
// exactly opposite terms of the waves at a reflecting wall leave the rounding
// error of one product as a flux through the wall.
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }

// The update of patch p by the whole CTA (one call per patch; the CTA may do
// several patches in turn).  nhist: the CTA's shared Newton-iteration counters.
template <class RP, int MX, int MY, int MBC, bool FWAVE, int NT, typename TW>
__device__ __forceinline__ void
step2_patch(double* __restrict__ q, double* __restrict__ qlast, const double* __restrict__ aux,
            double* __restrict__ regs, const PatchDesc* __restrict__ desc, const int p,
            const StepParams& sp, unsigned long long* __restrict__ cfl_bits, unsigned int* nhist)
{
    using G = Step2Geom<RP, MX, MY, MBC, TW, NT>;
    constexpr bool F32 = G::F32, REG = G::REG;
    static_assert(!RP::EXACT64 || G::REG, "exact solvers keep their FP64 fluctuations in registers");
    constexpr int NX = G::NX, NY = G::NY, NXY = G::NXY, MEQN = G::MEQN, MWAVES = G::MWAVES;
    constexpr int MAUX = G::MAUX, NEXTRA = G::NEXTRA, NI = G::NI, WSZ = G::WSZ;
    constexpr int MA = MAUX > 0 ? MAUX : 1;
    // flux2 / flux2fw interface ranges (padded): Godunov, cqxx, amdq+=cqxx, transverse
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
    double* FLX = As + G::AUXS * NXY;               // [MEQN][NY][NX] cell fluxes (FP32-wave path)
    double* red = FLX + (G::USE_FLX ? MEQN * NXY : 0);   // 64 doubles for reductions
    TW* W = reinterpret_cast<TW*>(red + 64);        // [WSZ][NI]  (SoA)
    TW* Tt = W + (size_t)WSZ * NI;                  // [TSZ][NI]
    TW* Qf = Tt + (size_t)G::TSZ * NI;              // [MEQN][NY][NX] q in TW (FP32-wave path)
    unsigned char* tflag = reinterpret_cast<unsigned char*>(Qf + (F32 ? MEQN * NXY : 0));

    const int tid = threadIdx.x;
    if (RP::EXACT64 && tid < 32) nhist[tid] = 0u;          // Newton iterations of this patch
    const PatchDesc pd = desc[p];
    const double dx = pd.dx, dy = pd.dy;
    const double dt = sp.inst_dt ? sp.dt * sp.inst_dt[pd.inst] : sp.dt;
    const double dtdx = dt / dx, dtdy = dt / dy;
    double* qg = q + (size_t)p * MEQN * NXY;
    // save_current_step: only the data time interpolation will read (coarser
    // levels of a subcycled step, patches with fine-grid neighbours)
    const bool save = sp.save_last && (pd.flags & PATCH_HAS_FINE_NBR);

    // ---- stage q (and aux) in shared memory --------------------------------
    unsigned bad = 0;        // STATUS_* found in this thread's cells
    for (int k = tid; k < MEQN * NXY; k += NT) {
        double v = qg[k];
        if (!isfinite(v)) bad |= STATUS_NONFINITE;
        if constexpr (RPDepth<RP>::value) { if (k < NXY && v < 0.0) bad |= STATUS_DEPTH; }
        Qs[k] = v;
        if (F32) Qf[k] = (TW)v;
        if (save) qlast[(size_t)p * MEQN * NXY + k] = v;
        FMs[k] = 0.0; FPs[k] = 0.0; GMs[k] = 0.0; GPs[k] = 0.0;
    }
    if (bad && sp.status) atomicOr(sp.status, bad);
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
    if constexpr (RPHooks<RP>::B4) {
        // user b4step2, cell by cell over the padded patch (cudaclaw_flux2.cu:111-150):
        // it may set the cell's aux from its q, position and time.  As the reference's
        // b4step2 it changes the patch's aux in place (the only write to the aux slab
        // during an update; each CTA writes its own patch)
        double* ag = const_cast<double*>(aux) + (size_t)p * G::AUXS * NXY;
        for (int c = tid; c < NXY; c += NT) {
            double qc[MEQN], ac[G::AUXS > 0 ? G::AUXS : 1];
            for (int m = 0; m < MEQN; m++) qc[m] = Qs[m * NXY + c];
            for (int a = 0; a < G::AUXS; a++) ac[a] = As[a * NXY + c];
            RP::b4step2(MBC, MX, MY, MEQN, qc, pd.xlower, pd.ylower, dx, dy, sp.t, dt, G::AUXS, ac,
                        c % NX - MBC + 1, c / NX - MBC + 1);
            for (int a = 0; a < G::AUXS; a++) { As[a * NXY + c] = ac[a]; ag[a * NXY + c] = ac[a]; }
        }
        __syncthreads();
    }

    const int mcapa = sp.mcapa;
    auto dtdx1d_x = [&](int ic, int jc) -> TW {
        return mcapa > 0 ? (TW)(dtdx / As[(mcapa - 1) * NXY + jc * NX + ic]) : (TW)dtdx;
    };
    auto dtdy1d_y = [&](int ic, int jc) -> TW {
        return mcapa > 0 ? (TW)(dtdy / As[(mcapa - 1) * NXY + jc * NX + ic]) : (TW)dtdy;
    };
    auto qload = [&](int m, int c) -> TW {
        if constexpr (F32) { return Qf[m * NXY + c]; }
        else { return (TW)Qs[m * NXY + c]; }
    };
    const TW gravw = (TW)sp.grav, drytolw = (TW)sp.dry_tolerance;

    // ---- time-sync flux store (before the update), FP64 ----------------------
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
            if constexpr (RP::EXACT64) { RP::cons_flux(face / 2, qv, sp.gamma, fl); }
            else { rpn2_cons_sw<double>(face / 2, qv, sp.grav, fl); }
            const int n = (face < 2) ? MY : MX;
            const double el = (face < 2) ? dy : dx;
            const int base = (face == 0) ? G::R_EF0 : (face == 1) ? G::R_EF1 : (face == 2) ? G::R_EF2 : G::R_EF3;
            const bool zero = (sp.reg_reset >> ((pd.face_type >> (2 * face)) & 3)) & 1;
            for (int m = 0; m < MEQN; m++) {
                double* r = &rg[base + j + m * n + k * n * MEQN];
                *r = (zero ? 0.0 : *r) + dt * el * fl[m];
            }
        }
    }

    double cflmax = 0.0;
    TW cflw = TW(0);

    // Reflecting walls of this patch (FP32-wave path).  Mirror symmetry makes the
    // mass flux through a wall exactly zero -- first-order part, second-order
    // correction and the transverse terms of the two rows (columns) beside it
    // cancel -- but FP32 waves only reproduce that cancellation to FP32 rounding,
    // which leaks about 1e-8 of the mass per step.  The FP32-wave path therefore
    // takes the exact value, zero, for the mass component (m = 0) at these faces;
    // the FP64 path keeps the reference's arithmetic.
    const int wallf = (F32 && RP::CONS_FLUX) ? (pd.phys_mask & sp.wall_faces) : 0;

    // g64: FP64 amdq, apdq of exact solvers (kept for the Godunov update)
    struct State { TW wave[MWAVES][MEQN]; TW s[MWAVES]; TW am[MEQN]; TW ap[MEQN]; TW ex[NEXTRA];
                   double g64[RP::EXACT64 ? 2 * MEQN : 1]; };

    // Normal solve of one interface (qL = cell cL, qR = cell cR).
    auto normal_solve = [&](int ixy, int cL, int cR, int k, bool cfl_range, TW d1, TW d0, State& st, double seed) {
        if constexpr (RP::EXACT64 && F32) {
            float qL[MEQN], qR[MEQN], w32[MWAVES][MEQN], s32[MWAVES], ex32[NEXTRA];
            double qL64[MEQN], qR64[MEQN], fL[MEQN], fR[MEQN], am64[MEQN], ap64[MEQN];
            for (int m = 0; m < MEQN; m++) {
                qL[m] = Qf[m * NXY + cL]; qR[m] = Qf[m * NXY + cR];
                qL64[m] = Qs[m * NXY + cL]; qR64[m] = Qs[m * NXY + cR];
                fL[m] = FLX[m * NXY + cL]; fR[m] = FLX[m * NXY + cR];
            }
            const EulerParams ep{sp.gamma, sp.newton_tol, seed};
            const int r = RP::solve_mixed(ixy, qL, qR, qL64, qR64, fL, fR, ep, w32, s32, am64, ap64, ex32);
            const int it = r & 0xff;
            atomicAdd(&nhist[it < 31 ? it : 31], 1u);
            if ((r & RP::NEWTON_FAILED) && sp.status) atomicOr(sp.status, (unsigned)STATUS_NEWTON);
            for (int mw = 0; mw < MWAVES; mw++) {
                st.s[mw] = (TW)s32[mw];
                for (int m = 0; m < MEQN; m++) st.wave[mw][m] = (TW)w32[mw][m];
            }
            for (int m = 0; m < MEQN; m++) {
                st.am[m] = (TW)am64[m]; st.ap[m] = (TW)ap64[m];
                st.g64[m] = am64[m]; st.g64[MEQN + m] = ap64[m];
            }
            for (int e = 0; e < NEXTRA; e++) st.ex[e] = (TW)ex32[e];
        } else if constexpr (RP::EXACT64) {
            double qL64[MEQN], qR64[MEQN], w64[MWAVES][MEQN], s64[MWAVES], am64[MEQN], ap64[MEQN], ex64[NEXTRA];
            for (int m = 0; m < MEQN; m++) { qL64[m] = Qs[m * NXY + cL]; qR64[m] = Qs[m * NXY + cR]; }
            const EulerParams ep{sp.gamma, sp.newton_tol, seed};
            const int r = RP::solve64(ixy, qL64, qR64, ep, w64, s64, am64, ap64, ex64);
            const int it = r & 0xff;
            atomicAdd(&nhist[it < 31 ? it : 31], 1u);
            if ((r & RP::NEWTON_FAILED) && sp.status) atomicOr(sp.status, (unsigned)STATUS_NEWTON);
            for (int mw = 0; mw < MWAVES; mw++) {
                st.s[mw] = (TW)s64[mw];
                for (int m = 0; m < MEQN; m++) st.wave[mw][m] = (TW)w64[mw][m];
            }
            for (int m = 0; m < MEQN; m++) {
                st.am[m] = (TW)am64[m]; st.ap[m] = (TW)ap64[m];
                st.g64[m] = am64[m]; st.g64[MEQN + m] = ap64[m];
            }
            for (int e = 0; e < NEXTRA; e++) st.ex[e] = (TW)ex64[e];
        } else {
            TW qL[MEQN], qR[MEQN], aL[MA], aR[MA];
            for (int m = 0; m < MEQN; m++) { qL[m] = qload(m, cL); qR[m] = qload(m, cR); }
            for (int a = 0; a < MAUX; a++) { aL[a] = (TW)As[a * NXY + cL]; aR[a] = (TW)As[a * NXY + cR]; }
            RP::template rpn2<TW>(ixy, qL, qR, aL, aR, st.wave, st.s, st.am, st.ap, st.ex, gravw);
        }
        for (int mw = 0; mw < MWAVES; mw++)
            for (int m = 0; m < MEQN; m++) W[(G::W_WAVE + mw * MEQN + m) * NI + k] = st.wave[mw][m];
        if (!REG) {
            for (int mw = 0; mw < MWAVES; mw++) W[(G::W_S + mw) * NI + k] = st.s[mw];
            for (int m = 0; m < MEQN; m++) { W[(G::W_AM + m) * NI + k] = st.am[m]; W[(G::W_AP + m) * NI + k] = st.ap[m]; }
            for (int e = 0; e < NEXTRA; e++) W[(G::W_EX + e) * NI + k] = st.ex[e];
        }
        if (cfl_range) {
            if (F32) {
                for (int mw = 0; mw < MWAVES; mw++) cflw = dmax1(dmax1(cflw, d1 * st.s[mw]), -(d0 * st.s[mw]));
            } else {
                for (int mw = 0; mw < MWAVES; mw++)
                    cflmax = dmax1(dmax1(cflmax, (double)(d1 * st.s[mw])), (double)(-(d0 * st.s[mw])));
            }
        }
    };
    auto restore = [&](int k, State& st) {
        if (REG) return;
        for (int mw = 0; mw < MWAVES; mw++) {
            for (int m = 0; m < MEQN; m++) st.wave[mw][m] = W[(G::W_WAVE + mw * MEQN + m) * NI + k];
            st.s[mw] = W[(G::W_S + mw) * NI + k];
        }
        for (int m = 0; m < MEQN; m++) { st.am[m] = W[(G::W_AM + m) * NI + k]; st.ap[m] = W[(G::W_AP + m) * NI + k]; }
        for (int e = 0; e < NEXTRA; e++) st.ex[e] = W[(G::W_EX + e) * NI + k];
    };

    // Limiter, second-order correction, fadd and transverse split of one interface.
    // Returns faddm/faddp (FP64) and writes the transverse terms into Tt.
    auto interface_update = [&](int ixy, int k, int cL, int cR, int pos, int lim_lo, int lim_hi,
                                bool god, bool cqr, bool acr, bool trr, TW dlo, TW dhi, TW dave,
                                const int* a1c, const int* a2c, const int* a3c, State& st,
                                double* faddm, double* faddp) {
        TW cq[MEQN];
        for (int m = 0; m < MEQN; m++) { cq[m] = TW(0); faddm[m] = 0.0; faddp[m] = 0.0; }
        // wall_lo: ghost on the left (low face), wall_hi: ghost on the right (high face)
        const bool wall_lo = wallf && pos == lim_lo && (wallf & (ixy == 1 ? 1 : 4));
        const bool wall_hi = wallf && pos == lim_hi && (wallf & (ixy == 1 ? 2 : 8));
        if (god) {
            if constexpr (RP::EXACT64) {
                for (int m = 0; m < MEQN; m++) { faddp[m] = faddp[m] - st.g64[MEQN + m]; faddm[m] = faddm[m] + st.g64[m]; }
            } else if constexpr (F32) {
                double am64[MEQN], ap64[MEQN];
                double qL[MEQN], qR[MEQN], aL[MA], aR[MA], fL[MEQN], fR[MEQN];
                for (int m = 0; m < MEQN; m++) {
                    qL[m] = Qs[m * NXY + cL]; qR[m] = Qs[m * NXY + cR];
                    if (G::USE_FLX) { fL[m] = FLX[m * NXY + cL]; fR[m] = FLX[m * NXY + cR]; }
                    else { fL[m] = 0.0; fR[m] = 0.0; }
                }
                for (int a = 0; a < MAUX; a++) { aL[a] = As[a * NXY + cL]; aR[a] = As[a * NXY + cR]; }
                RP::godunov64(ixy, qL, qR, aL, aR, fL, fR, st.ap, am64, ap64, sp.grav);
                // zero mass flux through a wall: the interior cell's fluctuation cancels its own flux
                if (wall_lo) { ap64[0] = fR[0]; am64[0] = (fR[0] - fL[0]) - fR[0]; }
                if (wall_hi) { am64[0] = 0.0 - fL[0]; ap64[0] = (fR[0] - fL[0]) + fL[0]; }
                for (int m = 0; m < MEQN; m++) { faddp[m] = faddp[m] - ap64[m]; faddm[m] = faddm[m] + am64[m]; }
            } else {
                for (int m = 0; m < MEQN; m++) { faddp[m] = faddp[m] - (double)st.ap[m]; faddm[m] = faddm[m] + (double)st.am[m]; }
            }
        }
        const bool second = FWAVE ? (sp.order1 != 1) : (sp.order1 == 2);
        if (second) {
            if (pos >= lim_lo && pos <= lim_hi) {
                // inline limiter (clawpack46_inlinelimiter.f:267-343) with unlimited neighbours;
                // the neighbours along the sweep are k -+ 1 (x) or k -+ (NX-2) (y)
                const int kstep = (ixy == 1) ? 1 : NX - 2;
                for (int mw = 0; mw < MWAVES; mw++) {
                    const int ml = sp.mthlim[mw];
                    if (ml == 0) continue;
                    TW wnorm2 = TW(0), dotl = TW(0), dotr = TW(0);
                    for (int m = 0; m < MEQN; m++) {
                        const TW w = st.wave[mw][m];
                        const TW wl = W[(G::W_WAVE + mw * MEQN + m) * NI + k - kstep];
                        const TW wr = W[(G::W_WAVE + mw * MEQN + m) * NI + k + kstep];
                        wnorm2 = wnorm2 + w * w;
                        dotl = dotl + wl * w;
                        dotr = dotr + w * wr;
                    }
                    if (wnorm2 == TW(0)) continue;
                    const TW r = (st.s[mw] > TW(0)) ? dotl / wnorm2 : dotr / wnorm2;
                    const TW wlim = limiter_phi<TW>(ml, r);
                    for (int m = 0; m < MEQN; m++) st.wave[mw][m] = wlim * st.wave[mw][m];
                }
            }
            if (cqr) {
                for (int m = 0; m < MEQN; m++) {
                    TW c = TW(0);
                    for (int mw = 0; mw < MWAVES; mw++) {
                        if (FWAVE)
                            c = add_rn(c, mul_rn(mul_rn(sgn1(st.s[mw]), sub_rn(TW(1), mul_rn(fabs(st.s[mw]), dave))),
                                                 st.wave[mw][m]));
                        else {
                            const TW sa = fabs(st.s[mw]);
                            c = add_rn(c, mul_rn(mul_rn(sa, sub_rn(TW(1), mul_rn(sa, dave))), st.wave[mw][m]));
                        }
                    }
                    if (m == 0 && (wall_lo || wall_hi)) c = TW(0);
                    cq[m] = c;
                    if (F32) {
                        const double h = 0.5 * (double)c;
                        faddm[m] = faddm[m] + h;
                        faddp[m] = faddp[m] + h;
                    } else {
                        faddm[m] = faddm[m] + (double)(TW(0.5) * c);
                        faddp[m] = faddp[m] + (double)(TW(0.5) * c);
                    }
                }
            }
        }
        unsigned char fl = 0;
        if (sp.order2 > 0 && trr) {
            TW am[MEQN], ap[MEQN];
            for (int m = 0; m < MEQN; m++) { am[m] = st.am[m]; ap[m] = st.ap[m]; }
            if (sp.order1 > 1 && sp.order2 == 2 && acr)
                for (int m = 0; m < MEQN; m++) { am[m] = am[m] + cq[m]; ap[m] = ap[m] - cq[m]; }
            TW qL[MEQN], qR[MEQN];
            for (int m = 0; m < MEQN; m++) { qL[m] = qload(m, cL); qR[m] = qload(m, cR); }
            constexpr bool BOTH = RPHooks<RP>::AUX_BOTH;
            TW a1[BOTH ? 2 * MA : MA], a2[BOTH ? 2 * MA : MA], a3[BOTH ? 2 * MA : MA], bm[MEQN], bp[MEQN];
            if constexpr (BOTH) {
                for (int h = 0; h < 2; h++)
                    for (int a = 0; a < MAUX; a++) {
                        a1[h * MA + a] = (TW)As[a * NXY + a1c[h]];
                        a2[h * MA + a] = (TW)As[a * NXY + a2c[h]];
                        a3[h * MA + a] = (TW)As[a * NXY + a3c[h]];
                    }
            } else {
                for (int a = 0; a < MAUX; a++) { a1[a] = (TW)As[a * NXY + a1c[0]]; a2[a] = (TW)As[a * NXY + a2c[0]]; a3[a] = (TW)As[a * NXY + a3c[0]]; }
            }
            RP::template rpt2<TW>(ixy, 1, qL, qR, a1, a2, a3, st.ex, am, bm, bp, gravw, drytolw);
            for (int m = 0; m < MEQN; m++) {
                Tt[(0 * MEQN + m) * NI + k] = TW(0.5) * dlo * bm[m];
                Tt[(1 * MEQN + m) * NI + k] = TW(0.5) * dlo * bp[m];
            }
            // (every if-constexpr body here is braced: inside a lambda of a template, nvcc
            // 12.9 also discards the statement that follows an unbraced discarded `for`)
            if constexpr (!BOTH) {
                for (int a = 0; a < MAUX; a++) { a1[a] = (TW)As[a * NXY + a1c[1]]; a2[a] = (TW)As[a * NXY + a2c[1]]; a3[a] = (TW)As[a * NXY + a3c[1]]; }
            }
            RP::template rpt2<TW>(ixy, 2, qL, qR, a1, a2, a3, st.ex, ap, bm, bp, gravw, drytolw);
            for (int m = 0; m < MEQN; m++) {
                Tt[(2 * MEQN + m) * NI + k] = TW(0.5) * dhi * bm[m];
                Tt[(3 * MEQN + m) * NI + k] = TW(0.5) * dhi * bp[m];
            }
            fl = 1;
        }
        tflag[k] = fl;
    };

    // clawpack46_fix_corners (clawpack46_step2.f:242-310): at a corner of the
    // cubed sphere (three blocks meet, no corner neighbour) the mbc x mbc corner
    // ghost cells take rotated copies of face ghost cells before each sweep
    // (sweep 0: x, 1: y).  Sources are face ghost cells, never corner cells, so
    // the copies are independent.
    const int bcc = (pd.flags / PATCH_BCC3) & 15;
    auto fix_corners = [&](int sweep) {
        for (int t = tid; t < 4 * MBC * MBC * MEQN; t += NT) {
            const int m = t / (4 * MBC * MBC), r = t % (4 * MBC * MBC);
            const int k = r / (MBC * MBC), ibc = 1 + (r % (MBC * MBC)) / MBC, jbc = 1 + r % MBC;
            if (!((bcc >> k) & 1)) continue;
            const int i1 = (k & 1) ? MX + ibc : 1 - ibc, j1 = (k & 2) ? MY + jbc : 1 - jbc;
            // int(ihat - jhat), int(ihat + jhat) with ihat = 0.5 or mx + 0.5, jhat = 0.5 or my + 0.5
            const int ih = (k & 1) ? MX : 0, jh = (k & 2) ? MY : 0;
            const int dmi = ih - jh, dpl = ih + jh + 1;
            const bool use_b = (sweep == 0 && (k == 0 || k == 3)) || (sweep == 1 && (k == 1 || k == 2));
            const int id = use_b ? j1 + dmi : -j1 + dpl, jd = use_b ? -i1 + dpl : i1 - dmi;
            const int dst = m * NXY + (j1 + MBC - 1) * NX + (i1 + MBC - 1);
            const int src = m * NXY + (jd + MBC - 1) * NX + (id + MBC - 1);
            Qs[dst] = Qs[src];
            if (F32) Qf[dst] = Qf[src];
        }
    };

    // cell fluxes for the FP64 remainder of the Godunov split
    auto cell_fluxes = [&](int ixy) {
        if constexpr (G::USE_FLX) {
            for (int c = tid; c < NXY; c += NT) {
                double qv[MEQN], fv[MEQN];
                for (int m = 0; m < MEQN; m++) qv[m] = Qs[m * NXY + c];
                RP::flux64(ixy, qv, RP::EXACT64 ? sp.gamma : sp.grav, fv);
                for (int m = 0; m < MEQN; m++) FLX[m * NXY + c] = fv[m];
            }
        }
    };

    // p*-seed of the exact solver for interface k of sweep ixy (all lanes of the
    // warp take part; k < 0 marks a lane without an interface)
    auto mlp_seed = [&](int ixy, int k) -> double {
        if constexpr (RP::EXACT64) {
            int cL = 0, cR = 1;
            if (k >= 0) {
                if (ixy == 1) { const int jc = 1 + k / (NX - 1), ic = 1 + k % (NX - 1); cL = jc * NX + ic - 1; cR = cL + 1; }
                else { const int jc = 1 + k / (NX - 2), ic = 1 + k % (NX - 2); cL = (jc - 1) * NX + ic; cR = cL + NX; }
            }
            double qL[MEQN], qR[MEQN];
            for (int m = 0; m < MEQN; m++) { qL[m] = Qs[m * NXY + cL]; qR[m] = Qs[m * NXY + cR]; }
            const typename RP::Prim P = RP::prim(ixy, qL, qR, sp.gamma);
            float x[MLP_IN];
            double pbase;
            mlp_features(P.rl, P.ul, P.pl, P.rr, P.ur, P.pr, sp.gamma, x, pbase);
            if (k < 0 || !(x[0] == x[0] && x[1] == x[1] && x[2] == x[2] && x[3] == x[3] && x[4] == x[4] && x[5] == x[5])) {
                x[0] = 1.0f; x[1] = 0.0f; x[2] = 1.0f; x[3] = 1.0f; x[4] = 0.0f; x[5] = 1.0f;
                k = -1;
            }
            const bool use = k >= 0 && mlp_gate(x);
            // the network runs per warp (mma.sync over its 32 interfaces): skip warps
            // without an interface past the gate (smooth flow, weak waves)
            if (!__any_sync(0xffffffffu, use)) return 0.0;
            const MlpView W(sp.mlp);
            MlpFrag h1, h2;
            mlp_warp_hidden<true>(W, x, h1, h2);
            const float y = mlp_warp_output(W, h2);
            if constexpr (F32) { return use ? pbase * (double)__expf(y) : 0.0; }
            else { return use ? pbase * fcb_exp((double)y) : 0.0; }
        } else {
            (void)ixy; (void)k;
            return 0.0;
        }
    };

    // x-sweep interface k -> row jc = 1 + k / (NX-1), interface ic = 1 + k % (NX-1)
    auto x1 = [&](int k, State& st, double seed) {
        const int jc = 1 + k / (NX - 1), ic = 1 + k % (NX - 1);
        const bool cr = (ic >= MBC && ic <= MX + MBC);
        normal_solve(1, jc * NX + ic - 1, jc * NX + ic, k, cr, cr ? dtdx1d_x(ic, jc) : TW(0),
                     cr ? dtdx1d_x(ic - 1, jc) : TW(0), st, seed);
    };
    auto x2 = [&](int k, State& st) {
        const int jc = 1 + k / (NX - 1), ic = 1 + k % (NX - 1);
        const TW dlo = dtdx1d_x(ic - 1, jc);
        const TW dhi = FWAVE ? dlo : dtdx1d_x(ic, jc);
        const TW dave = TW(0.5) * (dtdx1d_x(ic - 1, jc) + dtdx1d_x(ic, jc));
        // aux of cell i1 = ic-1 (amdq) / ic (apdq) on rows jc-1, jc, jc+1
        const int a1c[2] = {(jc - 1) * NX + ic - 1, (jc - 1) * NX + ic};
        const int a2c[2] = {jc * NX + ic - 1, jc * NX + ic};
        const int a3c[2] = {(jc + 1) * NX + ic - 1, (jc + 1) * NX + ic};
        double faddm[MEQN], faddp[MEQN];
        interface_update(1, k, jc * NX + ic - 1, jc * NX + ic, ic, MBC, MX + MBC,
                         ic >= GOD_LO && ic <= GOD_HI, ic >= CQ_LO && ic <= CQ_HI, ic >= AC_LO && ic <= AC_HI,
                         ic >= TR_LO && ic <= TR_HI, dlo, dhi, dave, a1c, a2c, a3c, st, faddm, faddp);
        for (int m = 0; m < MEQN; m++) {
            FMs[m * NXY + jc * NX + ic] = 0.0 + faddm[m];
            FPs[m * NXY + jc * NX + ic] = 0.0 + faddp[m];
        }
    };
    // y-sweep interface k -> row interface jc = 1 + k / (NX-2), column ic = 1 + k % (NX-2)
    auto y1 = [&](int k, State& st, double seed) {
        const int jc = 1 + k / (NX - 2), ic = 1 + k % (NX - 2);
        const bool cr = (jc >= MBC && jc <= MY + MBC);
        normal_solve(2, (jc - 1) * NX + ic, jc * NX + ic, k, cr, cr ? dtdy1d_y(ic, jc) : TW(0),
                     cr ? dtdy1d_y(ic, jc - 1) : TW(0), st, seed);
    };
    auto y2 = [&](int k, State& st) {
        const int jc = 1 + k / (NX - 2), ic = 1 + k % (NX - 2);
        const TW dlo = dtdy1d_y(ic, jc - 1);
        const TW dhi = FWAVE ? dlo : dtdy1d_y(ic, jc);
        const TW dave = TW(0.5) * (dtdy1d_y(ic, jc - 1) + dtdy1d_y(ic, jc));
        // aux of sweep cell i1 = jc-1 (amdq) / jc (apdq) on columns ic-1, ic, ic+1
        const int a1c[2] = {(jc - 1) * NX + ic - 1, jc * NX + ic - 1};
        const int a2c[2] = {(jc - 1) * NX + ic, jc * NX + ic};
        const int a3c[2] = {(jc - 1) * NX + ic + 1, jc * NX + ic + 1};
        double faddm[MEQN], faddp[MEQN];
        interface_update(2, k, (jc - 1) * NX + ic, jc * NX + ic, jc, MBC, MY + MBC,
                         jc >= GOD_LOY && jc <= GOD_HIY, jc >= CQ_LOY && jc <= CQ_HIY,
                         jc >= AC_LOY && jc <= AC_HIY, jc >= TR_LOY && jc <= TR_HIY, dlo, dhi, dave,
                         a1c, a2c, a3c, st, faddm, faddp);
        for (int m = 0; m < MEQN; m++) {
            GMs[m * NXY + jc * NX + ic] = GMs[m * NXY + jc * NX + ic] + faddm[m];
            GPs[m * NXY + jc * NX + ic] = GPs[m * NXY + jc * NX + ic] + faddp[m];
        }
    };
    // X3: gadd -> gm/gp.  gm(ic,jc) = ((0 + G2(row jc-1)) + G1(row jc)), gp identical.
    auto x3 = [&](int c) {
        const int jc = c / NX, ic = c % NX;
        if (ic < 1 || jc < 1) return;                    // accumulation range ic >= 1, rows >= 1
        for (int m = 0; m < MEQN; m++) {
            double g = 0.0;
            if (jc - 1 >= 1 && jc - 1 <= NY - 2) {       // row jc-1, its gadd(:,2)
                const int r = jc - 1;
                double v = 0.0;
                if (ic + 1 <= NX - 1) { const int kk = (r - 1) * (NX - 1) + ic; if (tflag[kk]) v = v - (double)Tt[(1 * MEQN + m) * NI + kk]; }
                { const int kk = (r - 1) * (NX - 1) + ic - 1; if (tflag[kk]) v = v - (double)Tt[(3 * MEQN + m) * NI + kk]; }
                g = g + v;
            }
            if (jc <= NY - 2) {                          // row jc, its gadd(:,1)
                const int r = jc;
                double v = 0.0;
                if (ic + 1 <= NX - 1) { const int kk = (r - 1) * (NX - 1) + ic; if (tflag[kk]) v = v - (double)Tt[(0 * MEQN + m) * NI + kk]; }
                { const int kk = (r - 1) * (NX - 1) + ic - 1; if (tflag[kk]) v = v - (double)Tt[(2 * MEQN + m) * NI + kk]; }
                g = g + v;
            }
            if (m == 0 && ((jc == MBC && (wallf & 4)) || (jc == MY + MBC && (wallf & 8)))) g = 0.0;
            GMs[m * NXY + c] = g;
            GPs[m * NXY + c] = g;
        }
    };
    // Y3: gadd -> fm/fp.  fm(ic,jc) = (fm + G2(col ic-1)) + G1(col ic)
    auto y3 = [&](int c) {
        const int jc = c / NX, ic = c % NX;
        if (jc < 1) return;
        const bool wall_edge = (ic == MBC && (wallf & 1)) || (ic == MX + MBC && (wallf & 2));
        for (int m = 0; m < MEQN; m++) {
            if (m == 0 && wall_edge) continue;
            double fm = FMs[m * NXY + c], fp = FPs[m * NXY + c];
            if (ic - 1 >= 1 && ic - 1 <= NX - 2) {
                const int col = ic - 1;
                double v = 0.0;
                if (jc + 1 <= NY - 1) { const int kk = jc * (NX - 2) + col - 1; if (tflag[kk]) v = v - (double)Tt[(1 * MEQN + m) * NI + kk]; }
                { const int kk = (jc - 1) * (NX - 2) + col - 1; if (tflag[kk]) v = v - (double)Tt[(3 * MEQN + m) * NI + kk]; }
                fm = fm + v; fp = fp + v;
            }
            if (ic >= 1 && ic <= NX - 2) {
                const int col = ic;
                double v = 0.0;
                if (jc + 1 <= NY - 1) { const int kk = jc * (NX - 2) + col - 1; if (tflag[kk]) v = v - (double)Tt[(0 * MEQN + m) * NI + kk]; }
                { const int kk = (jc - 1) * (NX - 2) + col - 1; if (tflag[kk]) v = v - (double)Tt[(2 * MEQN + m) * NI + kk]; }
                fm = fm + v; fp = fp + v;
            }
            FMs[m * NXY + c] = fm;
            FPs[m * NXY + c] = fp;
        }
    };

    // =================== x-sweeps (clawpack46_step2.f:113-167) ===================
    State st;
    if (bcc) { fix_corners(0); __syncthreads(); }
    cell_fluxes(1);
    if constexpr (RP::EXACT64 && F32) { __syncthreads(); }   // the exact solver reads the cell fluxes
    {
        const double seed = (RP::EXACT64 && sp.mlp) ? mlp_seed(1, tid < G::NIX ? tid : -1) : 0.0;
        if (REG) { if (tid < G::NIX) x1(tid, st, seed); }
        else for (int k = tid; k < G::NIX; k += NT) x1(k, st, 0.0);
    }
    __syncthreads();
    if (REG) { if (tid < G::NIX) x2(tid, st); }
    else for (int k = tid; k < G::NIX; k += NT) { restore(k, st); x2(k, st); }
    __syncthreads();
    if (bcc) { fix_corners(1); __syncthreads(); }
    // X3 and the y-sweep normal solves touch disjoint data: one phase
    for (int c = tid; c < NXY; c += NT) x3(c);
    cell_fluxes(2);
    if constexpr (RP::EXACT64 && F32) { __syncthreads(); }
    // =================== y-sweeps (clawpack46_step2.f:182-236) ===================
    {
        const double seed = (RP::EXACT64 && sp.mlp) ? mlp_seed(2, tid < G::NIY ? tid : -1) : 0.0;
        if (REG) { if (tid < G::NIY) y1(tid, st, seed); }
        else for (int k = tid; k < G::NIY; k += NT) y1(k, st, 0.0);
    }
    __syncthreads();
    if (REG) { if (tid < G::NIY) y2(tid, st); }
    else for (int k = tid; k < G::NIY; k += NT) { restore(k, st); y2(k, st); }
    __syncthreads();
    for (int c = tid; c < NXY; c += NT) y3(c);
    __syncthreads();

    // ---- time-sync wave accumulation (clawpack46_time_sync.f:163-226), FP64 ----
    if (sp.accumulate_waves) {
        const double dtdyv = dt * dy, dtdxv = dt * dx;
        // registers of a face reset since the last update start from zero
        auto z = [&](int face) { return ((sp.reg_reset >> ((pd.face_type >> (2 * face)) & 3)) & 1) != 0; };
        const bool z0 = z(0), z1 = z(1), z2 = z(2), z3 = z(3);
        for (int it = tid; it < (MY + MX) * MEQN; it += NT) {
            if (it < MY * MEQN) {
                const int j = it % MY, m = it / MY;
                const int jc = MBC + j;
                const int cl = m * NXY + jc * NX + MBC, cr = m * NXY + jc * NX + MX + MBC;
                double* r;
                r = &rg[G::R_FP0 + j + m * MY]; *r = (z0 ? 0.0 : *r) - dtdyv * FPs[cl];
                r = &rg[G::R_FM0 + j + m * MY]; *r = (z0 ? 0.0 : *r) + dtdyv * FMs[cl];
                r = &rg[G::R_FP1 + j + m * MY]; *r = (z1 ? 0.0 : *r) - dtdyv * FPs[cr];
                r = &rg[G::R_FM1 + j + m * MY]; *r = (z1 ? 0.0 : *r) + dtdyv * FMs[cr];
            } else {
                const int i2 = it - MY * MEQN;
                const int i = i2 % MX, m = i2 / MX;
                const int ic = MBC + i;
                const int cb = m * NXY + MBC * NX + ic, ct = m * NXY + (MY + MBC) * NX + ic;
                double* r;
                r = &rg[G::R_GP0 + i + m * MX]; *r = (z2 ? 0.0 : *r) - dtdxv * GPs[cb];
                r = &rg[G::R_GM0 + i + m * MX]; *r = (z2 ? 0.0 : *r) + dtdxv * GMs[cb];
                r = &rg[G::R_GP1 + i + m * MX]; *r = (z3 ? 0.0 : *r) - dtdxv * GPs[ct];
                r = &rg[G::R_GM1 + i + m * MX]; *r = (z3 ? 0.0 : *r) + dtdxv * GMs[ct];
            }
        }
    }

    // ---- q update over i,j = 1-mbc..mx+mbc-1 (clawpack46_step2_wrap.f:107-125) ----
    if constexpr (RPHooks<RP>::SRC) {
        // with a user src2 (clawpack46_update, fc2d_clawpack46.cpp:436-441: src2 after
        // step2), every padded cell gets its updated q (cells the update skips keep
        // theirs) passed through the cell-wise source term before it is stored
        for (int c = tid; c < NXY; c += NT) {
            const int jc = c / NX, ic = c % NX;
            double qc[MEQN], ac[G::AUXS > 0 ? G::AUXS : 1];
            for (int m = 0; m < MEQN; m++) {
                const int b = m * NXY;
                double v = Qs[b + c];
                if (ic <= NX - 2 && jc <= NY - 2) {
                    if (mcapa == 0)
                        v = v - dtdx * (FMs[b + c + 1] - FPs[b + c]) - dtdy * (GMs[b + c + NX] - GPs[b + c]);
                    else
                        v = v - (dtdx * (FMs[b + c + 1] - FPs[b + c]) + dtdy * (GMs[b + c + NX] - GPs[b + c])) /
                                    As[(mcapa - 1) * NXY + c];
                }
                qc[m] = v;
            }
            for (int a = 0; a < G::AUXS; a++) ac[a] = As[a * NXY + c];
            RP::src2(MBC, MX, MY, MEQN, qc, pd.xlower, pd.ylower, dx, dy, sp.t, dt, G::AUXS, ac, ic - MBC + 1,
                     jc - MBC + 1);
            for (int m = 0; m < MEQN; m++) qg[m * NXY + c] = qc[m];
        }
    } else
    for (int k = tid; k < MEQN * NXY; k += NT) {
        const int m = k / NXY, c = k % NXY;
        const int jc = c / NX, ic = c % NX;
        if (ic <= NX - 2 && jc <= NY - 2) {
            const int b = m * NXY;
            double v = Qs[k];
            if (mcapa == 0)
                v = v - dtdx * (FMs[b + c + 1] - FPs[b + c]) - dtdy * (GMs[b + c + NX] - GPs[b + c]);
            else
                v = v - (dtdx * (FMs[b + c + 1] - FPs[b + c]) + dtdy * (GMs[b + c + NX] - GPs[b + c])) /
                            As[(mcapa - 1) * NXY + c];
            qg[k] = v;
        } else if (bcc) {
            // cells the update skips keep the step's (corner-fixed) values, as the
            // reference fixes the corners of q in place
            const int kx = ic >= MX + MBC ? 1 : (ic < MBC ? 0 : -1);
            const int ky = jc >= MY + MBC ? 1 : (jc < MBC ? 0 : -1);
            if (kx >= 0 && ky >= 0 && ((bcc >> (kx + 2 * ky)) & 1)) qg[k] = Qs[k];
        }
    }

    // ---- CFL maximum: warp shuffles, then one atomic per CTA -----------------
    if (F32) cflmax = (double)cflw;
    for (int off = 16; off > 0; off >>= 1) cflmax = dmax1(cflmax, __shfl_xor_sync(0xffffffffu, cflmax, off));
    if ((tid & 31) == 0) red[tid >> 5] = cflmax;
    __syncthreads();
    if (tid < 32) {
        double v = (tid < NT / 32) ? red[tid] : 0.0;
        for (int off = 16; off > 0; off >>= 1) v = dmax1(v, __shfl_xor_sync(0xffffffffu, v, off));
        if (tid == 0) {
            unsigned long long bits = (unsigned long long)__double_as_longlong(v);
            if (v != v) bits = 0x7ff8000000000000ull;   // NaN (e.g. negative depth) wins the max
            atomicMax(cfl_bits + pd.inst, bits);
        }
    }
    if constexpr (RP::EXACT64) {
        if (tid < 32 && sp.newton_hist && nhist[tid]) atomicAdd(&sp.newton_hist[tid], (unsigned long long)nhist[tid]);
    }
}

// The fused update of npatch patches starting at slot p0.  One CTA per patch, or
// (PERSIST) a grid of a few CTAs per SM, each taking patches p0 + blockIdx.x,
// + gridDim.x, ... in turn, its shared memory reused patch after patch.
// Parameter block of relative patch b of a launch over lg.nlev levels.
__device__ __forceinline__ int group_slot(const LevelGroup& lg, int b)
{
    int k = 0;
    for (int i = 1; i < lg.nlev; i++) k += (b >= lg.start[i]) ? 1 : 0;
    return lg.nlev - 1 - k;
}

template <class RP, int MX, int MY, int MBC, bool FWAVE, int NT, typename TW, int MINB = 2, bool PERSIST = false>
__global__ void __launch_bounds__(NT, MINB)
step2_kernel(double* __restrict__ q, double* __restrict__ qlast, const double* __restrict__ aux,
             double* __restrict__ regs, const PatchDesc* __restrict__ desc, int p0, int npatch,
             const StepParams* __restrict__ spp, const LevelGroup lg, unsigned long long* __restrict__ cfl_bits)
{
    grid_dependency_wait();         // programmatic launch: the previous grid's writes are visible
    grid_launch_dependents();
    // per-launch parameters live in device memory (graph replay); a launch over
    // several levels holds one block per level, highest level first
    __shared__ unsigned int nhist[RP::EXACT64 ? 32 : 1];
    if constexpr (!PERSIST) {
        (void)npatch;
        const int p = p0 + (int)blockIdx.x;
        const StepParams sp = spp[group_slot(lg, (int)blockIdx.x)];
        step2_patch<RP, MX, MY, MBC, FWAVE, NT, TW>(q, qlast, aux, regs, desc, p, sp, cfl_bits, nhist);
    } else {
        for (int b = blockIdx.x; b < npatch; b += gridDim.x) {
            const int p = p0 + b;
            const StepParams sp = spp[group_slot(lg, b)];
            step2_patch<RP, MX, MY, MBC, FWAVE, NT, TW>(q, qlast, aux, regs, desc, p, sp, cfl_bits, nhist);
            __syncthreads();   // the next patch restages the shared memory
        }
    }
}

}  // namespace fcb
