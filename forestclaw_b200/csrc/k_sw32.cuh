// k_sw32.cuh -- the FP32-wave shallow-water update (Roe solver with the Harten-Hyman
// entropy fix) specialised for the configuration of the radial-dam runs: second-order
// corrections with one limiter for every wave (method(2) = 2), transverse corrections
// of second order (method(3) = 2), no capacity and no aux.  The host installs it only
// for such a solver (Step2Variant::spec); every other configuration runs step2_kernel.
//
// The arithmetic of the waves is the generic FP32-wave kernel's (the same rpn2 / rpt2
// / limiter / correction code on the same FP32 states); what changes is the layout:
//
//   * q arrives by one bulk asynchronous copy (cp.async.bulk, completion on an
//     mbarrier) instead of per-thread loads; the persistent form requests the next
//     patch of its CTA while the current one computes (two q buffers);
//   * the FP64 cell fluxes of both directions are computed once per cell
//     (f_x = (hu, hu^2/h + g h^2/2, hu hv/h), f_y = (hv, hu hv/h, hv^2/h + g h^2/2),
//     three planes);
//   * the flux arrays fm/fp (gm/gp) of clawpack46_step2.f are held as one FP64 plane
//     per direction, GX = fp and GY = gp: inside the Godunov range of a sweep
//     fm = (f(cell right) - f(cell left)) + fp, since the FP32-wave split takes
//     amdq as the FP64 remainder f(qR) - f(qL) - apdq; elsewhere fm = fp.  The update
//     q -= dt/dx (fm(i+1) - fp(i)) + dt/dy (gm(j+1) - gp(j)) then telescopes over the
//     cells exactly as before, so mass is conserved to FP64 round-off;
//   * the method flags and the limiter are compile-time constants, and every
//     interface carries transverse terms (the reference's transverse range covers
//     all interfaces of the padded sweep for method(3) = 2), so no per-interface
//     flags are stored.
//
// Walls (mthbc = 3): the mass component of the flux through a reflecting wall is
// exactly zero, as in the generic FP32-wave kernel (fm = -f(interior) at a high wall,
// fp = -f(interior) at a low wall).
#pragma once
#include <cuda_runtime.h>
#include "k_step2.cuh"

namespace fcb {

template <int MX, int NT_, bool PERSIST>
struct SW32Geom {
    static constexpr int MY = MX, MBC = 2, MEQN = 3, NX = MX + 2 * MBC, NY = MY + 2 * MBC, NXY = NX * NY;
    static constexpr int NIX = (NY - 2) * (NX - 1), NIY = (NX - 2) * (NY - 1);
    static constexpr int NI = NIX > NIY ? NIX : NIY;
    static constexpr int NT = NT_;
    static_assert(NT >= NI, "one thread per interface of a sweep");
    static constexpr int QB = MEQN * NXY;                       // doubles of one patch's q
    static constexpr int NBUF = PERSIST ? 2 : 1;
    static constexpr unsigned QBYTES = QB * 8u;                 // bulk copy size (a multiple of 16)
    static_assert(QBYTES % 16 == 0, "bulk copies move multiples of 16 bytes");
    // shared memory, bytes (every FP64 block a multiple of 16 bytes long)
    static constexpr size_t OFF_Q = 0;                          // [NBUF][MEQN][NXY] double
    static constexpr size_t OFF_FL = OFF_Q + (size_t)NBUF * QBYTES;   // FXX, FYY, FXY [NXY] double
    static constexpr size_t OFF_GX = OFF_FL + 3 * (size_t)NXY * 8;   // [MEQN][NXY] double
    static constexpr size_t OFF_GY = OFF_GX + (size_t)QB * 8;
    static constexpr size_t OFF_RED = OFF_GY + (size_t)QB * 8;       // 64 doubles
    static constexpr size_t OFF_BAR = OFF_RED + 64 * 8;              // 2 mbarriers + flag
    static constexpr size_t OFF_W = OFF_BAR + 32;                    // [7][NI] float
    static constexpr size_t OFF_T = OFF_W + 7 * (size_t)NI * 4;      // [12][NI] float
    static constexpr size_t BYTES = OFF_T + 12 * (size_t)NI * 4;
};

// ---- bulk copy global -> shared with an mbarrier (sm_90+ PTX) -------------------
__device__ __forceinline__ unsigned smem_u32(const void* p)
{
    return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
// Thread 0: expect `bytes` on the barrier and start the copy.  The fence orders the
// CTA's earlier generic-proxy accesses of the buffer before the async-proxy writes.
__device__ __forceinline__ void bulk_load(unsigned long long* bar, void* dst, const void* src, unsigned bytes)
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
// Wait for phase `parity` of the barrier to complete, at most `limit` polls.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, int limit)
{
    for (int i = 0; i < limit; i++) {
        unsigned done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Polls of a staging wait before the CTA gives up (each poll may suspend the thread
// for a while in hardware): far beyond any copy of a few KB, short of a hang.
constexpr int SW32_WAIT_LIMIT = 1 << 20;

// The update of patch p, q already in Qs (shared memory).
template <int MX, int NT, int LIM, bool PERSIST>
__device__ __forceinline__ void sw32_patch(unsigned char* sm, const double* __restrict__ Qs, double* __restrict__ q,
                                           double* __restrict__ qlast, double* __restrict__ regs,
                                           const PatchDesc& pd, const int p, const StepParams& sp,
                                           unsigned long long* __restrict__ cfl_bits)
{
    using G = SW32Geom<MX, NT, PERSIST>;
    using R = Step2Geom<RPShallowRoe, MX, MX, 2, float, NT>;    // register layout
    constexpr int MY = MX, MBC = 2, NX = G::NX, NY = G::NY, NXY = G::NXY, NI = G::NI;
    double* FXX = reinterpret_cast<double*>(sm + G::OFF_FL);
    double* FYY = FXX + NXY;
    double* FXY = FYY + NXY;
    double* GX = reinterpret_cast<double*>(sm + G::OFF_GX);
    double* GY = reinterpret_cast<double*>(sm + G::OFF_GY);
    double* red = reinterpret_cast<double*>(sm + G::OFF_RED);
    float* W = reinterpret_cast<float*>(sm + G::OFF_W);
    float* Tt = reinterpret_cast<float*>(sm + G::OFF_T);

    const int tid = threadIdx.x;
    const double dx = pd.dx, dy = pd.dy;
    const double dt = sp.inst_dt ? sp.dt * sp.inst_dt[pd.inst] : sp.dt;
    const double dtdx = dt / dx, dtdy = dt / dy;
    const double grav = sp.grav;
    double* qg = q + (size_t)p * G::QB;
    const bool save = sp.save_last && (pd.flags & PATCH_HAS_FINE_NBR);
    const int wallf = pd.phys_mask & sp.wall_faces;

    // normal fluxes of a cell: x (hu, FXX, FXY), y (hv, FXY, FYY)
    auto fx = [&](int m, int c) -> double { return m == 0 ? Qs[NXY + c] : (m == 1 ? FXX[c] : FXY[c]); };
    auto fy = [&](int m, int c) -> double { return m == 0 ? Qs[2 * NXY + c] : (m == 1 ? FXY[c] : FYY[c]); };

    // ---- cells: status, FP64 fluxes, faces no sweep writes ----------------------
    unsigned bad = 0;
    for (int c = tid; c < NXY; c += NT) {
        const double h = Qs[c], hu = Qs[NXY + c], hv = Qs[2 * NXY + c];
        if (!isfinite(h) || !isfinite(hu) || !isfinite(hv)) bad |= STATUS_NONFINITE;
        if (h < 0.0) bad |= STATUS_DEPTH;
        const double inv = 1.0 / h;
        FXX[c] = hu * hu * inv + 0.5 * grav * h * h;
        FYY[c] = hv * hv * inv + 0.5 * grav * h * h;
        FXY[c] = hu * hv * inv;
        const int ic = c % NX, jc = c / NX;
        if (ic == 0 || jc == 0)
            for (int m = 0; m < 3; m++) { GX[m * NXY + c] = 0.0; GY[m * NXY + c] = 0.0; }
    }
    if (save) {
        double* ql = qlast + (size_t)p * G::QB;
        for (int k = tid; k < G::QB; k += NT) ql[k] = Qs[k];
    }
    if (bad && sp.status) atomicOr(sp.status, bad);

    // ---- time-sync flux store (clawpack46_time_sync.f:37-90), FP64 ---------------
    double* rg = regs + (size_t)p * R::NREG;
    if (sp.store_flux) {
        for (int it = tid; it < 2 * 2 * MY + 2 * 2 * MX; it += NT) {
            int face, j, k;
            if (it < 4 * MY) { face = it / (2 * MY); int r = it % (2 * MY); j = r / 2; k = r % 2; }
            else { int r2 = it - 4 * MY; face = 2 + r2 / (2 * MX); int r = r2 % (2 * MX); j = r / 2; k = r % 2; }
            int ic, jc;
            if (face == 0) { ic = MBC - k; jc = MBC + j; }
            else if (face == 1) { ic = MX + MBC - 1 + k; jc = MBC + j; }
            else if (face == 2) { ic = MBC + j; jc = MBC - k; }
            else { ic = MBC + j; jc = MY + MBC - 1 + k; }
            double qv[3], fl[3];
            for (int m = 0; m < 3; m++) qv[m] = Qs[m * NXY + jc * NX + ic];
            rpn2_cons_sw<double>(face / 2, qv, grav, fl);
            const int n = (face < 2) ? MY : MX;
            const double el = (face < 2) ? dy : dx;
            const int base = (face == 0) ? R::R_EF0 : (face == 1) ? R::R_EF1 : (face == 2) ? R::R_EF2 : R::R_EF3;
            const bool zero = (sp.reg_reset >> ((pd.face_type >> (2 * face)) & 3)) & 1;
            for (int m = 0; m < 3; m++) {
                double* r = &rg[base + j + m * n + k * n * 3];
                *r = (zero ? 0.0 : *r) + dt * el * fl[m];
            }
        }
    }
    __syncthreads();

    const float gravw = (float)grav, drytolw = (float)sp.dry_tolerance;
    const float dtdxw = (float)dtdx, dtdyw = (float)dtdy;
    float cflw = 0.0f;
    float wave[3][3], s[3], am[3], ap[3], ex[3];

    // normal solve of interface k (cells cL, cR) of sweep ixy; waves to W
    auto normal = [&](int ixy, int k, int cL, int cR, bool cfl_range, float d) {
        float qL[3], qR[3];
        for (int m = 0; m < 3; m++) { qL[m] = (float)Qs[m * NXY + cL]; qR[m] = (float)Qs[m * NXY + cR]; }
        RPShallowRoe::rpn2<float>(ixy, qL, qR, nullptr, nullptr, wave, s, am, ap, ex, gravw);
        const int mv = ixy == 1 ? 2 : 1;
        W[0 * NI + k] = wave[0][0]; W[1 * NI + k] = wave[0][1]; W[2 * NI + k] = wave[0][2];
        W[3 * NI + k] = wave[1][mv];
        W[4 * NI + k] = wave[2][0]; W[5 * NI + k] = wave[2][1]; W[6 * NI + k] = wave[2][2];
        if (cfl_range)
            for (int mw = 0; mw < 3; mw++) cflw = dmax1(dmax1(cflw, d * s[mw]), -(d * s[mw]));
    };
    // wave mw, field m of interface kk from W (sweep ixy)
    auto wload = [&](int ixy, int mw, int m, int kk) -> float {
        if (mw == 1) return m == (ixy == 1 ? 2 : 1) ? W[3 * NI + kk] : 0.0f;
        return W[(mw == 0 ? 0 : 4) * NI + m * NI + kk];
    };

    // limiter, second-order correction, Godunov split, transverse split of interface k;
    // returns fp (FP64) and writes the transverse terms
    auto second = [&](int ixy, int k, int kstep, int cL, int cR, int pos, bool god, bool acr, float d, double* fpo) {
        const bool wall_lo = pos == MBC && (wallf & (ixy == 1 ? 1 : 4));
        const bool wall_hi = pos == MX + MBC && (wallf & (ixy == 1 ? 2 : 8));
        if (pos >= MBC && pos <= MX + MBC) {
            // inline limiter (clawpack46_inlinelimiter.f:267-343), neighbours k -+ kstep
            for (int mw = 0; mw < 3; mw++) {
                float wnorm2 = 0.0f, dotl = 0.0f, dotr = 0.0f;
                for (int m = 0; m < 3; m++) {
                    const float w = wave[mw][m];
                    const float wl = wload(ixy, mw, m, k - kstep), wr = wload(ixy, mw, m, k + kstep);
                    wnorm2 = wnorm2 + w * w;
                    dotl = dotl + wl * w;
                    dotr = dotr + w * wr;
                }
                if (wnorm2 == 0.0f) continue;
                const float r = (s[mw] > 0.0f) ? dotl / wnorm2 : dotr / wnorm2;
                const float wlim = limiter_phi<float>(LIM, r);
                for (int m = 0; m < 3; m++) wave[mw][m] = wlim * wave[mw][m];
            }
        }
        float cq[3];
        for (int m = 0; m < 3; m++) {
            float c = 0.0f;
            for (int mw = 0; mw < 3; mw++) {
                const float sa = fabsf(s[mw]);
                c = add_rn(c, mul_rn(mul_rn(sa, sub_rn(1.0f, mul_rn(sa, d))), wave[mw][m]));
            }
            if (m == 0 && (wall_lo || wall_hi)) c = 0.0f;
            cq[m] = c;
        }
        for (int m = 0; m < 3; m++) {
            double f = 0.0;
            if (god) {
                const double fL = ixy == 1 ? fx(m, cL) : fy(m, cL), fR = ixy == 1 ? fx(m, cR) : fy(m, cR);
                double ap64 = (double)ap[m];
                if (m == 0 && wall_lo) ap64 = fR;
                if (m == 0 && wall_hi) ap64 = (fR - fL) + fL;
                f = f - ap64;
            }
            fpo[m] = f + 0.5 * (double)cq[m];
        }
        if (acr)
            for (int m = 0; m < 3; m++) { am[m] = am[m] + cq[m]; ap[m] = ap[m] - cq[m]; }
        float bm[3], bp[3];
        RPShallowRoe::rpt2<float>(ixy, 1, nullptr, nullptr, nullptr, nullptr, nullptr, ex, am, bm, bp, gravw, drytolw);
        for (int m = 0; m < 3; m++) { Tt[(0 + m) * NI + k] = 0.5f * d * bm[m]; Tt[(3 + m) * NI + k] = 0.5f * d * bp[m]; }
        RPShallowRoe::rpt2<float>(ixy, 2, nullptr, nullptr, nullptr, nullptr, nullptr, ex, ap, bm, bp, gravw, drytolw);
        for (int m = 0; m < 3; m++) { Tt[(6 + m) * NI + k] = 0.5f * d * bm[m]; Tt[(9 + m) * NI + k] = 0.5f * d * bp[m]; }
    };

    // =================== x-sweeps (clawpack46_step2.f:113-167) ===================
    const int kx = tid, jx = 1 + kx / (NX - 1), ix = 1 + kx % (NX - 1);
    const int ky = tid, jy = 1 + ky / (NX - 2), iy = 1 + ky % (NX - 2);
    if (kx < G::NIX) normal(1, kx, jx * NX + ix - 1, jx * NX + ix, ix >= MBC && ix <= MX + MBC, dtdxw);
    __syncthreads();
    if (kx < G::NIX) {
        double fpv[3];
        second(1, kx, 1, jx * NX + ix - 1, jx * NX + ix, ix, ix <= NX - 2, ix <= NX - 2, dtdxw, fpv);
        for (int m = 0; m < 3; m++) GX[m * NXY + jx * NX + ix] = 0.0 + fpv[m];
    }
    __syncthreads();
    // transverse terms of the x-sweep into the y-faces: gp = gm = this (before the y-sweep).
    // The faces read later are those of the y-sweep's interfaces (columns 1..NX-2, rows
    // 1..NY-1), one per thread, numbered as the y-interfaces; faces in column 0 or row 0
    // stay zero.
    if (tid < G::NIY) {
        const int jc = jy, ic = iy, c = jc * NX + ic;
        for (int m = 0; m < 3; m++) {
            double g = 0.0;
            if (jc - 1 >= 1 && jc - 1 <= NY - 2) {       // row jc-1, its gadd(:,2)
                const int r = jc - 1;
                double v = 0.0;
                if (ic + 1 <= NX - 1) v = v - (double)Tt[(3 + m) * NI + (r - 1) * (NX - 1) + ic];
                v = v - (double)Tt[(9 + m) * NI + (r - 1) * (NX - 1) + ic - 1];
                g = g + v;
            }
            if (jc <= NY - 2) {                          // row jc, its gadd(:,1)
                const int r = jc;
                double v = 0.0;
                if (ic + 1 <= NX - 1) v = v - (double)Tt[(0 + m) * NI + (r - 1) * (NX - 1) + ic];
                v = v - (double)Tt[(6 + m) * NI + (r - 1) * (NX - 1) + ic - 1];
                g = g + v;
            }
            if (m == 0 && ((jc == MBC && (wallf & 4)) || (jc == MY + MBC && (wallf & 8)))) g = 0.0;
            GY[m * NXY + c] = g;
        }
    }
    // =================== y-sweeps (clawpack46_step2.f:182-236) ===================
    if (ky < G::NIY) normal(2, ky, (jy - 1) * NX + iy, jy * NX + iy, jy >= MBC && jy <= MY + MBC, dtdyw);
    __syncthreads();
    if (ky < G::NIY) {
        double fpv[3];
        second(2, ky, NX - 2, (jy - 1) * NX + iy, jy * NX + iy, jy, jy <= NY - 2, jy <= NY - 2, dtdyw, fpv);
        for (int m = 0; m < 3; m++) GY[m * NXY + jy * NX + iy] = GY[m * NXY + jy * NX + iy] + fpv[m];
    }
    __syncthreads();
    // transverse terms of the y-sweep into the x-faces: the faces of the x-sweep's interfaces
    // (columns 1..NX-1, rows 1..NY-2), one per thread; faces in column 0 get none
    if (tid < G::NIX) {
        const int jc = jx, ic = ix, c = jc * NX + ic;
        const bool wall_edge = (ic == MBC && (wallf & 1)) || (ic == MX + MBC && (wallf & 2));
        for (int m = 0; m < 3; m++) {
            if (m == 0 && wall_edge) continue;
            double g = GX[m * NXY + c];
            if (ic - 1 >= 1 && ic - 1 <= NX - 2) {
                const int col = ic - 1;
                double v = 0.0;
                if (jc + 1 <= NY - 1) v = v - (double)Tt[(3 + m) * NI + jc * (NX - 2) + col - 1];
                v = v - (double)Tt[(9 + m) * NI + (jc - 1) * (NX - 2) + col - 1];
                g = g + v;
            }
            if (ic >= 1 && ic <= NX - 2) {
                const int col = ic;
                double v = 0.0;
                if (jc + 1 <= NY - 1) v = v - (double)Tt[(0 + m) * NI + jc * (NX - 2) + col - 1];
                v = v - (double)Tt[(6 + m) * NI + (jc - 1) * (NX - 2) + col - 1];
                g = g + v;
            }
            GX[m * NXY + c] = g;
        }
    }
    __syncthreads();

    // flux arrays of face f (cell f is right of / above the face)
    auto fm_x = [&](int m, int f) -> double {
        const int jc = f / NX, ic = f % NX;
        if (jc < 1 || jc > NY - 2 || ic < 1 || ic > NX - 2) return GX[m * NXY + f];
        if (m == 0 && (wallf & 2) && ic == MX + MBC) return 0.0 - fx(0, f - 1);
        return (fx(m, f) - fx(m, f - 1)) + GX[m * NXY + f];
    };
    auto gm_y = [&](int m, int f) -> double {
        const int jc = f / NX, ic = f % NX;
        if (jc < 1 || jc > NY - 2 || ic < 1 || ic > NX - 2) return GY[m * NXY + f];
        if (m == 0 && (wallf & 8) && jc == MY + MBC) return 0.0 - fy(0, f - NX);
        return (fy(m, f) - fy(m, f - NX)) + GY[m * NXY + f];
    };

    // ---- time-sync wave accumulation (clawpack46_time_sync.f:163-226), FP64 ----
    if (sp.accumulate_waves) {
        const double dtdyv = dt * dy, dtdxv = dt * dx;
        // registers of a face reset since the last update start from zero
        auto z = [&](int face) { return ((sp.reg_reset >> ((pd.face_type >> (2 * face)) & 3)) & 1) != 0; };
        const bool z0 = z(0), z1 = z(1), z2 = z(2), z3 = z(3);
        for (int it = tid; it < (MY + MX) * 3; it += NT) {
            if (it < MY * 3) {
                const int j = it % MY, m = it / MY;
                const int jc = MBC + j;
                const int cl = jc * NX + MBC, cr = jc * NX + MX + MBC;
                double* r;
                r = &rg[R::R_FP0 + j + m * MY]; *r = (z0 ? 0.0 : *r) - dtdyv * GX[m * NXY + cl];
                r = &rg[R::R_FM0 + j + m * MY]; *r = (z0 ? 0.0 : *r) + dtdyv * fm_x(m, cl);
                r = &rg[R::R_FP1 + j + m * MY]; *r = (z1 ? 0.0 : *r) - dtdyv * GX[m * NXY + cr];
                r = &rg[R::R_FM1 + j + m * MY]; *r = (z1 ? 0.0 : *r) + dtdyv * fm_x(m, cr);
            } else {
                const int i2 = it - MY * 3;
                const int i = i2 % MX, m = i2 / MX;
                const int ic = MBC + i;
                const int cb = MBC * NX + ic, ct = (MY + MBC) * NX + ic;
                double* r;
                r = &rg[R::R_GP0 + i + m * MX]; *r = (z2 ? 0.0 : *r) - dtdxv * GY[m * NXY + cb];
                r = &rg[R::R_GM0 + i + m * MX]; *r = (z2 ? 0.0 : *r) + dtdxv * gm_y(m, cb);
                r = &rg[R::R_GP1 + i + m * MX]; *r = (z3 ? 0.0 : *r) - dtdxv * GY[m * NXY + ct];
                r = &rg[R::R_GM1 + i + m * MX]; *r = (z3 ? 0.0 : *r) + dtdxv * gm_y(m, ct);
            }
        }
    }

    // ---- q update over i,j = 1-mbc..mx+mbc-1 (clawpack46_step2_wrap.f:107-125) ----
    // (fm_x / gm_y of the cell's right and top faces written out: one flux plane per field)
    for (int k = tid; k < G::QB; k += NT) {
        const int m = k / NXY, c = k - m * NXY;
        const int jc = c / NX, ic = c - jc * NX;
        if (ic > NX - 2 || jc > NY - 2) continue;
        const double* fxp = m == 0 ? Qs + NXY : (m == 1 ? FXX : FXY);
        const double* fyp = m == 0 ? Qs + 2 * NXY : (m == 1 ? FXY : FYY);
        const double* gx = GX + m * NXY;
        const double* gy = GY + m * NXY;
        double fmv = gx[c + 1];
        if (jc >= 1 && ic + 1 <= NX - 2)
            fmv = (m == 0 && (wallf & 2) && ic + 1 == MX + MBC) ? 0.0 - fxp[c] : (fxp[c + 1] - fxp[c]) + fmv;
        double gmv = gy[c + NX];
        if (ic >= 1 && ic <= NX - 2 && jc + 1 <= NY - 2)
            gmv = (m == 0 && (wallf & 8) && jc + 1 == MY + MBC) ? 0.0 - fyp[c] : (fyp[c + NX] - fyp[c]) + gmv;
        qg[k] = Qs[k] - dtdx * (fmv - gx[c]) - dtdy * (gmv - gy[c]);
    }

    // ---- CFL maximum: warp shuffles, then one atomic per CTA -----------------
    double cflmax = (double)cflw;
    for (int off = 16; off > 0; off >>= 1) cflmax = dmax1(cflmax, __shfl_xor_sync(0xffffffffu, cflmax, off));
    if ((tid & 31) == 0) red[tid >> 5] = cflmax;
    __syncthreads();
    if (tid < 32) {
        double v = (tid < NT / 32) ? red[tid] : 0.0;
        for (int off = 16; off > 0; off >>= 1) v = dmax1(v, __shfl_xor_sync(0xffffffffu, v, off));
        if (tid == 0) {
            unsigned long long bits = (unsigned long long)__double_as_longlong(v);
            if (v != v) bits = 0x7ff8000000000000ull;
            atomicMax(cfl_bits + pd.inst, bits);
        }
    }
}

// The fused update of npatch patches from slot p0: one CTA per patch, or (PERSIST) a
// grid of resident CTAs taking patches p0 + blockIdx.x, + gridDim.x, ... with the
// next patch's q requested while the current one computes.
template <int MX, int NT, int MINB, int LIM, bool PERSIST>
__global__ void __launch_bounds__(NT, MINB)
sw32_kernel(double* __restrict__ q, double* __restrict__ qlast, const double* __restrict__ aux,
            double* __restrict__ regs, const PatchDesc* __restrict__ desc, int p0, int npatch,
            const StepParams* __restrict__ spp, const LevelGroup lg, unsigned long long* __restrict__ cfl_bits)
{
    (void)aux;
    using G = SW32Geom<MX, NT, PERSIST>;
    extern __shared__ __align__(128) unsigned char sm[];
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(sm + G::OFF_BAR);
    int* stop = reinterpret_cast<int*>(sm + G::OFF_BAR + 16);
    double* qbuf = reinterpret_cast<double*>(sm + G::OFF_Q);
    grid_dependency_wait();         // programmatic launch: the previous grid's writes are visible
    grid_launch_dependents();
    const int stride = PERSIST ? (int)gridDim.x : npatch;
    int b = blockIdx.x;
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        *stop = 0;
        mbar_fence_init();
    }
    __syncthreads();
    if (threadIdx.x == 0 && b < npatch) bulk_load(&bar[0], qbuf, q + (size_t)(p0 + b) * G::QB, G::QBYTES);
    unsigned phase[2] = {0u, 0u};
    for (int it = 0; b < npatch; b += stride, it++) {
        const int cur = PERSIST ? (it & 1) : 0;
        // the other buffer's last reader finished before the previous iteration's final barrier
        if (PERSIST && threadIdx.x == 0 && b + stride < npatch)
            bulk_load(&bar[cur ^ 1], qbuf + (size_t)(cur ^ 1) * G::QB, q + (size_t)(p0 + b + stride) * G::QB,
                      G::QBYTES);
        if (!mbar_wait(&bar[cur], phase[cur], SW32_WAIT_LIMIT)) atomicExch(stop, 1);
        phase[cur] ^= 1u;
        __syncthreads();
        if (*stop) break;
        const StepParams sp = spp[group_slot(lg, b)];
        const PatchDesc pd = desc[p0 + b];
        sw32_patch<MX, NT, LIM, PERSIST>(sm, qbuf + (size_t)cur * G::QB, q, qlast, regs, pd, p0 + b, sp, cfl_bits);
        __syncthreads();   // the next patch reuses the shared memory
    }
    if (*stop) {
        // a staging copy did not arrive: report it, and wait (bounded) for the copies
        // this CTA started before leaving
        if (threadIdx.x == 0) {
            const StepParams sp = spp[0];
            if (sp.status) atomicOr(sp.status, (unsigned)STATUS_STAGING);
            for (int k = 0; k < G::NBUF; k++) (void)mbar_wait(&bar[k], phase[k], SW32_WAIT_LIMIT);
        }
    }
}

template <int MX, int NT, int MINB, int LIM, bool PERSIST>
cudaError_t run_sw32_variant(double* q, double* qlast, const double* aux, double* regs, const PatchDesc* desc, int p0,
                             int npatch, const StepParams* sp, const LevelGroup& lg,
                             unsigned long long* cfl_bits, cudaStream_t st)
{
    using G = SW32Geom<MX, NT, PERSIST>;
    static bool attr_set = false;
    static int grid_cap = 0;
    auto kern = sw32_kernel<MX, NT, MINB, LIM, PERSIST>;
    if (!attr_set) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::BYTES);
        if (e != cudaSuccess) return e;
        if (PERSIST) {
            int dev = 0, nsm = 0, per_sm = 0;
            e = cudaGetDevice(&dev);
            if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
            if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, G::BYTES);
            if (e != cudaSuccess) return e;
            grid_cap = nsm * (per_sm > 0 ? per_sm : 1);
        }
        attr_set = true;
    }
    if (npatch <= 0) return cudaSuccess;
    const int grid = PERSIST ? (npatch < grid_cap ? npatch : grid_cap) : npatch;
    return launch_k(kern, grid, NT, G::BYTES, st, q, qlast, aux, regs, desc, p0, npatch, sp, lg, cfl_bits);
}

// Table entries: FP32-wave Roe shallow water, MXV x MXV patches (mbc 2), limiter LIM on every wave.
#define FCB_SW32_VARIANT(MXV, NT, MINB, LIM, PERSIST)                                                          \
    Step2Variant{FC2D_B200_PREC_FP32WAVE, FC2D_B200_RP_SW_ROE, MXV, MXV, 2, NT, MINB, 1,                        \
                 (int)SW32Geom<MXV, NT, PERSIST>::BYTES, PERSIST ? 1 : 0,                                       \
                 &run_sw32_variant<MXV, NT, MINB, LIM, PERSIST>, LIM}

}  // namespace fcb
