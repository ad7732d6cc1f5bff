/*
 * fc2d_b200_user.cuh -- application-supplied __device__ solvers for the fused update.
 *
 * The reference's GPU solver lets an app install its own device Riemann solvers and
 * b4step2 by function pointer: the app defines
 *     __device__ cudaclaw_cuda_rpn2_t my_rpn2_ptr = my_rpn2;
 * copies the pointer out with cudaMemcpyFromSymbol and stores it in the cudaclaw
 * vtable (fc2d_cudaclaw.h:156-162, typedefs fc2d_cudaclaw_cuda.h:52-73, e.g.
 * applications/cudaclaw/acoustics/2d/radial/user_cuda/rpn2acoustics.cu:36-86).
 * This header keeps those device signatures and offers two ways to register:
 *
 *   FC2D_B200_USER_SOLVER(name, rpn2, rpt2, b4step2, src2, meqn, mwaves, maux, mx)
 *       the solver functions are template arguments: the fused update kernel is
 *       instantiated in the app's translation unit with them inlined (fast path).
 *       b4step2 / src2 may be nullptr.  Defines
 *           extern "C" int name(fc2d_b200_solver_t* s);
 *
 *   FC2D_B200_USER_SOLVER_FNPTR(name, meqn, mwaves, maux, mx)
 *       the cudaclaw protocol: the kernel calls through device function pointers
 *       the app obtained with cudaMemcpyFromSymbol (slow path; the solver can be
 *       switched at run time).  Defines
 *           extern "C" int name(fc2d_b200_solver_t* s, fc2d_b200_cuda_rpn2_t rpn2,
 *                               fc2d_b200_cuda_rpt2_t rpt2, fc2d_b200_cuda_b4step2_t b4step2,
 *                               fc2d_b200_cuda_src2_t src2);
 *       (b4step2 / src2 may be NULL).  The pointers must come from the same
 *       translation unit (or device-linked module) as the macro: a kernel can only
 *       call device functions of its own module.
 *
 * Either registration function installs the kernel in the solver (which must have
 * been created with rp = FC2D_B200_RP_USER, precision FP64, time sync off, and the
 * same meqn / mwaves / maux / mx = my / mbc = 2) and returns an FC2D_B200_* status.
 * Conventions are cudaclaw's: idir = 0 (x) or 1 (y); wave[mw * meqn + m]; rpt2's
 * imp = 0 splits amdq, 1 splits apdq, and aux1/aux2/aux3 hold the aux of the rows
 * below / of / above the interface for both cells, [imp * maux + m] (cell left of
 * the interface first, cudaclaw_flux2.cu:682-694).  b4step2 and src2 are called per
 * cell (Fortran indices i, j over the padded patch, 1-mbc..mx+mbc) with that cell's
 * q[meqn] and aux[maux]: b4step2 before the sweeps (it may change aux), src2 after
 * the q update (it may change q; clawpack46_update calls src2 after step2,
 * fc2d_clawpack46.cpp:436-441).
 *
 * Build the app's .cu with
 *     nvcc -gencode arch=compute_100a,code=sm_100a -std=c++17 -fmad=false \
 *          -I<repo>/include -I<repo>/forestclaw_b200/csrc -shared -Xcompiler -fPIC ...
 * and link it against libfc2d_b200.so (-fmad=false keeps the FP64 arithmetic free
 * of contractions, as in the package's own FP64 kernels).
 */
#ifndef FC2D_B200_USER_CUH
#define FC2D_B200_USER_CUH

#include <cstddef>
#include <type_traits>
#include "fc2d_b200.h"
#include "k_step2_variant.cuh"

/* Device signatures of fc2d_cudaclaw_cuda.h:52-73 (b4step2, rpn2, rpt2) and the
 * cell-wise source term, which has b4step2's signature and may change q. */
typedef void (*fc2d_b200_cuda_b4step2_t)(int mbc, int mx, int my, int meqn, double q[], double xlower,
                                         double ylower, double dx, double dy, double time, double dt, int maux,
                                         double aux[], int i, int j);
typedef fc2d_b200_cuda_b4step2_t fc2d_b200_cuda_src2_t;
typedef void (*fc2d_b200_cuda_rpn2_t)(int idir, int meqn, int mwaves, int maux, double ql[], double qr[],
                                      double auxl[], double auxr[], double wave[], double s[], double amdq[],
                                      double apdq[]);
typedef void (*fc2d_b200_cuda_rpt2_t)(int idir, int meqn, int mwaves, int maux, double ql[], double qr[],
                                      double aux1[], double aux2[], double aux3[], int imp, double asdq[],
                                      double bmasdq[], double bpasdq[]);

namespace fcb {

/* Threads per CTA of a user kernel: one per interface of a sweep where that fits. */
template <int MX>
constexpr int user_threads() { return MX <= 8 ? 128 : (MX <= 16 ? 352 : 512); }

/* The cudaclaw-convention solver functions seen as one of the package's solver
 * structs (riemann.cuh): arrays of doubles in, waves as wave[mw][m]. */
template <int MEQN_, int MWAVES_, int MAUX_, class Impl>
struct RPUserBase {
    static constexpr int MEQN = MEQN_, MWAVES = MWAVES_, MAUX = MAUX_, NEXTRA = 1;
    static constexpr bool CONS_FLUX = false, EXACT64 = false;
    static constexpr bool USER_HOOKS = true, AUX_BOTH = true;
    static constexpr int MA = MAUX > 0 ? MAUX : 1;
    template <typename T>
    __device__ static void rpn2(int ixy, const T* qL, const T* qR, const T* auxL, const T* auxR,
                                T wave[MWAVES][MEQN], T s[MWAVES], T amdq[MEQN], T apdq[MEQN], T extra[NEXTRA], T grav)
    {
        (void)grav;
        double ql[MEQN], qr[MEQN], al[MA], ar[MA], w[MWAVES * MEQN], sv[MWAVES], am[MEQN], ap[MEQN];
        for (int m = 0; m < MEQN; m++) { ql[m] = (double)qL[m]; qr[m] = (double)qR[m]; }
        for (int a = 0; a < MAUX; a++) { al[a] = (double)auxL[a]; ar[a] = (double)auxR[a]; }
        Impl::call_rpn2(ixy - 1, MEQN, MWAVES, MAUX, ql, qr, al, ar, w, sv, am, ap);
        for (int mw = 0; mw < MWAVES; mw++) {
            s[mw] = (T)sv[mw];
            for (int m = 0; m < MEQN; m++) wave[mw][m] = (T)w[mw * MEQN + m];
        }
        for (int m = 0; m < MEQN; m++) { amdq[m] = (T)am[m]; apdq[m] = (T)ap[m]; }
        extra[0] = T(0);
    }
    template <typename T>
    __device__ static void rpt2(int ixy, int imp, const T* qL, const T* qR, const T* aux1, const T* aux2,
                                const T* aux3, const T extra[NEXTRA], const T* asdq, T* bm, T* bp, T grav, T drytol)
    {
        (void)extra; (void)grav; (void)drytol;
        double ql[MEQN], qr[MEQN], a1[2 * MA], a2[2 * MA], a3[2 * MA], as[MEQN], b1[MEQN], b2[MEQN];
        for (int m = 0; m < MEQN; m++) { ql[m] = (double)qL[m]; qr[m] = (double)qR[m]; as[m] = (double)asdq[m]; }
        for (int h = 0; h < 2; h++)
            for (int a = 0; a < MAUX; a++) {
                a1[h * MAUX + a] = (double)aux1[h * MA + a];
                a2[h * MAUX + a] = (double)aux2[h * MA + a];
                a3[h * MAUX + a] = (double)aux3[h * MA + a];
            }
        Impl::call_rpt2(ixy - 1, MEQN, MWAVES, MAUX, ql, qr, a1, a2, a3, imp - 1, as, b1, b2);
        for (int m = 0; m < MEQN; m++) { bm[m] = (T)b1[m]; bp[m] = (T)b2[m]; }
    }
};

/* Fast path: the functions are template arguments and inline into the kernel. */
template <auto RPN2, auto RPT2, auto B4, auto SRC, int MEQN_, int MWAVES_, int MAUX_>
struct RPUser : RPUserBase<MEQN_, MWAVES_, MAUX_, RPUser<RPN2, RPT2, B4, SRC, MEQN_, MWAVES_, MAUX_>> {
    static constexpr bool HAS_B4STEP2 = !std::is_same<decltype(B4), std::nullptr_t>::value;
    static constexpr bool HAS_SRC2 = !std::is_same<decltype(SRC), std::nullptr_t>::value;
    template <class... A> __device__ static void call_rpn2(A... a) { RPN2(a...); }
    template <class... A> __device__ static void call_rpt2(A... a) { RPT2(a...); }
    template <class... A> __device__ static void b4step2(A... a) { B4(a...); }
    template <class... A> __device__ static void src2(A... a) { SRC(a...); }
};

/* Slow path: device function pointers read from a __constant__ record of the app's module. */
struct UserFnPtrs {
    fc2d_b200_cuda_rpn2_t rpn2;
    fc2d_b200_cuda_rpt2_t rpt2;
    fc2d_b200_cuda_b4step2_t b4step2;
    fc2d_b200_cuda_src2_t src2;
};
template <int MEQN_, int MWAVES_, int MAUX_, class Ptrs>
struct RPUserPtr : RPUserBase<MEQN_, MWAVES_, MAUX_, RPUserPtr<MEQN_, MWAVES_, MAUX_, Ptrs>> {
    static constexpr bool HAS_B4STEP2 = true, HAS_SRC2 = true;
    template <class... A> __device__ static void call_rpn2(A... a) { Ptrs::get().rpn2(a...); }
    template <class... A> __device__ static void call_rpt2(A... a) { Ptrs::get().rpt2(a...); }
    template <class... A> __device__ static void b4step2(A... a) { if (Ptrs::get().b4step2) Ptrs::get().b4step2(a...); }
    template <class... A> __device__ static void src2(A... a) { if (Ptrs::get().src2) Ptrs::get().src2(a...); }
};

}  // namespace fcb

/* The layout the package and the app must agree on (the kernel's parameter structs). */
#define FC2D_B200_USER_ABI ((int)fcb::device_abi())

#define FC2D_B200_USER_VARIANT_(RPT, MXV, PERSIST)                                                            \
    fcb::Step2Variant{FC2D_B200_PREC_FP64, FC2D_B200_RP_USER, MXV, MXV, 2, fcb::user_threads<MXV>(),             \
                      (MXV > 16 ? 1 : 2),                                                                     \
                      fcb::Step2Geom<RPT, MXV, MXV, 2, double, fcb::user_threads<MXV>()>::REG ? 1 : 0,        \
                      (int)fcb::Step2Geom<RPT, MXV, MXV, 2, double, fcb::user_threads<MXV>()>::SMEM_BYTES,     \
                      PERSIST,                                                                               \
                      &fcb::run_step2_variant<RPT, MXV, 2, false, fcb::user_threads<MXV>(), (MXV > 16 ? 1 : 2), \
                                              double, PERSIST>}
#define FC2D_B200_USER_TABLE_(RPT, MXV) FC2D_B200_USER_VARIANT_(RPT, MXV, 0), FC2D_B200_USER_VARIANT_(RPT, MXV, 1)

#define FC2D_B200_USER_SOLVER(NAME, RPN2, RPT2, B4STEP2, SRC2, MEQN, MWAVES, MAUX, MXV)                      \
    using NAME##_rp_t = fcb::RPUser<RPN2, RPT2, B4STEP2, SRC2, MEQN, MWAVES, MAUX>;                           \
    extern "C" int NAME(fc2d_b200_solver_t* s)                                                               \
    {                                                                                                        \
        static const fcb::Step2Variant table[] = {FC2D_B200_USER_TABLE_(NAME##_rp_t, MXV)};                  \
        return fc2d_b200_set_user_variants(s, table, (int)(sizeof(table) / sizeof(table[0])), FC2D_B200_USER_ABI, \
                                           MEQN, MWAVES, MAUX);                                              \
    }

#define FC2D_B200_USER_SOLVER_FNPTR(NAME, MEQN, MWAVES, MAUX, MXV)                                           \
    __constant__ fcb::UserFnPtrs NAME##_fnptrs;                                                              \
    struct NAME##_ptrs_t {                                                                                   \
        __device__ static const fcb::UserFnPtrs& get() { return NAME##_fnptrs; }                           \
    };                                                                                                       \
    using NAME##_rp_t = fcb::RPUserPtr<MEQN, MWAVES, MAUX, NAME##_ptrs_t>;                                    \
    extern "C" int NAME(fc2d_b200_solver_t* s, fc2d_b200_cuda_rpn2_t rpn2, fc2d_b200_cuda_rpt2_t rpt2,        \
                        fc2d_b200_cuda_b4step2_t b4step2, fc2d_b200_cuda_src2_t src2)                         \
    {                                                                                                        \
        if (!rpn2 || !rpt2) return FC2D_B200_EINVAL;                                                         \
        const fcb::UserFnPtrs p{rpn2, rpt2, b4step2, src2};                                                  \
        if (cudaMemcpyToSymbol(NAME##_fnptrs, &p, sizeof(p)) != cudaSuccess) return FC2D_B200_ECUDA;         \
        static const fcb::Step2Variant table[] = {FC2D_B200_USER_TABLE_(NAME##_rp_t, MXV)};                  \
        return fc2d_b200_set_user_variants(s, table, (int)(sizeof(table) / sizeof(table[0])), FC2D_B200_USER_ABI, \
                                           MEQN, MWAVES, MAUX);                                              \
    }

#endif
