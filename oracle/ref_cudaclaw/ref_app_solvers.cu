// ref_app_solvers.cu -- the reference's cudaclaw Riemann solvers, compiled from
// the reference tree for the pin harness (test infrastructure only).
//
// Each app's solver file is included as it lies in the reference tree, inside a
// namespace of its own (the files define same-named __constant__ parameters).
// The apps' own headers pull in the whole framework (p4est, libsc), which the
// solver functions do not use: their include guards are defined here so those
// headers are skipped, the cudaclaw solver headers supply the typedefs, and
// SC_MIN / SC_MAX / fclaw_global_essentialf get plain definitions.  The
// solver files include fc2d_cudaclaw_check.h (no include guard) themselves, so
// each namespace gets its own copy of its helper.
//   swirl      applications/cudaclaw/advection/2d/swirl/user_cuda/rpn2adv.cu, rpt2adv.cu
//   radialdam  applications/clawpack/shallow/2d/radialdam_cuda/user_cuda/rpn2shallow.cu (Roe)
//   shockbubble applications/cudaclaw/euler/2d/shockbubble/user_cuda/rp2euler.cu (Roe; its
//              transverse solver shockbubble_rpt2euler4 is evaluated point-wise below)
#include <stdio.h>
#include <stdlib.h>
#include "fc2d_cudaclaw.h"
#include "fc2d_cudaclaw_cuda.h"

#define SWIRL_USER_H
#define RADIALDAM_USER_H
#define SHOCKBUBBLE_USER_H
#define FCLAW_BASE_H
#define SC_MIN(a, b) (((a) < (b)) ? (a) : (b))
#define SC_MAX(a, b) (((a) > (b)) ? (a) : (b))
#define fclaw_global_essentialf(...) printf(__VA_ARGS__)

namespace ref_swirl {
#include "applications/cudaclaw/advection/2d/swirl/user_cuda/rpn2adv.cu"
#include "applications/cudaclaw/advection/2d/swirl/user_cuda/rpt2adv.cu"
}
namespace ref_radialdam {
#include "applications/clawpack/shallow/2d/radialdam_cuda/user_cuda/rpn2shallow.cu"
}
namespace ref_shockbubble {
#include "applications/cudaclaw/euler/2d/shockbubble/user_cuda/rp2euler.cu"
}

// bmasdq, bpasdq of n interfaces (states of the cells below / above, asdq), as
// cudaclaw's flux2 calls the transverse solver: idir 0 or 1, imp 0, no aux.
__global__ void pin_euler_rpt2_kernel(int idir, int n, const double* ql, const double* qr, const double* asdq,
                                      double* bm, double* bp)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    double l[4], r[4], a[4], m[4], p[4], aux[1] = {0.0};
    for (int c = 0; c < 4; c++) { l[c] = ql[4 * k + c]; r[c] = qr[4 * k + c]; a[c] = asdq[4 * k + c]; }
    ref_shockbubble::shockbubble_rpt2euler4(idir, 4, 3, 0, l, r, aux, aux, aux, 0, a, m, p);
    for (int c = 0; c < 4; c++) { bm[4 * k + c] = m[c]; bp[4 * k + c] = p[c]; }
}

#define PIN_CK2(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { err = e_; goto done; } } while (0)

// The reference's Euler transverse solver on n interfaces (host arrays, 4 doubles each);
// gamma sets the solver's constants as its setprob_cuda would.  Returns 0 or the CUDA error.
extern "C" int pin_ref_euler_rpt2(int idir, int n, double gamma, const double* ql, const double* qr,
                                  const double* asdq, double* bm, double* bp)
{
    cudaError_t err = cudaSuccess;
    double* d = nullptr;
    const size_t bytes = sizeof(double) * 4 * (size_t)n;
    const double gamma1 = gamma - 1.0;
    if (n <= 0 || (idir != 0 && idir != 1)) return -1;
    PIN_CK2(cudaMemcpyToSymbol(ref_shockbubble::s_gamma, &gamma, sizeof(double)));
    PIN_CK2(cudaMemcpyToSymbol(ref_shockbubble::s_gamma1, &gamma1, sizeof(double)));
    PIN_CK2(cudaMalloc(&d, 5 * bytes));
    PIN_CK2(cudaMemcpy(d, ql, bytes, cudaMemcpyHostToDevice));
    PIN_CK2(cudaMemcpy(d + 4 * (size_t)n, qr, bytes, cudaMemcpyHostToDevice));
    PIN_CK2(cudaMemcpy(d + 8 * (size_t)n, asdq, bytes, cudaMemcpyHostToDevice));
    pin_euler_rpt2_kernel<<<(n + 127) / 128, 128>>>(idir, n, d, d + 4 * (size_t)n, d + 8 * (size_t)n,
                                                    d + 12 * (size_t)n, d + 16 * (size_t)n);
    PIN_CK2(cudaGetLastError());
    PIN_CK2(cudaMemcpy(bm, d + 12 * (size_t)n, bytes, cudaMemcpyDeviceToHost));
    PIN_CK2(cudaMemcpy(bp, d + 16 * (size_t)n, bytes, cudaMemcpyDeviceToHost));
done:
    if (d) cudaFree(d);
    return (int)err;
}

// Device pointers of solver pair `id` (0 swirl advection, 1 radialdam Roe) with
// its parameters set; returns 0, or -1 for an unknown id.
extern "C" int pin_ref_solver(int id, double grav, double dry_tolerance, double sea_level,
                              cudaclaw_cuda_rpn2_t* rpn2, cudaclaw_cuda_rpt2_t* rpt2)
{
    (void)dry_tolerance; (void)sea_level;
    switch (id) {
    case 0:
        ref_swirl::swirl_assign_rpn2(rpn2);
        ref_swirl::swirl_assign_rpt2(rpt2);
        return 0;
    case 1:
        ref_radialdam::radialdam_setprob_cuda(grav);
        ref_radialdam::radialdam_assign_rpn2(rpn2);
        ref_radialdam::radialdam_assign_rpt2(rpt2);
        return 0;
    default:
        return -1;
    }
}
