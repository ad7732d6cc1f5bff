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
#include <stdio.h>
#include <stdlib.h>
#include "fc2d_cudaclaw.h"
#include "fc2d_cudaclaw_cuda.h"

#define SWIRL_USER_H
#define RADIALDAM_USER_H
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
