// k_step2_f64_adv.cu -- FP64 instantiations (built with -fmad=false: bitwise equal to the FP64 CPU path)
// of the fused update for scalar advection (plane and manifold): the patch-to-CTA variants of each patch size
// (one CTA per patch, then the persistent forms).
#include "k_step2_variant.cuh"
#include "fc2d_b200.h"

namespace fcb {

const Step2Variant* step2_table_f64_adv(int* n)
{
    static const Step2Variant table[] = {
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP64, FC2D_B200_RP_ADVECTION, RPAdvection, 32, false, 512, 2, double),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP64, FC2D_B200_RP_ADVECTION, RPAdvection, 32, false, 256, 2, double),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP64, FC2D_B200_RP_ADVECTION, RPAdvection, 32, false, 256, 4, double),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP64, FC2D_B200_RP_ADVECTION, RPAdvection, 32, false, 1024, 1, double),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP64, FC2D_B200_RP_ADVECTION, RPAdvection, 16, false, 416, 2, double),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP64, FC2D_B200_RP_ADVECTION, RPAdvection, 16, false, 352, 2, double),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP64, FC2D_B200_RP_ADVECTION, RPAdvection, 16, false, 256, 3, double),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP64, FC2D_B200_RP_ADVECTION, RPAdvection, 8, false, 160, 2, double),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP64, FC2D_B200_RP_ADVECTION, RPAdvection, 8, false, 128, 4, double),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP64, FC2D_B200_RP_ADVECTION, RPAdvection, 8, false, 64, 8, double),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP64, FC2D_B200_RP_ADVECTION_MANIFOLD, RPAdvectionManifold, 32, false, 512, 2, double),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP64, FC2D_B200_RP_ADVECTION_MANIFOLD, RPAdvectionManifold, 32, false, 256, 2, double),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP64, FC2D_B200_RP_ADVECTION_MANIFOLD, RPAdvectionManifold, 32, false, 256, 4, double),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP64, FC2D_B200_RP_ADVECTION_MANIFOLD, RPAdvectionManifold, 32, false, 1024, 1, double),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP64, FC2D_B200_RP_ADVECTION_MANIFOLD, RPAdvectionManifold, 16, false, 416, 2, double),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP64, FC2D_B200_RP_ADVECTION_MANIFOLD, RPAdvectionManifold, 16, false, 352, 2, double),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP64, FC2D_B200_RP_ADVECTION_MANIFOLD, RPAdvectionManifold, 16, false, 256, 3, double),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP64, FC2D_B200_RP_ADVECTION_MANIFOLD, RPAdvectionManifold, 8, false, 160, 2, double),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP64, FC2D_B200_RP_ADVECTION_MANIFOLD, RPAdvectionManifold, 8, false, 128, 4, double),
        FCB_STEP2_VARIANT_P(FC2D_B200_PREC_FP64, FC2D_B200_RP_ADVECTION, RPAdvection, 32, false, 512, 2, double),
        FCB_STEP2_VARIANT_P(FC2D_B200_PREC_FP64, FC2D_B200_RP_ADVECTION, RPAdvection, 32, false, 1024, 1, double),
        FCB_STEP2_VARIANT_P(FC2D_B200_PREC_FP64, FC2D_B200_RP_ADVECTION, RPAdvection, 16, false, 416, 2, double),
        FCB_STEP2_VARIANT_P(FC2D_B200_PREC_FP64, FC2D_B200_RP_ADVECTION, RPAdvection, 8, false, 160, 2, double),
        FCB_STEP2_VARIANT_P(FC2D_B200_PREC_FP64, FC2D_B200_RP_ADVECTION_MANIFOLD, RPAdvectionManifold, 32, false, 512, 2, double),
        FCB_STEP2_VARIANT_P(FC2D_B200_PREC_FP64, FC2D_B200_RP_ADVECTION_MANIFOLD, RPAdvectionManifold, 32, false, 1024, 1, double),
        FCB_STEP2_VARIANT_P(FC2D_B200_PREC_FP64, FC2D_B200_RP_ADVECTION_MANIFOLD, RPAdvectionManifold, 16, false, 416, 2, double),
        FCB_STEP2_VARIANT_P(FC2D_B200_PREC_FP64, FC2D_B200_RP_ADVECTION_MANIFOLD, RPAdvectionManifold, 8, false, 160, 2, double),
    };
    *n = (int)(sizeof(table) / sizeof(table[0]));
    return table;
}

}  // namespace fcb
