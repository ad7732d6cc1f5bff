// k_step2_f64_euler.cu -- FP64 instantiations (built with -fmad=false: bitwise equal to the FP64 CPU path)
// of the fused update for Euler, exact Riemann solver: the patch-to-CTA variants of each patch size
// (one CTA per patch, then the persistent forms).
#include "k_step2_variant.cuh"
#include "fc2d_b200.h"

namespace fcb {

const Step2Variant* step2_table_f64_euler(int* n)
{
    static const Step2Variant table[] = {
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP64, FC2D_B200_RP_EULER_EXACT, RPEulerExact, 16, false, 352, 1, double),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP64, FC2D_B200_RP_EULER_EXACT, RPEulerExact, 16, false, 384, 1, double),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP64, FC2D_B200_RP_EULER_EXACT, RPEulerExact, 8, false, 128, 2, double),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP64, FC2D_B200_RP_EULER_EXACT, RPEulerExact, 8, false, 128, 1, double),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP64, FC2D_B200_RP_EULER_EXACT, RPEulerExact, 8, false, 160, 2, double),
        FCB_STEP2_VARIANT_P(FC2D_B200_PREC_FP64, FC2D_B200_RP_EULER_EXACT, RPEulerExact, 16, false, 352, 1, double),
        FCB_STEP2_VARIANT_P(FC2D_B200_PREC_FP64, FC2D_B200_RP_EULER_EXACT, RPEulerExact, 8, false, 128, 2, double),
    };
    *n = (int)(sizeof(table) / sizeof(table[0]));
    return table;
}

}  // namespace fcb
