// k_step2_f32w_sw.cu -- FP32-wave instantiations (built with --use_fast_math; FP64 accumulation)
// of the fused update for shallow water (Roe and f-wave): the specialised Roe kernel first, then the
// patch-to-CTA variants of each patch size (one CTA per patch, then the persistent forms).
#include "k_step2_variant.cuh"
#include "k_sw32.cuh"
#include "fc2d_b200.h"

namespace fcb {

const Step2Variant* step2_table_f32w_sw(int* n)
{
    static const Step2Variant table[] = {
        // Roe with the MC limiter on every wave and second-order transverse terms (k_sw32.cuh)
        FCB_SW32_VARIANT(16, 352, 2, 4, false),
        FCB_SW32_VARIANT(16, 352, 3, 4, false),
        FCB_SW32_VARIANT(16, 384, 2, 4, false),
        FCB_SW32_VARIANT(16, 352, 2, 4, true),
        FCB_SW32_VARIANT(16, 352, 3, 4, true),
        FCB_SW32_VARIANT(8, 128, 4, 4, false),
        FCB_SW32_VARIANT(8, 128, 8, 4, false),
        FCB_SW32_VARIANT(8, 128, 6, 4, true),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP32WAVE, FC2D_B200_RP_SW_ROE, RPShallowRoe, 16, false, 416, 2, float),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP32WAVE, FC2D_B200_RP_SW_ROE, RPShallowRoe, 16, false, 352, 2, float),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP32WAVE, FC2D_B200_RP_SW_ROE, RPShallowRoe, 16, false, 352, 1, float),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP32WAVE, FC2D_B200_RP_SW_ROE, RPShallowRoe, 16, false, 256, 3, float),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP32WAVE, FC2D_B200_RP_SW_ROE, RPShallowRoe, 16, false, 192, 4, float),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP32WAVE, FC2D_B200_RP_SW_ROE, RPShallowRoe, 8, false, 160, 2, float),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP32WAVE, FC2D_B200_RP_SW_ROE, RPShallowRoe, 8, false, 128, 4, float),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP32WAVE, FC2D_B200_RP_SW_ROE, RPShallowRoe, 8, false, 160, 4, float),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP32WAVE, FC2D_B200_RP_SW_ROE, RPShallowRoe, 8, false, 64, 8, float),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP32WAVE, FC2D_B200_RP_SW_FWAVE, RPShallowFWave, 16, true, 416, 2, float),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP32WAVE, FC2D_B200_RP_SW_FWAVE, RPShallowFWave, 16, true, 352, 2, float),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP32WAVE, FC2D_B200_RP_SW_FWAVE, RPShallowFWave, 16, true, 352, 1, float),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP32WAVE, FC2D_B200_RP_SW_FWAVE, RPShallowFWave, 16, true, 256, 3, float),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP32WAVE, FC2D_B200_RP_SW_FWAVE, RPShallowFWave, 16, true, 192, 4, float),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP32WAVE, FC2D_B200_RP_SW_FWAVE, RPShallowFWave, 8, true, 160, 2, float),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP32WAVE, FC2D_B200_RP_SW_FWAVE, RPShallowFWave, 8, true, 128, 4, float),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP32WAVE, FC2D_B200_RP_SW_FWAVE, RPShallowFWave, 8, true, 160, 4, float),
        FCB_STEP2_VARIANT(FC2D_B200_PREC_FP32WAVE, FC2D_B200_RP_SW_FWAVE, RPShallowFWave, 8, true, 64, 8, float),
        FCB_STEP2_VARIANT_P(FC2D_B200_PREC_FP32WAVE, FC2D_B200_RP_SW_ROE, RPShallowRoe, 16, false, 416, 2, float),
        FCB_STEP2_VARIANT_P(FC2D_B200_PREC_FP32WAVE, FC2D_B200_RP_SW_ROE, RPShallowRoe, 16, false, 352, 2, float),
        FCB_STEP2_VARIANT_P(FC2D_B200_PREC_FP32WAVE, FC2D_B200_RP_SW_ROE, RPShallowRoe, 8, false, 160, 2, float),
        FCB_STEP2_VARIANT_P(FC2D_B200_PREC_FP32WAVE, FC2D_B200_RP_SW_ROE, RPShallowRoe, 8, false, 160, 4, float),
        FCB_STEP2_VARIANT_P(FC2D_B200_PREC_FP32WAVE, FC2D_B200_RP_SW_FWAVE, RPShallowFWave, 16, true, 416, 2, float),
        FCB_STEP2_VARIANT_P(FC2D_B200_PREC_FP32WAVE, FC2D_B200_RP_SW_FWAVE, RPShallowFWave, 16, true, 352, 2, float),
        FCB_STEP2_VARIANT_P(FC2D_B200_PREC_FP32WAVE, FC2D_B200_RP_SW_FWAVE, RPShallowFWave, 8, true, 160, 2, float),
        FCB_STEP2_VARIANT_P(FC2D_B200_PREC_FP32WAVE, FC2D_B200_RP_SW_FWAVE, RPShallowFWave, 8, true, 160, 4, float),
    };
    *n = (int)(sizeof(table) / sizeof(table[0]));
    return table;
}

}  // namespace fcb
