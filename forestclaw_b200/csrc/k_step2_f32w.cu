// k_step2_f32w.cu -- FP32-wave instantiations of the fused update (k_step2.cuh).
// Waves, speeds, limiter, second-order correction and transverse splitting in
// FP32 (fast intrinsics: this unit is built with --use_fast_math); flux arrays,
// q update, time-sync registers and the Godunov split remainder in FP64.
#include "k_step2.cuh"
#include "kernels.h"
#include "fc2d_b200.h"

namespace fcb {

template <class RP, int MX, int MY, int MBC, bool FW, int NT, int MINB = 2>
static cudaError_t run_step2_f32(const Dims& d, double* q, double* qlast, const double* aux, double* regs,
                                 const PatchDesc* desc, int p0, int npatch, const StepParams* sp,
                                 unsigned long long* cfl_bits, cudaStream_t st)
{
    using G = Step2Geom<RP, MX, MY, MBC, float, NT>;
    static bool attr_set = false;
    auto kern = step2_kernel<RP, MX, MY, MBC, FW, NT, float, MINB>;
    if (!attr_set) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::SMEM_BYTES);
        if (e != cudaSuccess) return e;
        attr_set = true;
    }
    (void)d;
    if (npatch <= 0) return cudaSuccess;
    kern<<<npatch, NT, G::SMEM_BYTES, st>>>(q, qlast, aux, regs, desc, p0, sp, cfl_bits);
    return cudaGetLastError();
}

#define FCB_CASE32(RPID, RPT, MXV, MYV, MBCV, FW, NT)                                                       \
    if (rp == RPID && d.mx == MXV && d.my == MYV && d.mbc == MBCV)                                          \
        return run_step2_f32<RPT, MXV, MYV, MBCV, FW, NT>(d, q, qlast, aux, regs, desc, p0, npatch, sp, cfl_bits, st);

cudaError_t launch_step2_f32w(int rp, const Dims& d, double* q, double* qlast, const double* aux, double* regs,
                              const PatchDesc* desc, int p0, int npatch, const StepParams* sp,
                              unsigned long long* cfl_bits, cudaStream_t st)
{
    FCB_CASE32(FC2D_B200_RP_ADVECTION, RPAdvection, 32, 32, 2, false, 512)
    FCB_CASE32(FC2D_B200_RP_ADVECTION, RPAdvection, 16, 16, 2, false, 416)
    FCB_CASE32(FC2D_B200_RP_SW_ROE, RPShallowRoe, 16, 16, 2, false, 416)
    FCB_CASE32(FC2D_B200_RP_SW_ROE, RPShallowRoe, 8, 8, 2, false, 160)
    FCB_CASE32(FC2D_B200_RP_SW_FWAVE, RPShallowFWave, 16, 16, 2, true, 416)
    FCB_CASE32(FC2D_B200_RP_SW_FWAVE, RPShallowFWave, 8, 8, 2, true, 160)
    if (rp == FC2D_B200_RP_EULER_EXACT && d.mx == 16 && d.my == 16 && d.mbc == 2)
        return run_step2_f32<RPEulerExact, 16, 16, 2, false, 352, 1>(d, q, qlast, aux, regs, desc, p0, npatch, sp,
                                                                     cfl_bits, st);
    FCB_CASE32(FC2D_B200_RP_EULER_EXACT, RPEulerExact, 8, 8, 2, false, 128)
    return cudaErrorInvalidValue;
}

bool step2_f32w_supported(int rp, int mx, int my, int mbc)
{
    if (mbc != 2 || mx != my) return false;
    if (rp == FC2D_B200_RP_ADVECTION) return mx == 32 || mx == 16;
    if (rp == FC2D_B200_RP_SW_ROE || rp == FC2D_B200_RP_SW_FWAVE || rp == FC2D_B200_RP_EULER_EXACT)
        return mx == 16 || mx == 8;
    return false;
}

}  // namespace fcb
