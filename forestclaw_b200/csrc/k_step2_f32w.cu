// k_step2_f32w.cu -- FP32-wave instantiations of the fused update (see k_step2.cuh).
#include "kernels.h"
#include "fc2d_b200.h"

namespace fcb {

cudaError_t launch_step2_f32w(int rp, const Dims& d, double* q, double* qlast, const double* aux, double* regs,
                              const PatchDesc* desc, int p0, int npatch, const StepParams& sp,
                              unsigned long long* cfl_bits, cudaStream_t st)
{
    (void)rp; (void)d; (void)q; (void)qlast; (void)aux; (void)regs; (void)desc; (void)p0; (void)npatch;
    (void)sp; (void)cfl_bits; (void)st;
    return cudaErrorInvalidValue;
}

bool step2_f32w_supported(int rp, int mx, int my, int mbc)
{
    (void)rp; (void)mx; (void)my; (void)mbc;
    return false;
}

}  // namespace fcb
