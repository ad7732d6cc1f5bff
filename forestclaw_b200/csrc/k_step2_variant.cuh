// k_step2_variant.cuh -- launchers of the fused update, one per patch-to-CTA mapping.
//
// A variant fixes how one patch maps onto its CTA: NT threads and a
// __launch_bounds__ occupancy target of MINB CTAs per SM (which caps the
// registers per thread).  With NT >= the interfaces of a sweep every interface
// has its own thread and its normal solve stays in registers (REG); with fewer
// threads the CTA strides over the interfaces and keeps the per-interface record
// in shared memory.  The arithmetic of every interface and the order of all
// accumulations are the same in every variant, so the FP64 variants give
// identical bits; the autotuner (host side) picks the fastest for a forest.
#pragma once
#include "fcb_launch.cuh"
#include "k_step2.cuh"
#include "kernels.h"

namespace fcb {

template <class RP, int MX, int MBC, bool FW, int NT, int MINB, typename TW, bool PERSIST = false>
cudaError_t run_step2_variant(double* q, double* qlast, const double* aux, double* regs, const PatchDesc* desc,
                              int p0, int npatch, const StepParams* sp, const LevelGroup& lg,
                              unsigned long long* cfl_bits,
                              cudaStream_t st)
{
    using G = Step2Geom<RP, MX, MX, MBC, TW, NT>;
    static bool attr_set = false;
    static int grid_cap = 0;   // persistent: resident CTAs of the whole device
    auto kern = step2_kernel<RP, MX, MX, MBC, FW, NT, TW, MINB, PERSIST>;
    if (!attr_set) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::SMEM_BYTES);
        if (e != cudaSuccess) return e;
        if (PERSIST) {
            int dev = 0, nsm = 0, per_sm = 0;
            e = cudaGetDevice(&dev);
            if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
            if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, G::SMEM_BYTES);
            if (e != cudaSuccess) return e;
            grid_cap = nsm * (per_sm > 0 ? per_sm : 1);
        }
        attr_set = true;
    }
    if (npatch <= 0) return cudaSuccess;
    const int grid = PERSIST ? (npatch < grid_cap ? npatch : grid_cap) : npatch;
    return launch_k(kern, grid, NT, G::SMEM_BYTES, st, q, qlast, aux, regs, desc, p0, npatch, sp, lg, cfl_bits);
}

// One table entry: precision, solver id, square patch size MXV (mbc 2), threads, min CTAs per SM.
#define FCB_STEP2_VARIANT(PREC, RPID, RPT, MXV, FW, NT, MINB, TW)                                           \
    Step2Variant{PREC, RPID, MXV, MXV, 2, NT, MINB, Step2Geom<RPT, MXV, MXV, 2, TW, NT>::REG ? 1 : 0,       \
                 (int)Step2Geom<RPT, MXV, MXV, 2, TW, NT>::SMEM_BYTES, 0,                                   \
                 &run_step2_variant<RPT, MXV, 2, FW, NT, MINB, TW, false>}
// The same mapping as a persistent kernel: a grid of resident CTAs looping over the patches.
#define FCB_STEP2_VARIANT_P(PREC, RPID, RPT, MXV, FW, NT, MINB, TW)                                         \
    Step2Variant{PREC, RPID, MXV, MXV, 2, NT, MINB, Step2Geom<RPT, MXV, MXV, 2, TW, NT>::REG ? 1 : 0,       \
                 (int)Step2Geom<RPT, MXV, MXV, 2, TW, NT>::SMEM_BYTES, 1,                                   \
                 &run_step2_variant<RPT, MXV, 2, FW, NT, MINB, TW, true>}

}  // namespace fcb
