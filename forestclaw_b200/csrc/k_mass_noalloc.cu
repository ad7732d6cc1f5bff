// k_mass_noalloc.cu -- mass diagnostic that allocates no device memory, for
// callers that may not allocate between steps (all device memory handed out by
// their own pool, or other streams that the synchronisation of cudaFree would
// stall).
//
// Same arithmetic as k_patch_mass + the host Kahan loop of fc2d_b200_mass
// (fclaw2d_clawpatch46_diagnostics.f:13-55): per patch and field a Kahan sum of
// q*dx*dy over interior cells in (j, i) order, then per field a Kahan sum of the
// patch partials in patch order.  The partials and the per-field results go to
// a fixed file-scope device array instead of a cudaMalloc'd buffer.
//
// Scratch layout (doubles): [0, np*meqn) patch partials, [np*meqn, np*meqn+meqn)
// the per-field sums.  No element has to start at zero: each call writes every
// element it reads before reading it.
#include <cuda_runtime.h>
#include "kernels.h"

namespace fcb {

static __device__ __align__(256) double g_mass_scratch[MASS_SCRATCH_DOUBLES];

__global__ void k_patch_mass_scratch(const double* __restrict__ q, const PatchDesc* __restrict__ desc, int mx,
                                     int my, int mbc, int meqn, double* __restrict__ scratch)
{
    const int p = blockIdx.x, m = threadIdx.x;
    if (m >= meqn) return;
    const int nx = mx + 2 * mbc, ny = my + 2 * mbc;
    const PatchDesc pd = desc[p];
    const double area = pd.dx * pd.dy;
    const double* qp = q + ((size_t)p * meqn + m) * nx * ny;
    double sum = 0.0, comp = 0.0;
    for (int j = 0; j < my; j++)
        for (int i = 0; i < mx; i++) {
            double y = qp[(j + mbc) * nx + i + mbc] * area - comp;
            double t = sum + y;
            comp = (t - sum) - y;
            sum = t;
        }
    scratch[(size_t)p * meqn + m] = sum;
}

// One thread per field: Kahan over the patch partials in patch order.
__global__ void k_mass_reduce_scratch(int np, int meqn, double* __restrict__ scratch)
{
    const int m = threadIdx.x;
    if (m >= meqn) return;
    double sum = 0.0, comp = 0.0;
    for (int p = 0; p < np; p++) {
        const double y = scratch[(size_t)p * meqn + m] - comp;
        const double t = sum + y;
        comp = (t - sum) - y;
        sum = t;
    }
    scratch[(size_t)np * meqn + m] = sum;
}

cudaError_t mass_scratch_address(double** ptr)
{
    return cudaGetSymbolAddress((void**)ptr, g_mass_scratch);
}

void launch_mass_noalloc(const Dims& d, const double* q, const PatchDesc* desc, int np, double* scratch,
                         cudaStream_t st)
{
    if (np > 0) k_patch_mass_scratch<<<np, 32, 0, st>>>(q, desc, d.mx, d.my, d.mbc, d.meqn, scratch);
    k_mass_reduce_scratch<<<1, 32, 0, st>>>(np, d.meqn, scratch);
}

}  // namespace fcb
