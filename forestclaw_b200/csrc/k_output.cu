// k_output.cu -- device side of the VTK output: the point coordinates and the
// cell values of every patch, packed in the file's order, so one copy brings a
// frame to the host (fclaw2d_clawpatch_output_vtk.c:699-855: coordinate_cb,
// value_cb).  Built without FMA contraction: x = xlower + i dx is the same double
// the host computes; manifold points go through the cubed-sphere mapping of
// fcb_sphere.h.
#include "fcb_sphere.h"
#include "kernels.h"

namespace fcb {

// One CTA per output patch: order[b] = the patch slot written b-th.
__global__ void k_vtk_pack(const double* __restrict__ q, const PatchDesc* __restrict__ desc,
                           const int* __restrict__ order, int mx, int my, int mbc, int meqn, int manifold,
                           double* __restrict__ points, float* __restrict__ values)
{
    const int b = blockIdx.x, p = order[b];
    const PatchDesc pd = desc[p];
    const int nx = mx + 2 * mbc, ny = my + 2 * mbc;
    const int npt = (mx + 1) * (my + 1), ncell = mx * my;
    double* pt = points + (size_t)b * npt * 3;
    for (int k = threadIdx.x; k < npt; k += blockDim.x) {
        const int i = k % (mx + 1), j = k / (mx + 1);
        const double y = pd.ylower + j * pd.dy;
        const double x = pd.xlower + i * pd.dx;
        double xp = x, yp = y, zp = 0.0;
        if (manifold) cs_map(pd.block, x, y, &xp, &yp, &zp);
        pt[3 * k + 0] = xp;
        pt[3 * k + 1] = yp;
        pt[3 * k + 2] = zp;
    }
    const double* qp = q + (size_t)p * nx * ny * meqn;
    float* v = values + (size_t)b * ncell * meqn;
    for (int k = threadIdx.x; k < ncell * meqn; k += blockDim.x) {
        const int e = k % meqn, c = k / meqn, i = c % mx, j = c / mx;
        v[k] = __double2float_rn(qp[((size_t)e * ny + j + mbc) * nx + i + mbc]);
    }
}

void launch_vtk_pack(const Dims& d, const double* q, const PatchDesc* desc, const int* order, int npatch, int manifold,
                     double* points, float* values, cudaStream_t st)
{
    if (npatch > 0) k_vtk_pack<<<npatch, 256, 0, st>>>(q, desc, order, d.mx, d.my, d.mbc, d.meqn, manifold, points, values);
}

}  // namespace fcb
