// k_metric.cu -- cubed-sphere metric on the device: cell areas, capacity and
// edge velocities of the manifold advection app.
//
// Built without FMA contraction; the mapping (fcb_sphere.h) uses only + - * /
// and sqrt, so the areas and aux arrays equal the CPU oracle's bit for bit.
//
// Areas follow the reference's metric build:
//   from scratch  fclaw2d_metric_fort_compute_area_general (fclaw2d_metric_default_fort.f90:110-176):
//                 the sum, over the (2^(maxlevel-level))^2 sub-quads of a cell (ii outer,
//                 jj inner), of the bilinear-quad area of the mapped sub-quad corners;
//   from fine     fclaw2d_metric_fort_average_area (:690-755) for cells 0..mx+1 of a patch
//                 made by coarsening (children in igrid order, the last one covering a
//                 cell wins), the other cells from scratch (compute_area_ghost);
//   kept          copied.
// The area array of a patch covers -mbc..mx+mbc+1 (one ring more than q).
// aux (user46_setaux_manifold.f): kappa = area / (dx dy), x-edge velocity
// (psi(node(i,j+1)) - psi(node(i,j))) / dy, y-edge velocity -(psi(node(i+1,j)) - psi(node(i,j))) / dx
// (applications/clawpack/advection/2d/all/user46_setaux_manifold.f:20-110, sphere/psi.f).
#include "fcb_sphere.h"
#include "kernels.h"

namespace fcb {

// Areas of new patches (ops of kind 0 and 2 first in the op list): one warp per (op,
// cell).  A cell from scratch has (2^(maxlevel-level))^2 sub-quads: the lanes compute
// their areas (ii outer, jj inner; each corner mapped from the same arguments as in a
// column sweep) into shared memory in chunks of METRIC_CHUNK, and lane 0 adds each
// chunk in order, so the sum is the sequential one.
constexpr int METRIC_WARPS = 4, METRIC_CHUNK = 1024;
__global__ void __launch_bounds__(32 * METRIC_WARPS)
k_sphere_area(const MetricOp* __restrict__ ops, const PatchDesc* __restrict__ desc, int mx, int my, int mbc,
              int maxlevel, const double* __restrict__ oarea, double* __restrict__ narea)
{
    __shared__ double sub[METRIC_WARPS][METRIC_CHUNK];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const MetricOp op = ops[blockIdx.x];
    const int ax = mx + 2 * mbc + 2, ay = my + 2 * mbc + 2, na = ax * ay;
    const int k = blockIdx.y * METRIC_WARPS + w;
    if (k >= na) return;                                      // the whole warp
    double* a = narea + (size_t)op.dst * na;
    const PatchDesc pd = desc[op.dst];
    const int i = k % ax - mbc, j = k / ax - mbc;              // -mbc .. mx+mbc+1
    const bool interior = i >= 0 && i <= mx + 1 && j >= 0 && j <= my + 1;
    if (op.kind == 2 && interior) {
        // fclaw2d_metric_fort_average_area: child igrid covers coarse cells
        // (i, j) - (ig mx/2, jg my/2) in 0 .. mx/2+1; the last covering child wins
        if (lane != 0) return;
        int g = -1, ic = 0, jc = 0;
        for (int igrid = 0; igrid < 4; igrid++) {
            const int ig = igrid % 2, jg = igrid / 2;
            const int ii = i - ig * mx / 2, jj = j - jg * mx / 2;
            if (ii >= 0 && ii <= mx / 2 + 1 && jj >= 0 && jj <= my / 2 + 1) { g = igrid; ic = ii; jc = jj; }
        }
        const double* f = oarea + (size_t)op.src[g] * na;
        double sum = 0.0;
        for (int jj = 1; jj <= 2; jj++)
            for (int ii = 1; ii <= 2; ii++) {
                const int fi = (ic - 1) * 2 + ii, fj = (jc - 1) * 2 + jj;
                sum = sum + f[(fj + mbc) * ax + (fi + mbc)];
            }
        a[k] = sum;
        return;
    }
    // from scratch: fclaw2d_metric_fort_compute_area_general
    const int rf = 1 << (maxlevel - pd.level), block = pd.block;
    const long nsub = (long)rf * rf;
    const double dxf = pd.dx / rf, dyf = pd.dy / rf;
    const double xe = pd.xlower + (i - 1) * pd.dx, ye = pd.ylower + (j - 1) * pd.dy;
    double sum = 0.0;
    for (long s0 = 0; s0 < nsub; s0 += METRIC_CHUNK) {
        const int n = (int)(nsub - s0 < METRIC_CHUNK ? nsub - s0 : METRIC_CHUNK);
        for (int t = lane; t < n; t += 32) {
            const long sq = s0 + t;
            const int ii = (int)(sq / rf), jj = (int)(sq % rf);
            double p[4][3];
            cs_map(block, xe + ii * dxf, ye + jj * dyf, &p[0][0], &p[0][1], &p[0][2]);
            cs_map(block, xe + (ii + 1) * dxf, ye + jj * dyf, &p[1][0], &p[1][1], &p[1][2]);
            cs_map(block, xe + ii * dxf, ye + (jj + 1) * dyf, &p[2][0], &p[2][1], &p[2][2]);
            cs_map(block, xe + (ii + 1) * dxf, ye + (jj + 1) * dyf, &p[3][0], &p[3][1], &p[3][2]);
            sub[w][t] = cs_quad_area(p);
        }
        __syncwarp();
        if (lane == 0)
            for (int t = 0; t < n; t++) sum = sum + sub[w][t];
        __syncwarp();
    }
    if (lane == 0) a[k] = sum;
}

// Areas of kept patches (ops of kind 1): copied, one thread per (op, cell).
__global__ void k_sphere_area_copy(const MetricOp* __restrict__ ops, int na, const double* __restrict__ oarea,
                                   double* __restrict__ narea)
{
    const MetricOp op = ops[blockIdx.x];
    const int k = blockIdx.y * blockDim.x + threadIdx.x;
    if (k < na) narea[(size_t)op.dst * na + k] = oarea[(size_t)op.src[0] * na + k];
}

// aux of new patches (ops of kind 0 and 2): one thread per (op, cell).
__global__ void k_sphere_aux(const MetricOp* __restrict__ ops, const PatchDesc* __restrict__ desc, int mx, int my,
                             int mbc, const double* __restrict__ area, double* __restrict__ aux,
                             SphereFlow flow)
{
    const MetricOp op = ops[blockIdx.x];
    if (op.kind == 1) return;
    const int nx = mx + 2 * mbc, ny = my + 2 * mbc, nxy = nx * ny;
    const int ax = nx + 2, na = ax * (ny + 2);
    const PatchDesc pd = desc[op.dst];
    const int block = pd.block;
    const double* a = area + (size_t)op.dst * na;
    double* x = aux + (size_t)op.dst * 3 * nxy;
    const double dxdy = pd.dx * pd.dy;
    auto psi_node = [&](int i, int j) {
        double xp, yp, zp;
        cs_map(block, pd.xlower + (i - 1) * pd.dx, pd.ylower + (j - 1) * pd.dy, &xp, &yp, &zp);
        return cs_psi(flow.axis, flow.omega, xp, yp, zp);
    };
    const int k = blockIdx.y * blockDim.x + threadIdx.x;
    if (k < nxy) {
        const int i = k % nx + 1 - mbc, j = k / nx + 1 - mbc;
        x[k] = a[(j + mbc) * ax + (i + mbc)] / dxdy;
        const double p00 = psi_node(i, j);
        x[nxy + k] = (psi_node(i, j + 1) - p00) / pd.dy;
        x[2 * nxy + k] = -((psi_node(i + 1, j) - p00) / pd.dx);
    }
}

void launch_sphere_metric(const Dims& d, const MetricOp* ops, int nnew, int nkept, const PatchDesc* desc, int maxlevel,
                          const double* oarea, double* narea, double* aux, const SphereFlow& flow, cudaStream_t st)
{
    const int na = (d.mx + 2 * d.mbc + 2) * (d.my + 2 * d.mbc + 2);
    if (nnew > 0) {
        k_sphere_area<<<dim3(nnew, (na + METRIC_WARPS - 1) / METRIC_WARPS), 32 * METRIC_WARPS, 0, st>>>(
            ops, desc, d.mx, d.my, d.mbc, maxlevel, oarea, narea);
        k_sphere_aux<<<dim3(nnew, (d.nxy() + 127) / 128), 128, 0, st>>>(ops, desc, d.mx, d.my, d.mbc, narea, aux, flow);
    }
    if (nkept > 0) k_sphere_area_copy<<<dim3(nkept, (na + 255) / 256), 256, 0, st>>>(ops + nnew, na, oarea, narea);
}

}  // namespace fcb
