// An application's own device solvers, outside the package, registered through
// include/fc2d_b200_user.cuh: the radial acoustics Riemann pair of the reference's
// GPU app (applications/cudaclaw/acoustics/2d/radial/user_cuda/rpn2acoustics.cu:30-68,
// rpt2acoustics.cu:88-118, restated) and a damping source term q1 -= dt*rate*q1.
// Registered both ways: inlined into the fused update (acoustics_register_inline)
// and through device function pointers, the cudaclaw protocol (acoustics_register_by_pointer).
#include <cmath>
#include "fc2d_b200_user.cuh"

__constant__ double s_c, s_z, s_rate;

// setprob_cuda of the app: c = sqrt(bulk/rho), z = c rho, computed on the host
extern "C" int acoustics_set_params(double rho, double bulk, double rate)
{
    const double c = std::sqrt(bulk / rho), z = c * rho;
    if (cudaMemcpyToSymbol(s_c, &c, sizeof(double)) != cudaSuccess) return -1;
    if (cudaMemcpyToSymbol(s_z, &z, sizeof(double)) != cudaSuccess) return -1;
    if (cudaMemcpyToSymbol(s_rate, &rate, sizeof(double)) != cudaSuccess) return -1;
    return 0;
}

__device__ void rpn2acoustics(int idir, int meqn, int mwaves, int maux, double ql[], double qr[], double auxl[],
                              double auxr[], double wave[], double s[], double amdq[], double apdq[])
{
    const int mu = 1 + idir, mv = 2 - idir;
    s[0] = -s_c;
    s[1] = s_c;
    const double d0 = qr[0] - ql[0], d1 = qr[mu] - ql[mu];
    const double alpha1 = (-d0 + s_z * d1) / (2.0 * s_z);
    const double alpha2 = (d0 + s_z * d1) / (2.0 * s_z);
    wave[0] = -alpha1 * s_z;
    wave[mu] = alpha1;
    wave[mv] = 0;
    wave[meqn] = alpha2 * s_z;
    wave[meqn + mu] = alpha2;
    wave[meqn + mv] = 0;
    for (int m = 0; m < meqn; m++) {
        amdq[m] = s[0] * wave[m];
        apdq[m] = s[1] * wave[meqn + m];
    }
}

__device__ void rpt2acoustics(int idir, int meqn, int mwaves, int maux, double ql[], double qr[], double aux1[],
                              double aux2[], double aux3[], int imp, double asdq[], double bmasdq[], double bpasdq[])
{
    const int mu = 1 + idir, mv = 2 - idir;
    const double d0 = asdq[0], d1 = asdq[mv];
    const double alpha1 = (-d0 + s_z * d1) / (2.0 * s_z);
    const double alpha2 = (d0 + s_z * d1) / (2.0 * s_z);
    bmasdq[0] = s_c * alpha1 * s_z;
    bmasdq[mu] = 0;
    bmasdq[mv] = -s_c * alpha1;
    bpasdq[0] = s_c * alpha2 * s_z;
    bpasdq[mu] = 0;
    bpasdq[mv] = s_c * alpha2;
}

__device__ void damping_src2(int mbc, int mx, int my, int meqn, double q[], double xlower, double ylower, double dx,
                             double dy, double time, double dt, int maux, double aux[], int i, int j)
{
    q[0] = q[0] - dt * s_rate * q[0];
}

FC2D_B200_USER_SOLVER(acoustics_register_inline, rpn2acoustics, rpt2acoustics, nullptr, damping_src2, 3, 2, 0, 16)

// the cudaclaw way: device pointers to the functions, copied out with cudaMemcpyFromSymbol
FC2D_B200_USER_SOLVER_FNPTR(acoustics_register_fnptr, 3, 2, 0, 16)
__device__ fc2d_b200_cuda_rpn2_t acoustics_rpn2_ptr = rpn2acoustics;
__device__ fc2d_b200_cuda_rpt2_t acoustics_rpt2_ptr = rpt2acoustics;
__device__ fc2d_b200_cuda_src2_t acoustics_src2_ptr = damping_src2;

extern "C" int acoustics_register_by_pointer(fc2d_b200_solver_t* s)
{
    fc2d_b200_cuda_rpn2_t rpn2;
    fc2d_b200_cuda_rpt2_t rpt2;
    fc2d_b200_cuda_src2_t src2;
    if (cudaMemcpyFromSymbol(&rpn2, acoustics_rpn2_ptr, sizeof(rpn2)) != cudaSuccess) return FC2D_B200_ECUDA;
    if (cudaMemcpyFromSymbol(&rpt2, acoustics_rpt2_ptr, sizeof(rpt2)) != cudaSuccess) return FC2D_B200_ECUDA;
    if (cudaMemcpyFromSymbol(&src2, acoustics_src2_ptr, sizeof(src2)) != cudaSuccess) return FC2D_B200_ECUDA;
    return acoustics_register_fnptr(s, rpn2, rpt2, nullptr, src2);
}
