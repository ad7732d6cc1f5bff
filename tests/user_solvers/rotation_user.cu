// An application's own scalar advection pair and b4step2, registered through
// include/fc2d_b200_user.cuh: the swirl app's GPU Riemann solvers
// (applications/cudaclaw/advection/2d/swirl/user_cuda/rpn2adv.cu:5-27,
// rpt2adv.cu:4-22, restated) and a b4step2 in the form of its user_cuda/b4step2.cu:22-45
// with a quadratic stream function psi = omega ((x-1/2)^2 + (y-1/2)^2)/2 and the
// time factor vt = 1 - (t + dt/2)/2 (solid-body rotation slowing down).
#include "fc2d_b200_user.cuh"

__constant__ double s_omega;

extern "C" int rotation_set_params(double omega)
{
    return cudaMemcpyToSymbol(s_omega, &omega, sizeof(double)) == cudaSuccess ? 0 : -1;
}

__device__ void rpn2adv(int idir, int meqn, int mwaves, int maux, double ql[], double qr[], double auxl[],
                        double auxr[], double wave[], double s[], double amdq[], double apdq[])
{
    for (int m = 0; m < meqn; m++) wave[m] = qr[m] - ql[m];
    s[0] = auxr[idir];
    for (int m = 0; m < meqn; m++) {
        amdq[m] = (s[0] < 0 ? s[0] : 0) * wave[m];
        apdq[m] = (s[0] > 0 ? s[0] : 0) * wave[m];
    }
}

__device__ void rpt2adv(int idir, int meqn, int mwaves, int maux, double ql[], double qr[], double aux1[],
                        double aux2[], double aux3[], int imp, double asdq[], double bmasdq[], double bpasdq[])
{
    const int kv = 1 - idir;
    for (int m = 0; m < meqn; m++) {
        const double sm = aux2[imp * maux + kv], sp = aux3[imp * maux + kv];
        bmasdq[m] = (sm < 0 ? sm : 0) * asdq[m];
        bpasdq[m] = (sp > 0 ? sp : 0) * asdq[m];
    }
}

__device__ double rot_psi(double x, double y) { return s_omega * ((x - 0.5) * (x - 0.5) + (y - 0.5) * (y - 0.5)) / 2.0; }

__device__ void rotation_b4step2(int mbc, int mx, int my, int meqn, double q[], double xlower, double ylower,
                                 double dx, double dy, double time, double dt, int maux, double aux[], int i, int j)
{
    const double xll = xlower + (i - 1) * dx, yll = ylower + (j - 1) * dy;
    const double vt = 1.0 - (time + dt / 2.0) / 2.0;
    const double p1 = rot_psi(xll, yll + dy), p2 = rot_psi(xll, yll), p3 = rot_psi(xll + dx, yll);
    aux[0] = (p1 - p2) / dy;
    aux[1] = -(p3 - p2) / dx;
    aux[0] = aux[0] * vt;
    aux[1] = aux[1] * vt;
}

FC2D_B200_USER_SOLVER(rotation_register_inline, rpn2adv, rpt2adv, rotation_b4step2, nullptr, 1, 1, 2, 16)
