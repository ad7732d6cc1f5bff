// pin_harness.cu -- runs the reference's own CUDA patch update on host-supplied
// patches, so the CPU oracle's clawpack 4.6 update can be checked against code
// of the reference executed on a GPU.  Test infrastructure only (the checker of
// the oracle); nothing in the product links it.
//
// Built by oracle/Makefile (target ref) together with two files compiled from
// the reference tree where they lie:
//   src/solvers/fc2d_cudaclaw/cuda_source/cudaclaw_flux2.cu     update kernel
//       cudaclaw_flux2_and_update_batch (one CTA of 128 threads per patch,
//       blockIdx.z = patch; normal solves, wave limiting, second-order
//       corrections, transverse propagation, final update of the interior),
//       method constants set by cudaclaw_set_method_parameters (:46-53)
//   src/solvers/fc2d_cudaclaw/cuda_source/cudaclaw_limiters.cu  cudaclaw_limiter
// The launch follows cudaclaw_step2_batch (cudaclaw_step2.cu:178-209): block of
// FC2D_CUDACLAW_BLOCK_SIZE threads, grid (1, 1, patches), dynamic shared memory
// mwork * block doubles with mwork = max(4 meqn + 2 maux + mwaves + meqn mwaves,
// 5 meqn + 6 maux); per-patch scratch as cudaclaw_allocate_fluxes
// (cudaclaw_allocate.cu:44-90), speeds zeroed.
//
// The Riemann solvers are the reference's own cudaclaw app solvers
// (ref_app_solvers.cu): swirl advection and radialdam Roe shallow water.
#include <cuda_runtime.h>
#include <cstring>
#include <vector>
#include "fc2d_cudaclaw_cuda.h"
#include "cudaclaw_allocate.h"

__global__ void cudaclaw_flux2_and_update_batch(const int mx, const int my, const int meqn, const int mbc,
                                                const int maux, const int mwaves, const int mwork, const double dt,
                                                const double t, struct cudaclaw_fluxes* array_fluxes_struct_dev,
                                                double* maxcflblocks, cudaclaw_cuda_rpn2_t rpn2,
                                                cudaclaw_cuda_rpt2_t rpt2, cudaclaw_cuda_b4step2_t b4step2);
extern "C" void cudaclaw_set_method_parameters(int* order_in, int* mthlim_in, int mwaves, int use_fwaves_in);
__device__ double cudaclaw_limiter(int lim_choice, double r);

extern "C" int pin_ref_solver(int id, double grav, double dry_tolerance, double sea_level,
                              cudaclaw_cuda_rpn2_t* rpn2, cudaclaw_cuda_rpt2_t* rpt2);

__global__ void pin_limiter_kernel(int lim, const double* r, double* phi, int n)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) phi[k] = cudaclaw_limiter(lim, r[k]);
}

#define PIN_CK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { err = e_; goto done; } } while (0)

extern "C" {

// One update of npatch patches with reference solver pair `solver`
// (pin_ref_solver): q[npatch][meqn][ny][nx] in/out (i fastest, mbc ghost cells),
// aux[npatch][maux][ny][nx], dx[p], dy[p], mthlim[mwaves], prm = (grav,
// dry_tolerance, sea_level); cfl[p] = what the kernel stores per block.
// Returns 0, -1 for a bad argument, or the CUDA error code.
int pin_cudaclaw_step(int solver, int mx, int my, int mbc, int meqn, int maux, int mwaves, int use_fwaves,
                      int npatch, const int* order, const int* mthlim, double dt, const double* dx, const double* dy,
                      const double* prm, double* q, const double* aux, double* cfl)
{
    if (mwaves < 1 || mwaves > FC2D_CUDACLAW_MWAVES || meqn < 1 || maux < 0 || npatch < 1 || mbc < 2) return -1;
    const size_t size = (size_t)(2 * mbc + mx) * (2 * mbc + my);
    cudaError_t err = cudaSuccess;
    std::vector<cudaclaw_fluxes_t> F(npatch);
    std::vector<void*> allocs;
    double *qd = nullptr, *ad = nullptr, *cd = nullptr;
    cudaclaw_fluxes_t* Fd = nullptr;
    cudaclaw_cuda_rpn2_t rpn2 = nullptr;
    cudaclaw_cuda_rpt2_t rpt2 = nullptr;
    int ord[2] = {order[0], order[1]};
    std::vector<int> lim(mthlim, mthlim + mwaves);
    const int mwork1 = 4 * meqn + 2 * maux + mwaves + meqn * mwaves, mwork2 = 5 * meqn + 6 * maux;
    const int mwork = mwork1 > mwork2 ? mwork1 : mwork2;
    const int block = FC2D_CUDACLAW_BLOCK_SIZE;
    if (pin_ref_solver(solver, prm[0], prm[1], prm[2], &rpn2, &rpt2) != 0) return -1;
    PIN_CK(cudaMalloc(&qd, sizeof(double) * npatch * meqn * size));
    PIN_CK(cudaMalloc(&ad, sizeof(double) * npatch * (maux > 0 ? maux : 1) * size));
    PIN_CK(cudaMalloc(&cd, sizeof(double) * npatch));
    PIN_CK(cudaMalloc(&Fd, sizeof(cudaclaw_fluxes_t) * npatch));
    PIN_CK(cudaMemcpy(qd, q, sizeof(double) * npatch * meqn * size, cudaMemcpyHostToDevice));
    if (maux > 0) PIN_CK(cudaMemcpy(ad, aux, sizeof(double) * npatch * maux * size, cudaMemcpyHostToDevice));
    for (int p = 0; p < npatch; p++) {
        cudaclaw_fluxes_t& f = F[p];
        std::memset(&f, 0, sizeof(f));
        f.num = meqn * size; f.num_aux = maux * size;
        f.num_waves = 2 * mwaves * meqn * size; f.num_speeds = 2 * mwaves * size;
        f.num_bytes = f.num * sizeof(double); f.num_bytes_aux = f.num_aux * sizeof(double);
        f.num_bytes_waves = f.num_waves * sizeof(double); f.num_bytes_speeds = f.num_speeds * sizeof(double);
        f.qold_dev = qd + (size_t)p * meqn * size;
        f.aux_dev = ad + (size_t)p * maux * size;
        double** bufs[8] = {&f.fp_dev, &f.fm_dev, &f.gp_dev, &f.gm_dev, &f.apdq_dev, &f.amdq_dev, &f.bpdq_dev, &f.bmdq_dev};
        for (double** b : bufs) { PIN_CK(cudaMalloc(b, f.num_bytes)); allocs.push_back(*b); PIN_CK(cudaMemset(*b, 0, f.num_bytes)); }
        PIN_CK(cudaMalloc(&f.waves_dev, f.num_bytes_waves)); allocs.push_back(f.waves_dev);
        PIN_CK(cudaMemset(f.waves_dev, 0, f.num_bytes_waves));
        PIN_CK(cudaMalloc(&f.speeds_dev, f.num_bytes_speeds)); allocs.push_back(f.speeds_dev);
        PIN_CK(cudaMemset(f.speeds_dev, 0, f.num_bytes_speeds));
        f.dx = dx[p]; f.dy = dy[p];
    }
    PIN_CK(cudaMemcpy(Fd, F.data(), sizeof(cudaclaw_fluxes_t) * npatch, cudaMemcpyHostToDevice));
    cudaclaw_set_method_parameters(ord, lim.data(), mwaves, use_fwaves);
    cudaclaw_flux2_and_update_batch<<<dim3(1, 1, npatch), dim3(block, 1, 1), sizeof(double) * mwork * block>>>(
        mx, my, meqn, mbc, maux, mwaves, mwork, dt, 0.0, Fd, cd, rpn2, rpt2, nullptr);
    PIN_CK(cudaGetLastError());
    PIN_CK(cudaDeviceSynchronize());
    PIN_CK(cudaMemcpy(q, qd, sizeof(double) * npatch * meqn * size, cudaMemcpyDeviceToHost));
    PIN_CK(cudaMemcpy(cfl, cd, sizeof(double) * npatch, cudaMemcpyDeviceToHost));
done:
    for (void* a : allocs) cudaFree(a);
    if (qd) cudaFree(qd);
    if (ad) cudaFree(ad);
    if (cd) cudaFree(cd);
    if (Fd) cudaFree(Fd);
    return (int)err;
}

// phi[k] = cudaclaw_limiter(lim, r[k])
int pin_cudaclaw_limiter(int lim, const double* r, double* phi, int n)
{
    cudaError_t err = cudaSuccess;
    double *rd = nullptr, *pd = nullptr;
    PIN_CK(cudaMalloc(&rd, sizeof(double) * n));
    PIN_CK(cudaMalloc(&pd, sizeof(double) * n));
    PIN_CK(cudaMemcpy(rd, r, sizeof(double) * n, cudaMemcpyHostToDevice));
    pin_limiter_kernel<<<(n + 127) / 128, 128>>>(lim, rd, pd, n);
    PIN_CK(cudaGetLastError());
    PIN_CK(cudaMemcpy(phi, pd, sizeof(double) * n, cudaMemcpyDeviceToHost));
done:
    if (rd) cudaFree(rd);
    if (pd) cudaFree(pd);
    return (int)err;
}

}  // extern "C"
