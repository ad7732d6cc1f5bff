// k_mlp.cu -- training and evaluation kernels of the p*-seed network.
//
// Training data: primitive interface states (rhoL, uL, pL, rhoR, uR, pR) in the
// normal frame, sampled from a forest (k_sample_interfaces).  Targets are the
// exact star pressures (Newton from the PVRS start, tolerance set by the
// caller) as y = log(p*/pbar).  The loss is the mean squared error of y.
//
// One training step over a minibatch of nb rows:
//   k_mlp_fwdbwd  : 128 rows per CTA (4 warps x 32 rows); forward on the tensor
//                   cores (mlp_warp_hidden, BF16 inputs, FP32 accumulation,
//                   accurate tanh), backward in FP32 with the activations of the
//                   forward (the BF16 rounding of the forward is passed straight
//                   through); each CTA writes its partial gradient
//   k_mlp_reduce  : sums the partial gradients in CTA order (deterministic)
//   k_mlp_adam    : Adam on the FP32 master parameters, then the BF16 blob
#include <cuda_runtime.h>
#include <stdint.h>
#include "k_mlp.cuh"
#include "k_tc.cuh"
#include "kernels.h"
#include "riemann.cuh"

namespace fcb {

enum { FB_ROWS = 128, FB_THREADS = 128 };
constexpr size_t FB_SMEM = sizeof(float) * ((size_t)FB_ROWS * MLP_IN + 3 * (size_t)FB_ROWS * (MLP_H + 1) + FB_ROWS + 4);

// ---- parameter vector -> device blob ------------------------------------------
__global__ void k_mlp_blob(const float* __restrict__ prm, void* __restrict__ blob)
{
    float* f = reinterpret_cast<float*>(blob);
    __nv_bfloat16* w1 = reinterpret_cast<__nv_bfloat16*>(reinterpret_cast<char*>(blob) + MLP_BLOB_W1_BYTE);
    __nv_bfloat16* w2 = reinterpret_cast<__nv_bfloat16*>(reinterpret_cast<char*>(blob) + MLP_BLOB_W2_BYTE);
    for (int k = threadIdx.x; k < 256; k += blockDim.x) {
        float v = 0.0f;
        if (k < 64) v = prm[MLP_OFF_B1 + k];
        else if (k < 128) v = prm[MLP_OFF_B2 + k - 64];
        else if (k < 192) v = prm[MLP_OFF_W3 + k - 128];
        else if (k == 192) v = prm[MLP_OFF_B3];
        f[k] = v;
    }
    for (int k = threadIdx.x; k < 64 * 16; k += blockDim.x) {
        const int n = k / 16, c = k % 16;
        w1[k] = __float2bfloat16_rn(c < MLP_IN ? prm[MLP_OFF_W1 + n * MLP_IN + c] : 0.0f);
    }
    for (int k = threadIdx.x; k < 64 * 64; k += blockDim.x) w2[k] = __float2bfloat16_rn(prm[MLP_OFF_W2 + k]);
    // the tcgen05 operand copies: W1 (kchunks 2) then W2 (kchunks 8)
    char* tc = reinterpret_cast<char*>(blob) + MLP_BLOB_TC_BYTE;
    for (int k = threadIdx.x; k < 64 * 16; k += blockDim.x) {
        const int n = k / 16, c = k % 16;
        *reinterpret_cast<__nv_bfloat16*>(tc + kmajor_off(n, c, 2)) =
            __float2bfloat16_rn(c < MLP_IN ? prm[MLP_OFF_W1 + n * MLP_IN + c] : 0.0f);
    }
    for (int k = threadIdx.x; k < 64 * 64; k += blockDim.x)
        *reinterpret_cast<__nv_bfloat16*>(tc + 64 * 16 * 2 + kmajor_off(k / 64, k % 64, 8)) =
            __float2bfloat16_rn(prm[MLP_OFF_W2 + k]);
}

// ---- targets: exact star pressure of every sample ------------------------------
__global__ void k_mlp_targets(const double* __restrict__ prim, int n, double gam, double tol, float* __restrict__ X,
                              float* __restrict__ Y, int* __restrict__ iters)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const double* w = prim + (size_t)k * 6;
    float x[MLP_IN];
    double pbase;
    mlp_features(w[0], w[1], w[2], w[3], w[4], w[5], gam, x, pbase);
    int it = 0;
    const double ps = RPEulerExact::pstar(w[0], w[1], w[2], w[3], w[4], w[5], gam, tol, 0.0, it);
    for (int c = 0; c < MLP_IN; c++) X[(size_t)k * MLP_IN + c] = x[c];
    Y[k] = (float)log(ps / pbase);
    if (iters) iters[k] = it & 0xff;
}

// The training forward of one tile of FB_ROWS rows (row = threadIdx.x holds x) on the
// tcgen05 tensor cores: H1 and H2 (accurate tanh, FP32) to sH1 / sH2, the output y of the
// row returned.  ops: 30 KB of shared memory for the operands (16-byte aligned).
__device__ float mlp_tc_forward(const MlpView& W, const float x[MLP_IN], int row, char* ops,
                                float (*sH1)[MLP_H + 1], float (*sH2)[MLP_H + 1], unsigned* status)
{
    __shared__ unsigned long long s_bar;
    __shared__ uint32_t s_tmem;
    constexpr int NCOL = 128;
    const int tid = threadIdx.x, warp = tid >> 5;
    char* b1 = ops;                        // 64 x 16 bf16 (kchunks 2)
    char* b2 = b1 + 2048;                  // 64 x 64 (kchunks 8)
    char* a1 = b2 + 8192;                  // 128 x 16
    char* a2 = a1 + 4096;                  // 128 x 64
    if (warp == 0) tc_alloc(&s_tmem, NCOL);
    if (tid == 0) tc_bar_init(&s_bar);
    for (int k = 0; k < 16; k++)
        *reinterpret_cast<uint16_t*>(a1 + kmajor_off(row, k, 2)) = bf16_bits(k < MLP_IN ? x[k] : 0.0f);
    {   // W1 | W2 in core-matrix order, 16 bytes per load
        const uint4* src = reinterpret_cast<const uint4*>(reinterpret_cast<const char*>(W.f) + MLP_BLOB_TC_BYTE);
        uint4* dst = reinterpret_cast<uint4*>(b1);
        for (int e = tid; e < MLP_BLOB_TC_LEN / 16; e += FB_THREADS) dst[e] = src[e];
    }
    tc_publish();
    const uint32_t tm = s_tmem, lanes = tm + ((uint32_t)(warp * 32) << 16);
    if (tid == 0) {
        tc_mma(tm, smem_desc(a1, 256), smem_desc(b1, 256), tc_idesc(FB_ROWS, 64), 0);
        tc_commit(&s_bar);
    }
    bool ok = __syncthreads_and(tc_wait(&s_bar, 0));
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    float y = 0.0f;
    if (ok) {
        for (int c0 = 0; c0 < 64; c0 += 16) {
            float v[16];
            tc_ld16(lanes + c0, v);
            for (int k = 0; k < 16; k++) {
                const float h = mlp_act<false>(v[k] + W.f[MLP_BLOB_F_B1 + c0 + k]);
                sH1[row][c0 + k] = h;
                *reinterpret_cast<uint16_t*>(a2 + kmajor_off(row, c0 + k, 8)) = bf16_bits(h);
            }
        }
        tc_publish();
        if (tid == 0) {
            for (int kk = 0; kk < 4; kk++)
                tc_mma(tm + 64, smem_desc(a2 + kk * 256, 1024), smem_desc(b2 + kk * 256, 1024), tc_idesc(FB_ROWS, 64),
                       kk > 0);
            tc_commit(&s_bar);
        }
        ok = __syncthreads_and(tc_wait(&s_bar, 1));
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    }
    if (ok) {
        for (int c0 = 0; c0 < 64; c0 += 16) {
            float v[16];
            tc_ld16(lanes + 64 + c0, v);
            for (int k = 0; k < 16; k++) {
                const float h = mlp_act<false>(v[k] + W.f[MLP_BLOB_F_B2 + c0 + k]);
                sH2[row][c0 + k] = h;
                y = y + W.f[MLP_BLOB_F_W3 + c0 + k] * h;
            }
        }
        y = y + W.f[MLP_BLOB_F_B3];
    } else {
        if (tid == 0 && status) atomicOr(status, (unsigned)STATUS_TENSOR);
        (void)tc_wait(&s_bar, 0);
        (void)tc_wait(&s_bar, 1);
        for (int c = 0; c < MLP_H; c++) { sH1[row][c] = 0.0f; sH2[row][c] = 0.0f; }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) tc_dealloc(tm, NCOL);
    return y;
}

// ---- forward + backward of one minibatch ---------------------------------------
// The forward of the CTA's 128 rows runs on the tcgen05 tensor cores (the tiles of
// k_mlp_tc.cu, with the training's accurate tanh): the BF16 operands sit in the dZ
// area of shared memory, which the backward uses only afterwards, and the FP32
// accumulators in 128 TMEM columns.  A commit that does not arrive sets STATUS_TENSOR.
// The backward is FP32 on the CUDA cores.
__global__ void __launch_bounds__(FB_THREADS)
k_mlp_fwdbwd(const float* __restrict__ X, const float* __restrict__ Y, const int* __restrict__ idx, int nb,
             const void* __restrict__ blob, const float* __restrict__ prm, float* __restrict__ partial,
             float* __restrict__ loss_partial, unsigned* __restrict__ status)
{
    extern __shared__ float fb_smem[];
    float (*sX)[MLP_IN] = reinterpret_cast<float (*)[MLP_IN]>(fb_smem);
    float (*sH1)[MLP_H + 1] = reinterpret_cast<float (*)[MLP_H + 1]>(fb_smem + FB_ROWS * MLP_IN);
    float (*sH2)[MLP_H + 1] = sH1 + FB_ROWS;
    float (*sD)[MLP_H + 1] = sH2 + FB_ROWS;       // dZ2, then dZ1
    float* sdy = reinterpret_cast<float*>(sD + FB_ROWS);
    float* sred = sdy + FB_ROWS;
    const MlpView W(blob);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int row = warp * 32 + lane;                 // row of this CTA
    const int r = blockIdx.x * FB_ROWS + row;         // row of the minibatch
    const bool valid = r < nb;
    float x[MLP_IN];
    float t = 0.0f;
    if (valid) {
        const int s = idx ? idx[r] : r;
        for (int c = 0; c < MLP_IN; c++) x[c] = X[(size_t)s * MLP_IN + c];
        t = Y[s];
    } else {
        x[0] = 1.0f; x[1] = 0.0f; x[2] = 1.0f; x[3] = 1.0f; x[4] = 0.0f; x[5] = 1.0f;
    }
    for (int c = 0; c < MLP_IN; c++) sX[row][c] = valid ? x[c] : 0.0f;
    const float y = mlp_tc_forward(W, x, row, reinterpret_cast<char*>(sD), sH1, sH2, status);
    const float e = valid ? (y - t) : 0.0f;
    sdy[row] = 2.0f * e / (float)nb;
    // loss partial (sum of e^2 / nb over the CTA)
    {
        float l = e * e / (float)nb;
        for (int off = 16; off > 0; off >>= 1) l += __shfl_xor_sync(0xffffffffu, l, off);
        if (lane == 0) sred[warp] = l;
    }
    __syncthreads();
    float* gp = partial + (size_t)blockIdx.x * MLP_NPARAM;
    if (tid == 0) loss_partial[blockIdx.x] = sred[0] + sred[1] + sred[2] + sred[3];
    // dZ2[r][i] = dy[r] w3[i] (1 - H2^2)
    for (int k = tid; k < FB_ROWS * MLP_H; k += FB_THREADS) {
        const int rr = k / MLP_H, i = k % MLP_H;
        const float h = sH2[rr][i];
        sD[rr][i] = sdy[rr] * prm[MLP_OFF_W3 + i] * (1.0f - h * h);
    }
    // output layer gradients
    if (tid < MLP_H) {
        float s = 0.0f;
        for (int rr = 0; rr < FB_ROWS; rr++) s += sdy[rr] * sH2[rr][tid];
        gp[MLP_OFF_W3 + tid] = s;
    } else if (tid == MLP_H) {
        float s = 0.0f;
        for (int rr = 0; rr < FB_ROWS; rr++) s += sdy[rr];
        gp[MLP_OFF_B3] = s;
    }
    __syncthreads();
    // dW2[i][j] = sum_r dZ2[r][i] H1[r][j], db2[i] = sum_r dZ2[r][i]
    for (int k = tid; k < MLP_H * MLP_H; k += FB_THREADS) {
        const int i = k / MLP_H, j = k % MLP_H;
        float s = 0.0f;
        for (int rr = 0; rr < FB_ROWS; rr++) s += sD[rr][i] * sH1[rr][j];
        gp[MLP_OFF_W2 + k] = s;
    }
    if (tid < MLP_H) {
        float s = 0.0f;
        for (int rr = 0; rr < FB_ROWS; rr++) s += sD[rr][tid];
        gp[MLP_OFF_B2 + tid] = s;
    }
    // dZ1[r][j] = (sum_i dZ2[r][i] W2[i][j]) (1 - H1^2), in registers, then back to sD
    float dz1[FB_ROWS * MLP_H / FB_THREADS];
    for (int q = 0; q < FB_ROWS * MLP_H / FB_THREADS; q++) {
        const int k = tid + q * FB_THREADS, rr = k / MLP_H, j = k % MLP_H;
        float s = 0.0f;
        for (int i = 0; i < MLP_H; i++) s += sD[rr][i] * prm[MLP_OFF_W2 + i * MLP_H + j];
        const float h = sH1[rr][j];
        dz1[q] = s * (1.0f - h * h);
    }
    __syncthreads();
    for (int q = 0; q < FB_ROWS * MLP_H / FB_THREADS; q++) {
        const int k = tid + q * FB_THREADS;
        sD[k / MLP_H][k % MLP_H] = dz1[q];
    }
    __syncthreads();
    // dW1[j][c] = sum_r dZ1[r][j] x[r][c], db1[j] = sum_r dZ1[r][j]
    for (int k = tid; k < MLP_H * MLP_IN; k += FB_THREADS) {
        const int j = k / MLP_IN, c = k % MLP_IN;
        float s = 0.0f;
        for (int rr = 0; rr < FB_ROWS; rr++) s += sD[rr][j] * sX[rr][c];
        gp[MLP_OFF_W1 + k] = s;
    }
    if (tid < MLP_H) {
        float s = 0.0f;
        for (int rr = 0; rr < FB_ROWS; rr++) s += sD[rr][tid];
        gp[MLP_OFF_B1 + tid] = s;
    }
}

__global__ void k_mlp_reduce(const float* __restrict__ partial, const float* __restrict__ loss_partial, int nblk,
                             float* __restrict__ grad, float* __restrict__ loss)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < MLP_NPARAM) {
        float s = 0.0f;
        for (int b = 0; b < nblk; b++) s += partial[(size_t)b * MLP_NPARAM + k];
        grad[k] = s;
    }
    if (k == 0 && loss) {
        float s = 0.0f;
        for (int b = 0; b < nblk; b++) s += loss_partial[b];
        *loss = s;
    }
}

__global__ void k_mlp_adam(float* __restrict__ prm, const float* __restrict__ grad, float* __restrict__ m,
                           float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= MLP_NPARAM) return;
    const float gk = grad[k];
    const float mk = b1 * m[k] + (1.0f - b1) * gk;
    const float vk = b2 * v[k] + (1.0f - b2) * gk * gk;
    m[k] = mk;
    v[k] = vk;
    prm[k] = prm[k] - lr * (mk / c1) / (sqrtf(vk / c2) + eps);
}

// ---- evaluation: the deployed forward (approximate tanh, as in the solver) -------
__global__ void k_mlp_predict(const float* __restrict__ X, int n, const void* __restrict__ blob, float* __restrict__ Y)
{
    const MlpView W(blob);
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = r < n;
    float x[MLP_IN];
    for (int c = 0; c < MLP_IN; c++) x[c] = valid ? X[(size_t)r * MLP_IN + c] : (c == 1 || c == 4 ? 0.0f : 1.0f);
    MlpFrag h1, h2;
    mlp_warp_hidden<true>(W, x, h1, h2);
    const float y = mlp_warp_output(W, h2);
    if (valid) Y[r] = y;
}

// Newton iterations from the PVRS start (Yseed null) or from the network's start on
// the gated interfaces.
__global__ void k_mlp_newton_iters(const double* __restrict__ prim, const float* __restrict__ X,
                                   const float* __restrict__ Yseed, int n, double gam, double tol, int* __restrict__ iters)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const double* w = prim + (size_t)k * 6;
    double seed = 0.0;
    if (Yseed) {
        float x[MLP_IN];
        double pbase;
        mlp_features(w[0], w[1], w[2], w[3], w[4], w[5], gam, x, pbase);
        if (mlp_gate(x)) seed = pbase * fcb_exp((double)Yseed[k]);
    }
    int it = 0;
    RPEulerExact::pstar(w[0], w[1], w[2], w[3], w[4], w[5], gam, tol, seed, it);
    iters[k] = it & 0xff;
}

// ---- uniform sample of the normal-direction interfaces of a forest ---------------
__device__ __forceinline__ unsigned long long splitmix64(unsigned long long z)
{
    z += 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

__global__ void k_sample_interfaces(const double* __restrict__ q, int np, int mx, int my, int mbc, double gam,
                                    unsigned long long seed, int n, double* __restrict__ prim)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int nx = mx + 2 * mbc, ny = my + 2 * mbc, nxy = nx * ny;
    const int nfx = (mx + 1) * my, nfy = mx * (my + 1);
    const unsigned long long h1 = splitmix64(seed ^ (0x632be59bd9b4e019ULL * (unsigned long long)(k + 1)));
    const unsigned long long h2 = splitmix64(h1);
    const int p = (int)(h1 % (unsigned long long)np);
    const int f = (int)(h2 % (unsigned long long)(nfx + nfy));
    int cl, cr, ixy;
    if (f < nfx) {   // x-face between cells (i-1, j) and (i, j), i = 1..mx+1
        const int i = 1 + f % (mx + 1), j = 1 + f / (mx + 1);
        cl = (j + mbc - 1) * nx + (i - 1 + mbc - 1);
        cr = (j + mbc - 1) * nx + (i + mbc - 1);
        ixy = 1;
    } else {
        const int f2 = f - nfx;
        const int i = 1 + f2 % mx, j = 1 + f2 / mx;
        cl = (j - 1 + mbc - 1) * nx + (i + mbc - 1);
        cr = (j + mbc - 1) * nx + (i + mbc - 1);
        ixy = 2;
    }
    const double* qp = q + (size_t)p * 4 * nxy;
    double qL[4], qR[4];
    for (int m = 0; m < 4; m++) { qL[m] = qp[m * nxy + cl]; qR[m] = qp[m * nxy + cr]; }
    const RPEulerExact::Prim P = RPEulerExact::prim(ixy, qL, qR, gam);
    double* o = prim + (size_t)k * 6;
    o[0] = P.rl; o[1] = P.ul; o[2] = P.pl; o[3] = P.rr; o[4] = P.ur; o[5] = P.pr;
}

// ---- launch wrappers ---------------------------------------------------------------
static inline int nblk(int n, int b) { return (n + b - 1) / b; }

cudaError_t mlp_setup()
{
    return cudaFuncSetAttribute(k_mlp_fwdbwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)FB_SMEM);
}
void launch_mlp_blob(const float* prm, void* blob, cudaStream_t st) { k_mlp_blob<<<1, 256, 0, st>>>(prm, blob); }
void launch_mlp_targets(const double* prim, int n, double gam, double tol, float* X, float* Y, int* iters,
                        cudaStream_t st)
{
    if (n > 0) k_mlp_targets<<<nblk(n, 128), 128, 0, st>>>(prim, n, gam, tol, X, Y, iters);
}
int mlp_fwdbwd_blocks(int nb) { return nblk(nb, FB_ROWS); }
void launch_mlp_step(const float* X, const float* Y, const int* idx, int nb, void* blob, float* prm, float* grad,
                     float* m, float* v, float* partial, float* loss_partial, float* loss, float lr, int step,
                     bool update, unsigned* status, cudaStream_t st)
{
    const int nb_blk = nblk(nb, FB_ROWS);
    k_mlp_fwdbwd<<<nb_blk, FB_THREADS, FB_SMEM, st>>>(X, Y, idx, nb, blob, prm, partial, loss_partial, status);
    k_mlp_reduce<<<nblk(MLP_NPARAM, 256), 256, 0, st>>>(partial, loss_partial, nb_blk, grad, loss);
    if (!update) return;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
    k_mlp_adam<<<nblk(MLP_NPARAM, 256), 256, 0, st>>>(prm, grad, m, v, lr, b1, b2, 1e-8f, c1, c2);
    k_mlp_blob<<<1, 256, 0, st>>>(prm, blob);
}
void launch_mlp_predict(const float* X, int n, const void* blob, float* Y, cudaStream_t st)
{
    if (n > 0) k_mlp_predict<<<nblk(n, 128), 128, 0, st>>>(X, n, blob, Y);
}
void launch_mlp_newton_iters(const double* prim, const float* X, const float* Yseed, int n, double gam, double tol,
                             int* iters, cudaStream_t st)
{
    if (n > 0) k_mlp_newton_iters<<<nblk(n, 128), 128, 0, st>>>(prim, X, Yseed, n, gam, tol, iters);
}
void launch_sample_interfaces(const Dims& d, const double* q, int np, double gam, unsigned long long seed, int n,
                              double* prim, cudaStream_t st)
{
    if (n > 0 && np > 0)
        k_sample_interfaces<<<nblk(n, 128), 128, 0, st>>>(q, np, d.mx, d.my, d.mbc, gam, seed, n, prim);
}

}  // namespace fcb
