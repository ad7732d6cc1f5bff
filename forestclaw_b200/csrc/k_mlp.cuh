// k_mlp.cuh -- the p*-seed network of the exact Euler solver (device side).
//
// A 6 -> 64 -> 64 -> 1 perceptron with tanh hidden layers predicts the
// correction y = log(p* / p_pvrs) of the PVRS estimate for one interface from the
// normalised primitive states
//   x = (rhoL/rbar, uL/cbar, pL/pbar, rhoR/rbar, uR/cbar, pR/pbar),
//   rbar = (rhoL + rhoR)/2, pbar = (pL + pR)/2, cbar = sqrt(pbar/rbar),
// and the Newton iteration starts from p0 = p_pvrs exp(y) where the wave strength
// |dp|/pbar + |du|/cbar exceeds MLP_GATE (p_pvrs is floored at 1e-3 pbar).  Weights are BF16, the
// two hidden layers run on the tensor cores (mma.sync m16n8k16, BF16 inputs,
// FP32 accumulation), one warp evaluating 32 interfaces at a time; the output
// layer is an FP32 dot product.
//
// Parameter vector (FP32 master copy, MLP_NPARAM floats):
//   W1[64][6] | b1[64] | W2[64][64] | b2[64] | w3[64] | b3
// Device blob used by the kernels (MLP_BLOB_BYTES):
//   floats b1[64] b2[64] w3[64] b3 (padded to 256 floats) | bf16 W1[64][16]
//   (input columns 6..15 zero) | bf16 W2[64][64]
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include "fcb_common.h"

namespace fcb {


struct MlpView {
    const float* f;          // b1, b2, w3, b3
    const uint32_t* w1;      // bf16 pairs, [64][8] words (16 columns)
    const uint32_t* w2;      // bf16 pairs, [64][32] words
    __device__ explicit MlpView(const void* blob)
        : f(reinterpret_cast<const float*>(blob)),
          w1(reinterpret_cast<const uint32_t*>(reinterpret_cast<const char*>(blob) + MLP_BLOB_W1_BYTE)),
          w2(reinterpret_cast<const uint32_t*>(reinterpret_cast<const char*>(blob) + MLP_BLOB_W2_BYTE)) {}
};

// Normalised features of one interface (primitive states) and the base pressure
// the network corrects: the PVRS estimate, floored at 1e-3 pbar.
__device__ __forceinline__ void mlp_features(double rl, double ul, double pl, double rr, double ur, double pr,
                                             double gam, float x[MLP_IN], double& pbase)
{
    const double rb = 0.5 * (rl + rr);
    const double pbar = 0.5 * (pl + pr);
    const double cb = sqrt(pbar / rb);
    x[0] = (float)(rl / rb); x[1] = (float)(ul / cb); x[2] = (float)(pl / pbar);
    x[3] = (float)(rr / rb); x[4] = (float)(ur / cb); x[5] = (float)(pr / pbar);
    const double al = sqrt(gam * pl / rl), ar = sqrt(gam * pr / rr);
    const double ppv = pbar - 0.125 * (ur - ul) * (rl + rr) * (al + ar);
    pbase = ppv > 1e-3 * pbar ? ppv : 1e-3 * pbar;
}

// Wave strength |dp|/pbar + |du|/cbar of the normalised features.
__device__ __forceinline__ bool mlp_gate(const float x[MLP_IN])
{
    return fabsf(x[5] - x[2]) + fabsf(x[4] - x[1]) > (float)MLP_GATE;
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi)
{
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ void mma_bf16_16816(float d[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                               uint32_t b0, uint32_t b1)
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};\n"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

template <bool APPROX>
__device__ __forceinline__ float mlp_act(float z)
{
    if constexpr (APPROX) {
        float r;
        asm("tanh.approx.f32 %0, %1;" : "=f"(r) : "f"(z));
        return r;
    } else {
        return tanhf(z);
    }
}

// Hidden activations of the 32 rows of one warp, in mma C-fragment layout:
// h[mt][nt][c]: row 16 mt + g (+8 for c = 2, 3), column 8 nt + 2 t + (c & 1),
// g = lane / 4, t = lane % 4.
struct MlpFrag { float h[2][8][4]; };

__device__ __forceinline__ float mlp_pick(const float v[MLP_IN], int c) { return c < MLP_IN ? v[c] : 0.0f; }

// Layer 1 and 2 of the warp's 32 rows (row r = lane r's x).  h1 and h2 receive the
// activations; the caller needs all 32 lanes converged.
template <bool APPROX>
__device__ __forceinline__ void mlp_warp_hidden(const MlpView& W, const float x[MLP_IN], MlpFrag& h1, MlpFrag& h2)
{
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    // ---- layer 1: A rows from the lanes that own them (columns 2t, 2t+1; 6..15 zero)
    uint32_t a1[2][2];
    for (int mt = 0; mt < 2; mt++)
        for (int half = 0; half < 2; half++) {
            const int src = 16 * mt + g + 8 * half;
            float v[MLP_IN];
            for (int c = 0; c < MLP_IN; c++) v[c] = __shfl_sync(0xffffffffu, x[c], src);
            a1[mt][half] = pack_bf16(mlp_pick(v, 2 * t), mlp_pick(v, 2 * t + 1));
        }
    for (int nt = 0; nt < 8; nt++) {
        const uint32_t b0 = __ldg(&W.w1[(8 * nt + g) * 8 + t]);
        const float bb0 = __ldg(&W.f[MLP_BLOB_F_B1 + 8 * nt + 2 * t]), bb1 = __ldg(&W.f[MLP_BLOB_F_B1 + 8 * nt + 2 * t + 1]);
        for (int mt = 0; mt < 2; mt++) {
            float d[4] = {bb0, bb1, bb0, bb1};
            mma_bf16_16816(d, a1[mt][0], a1[mt][1], 0u, 0u, b0, 0u);
            for (int c = 0; c < 4; c++) h1.h[mt][nt][c] = mlp_act<APPROX>(d[c]);
        }
    }
    // ---- layer 2: the C fragments of layer 1 are the A fragments of layer 2
    uint32_t a2[2][4][4];
    for (int mt = 0; mt < 2; mt++)
        for (int kk = 0; kk < 4; kk++) {
            a2[mt][kk][0] = pack_bf16(h1.h[mt][2 * kk][0], h1.h[mt][2 * kk][1]);
            a2[mt][kk][1] = pack_bf16(h1.h[mt][2 * kk][2], h1.h[mt][2 * kk][3]);
            a2[mt][kk][2] = pack_bf16(h1.h[mt][2 * kk + 1][0], h1.h[mt][2 * kk + 1][1]);
            a2[mt][kk][3] = pack_bf16(h1.h[mt][2 * kk + 1][2], h1.h[mt][2 * kk + 1][3]);
        }
    for (int nt = 0; nt < 8; nt++) {
        const float bb0 = __ldg(&W.f[MLP_BLOB_F_B2 + 8 * nt + 2 * t]), bb1 = __ldg(&W.f[MLP_BLOB_F_B2 + 8 * nt + 2 * t + 1]);
        float d[2][4] = {{bb0, bb1, bb0, bb1}, {bb0, bb1, bb0, bb1}};
        for (int kk = 0; kk < 4; kk++) {
            const uint32_t b0 = __ldg(&W.w2[(8 * nt + g) * 32 + 8 * kk + t]);
            const uint32_t b1 = __ldg(&W.w2[(8 * nt + g) * 32 + 8 * kk + 4 + t]);
            for (int mt = 0; mt < 2; mt++) mma_bf16_16816(d[mt], a2[mt][kk][0], a2[mt][kk][1], a2[mt][kk][2], a2[mt][kk][3], b0, b1);
        }
        for (int mt = 0; mt < 2; mt++)
            for (int c = 0; c < 4; c++) h2.h[mt][nt][c] = mlp_act<APPROX>(d[mt][c]);
    }
}

// Output layer: y of the lane's own row.
__device__ __forceinline__ float mlp_warp_output(const MlpView& W, const MlpFrag& h2)
{
    const int lane = threadIdx.x & 31, t = lane & 3;
    float ys[2][2];
    for (int mt = 0; mt < 2; mt++) {
        float lo = 0.0f, hi = 0.0f;
        for (int nt = 0; nt < 8; nt++) {
            const float w0 = __ldg(&W.f[MLP_BLOB_F_W3 + 8 * nt + 2 * t]), w1 = __ldg(&W.f[MLP_BLOB_F_W3 + 8 * nt + 2 * t + 1]);
            lo = lo + w0 * h2.h[mt][nt][0] + w1 * h2.h[mt][nt][1];
            hi = hi + w0 * h2.h[mt][nt][2] + w1 * h2.h[mt][nt][3];
        }
        lo += __shfl_xor_sync(0xffffffffu, lo, 1);
        lo += __shfl_xor_sync(0xffffffffu, lo, 2);
        hi += __shfl_xor_sync(0xffffffffu, hi, 1);
        hi += __shfl_xor_sync(0xffffffffu, hi, 2);
        ys[mt][0] = lo; ys[mt][1] = hi;
    }
    const int mt = lane >> 4, rr = lane & 15, src = (rr & 7) * 4, half = rr >> 3;
    const float s00 = __shfl_sync(0xffffffffu, ys[0][0], src), s01 = __shfl_sync(0xffffffffu, ys[0][1], src);
    const float s10 = __shfl_sync(0xffffffffu, ys[1][0], src), s11 = __shfl_sync(0xffffffffu, ys[1][1], src);
    const float y = mt == 0 ? (half ? s01 : s00) : (half ? s11 : s10);
    return y + __ldg(&W.f[MLP_BLOB_F_B3]);
}

}  // namespace fcb
