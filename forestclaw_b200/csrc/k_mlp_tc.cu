// k_mlp_tc.cu -- batched evaluation of the p*-seed network on the 5th-generation
// tensor cores (tcgen05): one CTA of 128 threads per tile of 128 interface states.
//
// Layer 1 (128 x 16 states, 6 input columns and 10 zero columns, times W1^T) and
// layer 2 (128 x 64 activations times W2^T, four K = 16 steps) are tcgen05.mma of
// kind f16 with BF16 operands in shared memory and FP32 accumulators in tensor memory
// (TMEM: columns 0..63 layer 1, 64..127 layer 2); one thread issues the MMAs and
// commits them to an mbarrier, every warp reads its 32 rows back with tcgen05.ld
// (warp w owns TMEM lanes 32 w .. 32 w + 31), adds the bias and applies tanh.approx;
// the output layer is an FP32 dot product per row.  This is the deployed forward of
// k_mlp.cuh (the same BF16 weights and activations); the FP32 sums run in the tensor
// core's order, so results agree with the per-warp mma.sync form to FP32 rounding.
//
// Operands are K-major without swizzle: 8 x 8 BF16 core matrices of 128 contiguous
// bytes (8 rows of 16 bytes), the K-neighbour core matrix 128 bytes on (leading byte
// offset) and the next 8 rows kchunks * 128 bytes on (stride byte offset).
//
// Every wait is bounded: a commit that does not arrive sets STATUS_TENSOR in the
// status word, the CTA waits (bounded) for its MMA once more, frees its TMEM and
// returns without writing the rest of its results.
#include <cuda_bf16.h>
#include "kernels.h"
#include "k_mlp.cuh"
#include "k_tc.cuh"

namespace fcb {

namespace {

constexpr int TC_ROWS = 128;                 // states per tile (MMA M)
constexpr int TC_COLS = 128;                 // TMEM columns: layer 1 at 0, layer 2 at 64
// dynamic shared memory per CTA: the operands need 30 KB; asking for 56 KB keeps at
// most four CTAs on an SM, so the 4 x 128 TMEM columns they allocate always fit
constexpr int TC_SMEM = 56 * 1024;

struct TcSmem {
    uint16_t b1[64 * 16];                    // W1 [n][k]             (kchunks 2)
    uint16_t b2[64 * 64];                    // W2 [n][k]             (kchunks 8), right after W1
    uint16_t a1[TC_ROWS * 16];               // states, bf16          (kchunks 2)
    uint16_t a2[TC_ROWS * 64];               // layer-1 activations   (kchunks 8)
    float bias[256];                         // b1, b2, w3, b3
    unsigned long long bar;                  // MMA completion
    uint32_t tmem;                           // TMEM base written by tcgen05.alloc
};

}  // namespace

// A grid of resident CTAs (at most four per SM) loops over the tiles: the weights are
// staged once per CTA, then per tile the states, layer 1, the activations, layer 2 and
// the output; the mbarrier's phase flips with each commit.
__global__ void __launch_bounds__(TC_ROWS)
k_mlp_predict_tc(const float* __restrict__ X, int n, const void* __restrict__ blob, float* __restrict__ Y,
                 unsigned* __restrict__ status)
{
    extern __shared__ __align__(1024) unsigned char tc_raw[];
    TcSmem& S = *reinterpret_cast<TcSmem*>(tc_raw);
    const int tid = threadIdx.x, warp = tid >> 5;
    if (warp == 0) {                                           // TMEM for the CTA, allocated by one warp
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&S.tmem)),
                     "r"(TC_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&S.bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // ---- the weights and biases, once ----
    const float* bf = reinterpret_cast<const float*>(blob);
    char* a1 = reinterpret_cast<char*>(S.a1);
    char* a2 = reinterpret_cast<char*>(S.a2);
    char* b1 = reinterpret_cast<char*>(S.b1);
    char* b2 = reinterpret_cast<char*>(S.b2);
    {   // W1 | W2 in core-matrix order (the blob's tensor-core copy), 16 bytes per load
        const uint4* src = reinterpret_cast<const uint4*>(reinterpret_cast<const char*>(blob) + MLP_BLOB_TC_BYTE);
        uint4* dst = reinterpret_cast<uint4*>(b1);
        for (int e = tid; e < MLP_BLOB_TC_LEN / 16; e += TC_ROWS) dst[e] = src[e];
    }
    for (int e = tid; e < 256; e += TC_ROWS) S.bias[e] = bf[e];
    tc_publish();
    const uint32_t tm = S.tmem;
    const uint32_t lanes = tm + ((uint32_t)(warp * 32) << 16);  // this warp's TMEM lanes
    const int ntiles = (n + TC_ROWS - 1) / TC_ROWS;
    unsigned phase = 0;
    bool ok = true;
    for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const int r = tile * TC_ROWS + tid;
        const bool valid = r < n;
        for (int k = 0; k < 16; k++) {
            // rows past the end hold a neutral state (unit densities and pressures, no velocity)
            const float x = k >= MLP_IN ? 0.0f : (valid ? X[(size_t)r * MLP_IN + k] : (k == 1 || k == 4 ? 0.0f : 1.0f));
            *reinterpret_cast<uint16_t*>(a1 + kmajor_off(tid, k, 2)) = bf16_bits(x);
        }
        tc_publish();
        // ---- layer 1: D[0..63] = A1 W1^T (M 128, N 64, K 16) ----
        if (tid == 0) {
            tc_mma(tm, smem_desc(a1, 256), smem_desc(b1, 256), tc_idesc(TC_ROWS, 64), 0);
            tc_commit(&S.bar);
        }
        ok = __syncthreads_and(tc_wait(&S.bar, phase));
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (!ok) break;
        for (int c0 = 0; c0 < 64; c0 += 16) {
            float v[16];
            tc_ld16(lanes + c0, v);
            for (int k = 0; k < 16; k++)
                *reinterpret_cast<uint16_t*>(a2 + kmajor_off(tid, c0 + k, 8)) =
                    bf16_bits(tanh_approx(v[k] + S.bias[MLP_BLOB_F_B1 + c0 + k]));
        }
        tc_publish();
        // ---- layer 2: D[64..127] = A2 W2^T (M 128, N 64, K 64 in four steps of 16) ----
        if (tid == 0) {
            for (int kk = 0; kk < 4; kk++)
                tc_mma(tm + 64, smem_desc(a2 + kk * 256, 1024), smem_desc(b2 + kk * 256, 1024), tc_idesc(TC_ROWS, 64),
                       kk > 0);
            tc_commit(&S.bar);
        }
        ok = __syncthreads_and(tc_wait(&S.bar, phase));
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (!ok) break;
        // ---- output layer: FP32 dot product of the row with w3 ----
        float y = 0.0f;
        for (int c0 = 0; c0 < 64; c0 += 16) {
            float v[16];
            tc_ld16(lanes + 64 + c0, v);
            for (int k = 0; k < 16; k++)
                y = y + S.bias[MLP_BLOB_F_W3 + c0 + k] * tanh_approx(v[k] + S.bias[MLP_BLOB_F_B2 + c0 + k]);
        }
        if (valid) Y[r] = y + S.bias[MLP_BLOB_F_B3];
        // the tile's TMEM reads and shared-memory operands are done before the next tile
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
    }
    if (!ok) {
        // a commit that did not arrive: report it and give the MMA in flight one more
        // bounded wait before the TMEM is freed
        if (tid == 0 && status) atomicOr(status, (unsigned)STATUS_TENSOR);
        (void)tc_wait(&S.bar, phase ^ 1u);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tm), "r"(TC_COLS) : "memory");
}

cudaError_t mlp_tc_setup()
{
    return cudaFuncSetAttribute(k_mlp_predict_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM);
}

void launch_mlp_predict_tc(const float* X, int n, const void* blob, float* Y, unsigned* status, cudaStream_t st)
{
    static_assert(sizeof(TcSmem) <= (size_t)TC_SMEM, "operands fit the dynamic shared memory");
    if (n <= 0) return;
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int ntiles = (n + TC_ROWS - 1) / TC_ROWS, grid = ntiles < 4 * sms ? ntiles : 4 * sms;
    k_mlp_predict_tc<<<grid, TC_ROWS, TC_SMEM, st>>>(X, n, blob, Y, status);
}

}  // namespace fcb
