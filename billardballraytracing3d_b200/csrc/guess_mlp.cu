// The learned Newton initial guess: a small MLP on the tcgen05 tensor cores.
//
// Network (per (ray, patch) pair): 41 inputs -> 128 -> 128 -> 128 -> 4, GELU
// (tanh form) on the hidden layers, BF16 weights and activations, FP32
// accumulation in tensor memory.  Inputs: the ray in the patch's local frame
// (closest-approach point to the patch centre and direction, 6), the patch
// box extents (3) and a learned 32-wide embedding of the patch.  Outputs:
// Newton start (u, v), the ray parameter as an offset from the closest
// approach in units of the patch size, and a confidence logit.
//
// Every kernel here is one CTA of 128 threads per 128-row tile (persistent
// over tiles); one thread issues the MMAs, all four warps run the epilogue
// on their 32 TMEM lanes.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "umma.cuh"

namespace bbrt {

using namespace umma;

constexpr long long kMbarLimit = 1LL << 24;   // polls before a wait reports failure

// ---- self-check of the operand layouts -------------------------------------
//
// One CTA computes D = A * B^T (A 128 x 64, B 128 x 64, both given row-major
// with K contiguous) four times, with A and B each staged K-major or MN-major.
// All four results must equal the plain product.
__global__ void __launch_bounds__(128) k_umma_check(const uint16_t* __restrict__ A, const uint16_t* __restrict__ B,
                                                    float* __restrict__ D, int* __restrict__ err) {
    extern __shared__ __align__(1024) uint8_t sm[];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tslot;
    uint8_t* tAk = sm;            // rows m, cols k  (128 x 64)
    uint8_t* tAm = sm + 16384;    // rows k, cols m  (64 x 128)
    uint8_t* tBk = sm + 32768;    // rows n, cols k
    uint8_t* tBm = sm + 49152;    // rows k, cols n
    const int tid = threadIdx.x, warp = tid >> 5;
    for (int idx = tid; idx < 128 * 64; idx += 128) {
        const int r = idx >> 6, k = idx & 63;
        *reinterpret_cast<uint16_t*>(tAk + tile_off(r, k, 64)) = A[idx];
        *reinterpret_cast<uint16_t*>(tAm + tile_off(k, r, 128)) = A[idx];
        *reinterpret_cast<uint16_t*>(tBk + tile_off(r, k, 64)) = B[idx];
        *reinterpret_cast<uint16_t*>(tBm + tile_off(k, r, 128)) = B[idx];
    }
    fence_async_smem();
    if (warp == 0) tmem_alloc(smem_u32(&tslot), 128);
    if (tid == 0) mbar_init(smem_u32(&mbar), 1);
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = tslot;
    bool ok = true;
    for (int v = 0; v < 4 && ok; ++v) {
        const bool amn = v & 1, bmn = (v >> 1) & 1;
        if (tid == 0) {
            const uint32_t id = idesc_bf16(128, 128, amn, bmn);
            for (int k = 0; k < 4; ++k) {
                const uint64_t a = amn ? mnmajor_desc(smem_u32(tAm), 128, k) : kmajor_desc(smem_u32(tAk), 64, k);
                const uint64_t b = bmn ? mnmajor_desc(smem_u32(tBm), 128, k) : kmajor_desc(smem_u32(tBk), 64, k);
                mma(tmem, a, b, id, k > 0);
            }
            commit(smem_u32(&mbar));
        }
        ok = mbar_wait(smem_u32(&mbar), static_cast<uint32_t>(v & 1), kMbarLimit);
        fence_after_sync();
        if (!ok) {
            atomicOr(err, 1);
        } else {
            const int row = warp * 32 + (tid & 31);
            for (int c = 0; c < 8; ++c) {
                float x[16];
                tmem_ld16(tmem + (static_cast<uint32_t>(warp * 32) << 16) + c * 16, x);
                for (int j = 0; j < 16; ++j) D[(static_cast<long long>(v) * 128 + row) * 128 + c * 16 + j] = x[j];
            }
        }
        fence_before_sync();
        __syncthreads();
        fence_after_sync();
    }
    if (warp == 0) tmem_free(tmem, 128);
}

int launch_umma_check(const uint16_t* A, const uint16_t* B, float* D, int* err, cudaStream_t st) {
    const int smem = 65536;
    cudaError_t e = cudaFuncSetAttribute(k_umma_check, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return static_cast<int>(e);
    k_umma_check<<<1, 128, smem, st>>>(A, B, D, err);
    return static_cast<int>(cudaGetLastError());
}

}  // namespace bbrt
