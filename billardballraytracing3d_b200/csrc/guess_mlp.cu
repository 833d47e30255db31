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

#include "guess.h"
#include "umma.cuh"

namespace bbrt {

using namespace umma;

constexpr long long kMbarLimit = kMbarDefault;   // the self-check's bound (about 2 s of SM cycles)

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

// ---- the network -------------------------------------------------------------

__device__ __forceinline__ float gelu_f(float z) {
    return 0.5f * z * (1.0f + tanhf(kGeluC * (z + kGeluA * z * z * z)));
}
__device__ __forceinline__ float gelu_grad_f(float z) {
    const float th = tanhf(kGeluC * (z + kGeluA * z * z * z));
    return 0.5f * (1.0f + th) + 0.5f * z * (1.0f - th * th) * kGeluC * (1.0f + 3.0f * kGeluA * z * z);
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
}

// Sum over the 32 lanes of a warp (every lane gets the total).
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// 16 values of one row as BF16 into a core-blocked tile with C columns.
__device__ __forceinline__ void put_row16(uint8_t* tile, int row, int c0, int C, const float* v) {
    uint32_t p[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) p[j] = pack_bf16(v[2 * j], v[2 * j + 1]);
    *reinterpret_cast<uint4*>(tile + tile_off(row, c0, C)) = make_uint4(p[0], p[1], p[2], p[3]);
    *reinterpret_cast<uint4*>(tile + tile_off(row, c0 + 8, C)) = make_uint4(p[4], p[5], p[6], p[7]);
}

// Hidden-layer epilogue: row `row` of Z (TMEM columns zc..zc+127) plus bias,
// GELU, to BF16 in tile `out` (128 columns).
__device__ __forceinline__ void ep_gelu(uint32_t lane_base, int zc, const float* bias, uint8_t* out, int row) {
    for (int c = 0; c < 8; ++c) {
        float z[16];
        tmem_ld16(lane_base + zc + c * 16, z);
#pragma unroll
        for (int j = 0; j < 16; ++j) z[j] = gelu_f(z[j] + bias[c * 16 + j]);
        put_row16(out, row, c * 16, kH, z);
    }
}

// One stage boundary: operands written and fenced by every thread, TMEM reads
// done; thread 0 issues the MMAs of `issue` and commits; everyone waits, at
// most `limit` SM cycles.  Returns false (uniformly) when the wait timed out;
// a thread whose wait gave up waits once more, with the default bound, so
// that the MMAs already issued have finished with their operands and their
// accumulator before the caller leaves and frees tensor memory.
template <class Issue>
__device__ __forceinline__ bool mma_stage(uint32_t mbar, uint32_t& phase, long long limit, Issue&& issue) {
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    if (threadIdx.x == 0) {
        issue();
        commit(mbar);
    }
    const bool w = mbar_wait(mbar, phase, limit);
    if (!w) mbar_wait(mbar, phase, kMbarDefault);
    phase ^= 1u;
    const bool ok = __syncthreads_and(w) != 0;
    fence_after_sync();
    return ok;
}

// Adds dW (TMEM lane = output o, columns = inputs i, N columns) of this tile
// to G at [i][o] (rows of 128 outputs: coalesced across the warp).
__device__ __forceinline__ void ep_dw_oi(uint32_t lane_base, int col, int N, float* G, int row) {
    for (int c = 0; c < N / 16; ++c) {
        float g[16];
        tmem_ld16(lane_base + col + c * 16, g);
#pragma unroll
        for (int j = 0; j < 16; ++j) atomicAdd(G + (c * 16 + j) * kH + row, g[j]);
    }
}

// Backward hidden epilogue: dZ = dH (TMEM dhc) * gelu'(Z (TMEM zc) + bias),
// to BF16 in tile `out`; bias gradients summed over the warp's rows.
__device__ __forceinline__ void ep_dgelu(uint32_t lane_base, int dhc, int zc, const float* bias, uint8_t* out,
                                         int row, float* gb) {
    const int lane = threadIdx.x & 31;
    for (int c = 0; c < 8; ++c) {
        float dh[16], z[16];
        tmem_ld16(lane_base + dhc + c * 16, dh);
        tmem_ld16(lane_base + zc + c * 16, z);
#pragma unroll
        for (int j = 0; j < 16; ++j) dh[j] *= gelu_grad_f(z[j] + bias[c * 16 + j]);
        put_row16(out, row, c * 16, kH, dh);
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const float s = warp_sum(dh[j]);
            if (lane == j) atomicAdd(gb + c * 16 + j, s);
        }
    }
}

// Loads the BF16 weight image and the biases into shared memory.
__device__ __forceinline__ void load_weights(uint8_t* sm, const uint8_t* image, const float* P, int bias_off) {
    for (int k = threadIdx.x; k < kImageBytes / 16; k += blockDim.x)
        reinterpret_cast<uint4*>(sm)[k] = reinterpret_cast<const uint4*>(image)[k];
    float* sb = reinterpret_cast<float*>(sm + bias_off);
    for (int k = threadIdx.x; k < 3 * kH + kOut; k += blockDim.x)
        sb[k] = k < kH ? P[oB0 + k] : k < 2 * kH ? P[oB1 + k - kH] : k < 3 * kH ? P[oB2 + k - 2 * kH] : P[oB3 + k - 3 * kH];
}

// Input row (9 geometric features, the patch embedding, zero padding) to BF16.
__device__ __forceinline__ void put_input_row(uint8_t* tile, int row, const float* geo, const float* emb) {
    for (int c = 0; c < kIn / 16; ++c) {
        float v[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const int col = c * 16 + j;
            v[j] = col < kGeo ? geo[col] : (col < kGeo + kEmb && emb) ? emb[col - kGeo] : 0.0f;
        }
        put_row16(tile, row, c * 16, kIn, v);
    }
}

// Forward + backward of one batch; gradients added to G (W0..W2 as [i][o],
// W3 as [o][i], biases and embeddings as in P), loss added to *loss.
// TMEM: Z1 columns 0-127, Z2 128-255, Z3 256-383, scratch 384-511.
__global__ void __launch_bounds__(128, 1) k_mlp_train(MlpBatch Bt, MlpNet M) {
    extern __shared__ __align__(1024) uint8_t sm[];
    __shared__ __align__(8) uint64_t mbar_s;
    __shared__ uint32_t tslot;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    load_weights(sm, M.image, M.P, kTrainBias);
    const float* sb = reinterpret_cast<const float*>(sm + kTrainBias);
    uint8_t* tX = sm + kTrainX;
    uint8_t* tH1 = sm + kTrainH1;
    uint8_t* tH2 = sm + kTrainH2;
    uint8_t* tH3 = sm + kTrainH3;
    uint8_t* tG4 = sm + kTrainG4;
    const uint32_t aW0 = smem_u32(sm + iW0), aW1 = smem_u32(sm + iW1), aW2 = smem_u32(sm + iW2),
                   aW3 = smem_u32(sm + iW3);
    const uint32_t aX = smem_u32(tX), aH1 = smem_u32(tH1), aH2 = smem_u32(tH2), aH3 = smem_u32(tH3),
                   aG4 = smem_u32(tG4);
    if (warp == 0) tmem_alloc(smem_u32(&tslot), 512);
    if (tid == 0) mbar_init(smem_u32(&mbar_s), 1);
    fence_async_smem();
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tm = tslot, mbar = smem_u32(&mbar_s);
    const uint32_t lb = tm + (static_cast<uint32_t>(warp * 32) << 16);
    uint32_t phase = 0;
    bool ok = true;
    constexpr uint32_t ID_F = idesc_bf16(128, 128, false, false);
    constexpr uint32_t ID_F16 = idesc_bf16(128, 16, false, false);
    const int n_tiles = (Bt.B + 127) / 128;
    float* G = M.G;
    for (int tile = blockIdx.x; tile < n_tiles && ok; tile += gridDim.x) {
        const int r = tile * 128 + tid;
        const bool valid = r < Bt.B;
        const int s = valid ? (Bt.idx ? Bt.idx[r] : r) : 0;
        const int patch = valid ? Bt.pid[s] : 0;
        {
            float geo[kGeo];
#pragma unroll
            for (int k = 0; k < kGeo; ++k) geo[k] = valid ? Bt.feat[static_cast<long long>(s) * kGeo + k] : 0.0f;
            put_input_row(tX, tid, geo, valid ? M.P + oE + static_cast<long long>(patch) * kEmb : nullptr);
        }
        fence_async_smem();
        // ---- forward
        ok = mma_stage(mbar, phase, M.mbar_limit, [&] {
            for (int k = 0; k < kIn / 16; ++k) mma(tm, kmajor_desc(aX, kIn, k), kmajor_desc(aW0, kIn, k), ID_F, k > 0);
        });
        if (!ok) break;
        ep_gelu(lb, 0, sb, tH1, tid);
        fence_async_smem();
        ok = mma_stage(mbar, phase, M.mbar_limit, [&] {
            for (int k = 0; k < kH / 16; ++k) mma(tm + 128, kmajor_desc(aH1, kH, k), kmajor_desc(aW1, kH, k), ID_F, k > 0);
        });
        if (!ok) break;
        ep_gelu(lb, 128, sb + kH, tH2, tid);
        fence_async_smem();
        ok = mma_stage(mbar, phase, M.mbar_limit, [&] {
            for (int k = 0; k < kH / 16; ++k) mma(tm + 256, kmajor_desc(aH2, kH, k), kmajor_desc(aW2, kH, k), ID_F, k > 0);
        });
        if (!ok) break;
        ep_gelu(lb, 256, sb + 2 * kH, tH3, tid);
        fence_async_smem();
        ok = mma_stage(mbar, phase, M.mbar_limit, [&] {
            for (int k = 0; k < kH / 16; ++k) mma(tm + 384, kmajor_desc(aH3, kH, k), kmajor_desc(aW3, kH, k), ID_F16, k > 0);
        });
        if (!ok) break;
        // ---- outputs, loss and dZ4
        {
            float z[16];
            tmem_ld16(lb + 384, z);
            const float* b3 = sb + 3 * kH;
            const float u = z[0] + b3[0], v = z[1] + b3[1], sv = z[2] + b3[2], lg = z[3] + b3[3];
            float d[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) d[j] = 0.0f;
            float loss = 0.0f;
            if (valid) {
                const float y = Bt.lbl[s];
                const float* tg = Bt.tgt + static_cast<long long>(s) * 3;
                const float e0 = u - tg[0], e1 = v - tg[1], e2 = sv - tg[2];
                loss = y * (e0 * e0 + e1 * e1 + e2 * e2) + fmaxf(lg, 0.0f) - lg * y + log1pf(expf(-fabsf(lg)));
                loss *= Bt.inv_b;
                d[0] = 2.0f * y * e0 * Bt.inv_b;
                d[1] = 2.0f * y * e1 * Bt.inv_b;
                d[2] = 2.0f * y * e2 * Bt.inv_b;
                d[3] = (1.0f / (1.0f + expf(-lg)) - y) * Bt.inv_b;
                if (M.out) {
                    float* o = M.out + static_cast<long long>(r) * 4;
                    o[0] = u; o[1] = v; o[2] = sv; o[3] = lg;
                }
            }
            const float ls = warp_sum(loss);
            if (lane == 0) atomicAdd(M.loss, ls);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const float sj = warp_sum(d[j]);
                if (lane == j) atomicAdd(G + oB3 + j, sj);
            }
            put_row16(tG4, tid, 0, kOut, d);
        }
        fence_async_smem();
        // ---- backward, layer 3: dW3 = dZ4^T H3 (as [i][o] in TMEM, stored [o][i]), dH3 = dZ4 W3
        ok = mma_stage(mbar, phase, M.mbar_limit, [&] {
            for (int k = 0; k < 8; ++k)
                mma(tm + 384, mnmajor_desc(aH3, kH, k), mnmajor_desc(aG4, kOut, k), idesc_bf16(128, 16, true, true), k > 0);
        });
        if (!ok) break;
        {
            float g[16];
            tmem_ld16(lb + 384, g);
#pragma unroll
            for (int j = 0; j < 4; ++j) atomicAdd(G + oW3 + j * kH + tid, g[j]);
        }
        ok = mma_stage(mbar, phase, M.mbar_limit, [&] {
            mma(tm + 384, kmajor_desc(aG4, kOut, 0), mnmajor_desc(aW3, kH, 0), idesc_bf16(128, 128, false, true), false);
        });
        if (!ok) break;
        ep_dgelu(lb, 384, 256, sb + 2 * kH, tH3, tid, G + oB2);   // dZ3 over H3
        fence_async_smem();
        // ---- layer 2
        ok = mma_stage(mbar, phase, M.mbar_limit, [&] {
            for (int k = 0; k < 8; ++k)
                mma(tm + 384, mnmajor_desc(aH3, kH, k), mnmajor_desc(aH2, kH, k), idesc_bf16(128, 128, true, true), k > 0);
        });
        if (!ok) break;
        ep_dw_oi(lb, 384, kH, G + oW2, tid);
        ok = mma_stage(mbar, phase, M.mbar_limit, [&] {
            for (int k = 0; k < 8; ++k)
                mma(tm + 384, kmajor_desc(aH3, kH, k), mnmajor_desc(aW2, kH, k), idesc_bf16(128, 128, false, true), k > 0);
        });
        if (!ok) break;
        ep_dgelu(lb, 384, 128, sb + kH, tH2, tid, G + oB1);        // dZ2 over H2
        fence_async_smem();
        // ---- layer 1
        ok = mma_stage(mbar, phase, M.mbar_limit, [&] {
            for (int k = 0; k < 8; ++k)
                mma(tm + 384, mnmajor_desc(aH2, kH, k), mnmajor_desc(aH1, kH, k), idesc_bf16(128, 128, true, true), k > 0);
        });
        if (!ok) break;
        ep_dw_oi(lb, 384, kH, G + oW1, tid);
        ok = mma_stage(mbar, phase, M.mbar_limit, [&] {
            for (int k = 0; k < 8; ++k)
                mma(tm + 384, kmajor_desc(aH2, kH, k), mnmajor_desc(aW1, kH, k), idesc_bf16(128, 128, false, true), k > 0);
        });
        if (!ok) break;
        ep_dgelu(lb, 384, 0, sb, tH1, tid, G + oB0);                // dZ1 over H1
        fence_async_smem();
        // ---- layer 0: dW0 = dZ1^T X, dX = dZ1 W0 (embedding gradients)
        ok = mma_stage(mbar, phase, M.mbar_limit, [&] {
            for (int k = 0; k < 8; ++k)
                mma(tm + 384, mnmajor_desc(aH1, kH, k), mnmajor_desc(aX, kIn, k), idesc_bf16(128, 64, true, true), k > 0);
        });
        if (!ok) break;
        ep_dw_oi(lb, 384, kIn, G + oW0, tid);
        ok = mma_stage(mbar, phase, M.mbar_limit, [&] {
            for (int k = 0; k < 8; ++k)
                mma(tm + 384, kmajor_desc(aH1, kH, k), mnmajor_desc(aW0, kIn, k), idesc_bf16(128, 64, false, true), k > 0);
        });
        if (!ok) break;
        {
            float* ge = G + oE + static_cast<long long>(patch) * kEmb;
            for (int c = 0; c < kIn / 16; ++c) {
                float g[16];
                tmem_ld16(lb + 384 + c * 16, g);
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int col = c * 16 + j;
                    if (valid && col >= kGeo && col < kGeo + kEmb) atomicAdd(ge + col - kGeo, g[j]);
                }
            }
        }
    }
    if (!ok && tid == 0) atomicOr(M.err, 1);
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    if (warp == 0) tmem_free(tm, 512);
}

// Inference: guesses for the rows of a batch.  Rows come from `Rows` (a
// functor giving the 9 geometric features, the patch and the row's t offset
// and scale); outputs (u, v, t, logit) per row.
// TMEM: one 128-column accumulator reused by every layer.
template <class Rows>
__global__ void __launch_bounds__(128, 1) k_mlp_infer(Rows rows, long long n, const unsigned int* n_dev, MlpNet M,
                                                     double* __restrict__ out) {
    extern __shared__ __align__(1024) uint8_t sm[];
    __shared__ __align__(8) uint64_t mbar_s;
    __shared__ uint32_t tslot;
    // Graph launch: the row count is on the device; blocks without a tile
    // leave before loading weights or taking TMEM (uniform over the block).
    if (n_dev) n = *n_dev;
    if (blockIdx.x >= (n + 127) / 128) return;
    const int tid = threadIdx.x, warp = tid >> 5;
    load_weights(sm, M.image, M.P, kInferBias);
    const float* sb = reinterpret_cast<const float*>(sm + kInferBias);
    uint8_t* tX = sm + kInferX;
    uint8_t* tH = sm + kInferH;
    const uint32_t aW0 = smem_u32(sm + iW0), aW1 = smem_u32(sm + iW1), aW2 = smem_u32(sm + iW2),
                   aW3 = smem_u32(sm + iW3), aX = smem_u32(tX), aH = smem_u32(tH);
    if (warp == 0) tmem_alloc(smem_u32(&tslot), 128);
    if (tid == 0) mbar_init(smem_u32(&mbar_s), 1);
    fence_async_smem();
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tm = tslot, mbar = smem_u32(&mbar_s);
    const uint32_t lb = tm + (static_cast<uint32_t>(warp * 32) << 16);
    uint32_t phase = 0;
    bool ok = true;
    constexpr uint32_t ID_F = idesc_bf16(128, 128, false, false);
    const long long n_tiles = (n + 127) / 128;
    for (long long tile = blockIdx.x; tile < n_tiles && ok; tile += gridDim.x) {
        const long long r = tile * 128 + tid;
        const bool valid = r < n;
        float geo[kGeo];
        int patch = 0;
        double t0 = 0.0, scale = 0.0;
        if (valid) rows(r, geo, patch, t0, scale);
        else
            for (int k = 0; k < kGeo; ++k) geo[k] = 0.0f;
        put_input_row(tX, tid, geo, valid ? M.P + oE + static_cast<long long>(patch) * kEmb : nullptr);
        fence_async_smem();
        ok = mma_stage(mbar, phase, M.mbar_limit, [&] {
            for (int k = 0; k < kIn / 16; ++k) mma(tm, kmajor_desc(aX, kIn, k), kmajor_desc(aW0, kIn, k), ID_F, k > 0);
        });
        if (!ok) break;
        ep_gelu(lb, 0, sb, tH, tid);
        fence_async_smem();
        ok = mma_stage(mbar, phase, M.mbar_limit, [&] {
            for (int k = 0; k < kH / 16; ++k) mma(tm, kmajor_desc(aH, kH, k), kmajor_desc(aW1, kH, k), ID_F, k > 0);
        });
        if (!ok) break;
        ep_gelu(lb, 0, sb + kH, tH, tid);
        fence_async_smem();
        ok = mma_stage(mbar, phase, M.mbar_limit, [&] {
            for (int k = 0; k < kH / 16; ++k) mma(tm, kmajor_desc(aH, kH, k), kmajor_desc(aW2, kH, k), ID_F, k > 0);
        });
        if (!ok) break;
        ep_gelu(lb, 0, sb + 2 * kH, tH, tid);
        fence_async_smem();
        ok = mma_stage(mbar, phase, M.mbar_limit, [&] {
            for (int k = 0; k < kH / 16; ++k)
                mma(tm, kmajor_desc(aH, kH, k), kmajor_desc(aW3, kH, k), idesc_bf16(128, 16, false, false), k > 0);
        });
        if (!ok) break;
        float z[16];
        tmem_ld16(lb, z);
        if (valid) {
            const float* b3 = sb + 3 * kH;
            double* o = out + r * 4;
            o[0] = static_cast<double>(z[0] + b3[0]);
            o[1] = static_cast<double>(z[1] + b3[1]);
            o[2] = t0 + static_cast<double>(z[2] + b3[2]) * scale;
            o[3] = static_cast<double>(z[3] + b3[3]);
        }
    }
    if (!ok && tid == 0) atomicOr(M.err, 1);
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    if (warp == 0) tmem_free(tm, 128);
}

// Rows given directly as features (the check entry point): t offset 0, scale 1.
struct FeatureRows {
    const float* feat;
    const int* pid;
    __device__ void operator()(long long r, float* geo, int& patch, double& t0, double& scale) const {
        for (int k = 0; k < kGeo; ++k) geo[k] = feat[r * kGeo + k];
        patch = pid[r];
        t0 = 0.0;
        scale = 1.0;
    }
};

// Rows from the trace's Newton requests: the request's ray in its patch's frame.
struct RequestRows {
    const NewtonRequest* req;
    const double* o;
    const double* d;
    const int* obj_sub;
    const double* frame;
    __device__ void operator()(long long r, float* geo, int& patch, double& t0, double& scale) const {
        const NewtonRequest q = req[r];
        patch = obj_sub[q.obj];
        const double* f = frame + static_cast<long long>(patch) * kFrame;
        const double ox = o[3LL * q.ray], oy = o[3LL * q.ray + 1], oz = o[3LL * q.ray + 2];
        const double dx = d[3LL * q.ray], dy = d[3LL * q.ray + 1], dz = d[3LL * q.ray + 2];
        ray_features(f, ox, oy, oz, dx, dy, dz, geo, t0);
        scale = f[12];
    }
};

// FP32 master -> BF16 weight image in core-blocked order.
__global__ void k_pack_weights(const float* __restrict__ P, uint8_t* __restrict__ image) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < kH * kIn) {
        const int o = k / kIn, i = k % kIn;
        *reinterpret_cast<__nv_bfloat16*>(image + iW0 + tile_off(o, i, kIn)) = __float2bfloat16_rn(P[oW0 + k]);
    }
    if (k < kH * kH) {
        const int o = k / kH, i = k % kH;
        *reinterpret_cast<__nv_bfloat16*>(image + iW1 + tile_off(o, i, kH)) = __float2bfloat16_rn(P[oW1 + k]);
        *reinterpret_cast<__nv_bfloat16*>(image + iW2 + tile_off(o, i, kH)) = __float2bfloat16_rn(P[oW2 + k]);
    }
    if (k < kOut * kH) {
        const int o = k / kH, i = k % kH;
        *reinterpret_cast<__nv_bfloat16*>(image + iW3 + tile_off(o, i, kH)) = __float2bfloat16_rn(P[oW3 + k]);
    }
}

// One Adam step on every parameter (bias-corrected), gradients cleared after use.
__global__ void k_adam(float* __restrict__ P, float* __restrict__ G, float* __restrict__ m1, float* __restrict__ m2,
                       long long n, float lr, float b1, float b2, float eps, float c1, float c2) {
    const long long p = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (p >= n) return;
    const long long gi = grad_index(p);
    const float g = G[gi];
    const float a = b1 * m1[p] + (1.0f - b1) * g;
    const float b = b2 * m2[p] + (1.0f - b2) * g * g;
    m1[p] = a;
    m2[p] = b;
    P[p] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
}

// Training rows from recorded samples: features, targets (u, v, s) and label.
__global__ void k_make_rows(const GuessSample* __restrict__ S, long long n, const double* __restrict__ frame,
                            float* __restrict__ feat, int* __restrict__ pid, float* __restrict__ tgt,
                            float* __restrict__ lbl) {
    const long long k = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (k >= n) return;
    const GuessSample s = S[k];
    const double* f = frame + static_cast<long long>(s.patch) * kFrame;
    float geo[kGeo];
    double t0;
    ray_features(f, s.o[0], s.o[1], s.o[2], s.d[0], s.d[1], s.d[2], geo, t0);
    for (int j = 0; j < kGeo; ++j) feat[k * kGeo + j] = geo[j];
    pid[k] = s.patch;
    tgt[3 * k] = static_cast<float>(s.u);
    tgt[3 * k + 1] = static_cast<float>(s.v);
    tgt[3 * k + 2] = static_cast<float>((s.t - t0) / f[12]);
    lbl[k] = s.label ? 1.0f : 0.0f;
}

// ---- launchers ----------------------------------------------------------------

static int sm_count_cached() {
    static int n = 0;
    if (n == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 1;
    }
    return n;
}

cudaError_t mlp_pack(const float* P, uint8_t* image, cudaStream_t st) {
    k_pack_weights<<<(kH * kH + 255) / 256, 256, 0, st>>>(P, image);
    return cudaGetLastError();
}

cudaError_t mlp_train_batch(const MlpBatch& Bt, const MlpNet& M, cudaStream_t st) {
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, kTrainSmem);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    const int tiles = (Bt.B + 127) / 128;
    const int grid = tiles < sm_count_cached() ? tiles : sm_count_cached();
    if (grid <= 0) return cudaSuccess;
    k_mlp_train<<<grid, 128, kTrainSmem, st>>>(Bt, M);
    return cudaGetLastError();
}

cudaError_t mlp_adam(const MlpNet& M, float* m1, float* m2, long long n, float lr, int step, cudaStream_t st) {
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - powf(b1, static_cast<float>(step)), c2 = 1.0f - powf(b2, static_cast<float>(step));
    k_adam<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(M.P, M.G, m1, m2, n, lr, b1, b2, 1e-8f, c1, c2);
    return cudaGetLastError();
}

template <class Rows>
static cudaError_t infer(const Rows& rows, long long n, const MlpNet& M, double* out, cudaStream_t st,
                         const unsigned int* n_dev = nullptr) {
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k_mlp_infer<Rows>, cudaFuncAttributeMaxDynamicSharedMemorySize, kInferSmem);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    const long long tiles = (n + 127) / 128;
    const long long grid = tiles < sm_count_cached() ? tiles : sm_count_cached();
    if (grid <= 0) return cudaSuccess;
    k_mlp_infer<Rows><<<static_cast<unsigned>(grid), 128, kInferSmem, st>>>(rows, n, n_dev, M, out);
    return cudaGetLastError();
}

cudaError_t mlp_infer_features(const float* feat, const int* pid, long long n, const MlpNet& M, double* out,
                               cudaStream_t st) {
    return infer(FeatureRows{ feat, pid }, n, M, out, st);
}

cudaError_t mlp_infer_requests(const NewtonRequest* req, long long n, const double* o, const double* d,
                               const int* obj_sub, const double* frame, const MlpNet& M, double* out,
                               cudaStream_t st, const unsigned int* n_dev) {
    return infer(RequestRows{ req, o, d, obj_sub, frame }, n, M, out, st, n_dev);
}

cudaError_t mlp_make_rows(const GuessSample* S, long long n, const double* frame, float* feat, int* pid, float* tgt,
                          float* lbl, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    k_make_rows<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(S, n, frame, feat, pid, tgt, lbl);
    return cudaGetLastError();
}

}  // namespace bbrt
