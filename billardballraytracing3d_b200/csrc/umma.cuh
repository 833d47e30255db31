// Fifth-generation tensor core (tcgen05) building blocks for sm_100a:
// shared-memory matrix descriptors, the BF16 x BF16 -> FP32 MMA issued by one
// thread, its completion through an mbarrier, tensor-memory (TMEM)
// allocation and the TMEM -> register load of the accumulator.
//
// Operand tiles in shared memory use one layout, "core-blocked": a tile of
// R rows x C columns (C the contiguous dimension, 2-byte elements) is cut into
// 8 x 8 core matrices of 128 contiguous bytes (row r of a core at byte
// 16 * (r % 8), element c at 2 * (c % 8)); core (row group g, column group h)
// starts at byte (g * C / 8 + h) * 128.  Such a tile is a K-major operand when
// its columns run along K (rows = M or N), and an MN-major operand when its
// columns run along M or N (rows = K): the same bytes serve both, only the
// descriptor's two core strides swap roles.  No swizzling.
#pragma once

#include <cstdint>

namespace bbrt {
namespace umma {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Byte offset of element (r, c) in a core-blocked tile with C columns.
__host__ __device__ __forceinline__ uint32_t tile_off(int r, int c, int C) {
    return static_cast<uint32_t>((((r >> 3) * (C >> 3) + (c >> 3)) << 7) + ((r & 7) << 4) + ((c & 7) << 1));
}

// Shared-memory matrix descriptor (no swizzle): start address, leading and
// stride byte offsets (each >> 4), descriptor version 1.
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = static_cast<uint64_t>((addr >> 4) & 0x3FFFu);
    d |= static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16;
    d |= static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32;
    d |= static_cast<uint64_t>(1) << 46;
    return d;
}

// Descriptor of the k-th 16-wide K slice of a core-blocked tile with C columns.
//   K-major (columns along K): leading = next column group, stride = next row group.
//   MN-major (rows along K):   leading = next row group (K), stride = next column group (MN).
__device__ __forceinline__ uint64_t kmajor_desc(uint32_t tile, int C, int k) {
    const uint32_t rg = static_cast<uint32_t>(C >> 3) << 7;
    return sdesc(tile + static_cast<uint32_t>(k) * 256u, 128u, rg);
}
__device__ __forceinline__ uint64_t mnmajor_desc(uint32_t tile, int C, int k) {
    const uint32_t rg = static_cast<uint32_t>(C >> 3) << 7;
    return sdesc(tile + static_cast<uint32_t>(k) * 2u * rg, rg, 128u);
}

// Instruction descriptor, kind::f16: BF16 A and B, FP32 accumulator, M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, bool a_mn, bool b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
           (static_cast<uint32_t>(N >> 3) << 17) | (static_cast<uint32_t>(M >> 4) << 24);
}

// D (TMEM) [+]= A * B for one 16-deep K slice; issued by a single thread.
__device__ __forceinline__ void mma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, bool accumulate) {
    const uint32_t acc = accumulate ? 1u : 0u, z = 0u;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z));
}

// Arrive on the mbarrier once every MMA this thread issued so far has completed.
__device__ __forceinline__ void commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Waits for the phase with the given parity to complete; gives up after
// `max_cycles` SM clock cycles and returns false (the caller reports it).
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, long long max_cycles) {
    const long long start = clock64();
    while (clock64() - start < max_cycles) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Generic-proxy shared-memory writes made visible to the tensor core.
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// TMEM allocation by one whole warp; the base address is written to *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t base, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(ncols) : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane (warp w of the
// warpgroup reads lanes 32w..32w+31), waited for before returning.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}

}  // namespace umma
}  // namespace bbrt
