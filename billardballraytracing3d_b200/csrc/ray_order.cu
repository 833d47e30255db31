// Coherent processing order for a batch of rays.
//
// Rays are bucketed by an 18-bit key — the octant of the direction (3 bits)
// over a 15-bit Morton code of the origin quantised to 32 cells per axis
// inside a cube of four scene radii — with a counting sort: histogram,
// exclusive scan, scatter.  Warps then hold rays that start close together
// and head the same way, so their BVH walks and stage-1 patch tests follow
// the same paths.  Only the order in which rays are processed changes; every
// ray's result is written to its own index.
#include <cuda_runtime.h>

namespace bbrt {

constexpr int kOrderBits = 18;
constexpr int kOrderBuckets = 1 << kOrderBits;

__device__ __forceinline__ unsigned spread5(unsigned v) {
    // 5 bits -> every third bit
    v &= 31u;
    v = (v | (v << 8)) & 0x0000F00Fu;
    v = (v | (v << 4)) & 0x000C30C3u;
    v = (v | (v << 2)) & 0x00249249u;
    return v;
}

__device__ __forceinline__ unsigned ray_key(const double* o, const double* d, const double c[3], double inv_span) {
    unsigned q[3];
    for (int a = 0; a < 3; ++a) {
        double x = (o[a] - c[a]) * inv_span + 0.5;
        x = x < 0.0 ? 0.0 : (x > 0.999999 ? 0.999999 : x);
        if (!(x == x)) x = 0.0;   // NaN origin
        q[a] = static_cast<unsigned>(x * 32.0);
    }
    const unsigned morton = spread5(q[0]) | (spread5(q[1]) << 1) | (spread5(q[2]) << 2);
    const unsigned oct = (d[0] < 0.0 ? 1u : 0u) | (d[1] < 0.0 ? 2u : 0u) | (d[2] < 0.0 ? 4u : 0u);
    return (oct << 15) | morton;
}

__global__ void k_order_hist(const double* __restrict__ o, const double* __restrict__ d, long long n, double cx,
                             double cy, double cz, double inv_span, unsigned* __restrict__ keys,
                             unsigned* __restrict__ hist) {
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const double c[3] = { cx, cy, cz };
    const unsigned k = ray_key(o + 3 * i, d + 3 * i, c, inv_span);
    keys[i] = k;
    atomicAdd(hist + k, 1u);
}

// Exclusive scan of kOrderBuckets counts by one block of 1024 threads.
__global__ void __launch_bounds__(1024) k_order_scan(unsigned* __restrict__ hist) {
    constexpr int per = kOrderBuckets / 1024;
    __shared__ unsigned part[1024];
    const int t = threadIdx.x;
    unsigned* h = hist + t * per;
    unsigned s = 0;
    for (int k = 0; k < per; ++k) s += h[k];
    part[t] = s;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        const unsigned v = (t >= off) ? part[t - off] : 0u;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    unsigned run = part[t] - s;
    for (int k = 0; k < per; ++k) {
        const unsigned c = h[k];
        h[k] = run;
        run += c;
    }
}

__global__ void k_order_scatter(const unsigned* __restrict__ keys, long long n, unsigned* __restrict__ cursor,
                                int* __restrict__ order) {
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const unsigned pos = atomicAdd(cursor + keys[i], 1u);
    order[pos] = static_cast<int>(i);
}

size_t ray_order_workspace_bytes(long long n) {
    return sizeof(unsigned) * (static_cast<size_t>(n) + kOrderBuckets) + 512;
}

// order[n] receives the processing order.  `ws` holds ray_order_workspace_bytes(n).
cudaError_t ray_order(const double* o, const double* d, long long n, const double center[3], double radius,
                      void* ws, int* order, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    unsigned* hist = static_cast<unsigned*>(ws);
    unsigned* keys = hist + kOrderBuckets;
    cudaError_t e = cudaMemsetAsync(hist, 0, sizeof(unsigned) * kOrderBuckets, stream);
    if (e != cudaSuccess) return e;
    const double inv_span = radius > 0.0 ? 1.0 / (4.0 * radius) : 1.0;
    const unsigned blocks = static_cast<unsigned>((n + 255) / 256);
    k_order_hist<<<blocks, 256, 0, stream>>>(o, d, n, center[0], center[1], center[2], inv_span, keys, hist);
    k_order_scan<<<1, 1024, 0, stream>>>(hist);
    k_order_scatter<<<blocks, 256, 0, stream>>>(keys, n, hist, order);
    return cudaGetLastError();
}

}  // namespace bbrt
