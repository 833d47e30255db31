// Coherent processing order for a batch of rays.
//
// Rays are bucketed by an 18-bit key — the octant of the direction (3 bits)
// over a 15-bit Morton code, quantised to 32 cells per axis, of the point
// where the ray enters the sphere around the scene (or of its origin) — with
// a counting sort: histogram,
// exclusive scan (two passes), scatter.  Warps then hold rays that start close together
// and head the same way, so their BVH walks and stage-1 patch tests follow
// the same paths.  Only the order in which rays are processed changes; every
// ray's result is written to its own index.
#include <cuda_runtime.h>

#include "dscene.h"

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

// The point where a ray enters the sphere (c, r) around the scene — the origin
// when it starts inside or misses — so that rays which meet the scene at the
// same place in the same direction octant share a key.
__device__ __forceinline__ void entry_point(const double* o, const double* d, const double c[3], double r,
                                            double* p) {
    const double ox = o[0] - c[0], oy = o[1] - c[1], oz = o[2] - c[2];
    const double dd = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    const double b = ox * d[0] + oy * d[1] + oz * d[2];
    const double cc = ox * ox + oy * oy + oz * oz - r * r;
    const double disc = b * b - dd * cc;
    double t = 0.0;
    if (cc > 0.0 && dd > 0.0 && disc > 0.0) t = (-b - sqrt(disc)) / dd;
    if (!(t > 0.0)) t = 0.0;
    for (int a = 0; a < 3; ++a) p[a] = o[a] + t * d[a];
}

__global__ void k_order_hist(const double* __restrict__ o, const double* __restrict__ d, long long n, double cx,
                             double cy, double cz, double inv_span, double entry_r, unsigned* __restrict__ keys,
                             unsigned* __restrict__ hist) {
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const double c[3] = { cx, cy, cz };
    double p[3];
    if (entry_r > 0.0) entry_point(o + 3 * i, d + 3 * i, c, entry_r, p);
    else for (int a = 0; a < 3; ++a) p[a] = o[3 * i + a];
    const unsigned k = ray_key(p, d + 3 * i, c, inv_span);
    keys[i] = k;
    atomicAdd(hist + k, 1u);
}

// Exclusive scan of the kOrderBuckets counts in two passes of
// kOrderBuckets / 1024 blocks: each block scans its 1024 counts in place and
// records their total; then each block adds the totals of the blocks before it.
constexpr int kScanBlock = 1024;
constexpr int kScanBlocks = kOrderBuckets / kScanBlock;

// Block-wide exclusive scan of one value per thread (1024 threads); *total
// receives the block's sum.
__device__ __forceinline__ unsigned block_exclusive_scan(unsigned v, unsigned* warp_sums, unsigned* total) {
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    unsigned x = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const unsigned y = __shfl_up_sync(0xffffffffu, x, off);
        if (lane >= off) x += y;
    }
    if (lane == 31) warp_sums[w] = x;
    __syncthreads();
    if (w == 0) {
        unsigned s = warp_sums[lane];
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const unsigned y = __shfl_up_sync(0xffffffffu, s, off);
            if (lane >= off) s += y;
        }
        warp_sums[lane] = s;   // inclusive prefix of the warp totals
    }
    __syncthreads();
    if (total) *total = warp_sums[31];
    return x - v + (w > 0 ? warp_sums[w - 1] : 0u);
}

__global__ void __launch_bounds__(kScanBlock) k_order_scan_local(unsigned* __restrict__ hist,
                                                                 unsigned* __restrict__ block_sums) {
    __shared__ unsigned ws[32];
    __shared__ unsigned total;
    unsigned* h = hist + blockIdx.x * kScanBlock;
    const unsigned v = h[threadIdx.x];
    const unsigned ex = block_exclusive_scan(v, ws, &total);
    h[threadIdx.x] = ex;
    if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanBlock) k_order_scan_add(unsigned* __restrict__ hist,
                                                               const unsigned* __restrict__ block_sums) {
    __shared__ unsigned part[32];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    // sum of the totals of blocks [0, blockIdx.x)
    unsigned v = (t < static_cast<int>(blockIdx.x)) ? block_sums[t] : 0u;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    if (lane == 0) part[w] = v;
    __syncthreads();
    unsigned base = 0;
    for (int k = 0; k < 32; ++k) base += part[k];
    hist[blockIdx.x * kScanBlock + t] += base;
}

__global__ void k_order_scatter(const unsigned* __restrict__ keys, long long n, unsigned* __restrict__ cursor,
                                int* __restrict__ order, long long base) {
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const unsigned pos = atomicAdd(cursor + keys[i], 1u);
    order[pos] = static_cast<int>(base + i);
}

size_t ray_order_workspace_bytes(long long n) {
    return sizeof(unsigned) * (static_cast<size_t>(n) + kOrderBuckets + kScanBlocks) + 512;
}

// order[n] receives the processing order (ray indices plus `base`).  `ws`
// holds ray_order_workspace_bytes(n).  entry: key on the point where each ray
// enters the scene's sphere (else on its origin).
cudaError_t ray_order(const double* o, const double* d, long long n, const double center[3], double radius,
                      void* ws, int* order, cudaStream_t stream, bool entry, long long base) {
    if (n <= 0) return cudaSuccess;
    unsigned* hist = static_cast<unsigned*>(ws);
    unsigned* block_sums = hist + kOrderBuckets;
    unsigned* keys = block_sums + kScanBlocks;
    cudaError_t e = cudaMemsetAsync(hist, 0, sizeof(unsigned) * kOrderBuckets, stream);
    if (e != cudaSuccess) return e;
    // origins: a cube of four radii; entry points: the sphere's own cube
    const double inv_span = radius > 0.0 ? 1.0 / ((entry ? 2.0 : 4.0) * radius) : 1.0;
    const unsigned blocks = static_cast<unsigned>((n + 255) / 256);
    k_order_hist<<<blocks, 256, 0, stream>>>(o, d, n, center[0], center[1], center[2], inv_span,
                                             entry && radius > 0.0 ? radius : 0.0, keys, hist);
    k_order_scan_local<<<kScanBlocks, kScanBlock, 0, stream>>>(hist, block_sums);
    k_order_scan_add<<<kScanBlocks, kScanBlock, 0, stream>>>(hist, block_sums);
    k_order_scatter<<<blocks, 256, 0, stream>>>(keys, n, hist, order, base);
    return cudaGetLastError();
}

// ---- a round's Newton requests grouped by patch object ----------------------
//
// The same counting sort over the object index: the requests of one patch end
// up next to each other, so the lanes of a Newton warp share their patch's
// node-field loads.  Each request is solved on its own and written to its
// own (ray, entry), so only the order of the work changes.  With n_dev (a
// graph launch) the count is read on the device and n only sizes the grid.

// Bucket of a request: its object, refined (side > 1) by the side x side
// region of the patch that holds its stage-1 cell (key = cell * 6 + test).
__device__ __forceinline__ unsigned req_bucket(const NewtonRequest& q, int side, int nc) {
    if (side <= 1) return static_cast<unsigned>(q.obj);
    const int cell = q.key / 6, ci = cell / nc, cj = cell - ci * nc;
    return static_cast<unsigned>(q.obj) * side * side + (ci * side / nc) * side + (cj * side / nc);
}

__global__ void k_req_hist(const NewtonRequest* __restrict__ req, long long n, const unsigned* n_dev, int side,
                           int nc, unsigned* __restrict__ hist) {
    if (n_dev) n = *n_dev;
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    atomicAdd(hist + req_bucket(req[i], side, nc), 1u);
}

__global__ void k_req_scatter(const NewtonRequest* __restrict__ req, long long n, const unsigned* n_dev, int side,
                              int nc, unsigned* __restrict__ cursor, NewtonRequest* __restrict__ out) {
    if (n_dev) n = *n_dev;
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const NewtonRequest q = req[i];
    out[atomicAdd(cursor + req_bucket(q, side, nc), 1u)] = q;
}

// Largest object count the request sort handles (one bucket per object).
int request_sort_max_objects() { return kOrderBuckets; }

// out[0, count) = req[0, count) grouped by object, and within an object by
// the side x side region of its stage-1 cell (coarse_cells cells per patch
// side; side 1 when the buckets would not fit); `ws` holds
// ray_order_workspace_bytes(any n); n_objects <= request_sort_max_objects().
cudaError_t sort_requests(const NewtonRequest* req, long long n, const unsigned* n_dev, int n_objects, int side,
                          int coarse_cells, void* ws, NewtonRequest* out, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    if (n_objects < 1 || n_objects > kOrderBuckets) return cudaErrorInvalidValue;
    if (side < 1 || coarse_cells < 1 || static_cast<long long>(n_objects) * side * side > kOrderBuckets) side = 1;
    unsigned* hist = static_cast<unsigned*>(ws);
    unsigned* block_sums = hist + kOrderBuckets;
    const int buckets = n_objects * side * side;
    const int scan_blocks = (buckets + kScanBlock - 1) / kScanBlock;
    cudaError_t e = cudaMemsetAsync(hist, 0, sizeof(unsigned) * kScanBlock * scan_blocks, stream);
    if (e != cudaSuccess) return e;
    const unsigned blocks = static_cast<unsigned>((n + 255) / 256);
    k_req_hist<<<blocks, 256, 0, stream>>>(req, n, n_dev, side, coarse_cells, hist);
    k_order_scan_local<<<scan_blocks, kScanBlock, 0, stream>>>(hist, block_sums);
    k_order_scan_add<<<scan_blocks, kScanBlock, 0, stream>>>(hist, block_sums);
    k_req_scatter<<<blocks, 256, 0, stream>>>(req, n, n_dev, side, coarse_cells, hist, out);
    return cudaGetLastError();
}

}  // namespace bbrt
