// Rays into, and results out of, a scene set's one trace: member m owns the
// set's rays [off_m, off_m + n_m); the trace itself is the single-scene
// wavefront over the set's merged arrays (capi.cpp bbrt_trace_set).
#include "scene_set.h"

namespace bbrt {
namespace {

// The member owning set ray i: the last member whose range starts at or
// before i (ranges are contiguous and ascending; empty ones are skipped by
// taking the last).
__device__ __forceinline__ int member_of(const MemberIO* m, int n_members, long long i) {
    int lo = 0, hi = n_members - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (m[mid].off <= i) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__global__ void k_set_gather(SetIO io) {
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i >= io.n) return;
    const int k = member_of(io.m, io.n_members, i);
    const MemberIO& M = io.m[k];
    const long long j = i - M.off;
    for (int a = 0; a < 3; ++a) {
        io.o[3 * i + a] = M.o[3 * j + a];
        io.d[3 * i + a] = M.d[3 * j + a];
    }
    io.ray_member[i] = k;
}

__global__ void k_set_members(SetIO io) {
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i >= io.n) return;
    io.ray_member[i] = member_of(io.m, io.n_members, i);
}

__global__ void k_set_scatter(SetIO io) {
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i >= io.n) return;
    const MemberIO& M = io.m[io.ray_member[i]];
    const long long j = i - M.off;
    const int K = io.K;
    if (M.status) M.status[j] = io.status[i];
    if (M.bounce_count) M.bounce_count[j] = io.bounce_count[i];
    if (M.exit_dir) for (int a = 0; a < 3; ++a) M.exit_dir[3 * j + a] = io.exit_dir[3 * i + a];
    if (M.end_point) for (int a = 0; a < 3; ++a) M.end_point[3 * j + a] = io.end_point[3 * i + a];
    if (M.hit_object)
        for (int b = 0; b < K; ++b) {
            const int o = io.hit_object[i * K + b];
            M.hit_object[j * K + b] = o >= 0 ? o - M.obj_off : o;
        }
    if (M.hit_point) for (int b = 0; b < 3 * K; ++b) M.hit_point[j * 3 * K + b] = io.hit_point[i * 3 * K + b];
    if (M.hit_uv) for (int b = 0; b < 2 * K; ++b) M.hit_uv[j * 2 * K + b] = io.hit_uv[i * 2 * K + b];
    if (M.err_object) {
        const int o = io.err_object[i];
        M.err_object[j] = o >= 0 ? o - M.obj_off : o;
    }
    if (M.err_value) for (int a = 0; a < 2; ++a) M.err_value[2 * j + a] = io.err_value[2 * i + a];
    if (M.ray_work) for (int a = 0; a < 4; ++a) M.ray_work[4 * j + a] = io.ray_work[4 * i + a];
}

}  // namespace

cudaError_t set_gather(const SetIO& io, cudaStream_t st) {
    if (io.n <= 0) return cudaSuccess;
    k_set_gather<<<static_cast<unsigned>((io.n + 255) / 256), 256, 0, st>>>(io);
    return cudaGetLastError();
}

cudaError_t set_members(const SetIO& io, cudaStream_t st) {
    if (io.n <= 0) return cudaSuccess;
    k_set_members<<<static_cast<unsigned>((io.n + 255) / 256), 256, 0, st>>>(io);
    return cudaGetLastError();
}

cudaError_t set_scatter(const SetIO& io, cudaStream_t st) {
    if (io.n <= 0) return cudaSuccess;
    k_set_scatter<<<static_cast<unsigned>((io.n + 255) / 256), 256, 0, st>>>(io);
    return cudaGetLastError();
}

}  // namespace bbrt
