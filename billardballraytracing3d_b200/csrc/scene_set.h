// A scene set's per-member rays and outputs: the set traces all members'
// rays as one array (their ranges side by side); these descriptors move the
// rays in and the results out (scene_set.cu).
#pragma once

#include <cuda_runtime.h>

namespace bbrt {

struct MemberIO {
    const double* o = nullptr;   // the member's rays (device, [n][3])
    const double* d = nullptr;
    long long off = 0, n = 0;    // its range in the set's ray arrays
    int obj_off = 0;             // its first object in the set
    // its outputs (device, each may be null), laid out as bbrt_trace_out
    int* status = nullptr;
    int* bounce_count = nullptr;
    double* exit_dir = nullptr;
    double* end_point = nullptr;
    int* hit_object = nullptr;
    double* hit_point = nullptr;
    double* hit_uv = nullptr;
    int* err_object = nullptr;
    double* err_value = nullptr;
    long long* ray_work = nullptr;
};

struct SetIO {
    const MemberIO* m = nullptr;   // [n_members], device
    int n_members = 0;
    long long n = 0;               // rays in all
    int K = 0;                     // recorded bounces per ray
    // the set's arrays
    double* o = nullptr;
    double* d = nullptr;
    int* ray_member = nullptr;
    const int* status = nullptr;
    const int* bounce_count = nullptr;
    const double* exit_dir = nullptr;
    const double* end_point = nullptr;
    const int* hit_object = nullptr;
    const double* hit_point = nullptr;
    const double* hit_uv = nullptr;
    const int* err_object = nullptr;
    const double* err_value = nullptr;
    const long long* ray_work = nullptr;
};

// Copies every member's rays into the set's arrays and records each ray's member.
cudaError_t set_gather(const SetIO& io, cudaStream_t st);
// Records each set ray's member only (the rays are already in place).
cudaError_t set_members(const SetIO& io, cudaStream_t st);
// Copies the set's per-ray results to every member's outputs; object indices
// (hit and error objects) go back to the member's own numbering.
cudaError_t set_scatter(const SetIO& io, cudaStream_t st);

}  // namespace bbrt
