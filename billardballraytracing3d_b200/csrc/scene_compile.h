// Arguments of the GPU scene compile (scene_compile.cu), shared with the host
// code that uploads a scene's patch tables and reads the per-patch results.
#pragma once

#include <cuda_runtime.h>

namespace bbrt {

struct SetupArgs {
    int n_patches = 0;
    int cn = 0;                        // coarse grid points per axis
    const double* coarse_uv = nullptr; // [cn]
    const int* dims = nullptr;         // [n_patches][2] imax, jmax
    const long long* node_off = nullptr;   // into nodes: un[imax] vn[jmax] uw[imax] vw[jmax]
    const long long* field_off = nullptr;  // into fields: imax * jmax nodes x 12 doubles, node-major
    const double* nodes = nullptr;
    const double* fields = nullptr;
    double* c_xyz = nullptr;           // [n_patches][cn * cn][3]
    double* c_cell = nullptr;          // [n_patches][(cn - 1)^2][4] unit normal, sagitta
    double* patch_out = nullptr;       // [n_patches][10] box min xyz, max xyz, centroid xyz, padding
    // stage-1 cull tables (cell_box null: none)
    float* cell_box = nullptr;         // [n_patches][(cn - 1)^2][6], rounded outward
    float* block_box = nullptr;        // [n_patches][n_blocks_side^2][6]
    int block_cells = 4, n_blocks_side = 0;
    double* cull_stats = nullptr;      // [n_patches][3] longest triangle edge, largest |coordinate|, all finite
};

cudaError_t launch_patch_setup(const SetupArgs& A, int sm_count, cudaStream_t st);

}  // namespace bbrt
