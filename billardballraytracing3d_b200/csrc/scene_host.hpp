// Host side of a bbrt scene: per-object set-up, the BVH build and the
// flattened arrays that are uploaded to the GPU once per scene.
//
// The set-up arithmetic has to produce the same doubles as the reference's
// SurfacePatch / Triangle constructors and BVH builder, because the GPU's
// stage-1 decisions read the coarse grid, sagittas and boxes bit for bit.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/bbrt.h"

namespace bbrt {

// Upper bound on interpolation nodes per axis that the device Newton solve
// handles (per-thread basis arrays are sized to it; kDevMaxNodes in exact.cuh).
constexpr int kMaxNodes = 16;

// Number of double fields kept per node on the device, in this order:
// x y z  dxdu dydu dzdu  dxdv dydv dzdv  nuX nuY nuZ.
constexpr int kFields = 12;

struct BvhNode {
    double box[6];          // min xyz, max xyz
    int right;              // -1 for a leaf
    int start, count;       // leaf range into leaf_objects
    int axis;               // split axis of an internal node
};

struct HostScene {
    bbrt_config cfg{};
    int n_objects = 0;
    std::vector<int> kind;            // BBRT_OBJ_*
    std::vector<int> sub;             // index into the patch or triangle tables
    std::vector<long long> zone;      // zoneID (triangles: their object index)
    std::vector<double> box;          // [n_objects][6]
    std::vector<double> centroid;     // [n_objects][3]
    std::vector<double> padding;      // [n_objects] self_intersect_padding

    // patches
    int n_patches = 0;
    std::vector<int> patch_obj;       // object index of each patch
    int coarse_n = 0;
    std::vector<double> coarse_uv;    // [coarse_n] (the same for u and v, and every patch)
    std::vector<int> p_imax, p_jmax;
    std::vector<long long> p_node_off;   // into p_nodes: un[imax] vn[jmax] uw[imax] vw[jmax]
    std::vector<long long> p_field_off;  // into p_fields: imax*jmax nodes x kFields, node-major
    std::vector<double> p_nodes, p_fields;
    std::vector<double> c_xyz;        // [n_patches][coarse_n^2][3]
    std::vector<double> c_cell;       // [n_patches][(coarse_n-1)^2][4]: normal xyz, sagitta

    // triangles
    std::vector<double> tri;          // [n_tri][9]

    // BVH
    std::vector<BvhNode> nodes;
    std::vector<int> leaf_objects;
    int max_depth = 0;

    double scene_diagonal = 0.0;
    double max_patch_sagitta = 0.0;
};

// Builds every object's set-up, the BVH over objects in the given order and
// the scene scale.  Throws std::invalid_argument / std::runtime_error with
// the reference's wording on bad input.  The same in three steps:
//   build_host_tables   validation, object tables, patch node / field tables,
//                       triangle boxes and centroids
//   setup_patches_host  per patch: coarse grid, cell normals and sagittas,
//                       box, centroid, padding (the step the GPU can take over:
//                       scene_compile.cu)
//   finish_host_scene   BVH over the object boxes and centroids, scene scale
void build_host_scene(const bbrt_object_desc* objects, int n_objects, const bbrt_config& cfg,
                      HostScene& out);
void build_host_tables(const bbrt_object_desc* objects, int n_objects, const bbrt_config& cfg, HostScene& out);
void setup_patches_host(const bbrt_object_desc* objects, HostScene& S);
void finish_host_scene(HostScene& S);

// SurfacePatch::sample_grid (SurfacePatch.hpp:199-242).
void sample_grid(const bbrt_patch_desc& p, int n, double* xyz, double* normal, double* dxdu);

// Patch file parsing (SurfacePatch.hpp:313-371); throws std::runtime_error.
struct PatchFileData {
    int imax = 0, jmax = 0, kmax = 0;
    long long zone = 0;
    std::vector<double> un, vn;
    std::vector<double> f[13];        // x y z dxdu dydu dzdu dxdv dydv dzdv dS nuX nuY nuZ
    std::vector<int> mask;
    int edge_flags[4] = { 0, 0, 0, 0 };
};
void read_patch_file(const std::string& path, PatchFileData& out);
bbrt_patch_desc patch_desc_of(const PatchFileData& d);

}  // namespace bbrt

namespace bbrt {

// Conservative cull tables for stage 1 (float cell and block boxes, rounded
// outward) and the per-ray inflation constants (see DScene).
struct CullTables {
    bool enabled = false;
    int block_cells = 4, n_blocks_side = 0;
    std::vector<float> cell_box, block_box;
    double a = 0.0, h = 0.0, b = 0.0, coord = 0.0, radius = 0.0;
    double center[3] = { 0.0, 0.0, 0.0 };
};
void build_cull_tables(const HostScene& S, CullTables& out);
// The per-ray inflation constants and the on/off decision of the cull tables,
// from the longest triangle edge, the largest |coordinate| and whether every
// offset corner is finite (build_cull_tables, or the GPU scene compile, which
// computes those three per patch); sets C.enabled.
void cull_constants(const HostScene& S, double hmax, double cmax, bool finite, CullTables& C);

}  // namespace bbrt
