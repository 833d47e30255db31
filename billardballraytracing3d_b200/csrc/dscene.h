// Device-side scene view and launch descriptors shared by the host C ABI
// (capi.cpp) and the kernels (*.cu).  Plain pointers into one scene's device
// allocation; passed to kernels by value.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

namespace bbrt {

struct GuessSample;

struct DScene {
    int n_objects = 0;
    int n_nodes = 0;
    int coarse_n = 0;               // coarse grid is coarse_n x coarse_n for every patch
    int newton_max_iters = 20;
    double newton_tol = 1e-3;
    double scene_diagonal = 0.0;
    double max_patch_sagitta = 0.0;
    double eps_factor = 1e-9;       // kSelfIntersectEpsilonFactor
    double sag_factor = 5.0;        // kSagittaClearanceFactor
    double backface_tol = 1e-9;     // kBackfaceHitTol

    // BVH nodes renumbered breadth-first (the top levels come first) with
    // explicit children; the tree and its child order are the reference's.
    const double* node_box = nullptr;      // [n_nodes][6]  min xyz, max xyz
    const int* node_link = nullptr;        // [n_nodes][4]  internal: left, right, 0, axis
                                           //               leaf:     start, -1, count, 0
    const int* leaf_objects = nullptr;
    int smem_nodes = 0;                    // nodes [0, smem_nodes) staged in shared memory
    // FP32 copies of the node boxes (nearest rounding) for the FP32 node
    // test, and per axis a bound on |coordinate| over every node box (FP32,
    // rounded up, at least 2^-60); node_f32_ok = 0 when a bound exceeds 2^40
    // (the test then stays FP64).
    const float* node_box32 = nullptr;     // [n_nodes][6]
    float node_bound[3] = { 0.0f, 0.0f, 0.0f };
    int node_f32_ok = 0;

    // objects
    const int* obj_kind = nullptr;         // BBRT_OBJ_*
    const int* obj_sub = nullptr;          // patch or triangle index
    const double* obj_pad = nullptr;       // self_intersect_padding

    // patches
    const int* p_dims = nullptr;           // [n_patches][2] imax, jmax
    const long long* p_node_off = nullptr; // un[imax] vn[jmax] uw[imax] vw[jmax]
    const long long* p_field_off = nullptr;// node-major, 12 doubles per node
    const double* p_nodes = nullptr;
    const double* p_fields = nullptr;
    const float* p_nodes32 = nullptr;      // FP32 copies (same offsets) for the FP32 Newton phase
    const float* p_fields32 = nullptr;
    int precision = 0;                     // BBRT_PREC_*
    int max_nodes = 0;                     // largest node count per axis over the patches
    const double* coarse_uv = nullptr;     // [coarse_n]
    const double* c_xyz = nullptr;         // [n_patches][coarse_n^2][3]
    const double* c_cell = nullptr;        // [n_patches][(coarse_n-1)^2][4] normal xyz, sagitta
    const float* c_cell_box = nullptr;     // [n_patches][(coarse_n-1)^2][6] cell AABB (cull)
    const float* c_block_box = nullptr;    // [n_patches][n_blocks][6] block AABB (cull)
    int block_cells = 4;                   // a block is block_cells x block_cells cells
    int n_blocks_side = 0;                 // blocks per side
    // Conservative inflation of the cull boxes for a ray with origin o:
    //   L     = |o - cull_center| + cull_radius   (bounds |o - v| for every vertex v)
    //   delta = cull_a * (L + cull_h) + cull_b * (L + |o| + cull_coord)
    // cull_a covers the FP64 Moller-Trumbore rounding (hits accepted up to that
    // far outside a triangle), cull_b the FP32 slab test's own rounding.
    int cull_enabled = 0;
    double cull_a = 0.0, cull_h = 0.0, cull_b = 0.0, cull_coord = 0.0;
    double cull_center[3] = { 0.0, 0.0, 0.0 };
    double cull_radius = 0.0;

    // triangles
    const double* tri = nullptr;           // [n_tri][9]

    // Several scenes traced as one (a scene set): the member scenes' objects,
    // patches and BVH trees live in the arrays above side by side; member m's
    // tree starts at node m_root[m], and its scale and cull constants are
    // m_param[m * kMemberParams + ...] (see kMemberParams).  n_members == 0
    // for a single scene, whose tree starts at node 0.
    int n_members = 0;
    const int* m_root = nullptr;
    const double* m_param = nullptr;
};

// Per-member values of a scene set: scene diagonal, cull on (1) / off (0),
// cull_a, cull_h, cull_b, cull_coord, cull_radius, cull_center xyz.
constexpr int kMemberParams = 10;

// Counter slots of the per-launch statistics buffer (long long each).
enum StatSlot {
    ST_BOUNCES = 0, ST_QUERIES, ST_NODE_TESTS, ST_PATCH_TESTS, ST_CELL_TESTS, ST_TRI_TESTS,
    ST_NEWTON_ITERS, ST_NEWTON_ITERS_FP32, ST_HIST0,
    // share of the tail kernels (also included in the totals above)
    ST_TAIL_NODE_TESTS = ST_HIST0 + 8, ST_TAIL_CELL_TESTS, ST_TAIL_TRI_TESTS, ST_TAIL_NEWTON_ITERS, ST_TAIL_RAYS,
    // learned guess: Newton solves started from the network, and those that fell back to the triangle
    ST_GUESS_USED, ST_GUESS_FALLBACK,
    // learned form: patches whose Newton root lay outside the patch, taken as not hit
    ST_OFF_PATCH,
    // FP32 node test: node tests it left undecided (run in FP64)
    ST_NODE_F64,
    ST_COUNT
};

struct TraceArgs {
    const double* origins = nullptr;   // [n][3]
    const double* dirs = nullptr;      // [n][3]
    long long n = 0;
    int max_bounces = 0;
    int record = 0;                    // K
    int cull = 1;
    int* status = nullptr;
    int* bounce_count = nullptr;
    double* exit_dir = nullptr;
    double* end_point = nullptr;
    int* hit_object = nullptr;         // [n][K]
    double* hit_point = nullptr;       // [n][K][3]
    double* hit_uv = nullptr;          // [n][K][2]
    int* err_object = nullptr;
    double* err_value = nullptr;       // [n][2]
    long long* ray_work = nullptr;     // [n][4] node tests, box tests, MT tests, Newton iterations
    unsigned long long* hit_counts = nullptr;  // per object (plane source), may be null
    int count_from = 1;                // first bounce index that is counted
    long long* stats = nullptr;        // [ST_COUNT], may be null
    unsigned long long* work_counter = nullptr;  // persistent-launch ray counter (zeroed by host)
    // Training-sample recording (learned guess): converged Newton solves go to
    // samples[0, cap_pos), stage-1 misses to samples[cap_pos, cap_pos + cap_neg);
    // sample_count[1] / [0] count positives / negatives offered (may exceed the caps).
    GuessSample* samples = nullptr;
    unsigned long long* sample_count = nullptr;
    long long sample_cap_pos = 0, sample_cap_neg = 0;
    // Learned form: a patch whose Newton solve converges to a root outside
    // the patch's parameter domain (|u| or |v| > 1 + 1e-6) is taken as not
    // hit instead of failing the ray, unless the network placed a confident
    // hit well inside the patch (then the root is suspect and the failure
    // stands).  Off (0) in the plain and split forms, which keep the
    // reference's failure.
    int off_patch_miss = 0;
    // Scene set: the member scene of every ray ([n]); null for one scene.
    const int* ray_member = nullptr;
};

// Network outputs (u, v, t, logit) that place a confident hit well inside
// the patch: they veto the learned form's off-patch miss.
__host__ __device__ inline bool guess_inside(const double* g, double min_logit) {
    return g != nullptr && g[3] > min_logit && fabs(g[0]) <= 0.95 && fabs(g[1]) <= 0.95;
}

// A patch query of the current bounce whose stage-1 winner needs Newton.
struct NewtonRequest {
    int ray;      // ray index
    int entry;    // slot in the ray's resolved list
    int obj;      // object index of the patch
    int key;      // stage-1 winner
    double t0;    // stage-1 t
};

// Resolved Newton results of a ray's current query: res_obj[ray][k] and
// res_data[ray][k][kResData] = t, point xyz, normal xyz, u, v, ev0, ev1.
constexpr int kResolved = 4;
constexpr int kResData = 11;

// Workspace of the wavefront trace (advance / Newton rounds).
struct WaveArgs {
    double* o = nullptr;       // [n][3] ray state between rounds
    double* d = nullptr;
    double* end = nullptr;
    int* bounces = nullptr;
    int* nres = nullptr;
    int* res_obj = nullptr;    // [n][kResolved]
    int* res_err = nullptr;    // [n][kResolved]
    double* res_data = nullptr;  // [n][kResolved][kResData]
    const NewtonRequest* runnable = nullptr;   // previous round's requests (null: round 0, all rays)
    const int* order = nullptr;                // round 0 processing order (null: index order)
    long long n_runnable = 0;
    NewtonRequest* req = nullptr;              // this round's requests
    unsigned int* counters = nullptr;          // [0] requests of the round, [1] overflowed rays (cumulative),
                                               // [2] runnable rays fetched this round, [3] watchdog tripped
    int* overflow = nullptr;                   // rays whose query needs more than kResolved solves
    // Learned guess of this round's requests: guess[r] = (u, v, t, logit), or null.
    const double* guess = nullptr;
    const double* frame = nullptr;             // per-patch frames (size L at [12] of each 16)
    double guess_min_logit = 0.0;              // confidence needed to start Newton from the guess
    double guess_t_window = 0.5;               // accepted |t - t_stage1| in units of L
    int warp_stage1 = 1;                       // stage 1 of k_advance by the whole warp (else per lane)
    int half_stage1 = 1;                       // ... two patches at a time by half-warps where they fit
    int quarter_stage1 = 0;                    // ... four at a time by quarter-warps instead
    // Traversal state of a query suspended for a Newton solve, so that the
    // next round resumes it instead of replaying it from the root:
    // qs_int[ray][kQsInt] = stack depth (-1: none saved), leaf start, leaf
    // count, position in the leaf, best object, best resolved entry;
    // qs_dbl[ray][3] = best t, triangle u, v; qs_stack[ray][kSaveStack].
    int* qs_int = nullptr;
    double* qs_dbl = nullptr;
    int* qs_stack = nullptr;
    int resume_queries = 1;
    int group_newton = 0;                      // Newton solves by 8-lane groups when the patches allow it
    int child_test = -1;                       // k_advance tests a node's children with it (-1: when the
                                               // tree is larger than the shared-memory copy)
    // Graph-launched trace: the launch's item count (runnable rays, requests,
    // tail rays) is read from this device word instead of the host argument,
    // and the Newton kernel copies each request it solves to next_req (the
    // next round's runnable set); null in the host-driven trace.
    const unsigned int* count_dev = nullptr;
    NewtonRequest* next_req = nullptr;
    // k_advance stops (counters[3] set) once it has run this many SM cycles.
    long long watchdog_cycles = 1LL << 35;
    // k_advance and the warp-per-ray tail test BVH nodes in FP32
    // (node_box_f32), in FP64 only where the FP32 interval does not decide;
    // the visit sequence is unchanged.
    int node_f32 = 0;
    // k_advance: in a round with fewer rays than the grid's lanes, fewer
    // lanes of each warp take rays, spreading the round over every warp.
    int adapt_lanes = 0;
    // Rounds of at most this many Newton requests solve each with 8 lanes
    // (patches of at most 8 nodes per axis); 0: one request per thread always.
    long long newton_group_max = 0;
};

// Round counters of the wavefront trace in device memory: [0..3] as
// WaveArgs::counters; [4..7] are the round control of the graph-launched
// trace, written by k_wave_decide after each k_advance; [8..9] hand out the
// tail kernels' rays.  All start at zero for each trace.
constexpr int kWcNext = 4;     // requests solved this round, runnable next round (0: rounds end)
constexpr int kWcTail = 5;     // requests left to the tail kernel (the last, small round)
constexpr int kWcRounds = 6;   // rounds whose requests went to Newton
constexpr int kWcBound = 7;    // the round bound was reached
constexpr int kWcTailNext = 8; // next slot of the tail kernel (rays handed out one at a time)
constexpr int kWcOvfNext = 9;  // next slot of the overflow tail
constexpr int kWaveCounters = 10;

constexpr int kQsInt = 6;
constexpr int kSaveStack = 24;

struct QueryArgs {
    const double* origins = nullptr;
    const double* dirs = nullptr;
    long long n = 0;
    int mode = 0;          // BBRT_QUERY_*
    int object = 0;
    int cull = 1;
    void* out = nullptr;   // bbrt_hit[n]
};

}  // namespace bbrt
