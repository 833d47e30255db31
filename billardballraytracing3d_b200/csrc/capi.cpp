// C ABI of libbbrt_cuda.so (include/bbrt.h): scene lifetime, device upload,
// and the batch entry points that launch the trace kernels.
//
// Reference call sites replaced (manuelarturosantana/BillardBallRayTracing3D):
//   RayTracingDriver(dir) / (dir, prefix, first, last)   RayTracingDriver.hpp:91-114, 346-424
//   RayTracingDriver::trace_ray / run                     :172-242, :143-150
//   BVH::intersect, brute_force_intersect                 BVH.hpp:75-128, BruteForce.hpp:7-16
//   PlaneSourceDriver::run                                PlaneSourceDriver.hpp:79-109
//   BounceMapDriver::run                                  BounceMapDriver.hpp:103-259
//   SurfacePatch::load_patch_file / sample_grid           SurfacePatch.hpp:313-371, :199-242
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <initializer_list>
#include <limits>
#include <memory>
#include <mutex>
#include <numeric>
#include <random>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/bbrt.h"
#include "dscene.h"
#include "guess.h"
#include "scene_compile.h"
#include "scene_set.h"
#include "scene_host.hpp"

namespace bbrt {
cudaError_t launch_trace(const DScene& S, const TraceArgs& A, cudaStream_t stream, int sm_count);
size_t wave_workspace_bytes(long long n);
void wave_layout(void* ws, long long n, WaveArgs& W, NewtonRequest*& req_a, NewtonRequest*& req_b);
cudaError_t launch_advance(const DScene& S, const TraceArgs& A, const WaveArgs& W, int sm_count, int shape,
                           cudaStream_t stream);
cudaError_t launch_newton(const DScene& S, const TraceArgs& A, const WaveArgs& W, long long n_req,
                          cudaStream_t stream);
cudaError_t launch_wave_decide(unsigned int* counters, long long wave_tail, long long max_rounds,
                               cudaGraphConditionalHandle loop, cudaStream_t stream);
cudaError_t launch_resume_warp(const DScene& S, const TraceArgs& A, const WaveArgs& W, const NewtonRequest* reqs,
                               const int* rays, long long n, int sm_count, int shape, cudaStream_t stream);
cudaError_t launch_resume(const DScene& S, const TraceArgs& A, const WaveArgs& W, const NewtonRequest* reqs,
                          const int* rays, long long n, cudaStream_t stream);
size_t ray_order_workspace_bytes(long long n);
int request_sort_max_objects();
cudaError_t sort_requests(const NewtonRequest* req, long long n, const unsigned* n_dev, int n_objects, int side,
                          int coarse_cells, void* ws, NewtonRequest* out, cudaStream_t stream);
cudaError_t ray_order(const double* o, const double* d, long long n, const double center[3], double radius,
                      void* ws, int* order, cudaStream_t stream, bool entry, long long base);
cudaError_t launch_query(const DScene& S, const QueryArgs& Q, cudaStream_t stream);
cudaError_t noalloc_prepare();
cudaError_t launch_trace_noalloc(const DScene& S, TraceArgs A, bool count_hits, long long* hit_counts_out,
                                 long long* host_stats, cudaStream_t stream, int sm_count);
int launch_umma_check(const uint16_t* A, const uint16_t* B, float* D, int* err, cudaStream_t st);
cudaError_t launch_node_check(const DScene& S, const double* o, const double* d, const double* best, long long n,
                              const double* boxes, int* out, cudaStream_t stream);
cudaError_t launch_bounce_rays(const double* frames, const double* trig, int theta_n, int phi_n, long long n,
                               double* org, double* dir, cudaStream_t st);
cudaError_t launch_bounce_reduce(const int* status, const int* bounces, long long points, int dirs_per, int* max_out,
                                 int* err_out, int* best_out, cudaStream_t st);
}  // namespace bbrt

namespace {

thread_local std::string g_error;

int fail(int code, const std::string& msg) {
    g_error = msg;
    return code;
}

#define BBRT_CUDA(call)                                                                   \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return fail(BBRT_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// A grow-only device buffer, freed when it goes out of scope.
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    cudaError_t ensure(size_t n) {
        if (n <= bytes) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        cudaError_t e = cudaMalloc(&p, n);
        if (e == cudaSuccess) bytes = n;
        return e;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
};

}  // namespace

struct bbrt_scene {
    bbrt::HostScene host;
    bbrt::CullTables cull;
    bbrt::DScene dev;
    bool uploaded = false;
    bool device_ready = false;      // device, stream and events chosen
    bool tables_uploaded = false;   // patch node / field tables on the device
    bool setup_on_device = false;   // coarse grids, cells and cull boxes computed on (and kept only on) the GPU
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[4] = { nullptr, nullptr, nullptr, nullptr };
    std::vector<void*> allocs;
    long long device_bytes = 0;
    DevBuf stats, work, in_o, in_d, o_status, o_bounce, o_dir, o_end, o_hobj, o_hpt, o_huv, o_eobj, o_eval,
        counts, hits, wave, wave_ctr, o_work, order, order_ws;
    unsigned int* wave_ctr_host = nullptr;   // pinned copy of the round counters
    // per-launch timing of calls that collect statistics
    static constexpr int kTimerEvents = 96;
    cudaEvent_t kev[kTimerEvents] = {};
    int kev_used = 0;
    bool timing = false;
    long long rounds = 0, launches = 0;
    std::vector<std::pair<int, int>> kspans;   // (kernel kind, first event)
    std::mutex mu;
    // Graph-launched wavefront traces: instantiated graphs of recent argument
    // sets (most recent last), and the streams they are captured on.
    struct WaveGraph {
        std::vector<long long> key;
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        long long launches_fixed = 0, launches_round = 0;   // kernels outside / inside the round loop
    };
    static constexpr size_t kWaveGraphs = 4;
    std::vector<WaveGraph> wgraphs;
    cudaStream_t cap[2] = { nullptr, nullptr };

    // Learned Newton guess: network (FP32 master, BF16 image, Adam moments),
    // per-patch frames, per-request outputs of the current round.
    struct Guess {
        DevBuf P, G, m1, m2, image, loss, err, out, rows;
        const double* frame = nullptr;     // [n_patches][kFrame] (scene allocation)
        bool trained = false;
        long long steps = 0;
        double min_logit = 0.0, t_window = 0.5;
    } guess;
    // Launch schedule of this scene (library defaults until set or autotuned).
    bool tune_set = false;
    bbrt_tuning tune{};
    // Scene set (bbrt_scene_set): the members' ray ranges of the current call
    // ([M + 1] offsets), each member's ordering sphere ([M][4] centre, radius)
    // and the member of every ray; empty / null for a single scene.
    std::vector<long long> member_rays;
    std::vector<double> member_sphere;
    const int* ray_member = nullptr;
    // Per-kernel event timing without device counters (bbrt_trace BBRT_TIMES_ONLY).
    bool time_kernels = false;
    // Training-sample recording, set only inside bbrt_guess_train.
    bbrt::GuessSample* rec_samples = nullptr;
    unsigned long long* rec_count = nullptr;
    long long rec_cap_pos = 0, rec_cap_neg = 0;

    ~bbrt_scene() {
        for (void* p : allocs) cudaFree(p);
        for (DevBuf* b : { &stats, &work, &in_o, &in_d, &o_status, &o_bounce, &o_dir, &o_end, &o_hobj, &o_hpt,
                           &o_huv, &o_eobj, &o_eval, &counts, &hits, &wave, &wave_ctr, &o_work, &order, &order_ws,
                           &guess.P, &guess.G, &guess.m1, &guess.m2, &guess.image, &guess.loss, &guess.err,
                           &guess.out, &guess.rows })
            b->release();
        if (wave_ctr_host) cudaFreeHost(wave_ctr_host);
        for (WaveGraph& g : wgraphs) {
            if (g.exec) cudaGraphExecDestroy(g.exec);
            if (g.graph) cudaGraphDestroy(g.graph);
        }
        for (auto& c : cap)
            if (c) cudaStreamDestroy(c);
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
        for (auto& e : kev)
            if (e) cudaEventDestroy(e);
        if (stream) cudaStreamDestroy(stream);
    }

    template <class T>
    int alloc(size_t n, T*& dst) {
        void* p = nullptr;
        BBRT_CUDA(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)));
        allocs.push_back(p);
        device_bytes += static_cast<long long>(n * sizeof(T));
        dst = static_cast<T*>(p);
        return BBRT_OK;
    }

    template <class T>
    int upload(const std::vector<T>& v, const T*& dst) {
        if (v.empty()) { dst = nullptr; return BBRT_OK; }
        void* p = nullptr;
        BBRT_CUDA(cudaMalloc(&p, v.size() * sizeof(T)));
        allocs.push_back(p);
        device_bytes += static_cast<long long>(v.size() * sizeof(T));
        BBRT_CUDA(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
        dst = static_cast<const T*>(p);
        return BBRT_OK;
    }
};

namespace {

// Per-patch frame of the learned guess (16 doubles, see guess.h): node mean,
// mean dX/du made orthogonal to the mean normal, the normal, their cross
// product, half the box diagonal and the box half-extents over it.
std::vector<double> patch_frames(const bbrt::HostScene& H) {
    std::vector<double> fr(static_cast<size_t>(H.n_patches) * bbrt::kFrame, 0.0);
    for (int obj = 0; obj < H.n_objects; ++obj) {
        if (H.kind[obj] != BBRT_OBJ_PATCH) continue;
        const int q = H.sub[obj];
        const int nn = H.p_imax[q] * H.p_jmax[q];
        const double* F = H.p_fields.data() + H.p_field_off[q];
        double c[3] = { 0, 0, 0 }, tu[3] = { 0, 0, 0 }, nv[3] = { 0, 0, 0 };
        for (int k = 0; k < nn; ++k)
            for (int a = 0; a < 3; ++a) {
                c[a] += F[k * bbrt::kFields + a];
                tu[a] += F[k * bbrt::kFields + 3 + a];
                nv[a] += F[k * bbrt::kFields + 9 + a];
            }
        double ln = std::sqrt(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2]);
        if (!(ln > 0.0)) { nv[0] = 0; nv[1] = 0; nv[2] = 1; ln = 1.0; }
        for (int a = 0; a < 3; ++a) { c[a] /= nn; nv[a] /= ln; }
        const double dn = tu[0] * nv[0] + tu[1] * nv[1] + tu[2] * nv[2];
        for (int a = 0; a < 3; ++a) tu[a] -= dn * nv[a];
        double lt = std::sqrt(tu[0] * tu[0] + tu[1] * tu[1] + tu[2] * tu[2]);
        if (!(lt > 1e-300)) {
            const double ax[3] = { std::fabs(nv[0]) < 0.9 ? 1.0 : 0.0, std::fabs(nv[0]) < 0.9 ? 0.0 : 1.0, 0.0 };
            const double p = ax[0] * nv[0] + ax[1] * nv[1];
            for (int a = 0; a < 3; ++a) tu[a] = ax[a] - p * nv[a];
            lt = std::sqrt(tu[0] * tu[0] + tu[1] * tu[1] + tu[2] * tu[2]);
        }
        for (int a = 0; a < 3; ++a) tu[a] /= lt;
        const double t2[3] = { nv[1] * tu[2] - nv[2] * tu[1], nv[2] * tu[0] - nv[0] * tu[2], nv[0] * tu[1] - nv[1] * tu[0] };
        const double* b = H.box.data() + 6 * static_cast<size_t>(obj);
        const double ex[3] = { 0.5 * (b[3] - b[0]), 0.5 * (b[4] - b[1]), 0.5 * (b[5] - b[2]) };
        double L = std::sqrt(ex[0] * ex[0] + ex[1] * ex[1] + ex[2] * ex[2]);
        if (!(L > 0.0)) L = 1.0;
        double* f = fr.data() + static_cast<size_t>(q) * bbrt::kFrame;
        for (int a = 0; a < 3; ++a) {
            f[a] = c[a];
            f[3 + a] = tu[a];
            f[6 + a] = t2[a];
            f[9 + a] = nv[a];
            f[13 + a] = ex[a] / L;
        }
        f[12] = L;
    }
    return fr;
}

// Binds the scene to the current device: its stream and events.
int ensure_device(bbrt_scene* s) {
    if (s->device_ready) return BBRT_OK;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0)
        return fail(BBRT_ERR_CUDA, "bbrt: no CUDA device available (the trace path has no CPU fallback)");
    BBRT_CUDA(cudaGetDevice(&s->device));
    BBRT_CUDA(cudaDeviceGetAttribute(&s->sm_count, cudaDevAttrMultiProcessorCount, s->device));
    BBRT_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    // the allocation-free trace's module (scratch array and kernel) is loaded
    // here, so that bbrt_trace_noalloc itself never triggers a module load
    BBRT_CUDA(bbrt::noalloc_prepare());
    for (auto& e : s->ev) BBRT_CUDA(cudaEventCreate(&e));
    for (auto& e : s->kev) BBRT_CUDA(cudaEventCreate(&e));
    s->device_ready = true;
    return BBRT_OK;
}

// The patch tables every patch kernel reads (node counts, offsets, nodes and
// weights, node-major fields) and the coarse (u, v) values.
int upload_patch_tables(bbrt_scene* s) {
    if (s->tables_uploaded) return BBRT_OK;
    const bbrt::HostScene& H = s->host;
    bbrt::DScene& D = s->dev;
    std::vector<int> dims(2 * static_cast<size_t>(H.n_patches));
    for (int q = 0; q < H.n_patches; ++q) {
        dims[2 * q] = H.p_imax[q];
        dims[2 * q + 1] = H.p_jmax[q];
    }
    int rc;
    if ((rc = s->upload(dims, D.p_dims))) return rc;
    if ((rc = s->upload(H.p_node_off, D.p_node_off))) return rc;
    if ((rc = s->upload(H.p_field_off, D.p_field_off))) return rc;
    if ((rc = s->upload(H.p_nodes, D.p_nodes))) return rc;
    if ((rc = s->upload(H.p_fields, D.p_fields))) return rc;
    if ((rc = s->upload(H.coarse_uv, D.coarse_uv))) return rc;
    s->tables_uploaded = true;
    return BBRT_OK;
}

// The per-patch set-up of scene creation on the GPU (scene_compile.cu): the
// coarse grids, cell data and cull boxes stay in device memory; boxes,
// centroids and paddings come back for the host's BVH build, and the
// per-patch edge / coordinate bounds for the cull constants.
int device_setup(bbrt_scene* s) {
    int rc;
    if ((rc = ensure_device(s))) return rc;
    if ((rc = upload_patch_tables(s))) return rc;
    bbrt::HostScene& H = s->host;
    bbrt::DScene& D = s->dev;
    const int cn = H.coarse_n, nc = cn - 1, P = H.n_patches;
    bbrt::SetupArgs A;
    A.n_patches = P;
    A.cn = cn;
    A.coarse_uv = D.coarse_uv;
    A.dims = D.p_dims;
    A.node_off = D.p_node_off;
    A.field_off = D.p_field_off;
    A.nodes = D.p_nodes;
    A.fields = D.p_fields;
    const size_t per_xyz = 3 * static_cast<size_t>(cn) * cn, per_cell = 4 * static_cast<size_t>(nc) * nc;
    double *cx = nullptr, *cc = nullptr;
    if ((rc = s->alloc(per_xyz * P, cx))) return rc;
    if ((rc = s->alloc(per_cell * P, cc))) return rc;
    A.c_xyz = cx;
    A.c_cell = cc;
    DevBuf out, stats;
    BBRT_CUDA(out.ensure(sizeof(double) * 10 * std::max(P, 1)));
    A.patch_out = static_cast<double*>(out.p);
    const bool cull = H.cfg.cull && P > 0;
    int B = 4, NB = 0;
    if (cull) {
        B = std::max(4, static_cast<int>(std::ceil(std::sqrt(static_cast<double>(nc)))));
        NB = (nc + B - 1) / B;
        float *cb = nullptr, *bb = nullptr;
        if ((rc = s->alloc(static_cast<size_t>(P) * nc * nc * 6, cb))) return rc;
        if ((rc = s->alloc(static_cast<size_t>(P) * NB * NB * 6, bb))) return rc;
        A.cell_box = cb;
        A.block_box = bb;
        A.block_cells = B;
        A.n_blocks_side = NB;
        BBRT_CUDA(stats.ensure(sizeof(double) * 3 * P));
        A.cull_stats = static_cast<double*>(stats.p);
    }
    BBRT_CUDA(bbrt::launch_patch_setup(A, s->sm_count, s->stream));
    std::vector<double> po(10 * static_cast<size_t>(P)), cs(cull ? 3 * static_cast<size_t>(P) : 0);
    if (P > 0) BBRT_CUDA(cudaMemcpyAsync(po.data(), out.p, sizeof(double) * po.size(), cudaMemcpyDeviceToHost, s->stream));
    if (cull) BBRT_CUDA(cudaMemcpyAsync(cs.data(), stats.p, sizeof(double) * cs.size(), cudaMemcpyDeviceToHost, s->stream));
    BBRT_CUDA(cudaStreamSynchronize(s->stream));
    for (int q = 0; q < P; ++q) {
        const int k = H.patch_obj[q];
        std::memcpy(&H.box[6 * static_cast<size_t>(k)], &po[10 * static_cast<size_t>(q)], sizeof(double) * 6);
        std::memcpy(&H.centroid[3 * static_cast<size_t>(k)], &po[10 * static_cast<size_t>(q) + 6], sizeof(double) * 3);
        H.padding[k] = po[10 * static_cast<size_t>(q) + 9];
    }
    bbrt::finish_host_scene(H);
    D.c_xyz = cx;
    D.c_cell = cc;
    s->cull = bbrt::CullTables();
    if (cull) {
        double hmax = 0.0, cmax = 0.0;
        bool finite = true;
        for (int q = 0; q < P; ++q) {
            hmax = std::max(hmax, cs[3 * static_cast<size_t>(q)]);
            cmax = std::max(cmax, cs[3 * static_cast<size_t>(q) + 1]);
            finite = finite && cs[3 * static_cast<size_t>(q) + 2] != 0.0;
        }
        s->cull.block_cells = B;
        s->cull.n_blocks_side = NB;
        bbrt::cull_constants(H, hmax, cmax, finite, s->cull);
        D.c_cell_box = A.cell_box;
        D.c_block_box = A.block_box;
    }
    s->setup_on_device = true;
    return BBRT_OK;
}

// Per-axis bound on |coordinate| over a scene's node boxes for the FP32
// node test's error margin (rounded up to FP32, at least 2^-60); the FP32
// test is off for the scene when a bound exceeds 2^40 or a coordinate is
// not finite.
void node_bounds(const double* box, size_t n_values, bbrt::DScene& D) {
    double bound[3] = { std::ldexp(1.0, -60), std::ldexp(1.0, -60), std::ldexp(1.0, -60) };
    bool finite = true;
    for (size_t k = 0; k < n_values; ++k) {
        finite = finite && std::isfinite(box[k]);
        bound[k % 3] = std::max(bound[k % 3], std::fabs(box[k]));
    }
    D.node_f32_ok = finite ? 1 : 0;
    for (int a = 0; a < 3; ++a) {
        if (!(bound[a] <= std::ldexp(1.0, 40))) {
            D.node_f32_ok = 0;
            bound[a] = std::ldexp(1.0, 40);
        }
        float f = static_cast<float>(bound[a]);
        if (static_cast<double>(f) < bound[a]) f = std::nextafter(f, std::numeric_limits<float>::infinity());
        D.node_bound[a] = f;
    }
}

// Uploads a scene's BVH node tables: FP64 boxes and links, and the FP32
// boxes (nearest rounding) of the FP32 node test with their bounds.
int upload_node_tables(bbrt_scene* s, const std::vector<double>& nbox, const std::vector<int>& nlink) {
    bbrt::DScene& D = s->dev;
    int rc;
    if ((rc = s->upload(nbox, D.node_box))) return rc;
    if ((rc = s->upload(nlink, D.node_link))) return rc;
    const std::vector<float> box32(nbox.begin(), nbox.end());
    node_bounds(nbox.data(), nbox.size(), D);
    if ((rc = s->upload(box32, D.node_box32))) return rc;
    if (reinterpret_cast<uintptr_t>(D.node_box32) % 16 != 0)
        return fail(BBRT_ERR_CUDA, "bbrt_scene_upload: node box array not 16-byte aligned");
    return BBRT_OK;
}

int ensure_uploaded(bbrt_scene* s) {
    if (s->uploaded) return BBRT_OK;
    int rc0 = ensure_device(s);
    if (rc0) return rc0;
    if ((rc0 = upload_patch_tables(s))) return rc0;
    const bbrt::HostScene& H = s->host;
    bbrt::DScene& D = s->dev;
    D.n_objects = H.n_objects;
    D.n_nodes = static_cast<int>(H.nodes.size());
    D.coarse_n = H.coarse_n;
    D.newton_max_iters = H.cfg.newton_max_iters;
    D.newton_tol = H.cfg.newton_tol;
    D.scene_diagonal = H.scene_diagonal;
    D.max_patch_sagitta = H.max_patch_sagitta;
    D.eps_factor = H.cfg.self_intersect_eps_factor;
    D.sag_factor = H.cfg.sagitta_clearance_factor;
    D.backface_tol = H.cfg.backface_tol;
    // Renumber the depth-first tree breadth-first (children explicit), so the
    // top levels are the first nodes and can be staged in shared memory.
    const size_t nn = H.nodes.size();
    std::vector<int> bfs;
    bfs.reserve(nn);
    std::vector<int> newid(nn, -1);
    bfs.push_back(0);
    for (size_t h = 0; h < bfs.size(); ++h) {
        const bbrt::BvhNode& nd = H.nodes[bfs[h]];
        newid[bfs[h]] = static_cast<int>(h);
        if (nd.right >= 0) {
            bfs.push_back(bfs[h] + 1);   // left child follows its parent in the depth-first layout
            bfs.push_back(nd.right);
        }
    }
    std::vector<double> nbox(6 * nn);
    std::vector<int> nlink(4 * nn);
    for (size_t h = 0; h < nn; ++h) {
        const bbrt::BvhNode& nd = H.nodes[bfs[h]];
        std::memcpy(&nbox[6 * h], nd.box, sizeof(double) * 6);
        if (nd.right >= 0) {
            nlink[4 * h] = newid[bfs[h] + 1];
            nlink[4 * h + 1] = newid[nd.right];
            nlink[4 * h + 2] = 0;
            nlink[4 * h + 3] = nd.axis;
        } else {
            nlink[4 * h] = nd.start;
            nlink[4 * h + 1] = -1;
            nlink[4 * h + 2] = nd.count;
            nlink[4 * h + 3] = 0;
        }
    }
    // the traversal stack keeps a node index in 24 bits
    if (nn >= (static_cast<size_t>(1) << 24))
        return fail(BBRT_ERR_UNSUPPORTED, "bbrt_scene_upload: more than 16,777,215 BVH nodes");
    // up to 3400 nodes (64 bytes each, 217 KB) in shared memory; launch shapes
    // with several blocks per SM stage fewer
    D.smem_nodes = static_cast<int>(std::min<size_t>(nn, 3400));
    for (int q = 0; q < H.n_patches; ++q) D.max_nodes = std::max(D.max_nodes, std::max(H.p_imax[q], H.p_jmax[q]));
    int rc;
    if ((rc = upload_node_tables(s, nbox, nlink))) return rc;
    if ((rc = s->upload(H.leaf_objects, D.leaf_objects))) return rc;
    if ((rc = s->upload(H.kind, D.obj_kind))) return rc;
    if ((rc = s->upload(H.sub, D.obj_sub))) return rc;
    if ((rc = s->upload(H.padding, D.obj_pad))) return rc;
    {
        const std::vector<float> n32(H.p_nodes.begin(), H.p_nodes.end());
        const std::vector<float> f32(H.p_fields.begin(), H.p_fields.end());
        if ((rc = s->upload(n32, D.p_nodes32))) return rc;
        if ((rc = s->upload(f32, D.p_fields32))) return rc;
        // both Newton phases read a node's fields with 16-byte loads: every
        // node starts at a multiple of kFields values from an aligned base
        static_assert(bbrt::kFields % 4 == 0, "FP32 node records must be whole 16-byte units");
        if (reinterpret_cast<uintptr_t>(D.p_fields32) % 16 != 0 || reinterpret_cast<uintptr_t>(D.p_fields) % 16 != 0)
            return fail(BBRT_ERR_CUDA, "bbrt_scene_upload: field arrays not 16-byte aligned");
        const std::vector<double> fr = patch_frames(H);
        if ((rc = s->upload(fr, s->guess.frame))) return rc;
    }
    D.precision = H.cfg.precision;
    if (!s->setup_on_device) {
        if ((rc = s->upload(H.c_xyz, D.c_xyz))) return rc;
        if ((rc = s->upload(H.c_cell, D.c_cell))) return rc;
    }
    if ((rc = s->upload(H.tri, D.tri))) return rc;
    if (s->cull.enabled) {
        if (!s->setup_on_device) {
            if ((rc = s->upload(s->cull.cell_box, D.c_cell_box))) return rc;
            if ((rc = s->upload(s->cull.block_box, D.c_block_box))) return rc;
        }
        D.block_cells = s->cull.block_cells;
        D.n_blocks_side = s->cull.n_blocks_side;
        D.cull_enabled = 1;
        D.cull_a = s->cull.a;
        D.cull_h = s->cull.h;
        D.cull_b = s->cull.b;
        D.cull_coord = s->cull.coord;
        D.cull_radius = s->cull.radius;
        for (int a = 0; a < 3; ++a) D.cull_center[a] = s->cull.center[a];
    }
    // the kernels read node boxes, cell data and cull boxes with 8- and
    // 16-byte loads; every record starts at a whole multiple of 8 or 16 bytes
    // from its array's start, so the starts must be 16-byte aligned
    for (const void* p : std::initializer_list<const void*>{ D.node_box, D.c_cell, D.c_cell_box, D.c_block_box })
        if (reinterpret_cast<uintptr_t>(p) % 16 != 0)
            return fail(BBRT_ERR_CUDA, "bbrt_scene_upload: scene array not 16-byte aligned");
    BBRT_CUDA(s->stats.ensure(sizeof(long long) * bbrt::ST_COUNT));
    BBRT_CUDA(s->work.ensure(sizeof(unsigned long long)));
    s->uploaded = true;
    return BBRT_OK;
}

int create_scene(const bbrt_object_desc* objects, int n, const bbrt_config* cfg, bbrt_scene_t* out) {
    if (!out) return fail(BBRT_ERR_ARG, "bbrt_scene_create: out is NULL");
    *out = nullptr;
    bbrt_config c;
    bbrt_config_init(&c);
    if (cfg) c = *cfg;
    if (c.setup_on_device < -1 || c.setup_on_device > 1)
        return fail(BBRT_ERR_ARG, "bbrt_scene_create: setup_on_device must be -1, 0 or 1");
    bool on_device = c.setup_on_device == 1;
    if (c.setup_on_device == -1) {
        int ndev = 0;
        on_device = cudaGetDeviceCount(&ndev) == cudaSuccess && ndev > 0;
    }
    std::unique_ptr<bbrt_scene> s(new bbrt_scene());
    try {
        bbrt::build_host_tables(objects, n, c, s->host);
        if (s->host.n_patches == 0) on_device = false;   // triangles only: nothing to compile
        if (!on_device) {
            bbrt::setup_patches_host(objects, s->host);
            bbrt::finish_host_scene(s->host);
            bbrt::build_cull_tables(s->host, s->cull);
        }
    } catch (const std::invalid_argument& e) {
        return fail(BBRT_ERR_ARG, e.what());
    } catch (const std::runtime_error& e) {
        return fail(BBRT_ERR_FORMAT, e.what());
    } catch (const std::bad_alloc&) {
        return fail(BBRT_ERR_NOMEM, "bbrt_scene_create: out of host memory");
    }
    if (on_device) {
        int rc = BBRT_OK;
        try {
            rc = device_setup(s.get());
        } catch (const std::bad_alloc&) {
            return fail(BBRT_ERR_NOMEM, "bbrt_scene_create: out of host memory");
        }
        if (rc) return rc;
    }
    *out = s.release();
    return BBRT_OK;
}

// Reads a list of patch files and builds the scene from them.
int create_from_files(const std::vector<std::string>& paths, const bbrt_config* cfg, bbrt_scene_t* out) {
    std::vector<bbrt::PatchFileData> files(paths.size());
    try {
        for (size_t k = 0; k < paths.size(); ++k) bbrt::read_patch_file(paths[k], files[k]);
    } catch (const std::runtime_error& e) {
        const std::string m = e.what();
        return fail(m.find("cannot open") != std::string::npos ? BBRT_ERR_IO : BBRT_ERR_FORMAT, m);
    }
    std::vector<bbrt_patch_desc> pd(files.size());
    std::vector<bbrt_object_desc> od(files.size());
    for (size_t k = 0; k < files.size(); ++k) {
        pd[k] = bbrt::patch_desc_of(files[k]);
        od[k] = bbrt_object_desc{};
        od[k].kind = BBRT_OBJ_PATCH;
        od[k].patch = &pd[k];
    }
    return create_scene(od.data(), static_cast<int>(od.size()), cfg, out);
}

cudaStream_t pick_stream(bbrt_scene* s, void* stream) {
    return stream ? static_cast<cudaStream_t>(stream) : s->stream;
}

void fill_stats(bbrt_scene* s, const long long* st, long long n, float kernel_ms, float total_ms,
                bbrt_trace_stats* out) {
    std::memset(out, 0, sizeof *out);
    out->rays = n;
    out->bounces = st[bbrt::ST_BOUNCES];
    out->queries = st[bbrt::ST_QUERIES];
    out->node_tests = st[bbrt::ST_NODE_TESTS];
    out->patch_tests = st[bbrt::ST_PATCH_TESTS];
    out->cell_tests = st[bbrt::ST_CELL_TESTS];
    out->tri_tests = st[bbrt::ST_TRI_TESTS];
    out->newton_iters = st[bbrt::ST_NEWTON_ITERS];
    out->newton_iters_fp32 = st[bbrt::ST_NEWTON_ITERS_FP32];
    for (int k = 0; k < BBRT_RAY_STATUS_COUNT; ++k) out->status_hist[k] = st[bbrt::ST_HIST0 + k];
    out->kernel_ms = kernel_ms;
    out->total_ms = total_ms;
    out->tail_node_tests = st[bbrt::ST_TAIL_NODE_TESTS];
    out->tail_cell_tests = st[bbrt::ST_TAIL_CELL_TESTS];
    out->tail_tri_tests = st[bbrt::ST_TAIL_TRI_TESTS];
    out->tail_newton_iters = st[bbrt::ST_TAIL_NEWTON_ITERS];
    out->tail_rays = st[bbrt::ST_TAIL_RAYS];
    out->guess_used = st[bbrt::ST_GUESS_USED];
    out->guess_fallback = st[bbrt::ST_GUESS_FALLBACK];
    out->off_patch = st[bbrt::ST_OFF_PATCH];
    out->node_tests_fp64 = st[bbrt::ST_NODE_F64];
    double* dst[5] = { &out->order_ms, &out->advance_ms, &out->newton_ms, &out->tail_ms, &out->guess_ms };
    for (const auto& sp : s->kspans) {
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, s->kev[sp.second], s->kev[sp.second + 1]) == cudaSuccess) *dst[sp.first] += ms;
    }
    out->rounds = s->rounds;
    out->launches = s->launches;
}

enum { K_ORDER = 0, K_ADVANCE = 1, K_NEWTON = 2, K_TAIL = 3, K_GUESS = 4 };

// Records a pair of events around one launch when the call collects statistics.
template <class F>
cudaError_t timed(bbrt_scene* s, int kind, cudaStream_t st, F&& launch) {
    s->launches += (kind == K_ORDER) ? 4 : 1;   // ray ordering is four kernels
    if (!s->timing || s->kev_used + 2 > bbrt_scene::kTimerEvents) return launch();
    const int k = s->kev_used;
    cudaError_t e = cudaEventRecord(s->kev[k], st);
    if (e != cudaSuccess) return e;
    e = launch();
    if (e != cudaSuccess) return e;
    e = cudaEventRecord(s->kev[k + 1], st);
    if (e != cudaSuccess) return e;
    s->kspans.emplace_back(kind, k);
    s->kev_used += 2;
    return cudaSuccess;
}

// Batches at least this large run as a wavefront of advance / Newton rounds;
// smaller ones (and the last few rays of a wavefront) run one ray per thread
// to the end.
struct Tuning {
    long long wave_min_rays = 8192;   // smaller batches: one ray per thread to the end
    long long wave_tail = 4096;       // last requests finished one ray per warp
    int order_rays = 1;               // bucket rays by origin / direction before round 0
    int log_rounds = 0;               // print per-round counts and times to stderr
    int warp_tail = 1;                // finish the tail one warp per ray (else one thread per ray)
    int advance_shape = 3;            // k_advance launch shape (see launch_advance): 512 threads x 1 block per SM
    int warp_stage1 = 1;              // k_advance runs each patch's stage 1 with the whole warp
    int resume_queries = 1;           // suspended queries resume where they stopped (else replay from the root)
    int tail_shape = 0;               // k_resume_warp launch shape (see launch_resume_warp)
    int group_newton = 0;             // k_newton by 8-lane groups (exact, measured slower: off)
    int graph_rounds = 1;             // the rounds as one CUDA graph with a device-side loop
    int sort_requests = 1;            // group each round's Newton requests by patch before solving them
    int sort_side = 4;                // ... and within a patch by the side x side region of the stage-1 cell
    int order_entry = 1;              // round-0 order keyed on the scene-sphere entry point (else the origin)
    int child_test = -1;              // k_advance child tests: -1 when the BVH exceeds the staged nodes, 0 / 1
    int half_stage1 = 1;              // k_advance stage 1 of two patches at a time by half-warps
    int quarter_stage1 = 0;           // ... four at a time by quarter-warps
    int node_f32 = 1;                 // BVH nodes tested in FP32, FP64 where FP32 cannot decide (k_advance, tail)
    int adapt_lanes = 1;              // small k_advance rounds: fewer rays per warp, over every warp
    long long newton_group_max = 32768;  // smaller Newton rounds: 8 lanes per request
};

// Launch-shape knobs; defaults tuned on B200, overridable for experiments by
// the environment (BBRT_WAVE_MIN, BBRT_WAVE_TAIL, BBRT_ORDER_RAYS,
// BBRT_LOG_ROUNDS).  Read once per process.
const Tuning& tuning() {
    static const Tuning t = [] {
        Tuning v;
        if (const char* e = std::getenv("BBRT_WAVE_MIN")) v.wave_min_rays = std::atoll(e);
        if (const char* e = std::getenv("BBRT_WAVE_TAIL")) v.wave_tail = std::atoll(e);
        if (const char* e = std::getenv("BBRT_ORDER_RAYS")) v.order_rays = std::atoi(e);
        if (const char* e = std::getenv("BBRT_LOG_ROUNDS")) v.log_rounds = std::atoi(e);
        if (const char* e = std::getenv("BBRT_WARP_TAIL")) v.warp_tail = std::atoi(e);
        if (const char* e = std::getenv("BBRT_ADV_SHAPE")) v.advance_shape = std::atoi(e);
        if (const char* e = std::getenv("BBRT_WARP_S1")) v.warp_stage1 = std::atoi(e);
        if (const char* e = std::getenv("BBRT_RESUME")) v.resume_queries = std::atoi(e);
        if (const char* e = std::getenv("BBRT_TAIL_SHAPE")) v.tail_shape = std::atoi(e);
        if (const char* e = std::getenv("BBRT_GROUP_NEWTON")) v.group_newton = std::atoi(e);
        if (const char* e = std::getenv("BBRT_GRAPH")) v.graph_rounds = std::atoi(e);
        if (const char* e = std::getenv("BBRT_SORT_REQ")) v.sort_requests = std::atoi(e);
        if (const char* e = std::getenv("BBRT_SORT_SIDE")) v.sort_side = std::max(1, std::atoi(e));
        if (const char* e = std::getenv("BBRT_ORDER_ENTRY")) v.order_entry = std::atoi(e);
        if (const char* e = std::getenv("BBRT_CHILD_TEST")) v.child_test = std::atoi(e);
        if (const char* e = std::getenv("BBRT_HALF_S1")) v.half_stage1 = std::atoi(e);
        if (const char* e = std::getenv("BBRT_QUARTER_S1")) v.quarter_stage1 = std::atoi(e);
        if (const char* e = std::getenv("BBRT_NODE_F32")) v.node_f32 = std::atoi(e);
        if (const char* e = std::getenv("BBRT_ADAPT_LANES")) v.adapt_lanes = std::atoi(e);
        if (const char* e = std::getenv("BBRT_NEWTON_GROUP_MAX")) v.newton_group_max = std::atoll(e);
        return v;
    }();
    return t;
}

// Device view of a scene's network (parameters must be allocated).
bbrt::MlpNet guess_net(bbrt_scene* s) {
    bbrt::MlpNet M;
    M.image = static_cast<const uint8_t*>(s->guess.image.p);
    M.P = static_cast<float*>(s->guess.P.p);
    M.G = static_cast<float*>(s->guess.G.p);
    M.loss = static_cast<float*>(s->guess.loss.p);
    M.out = nullptr;
    M.err = static_cast<int*>(s->guess.err.p);
    M.mbar_limit = s->tune_set && s->tune.mma_wait_cycles > 0 ? s->tune.mma_wait_cycles : bbrt::kMbarDefault;
    return M;
}

// The wavefront trace: k_advance moves every runnable ray until its query
// meets a patch whose Newton solve is not yet known (or the ray finishes);
// k_newton solves all such requests; the rays that asked become the next
// round's runnable set.  Rounds end when no ray is waiting; a small last
// set, and rays whose query needed more solves than the resolved list holds,
// are finished by k_resume.
// Finishes the rays of `reqs` (or `rays`) from their saved state.
// The scene's schedule: its own once set or autotuned, else the library defaults.
bbrt_tuning scene_tuning(const bbrt_scene* s) {
    if (s->tune_set) return s->tune;
    const Tuning& T = tuning();
    bbrt_tuning t;
    t.advance_shape = T.advance_shape;
    t.warp_stage1 = T.warp_stage1;
    t.order_rays = T.order_rays;
    t.warp_tail = T.warp_tail;
    t.wave_tail = T.wave_tail;
    t.wave_min_rays = T.wave_min_rays;
    t.graph_rounds = T.graph_rounds;
    t.watchdog_cycles = 0;
    t.mma_wait_cycles = 0;
    return t;
}

// The k_advance watchdog and the tensor-core wait bound of a schedule
// (0 in the schedule: the defaults).
long long watchdog_cycles(const bbrt_tuning& T) { return T.watchdog_cycles > 0 ? T.watchdog_cycles : 1LL << 35; }
long long mma_wait_cycles(const bbrt_tuning& T) { return T.mma_wait_cycles > 0 ? T.mma_wait_cycles : bbrt::kMbarDefault; }

cudaError_t run_tail(bbrt_scene* s, const bbrt::TraceArgs& A, const bbrt::WaveArgs& W,
                     const bbrt::NewtonRequest* reqs, const int* rays, long long n, cudaStream_t st) {
    if (scene_tuning(s).warp_tail)
        return bbrt::launch_resume_warp(s->dev, A, W, reqs, rays, n, s->sm_count, tuning().tail_shape, st);
    return bbrt::launch_resume(s->dev, A, W, reqs, rays, n, st);
}

// Whether a round's Newton requests are grouped by patch before solving (one
// counting-sort bucket per object); the sort uses the ray-order workspace.
bool sort_round_requests(const bbrt_scene* s) {
    return tuning().sort_requests && s->host.n_objects >= 1 && s->host.n_objects <= bbrt::request_sort_max_objects();
}

// Round 0's processing order (s->order): rays bucketed by where they enter
// the scene's sphere; in a scene set, each member's rays among themselves
// in its own range, so that warps keep to one member's tree.
cudaError_t order_rays(bbrt_scene* s, const bbrt::TraceArgs& A, cudaStream_t st) {
    int* order = static_cast<int*>(s->order.p);
    const bool entry = tuning().order_entry != 0;
    if (s->member_rays.empty()) {
        const double radius = s->cull.radius > 0.0 ? s->cull.radius : s->host.scene_diagonal;
        return bbrt::ray_order(A.origins, A.dirs, A.n, s->cull.center, radius, s->order_ws.p, order, st, entry, 0);
    }
    for (size_t m = 0; m + 1 < s->member_rays.size(); ++m) {
        const long long off = s->member_rays[m], cnt = s->member_rays[m + 1] - off;
        if (cnt <= 0) continue;
        const double* sp = &s->member_sphere[4 * m];
        const cudaError_t e = bbrt::ray_order(A.origins + 3 * off, A.dirs + 3 * off, cnt, sp, sp[3], s->order_ws.p,
                                              order + off, st, entry, off);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// ---- the wavefront trace as one CUDA graph ------------------------------------

// Values a captured graph depends on, flattened (pointers and integers by
// value, doubles by bit pattern): a graph is reused only for an equal key.
struct GraphKey {
    std::vector<long long> v;
    template <class T>
    void put(T x) {
        if constexpr (std::is_pointer<T>::value) {
            v.push_back(static_cast<long long>(reinterpret_cast<intptr_t>(x)));
        } else if constexpr (std::is_floating_point<T>::value) {
            const double d = static_cast<double>(x);
            long long b = 0;
            std::memcpy(&b, &d, sizeof b);
            v.push_back(b);
        } else {
            v.push_back(static_cast<long long>(x));
        }
    }
};

// A launched graph-run of the wavefront: its kernel counts outside and inside the round loop.
struct GraphLaunch {
    bool on = false;
    long long fixed = 0, per_round = 0;
};

// Whether a graph-launched trace stopped on a device-side bound; sets the
// call's round and launch counts.  After the graph's work has completed.
int check_wave_graph(bbrt_scene* s, const GraphLaunch& g) {
    const unsigned int* c = s->wave_ctr_host;
    if (c[3]) return fail(BBRT_ERR_KERNEL, "bbrt_trace: a wavefront round ran past its watchdog and was stopped");
    if (c[bbrt::kWcBound]) return fail(BBRT_ERR_KERNEL, "bbrt_trace: wavefront round bound reached");
    s->rounds = 1 + static_cast<long long>(c[bbrt::kWcRounds]);
    s->launches = g.fixed + static_cast<long long>(c[bbrt::kWcRounds]) * g.per_round;
    return BBRT_OK;
}

// The wavefront trace captured as one graph:
//   [ray order] -> zero counters -> round 0 -> WHILE(loop) { round } -> tail -> overflow tail -> counters to host
// where a round is k_advance -> k_wave_decide -> [k_mlp_infer] -> k_newton.
// k_wave_decide takes the host loop's decision on the device (continue,
// hand the last small round to the tail, or stop) and sets the loop's
// condition, so no round waits for the host.  Every launch after round 0
// reads its item count from the counters; requests are written to req_a by
// k_advance and copied to req_b (the next round's runnable set) by k_newton.
int build_wave_graph(bbrt_scene* s, const bbrt::TraceArgs& A, const bbrt_tuning& T, bool learned,
                     long long max_rounds, bbrt_scene::WaveGraph& out) {
    for (auto& c : s->cap)
        if (!c) BBRT_CUDA(cudaStreamCreateWithFlags(&c, cudaStreamNonBlocking));
    const long long n = A.n;
    bbrt::WaveArgs W;
    bbrt::NewtonRequest *req_a = nullptr, *req_b = nullptr;
    bbrt::wave_layout(s->wave.p, n, W, req_a, req_b);
    unsigned int* c = static_cast<unsigned int*>(s->wave_ctr.p);
    W.counters = c;
    W.warp_stage1 = T.warp_stage1;
    W.resume_queries = tuning().resume_queries;
    W.child_test = tuning().child_test;
    W.half_stage1 = tuning().half_stage1;
    W.quarter_stage1 = tuning().quarter_stage1;
    W.node_f32 = tuning().node_f32;
    W.adapt_lanes = tuning().adapt_lanes;
    W.newton_group_max = tuning().newton_group_max;
    W.group_newton = tuning().group_newton;
    W.watchdog_cycles = watchdog_cycles(T);
    W.n_runnable = n;   // sizes the persistent grid; later rounds read their count
    if (T.order_rays) W.order = static_cast<const int*>(s->order.p);
    bbrt::WaveArgs W0 = W, Wr = W, Wn = W, Wt = W, Wo = W;
    W0.req = req_a;                        // round 0: every ray
    Wr.runnable = req_b;                   // later rounds: last round's requests
    Wr.req = req_a;
    Wr.count_dev = c + bbrt::kWcNext;
    // Newton solves req_b: the requests grouped by patch (sorted from req_a),
    // or copied there by k_newton itself as it solves them in place
    const bool sort = sort_round_requests(s);
    Wn.req = sort ? req_b : req_a;
    Wn.next_req = sort ? nullptr : req_b;
    Wn.count_dev = c + bbrt::kWcNext;
    double* gout = static_cast<double*>(s->guess.out.p);
    if (learned) {
        Wn.guess = gout;
        Wn.frame = s->guess.frame;
        Wn.guess_min_logit = s->guess.min_logit;
        Wn.guess_t_window = s->guess.t_window;
    }
    Wt.count_dev = c + bbrt::kWcTail;      // the last, small round's requests
    Wo.count_dev = c + 1;                  // rays that overflowed the resolved list
    const bbrt::MlpNet net = learned ? guess_net(s) : bbrt::MlpNet();
    auto round = [&](cudaStream_t q, const bbrt::WaveArgs& Wa, cudaGraphConditionalHandle loop) -> cudaError_t {
        cudaError_t e = bbrt::launch_advance(s->dev, A, Wa, s->sm_count, T.advance_shape, q);
        if (e == cudaSuccess) e = bbrt::launch_wave_decide(c, T.wave_tail, max_rounds, loop, q);
        if (e == cudaSuccess && sort)
            e = bbrt::sort_requests(req_a, n, c + bbrt::kWcNext, s->host.n_objects, tuning().sort_side,
                                    s->dev.coarse_n - 1, s->order_ws.p, req_b, q);
        if (e == cudaSuccess && learned)
            e = bbrt::mlp_infer_requests(Wn.req, n, W.o, W.d, s->dev.obj_sub, s->guess.frame, net, gout, q,
                                         c + bbrt::kWcNext);
        if (e == cudaSuccess) e = bbrt::launch_newton(s->dev, A, Wn, n, q);
        return e;
    };
    cudaStream_t cs = s->cap[0], cb = s->cap[1];
    BBRT_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed));
    cudaStreamCaptureStatus cst;
    cudaGraph_t cg = nullptr;
    cudaGraphConditionalHandle loop = 0;
    cudaError_t e = cudaStreamGetCaptureInfo(cs, &cst, nullptr, &cg, nullptr, nullptr);
    if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&loop, cg, 0, cudaGraphCondAssignDefault);
    if (e == cudaSuccess && T.order_rays) e = order_rays(s, A, cs);
    if (e == cudaSuccess) e = cudaMemsetAsync(c, 0, bbrt::kWaveCounters * sizeof(unsigned int), cs);
    if (e == cudaSuccess) e = round(cs, W0, loop);
    if (e == cudaSuccess) {
        const cudaGraphNode_t* deps = nullptr;
        size_t n_deps = 0;
        e = cudaStreamGetCaptureInfo(cs, &cst, nullptr, &cg, &deps, &n_deps);
        cudaGraphNodeParams cp = {};   // reserved fields zero
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = loop;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t cond = nullptr;
        if (e == cudaSuccess) e = cudaGraphAddNode(&cond, cg, deps, n_deps, &cp);
        if (e == cudaSuccess) e = cudaStreamUpdateCaptureDependencies(cs, &cond, 1, cudaStreamSetCaptureDependencies);
        if (e == cudaSuccess) {
            e = cudaStreamBeginCaptureToGraph(cb, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                              cudaStreamCaptureModeRelaxed);
            if (e == cudaSuccess) {
                cudaError_t eb = cudaMemsetAsync(c, 0, sizeof(unsigned int), cb);
                if (eb == cudaSuccess) eb = cudaMemsetAsync(c + 2, 0, sizeof(unsigned int), cb);
                if (eb == cudaSuccess) eb = round(cb, Wr, loop);
                cudaGraph_t body = nullptr;
                e = cudaStreamEndCapture(cb, &body);
                if (e == cudaSuccess) e = eb;
            }
        }
    }
    if (e == cudaSuccess) e = run_tail(s, A, Wt, req_a, nullptr, n, cs);
    if (e == cudaSuccess) e = run_tail(s, A, Wo, nullptr, W.overflow, n, cs);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(s->wave_ctr_host, c, bbrt::kWaveCounters * sizeof(unsigned int), cudaMemcpyDeviceToHost, cs);
    cudaGraph_t g = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(cs, &g);
    if (e == cudaSuccess) e = ee;
    cudaGraphExec_t x = nullptr;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&x, g, 0);
    if (e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return fail(BBRT_ERR_CUDA, std::string("bbrt_trace: wavefront graph: ") + cudaGetErrorString(e));
    }
    out.graph = g;
    out.exec = x;
    // advance, decide, [4 sort kernels], [infer], Newton
    const long long per_round = 3 + (learned ? 1 : 0) + (sort ? 4 : 0);
    out.launches_round = per_round;
    out.launches_fixed = (T.order_rays ? 4 : 0) + per_round + 2;
    return BBRT_OK;
}

// Launches the scene's graph for these arguments (captured on first use).
int launch_wave_graph(bbrt_scene* s, const bbrt::TraceArgs& A, const bbrt_tuning& T, cudaStream_t st,
                      GraphLaunch& used) {
    const long long n = A.n;
    const bool learned = s->host.cfg.guess == BBRT_GUESS_LEARNED && s->guess.trained;
    if (T.order_rays) {
        BBRT_CUDA(s->order_ws.ensure(bbrt::ray_order_workspace_bytes(n)));
        BBRT_CUDA(s->order.ensure(sizeof(int) * static_cast<size_t>(n)));
    }
    if (sort_round_requests(s)) BBRT_CUDA(s->order_ws.ensure(bbrt::ray_order_workspace_bytes(n)));
    if (learned) BBRT_CUDA(s->guess.out.ensure(sizeof(double) * 4 * static_cast<size_t>(n)));
    const long long max_rounds = 4 + static_cast<long long>(A.max_bounces + 1) * (s->host.n_objects + 1);
    GraphKey k;
    for (const void* p : std::initializer_list<const void*>{ static_cast<const void*>(A.origins), static_cast<const void*>(A.dirs),
                           static_cast<const void*>(A.status), static_cast<const void*>(A.bounce_count),
                           static_cast<const void*>(A.exit_dir), static_cast<const void*>(A.end_point),
                           static_cast<const void*>(A.hit_object), static_cast<const void*>(A.hit_point),
                           static_cast<const void*>(A.hit_uv), static_cast<const void*>(A.err_object),
                           static_cast<const void*>(A.err_value), static_cast<const void*>(A.ray_work),
                           static_cast<const void*>(A.hit_counts), static_cast<const void*>(A.stats),
                           static_cast<const void*>(A.work_counter), static_cast<const void*>(A.samples),
                           static_cast<const void*>(A.sample_count), s->wave.p, s->wave_ctr.p,
                           static_cast<const void*>(s->wave_ctr_host), s->order.p, s->order_ws.p, s->guess.out.p,
                           static_cast<const void*>(s->guess.frame), s->guess.image.p, s->guess.P.p,
                           s->guess.err.p })
        k.put(p);
    for (long long x : std::initializer_list<long long>{ A.n, static_cast<long long>(A.max_bounces), static_cast<long long>(A.record),
                         static_cast<long long>(A.cull), static_cast<long long>(A.count_from), A.sample_cap_pos,
                         A.sample_cap_neg, static_cast<long long>(s->dev.precision), static_cast<long long>(learned),
                         static_cast<long long>(T.advance_shape), static_cast<long long>(T.warp_stage1),
                         static_cast<long long>(T.order_rays), static_cast<long long>(T.warp_tail), T.wave_tail,
                         static_cast<long long>(tuning().resume_queries), static_cast<long long>(tuning().group_newton),
                         static_cast<long long>(tuning().tail_shape), static_cast<long long>(tuning().quarter_stage1),
                         static_cast<long long>(tuning().node_f32), static_cast<long long>(tuning().adapt_lanes),
                         tuning().newton_group_max, max_rounds,
                         static_cast<long long>(sort_round_requests(s)), watchdog_cycles(T), mma_wait_cycles(T),
                         static_cast<long long>(A.off_patch_miss) })
        k.put(x);
    k.put(s->guess.min_logit);
    k.put(s->guess.t_window);
    k.put(static_cast<const void*>(A.ray_member));
    for (long long r : s->member_rays) k.put(r);
    auto& gs = s->wgraphs;
    auto it = std::find_if(gs.begin(), gs.end(), [&](const bbrt_scene::WaveGraph& g) { return g.key == k.v; });
    if (it == gs.end()) {
        if (gs.size() == bbrt_scene::kWaveGraphs) {
            if (gs.front().exec) cudaGraphExecDestroy(gs.front().exec);
            if (gs.front().graph) cudaGraphDestroy(gs.front().graph);
            gs.erase(gs.begin());
        }
        bbrt_scene::WaveGraph g;
        const int rc = build_wave_graph(s, A, T, learned, max_rounds, g);
        if (rc) return rc;
        g.key = std::move(k.v);
        gs.push_back(std::move(g));
    } else if (it + 1 != gs.end()) {
        std::rotate(it, it + 1, gs.end());   // most recent last
    }
    used.on = true;
    used.fixed = gs.back().launches_fixed;
    used.per_round = gs.back().launches_round;
    BBRT_CUDA(cudaGraphLaunch(gs.back().exec, st));
    return BBRT_OK;
}

// One scene's wavefront trace as a resumable sequence, so that several
// scenes can advance round by round together (bbrt_trace_batch): begin()
// queues the ordering and round 0 and the readback of its counters; after
// that readback has completed, step() queues the next round (or the tail)
// until done; finish() runs the tail of rays that overflowed the resolved
// list.  run_wavefront() is the one-scene loop over the same steps.
struct WaveRun {
    bbrt_scene* s = nullptr;
    bbrt::TraceArgs A;
    cudaStream_t st = nullptr;
    bbrt_tuning T{};
    int log_rounds = 0;
    bbrt::WaveArgs W;
    bbrt::NewtonRequest *req_a = nullptr, *req_b = nullptr;
    long long round = 0, max_rounds = 0, overflowed = 0;
    bool done = false;
    GraphLaunch graph;   // graph-launched: check_wave_graph() after completion

    int begin(bbrt_scene* s_, const bbrt::TraceArgs& A_, cudaStream_t st_) {
        s = s_;
        A = A_;
        st = st_;
        const long long n = A.n;
        T = scene_tuning(s);
        log_rounds = tuning().log_rounds;
        BBRT_CUDA(s->wave.ensure(bbrt::wave_workspace_bytes(n)));
        BBRT_CUDA(s->wave_ctr.ensure(bbrt::kWaveCounters * sizeof(unsigned int)));
        if (!s->wave_ctr_host)
            BBRT_CUDA(cudaMallocHost(&s->wave_ctr_host, bbrt::kWaveCounters * sizeof(unsigned int)));
        if (T.graph_rounds) {
            done = true;
            return launch_wave_graph(s, A, T, st, graph);
        }
        bbrt::wave_layout(s->wave.p, n, W, req_a, req_b);
        if (sort_round_requests(s)) BBRT_CUDA(s->order_ws.ensure(bbrt::ray_order_workspace_bytes(n)));
        W.counters = static_cast<unsigned int*>(s->wave_ctr.p);
        W.warp_stage1 = T.warp_stage1;
        W.resume_queries = tuning().resume_queries;
        W.child_test = tuning().child_test;
        W.half_stage1 = tuning().half_stage1;
        W.quarter_stage1 = tuning().quarter_stage1;
        W.node_f32 = tuning().node_f32;
        W.adapt_lanes = tuning().adapt_lanes;
        W.newton_group_max = tuning().newton_group_max;
        W.group_newton = tuning().group_newton;
        W.watchdog_cycles = watchdog_cycles(T);
        W.runnable = nullptr;
        W.n_runnable = n;
        W.req = req_a;
        if (T.order_rays) {
            BBRT_CUDA(s->order_ws.ensure(bbrt::ray_order_workspace_bytes(n)));
            BBRT_CUDA(s->order.ensure(sizeof(int) * static_cast<size_t>(n)));
            BBRT_CUDA(timed(s, K_ORDER, st, [&] { return order_rays(s, A, st); }));
            W.order = static_cast<const int*>(s->order.p);
        }
        BBRT_CUDA(cudaMemsetAsync(W.counters, 0, bbrt::kWaveCounters * sizeof(unsigned int), st));
        // every round finishes at least one query or one Newton solve of each runnable ray
        max_rounds = 4 + static_cast<long long>(A.max_bounces + 1) * (s->host.n_objects + 1);
        return launch_round();
    }

    int launch_round() {
        if (log_rounds) BBRT_CUDA(cudaEventRecord(s->ev[2], st));
        BBRT_CUDA(cudaMemsetAsync(W.counters, 0, sizeof(unsigned int), st));
        BBRT_CUDA(cudaMemsetAsync(W.counters + 2, 0, sizeof(unsigned int), st));
        BBRT_CUDA(timed(s, K_ADVANCE, st,
                        [&] { return bbrt::launch_advance(s->dev, A, W, s->sm_count, T.advance_shape, st); }));
        ++s->rounds;
        if (log_rounds) BBRT_CUDA(cudaEventRecord(s->ev[3], st));
        BBRT_CUDA(cudaMemcpyAsync(s->wave_ctr_host, W.counters, 4 * sizeof(unsigned int), cudaMemcpyDeviceToHost, st));
        return BBRT_OK;
    }

    int step() {
        if (s->wave_ctr_host[3])
            return fail(BBRT_ERR_KERNEL, "bbrt_trace: a wavefront round ran past its watchdog and was stopped");
        const long long n_req = s->wave_ctr_host[0];
        overflowed = s->wave_ctr_host[1];
        if (log_rounds) {
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, s->ev[2], s->ev[3]);
            std::fprintf(stderr, "bbrt round %lld: runnable %lld advance %.3f ms -> requests %lld overflow %lld\n",
                         round, W.n_runnable, ms, n_req, overflowed);
        }
        if (n_req == 0) {
            done = true;
            return BBRT_OK;
        }
        if (n_req <= T.wave_tail) {
            BBRT_CUDA(timed(s, K_TAIL, st, [&] { return run_tail(s, A, W, W.req, nullptr, n_req, st); }));
            done = true;
            return BBRT_OK;
        }
        if (log_rounds) BBRT_CUDA(cudaEventRecord(s->ev[2], st));
        if (sort_round_requests(s)) {
            // group the requests by patch into the other list, which Newton
            // solves and the next round runs; the next requests go to this one
            bbrt::NewtonRequest* grouped = (W.req == req_a) ? req_b : req_a;
            BBRT_CUDA(timed(s, K_ORDER, st, [&] {
                return bbrt::sort_requests(W.req, n_req, nullptr, s->host.n_objects, tuning().sort_side,
                                           s->dev.coarse_n - 1, s->order_ws.p, grouped, st);
            }));
            W.req = grouped;
        }
        W.guess = nullptr;
        if (s->host.cfg.guess == BBRT_GUESS_LEARNED && s->guess.trained) {
            BBRT_CUDA(s->guess.out.ensure(sizeof(double) * 4 * static_cast<size_t>(n_req)));
            const bbrt::MlpNet net = guess_net(s);
            BBRT_CUDA(timed(s, K_GUESS, st, [&] {
                return bbrt::mlp_infer_requests(W.req, n_req, W.o, W.d, s->dev.obj_sub, s->guess.frame, net,
                                                static_cast<double*>(s->guess.out.p), st);
            }));
            W.guess = static_cast<const double*>(s->guess.out.p);
            W.frame = s->guess.frame;
            W.guess_min_logit = s->guess.min_logit;
            W.guess_t_window = s->guess.t_window;
        }
        BBRT_CUDA(timed(s, K_NEWTON, st, [&] { return bbrt::launch_newton(s->dev, A, W, n_req, st); }));
        if (log_rounds) {
            BBRT_CUDA(cudaEventRecord(s->ev[3], st));
            BBRT_CUDA(cudaEventSynchronize(s->ev[3]));
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, s->ev[2], s->ev[3]);
            std::fprintf(stderr, "bbrt round %lld: newton %.3f ms\n", round, ms);
        }
        W.runnable = W.req;
        W.n_runnable = n_req;
        W.req = (W.req == req_a) ? req_b : req_a;
        if (++round == max_rounds) return fail(BBRT_ERR_KERNEL, "bbrt_trace: wavefront round bound reached");
        return launch_round();
    }

    int finish() {
        if (graph.on) return BBRT_OK;   // the overflow tail is part of the graph
        if (overflowed > 0)
            BBRT_CUDA(timed(s, K_TAIL, st, [&] { return run_tail(s, A, W, nullptr, W.overflow, overflowed, st); }));
        return BBRT_OK;
    }
};

// `graph` describes a graph-launched trace (to be checked once its work has
// completed); graph.on is false for the host-driven rounds.
int run_wavefront(bbrt_scene* s, const bbrt::TraceArgs& A, cudaStream_t st, GraphLaunch& graph) {
    WaveRun w;
    int rc = w.begin(s, A, st);
    while (!rc && !w.done) {
        BBRT_CUDA(cudaStreamSynchronize(st));
        rc = w.step();
    }
    if (rc) return rc;
    graph = w.graph;
    return w.finish();
}

// Whether a trace of this scene runs the learned guess (its wavefront rounds do).
bool learned_trace(const bbrt_scene* s) {
    return s->host.cfg.guess == BBRT_GUESS_LEARNED && s->guess.trained && s->guess.err.p;
}

// Whether every tensor-core completion wait of a learned trace finished in
// time (the flag is cleared when the trace is prepared).  After the trace's
// work has completed.
int check_guess_waits(bbrt_scene* s, cudaStream_t st) {
    if (!learned_trace(s)) return BBRT_OK;
    int e = 0;
    BBRT_CUDA(cudaMemcpyAsync(&e, s->guess.err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    BBRT_CUDA(cudaStreamSynchronize(st));
    if (e) return fail(BBRT_ERR_KERNEL, "bbrt_trace: a tensor-core completion wait of the learned guess timed out");
    return BBRT_OK;
}

// Launches the trace kernel on device arrays.  hit_counts (device, may be
// null) receives per-object counts for bounces with index >= count_from.
// Trace arguments of one call and the per-call resets (statistics, ray
// counter, per-kernel timing); records the call's start event.
int prepare_trace(bbrt_scene* s, const double* d_o, const double* d_d, long long n, int max_bounces,
                  const bbrt_trace_out* out_dev, unsigned long long* hit_counts, int count_from, cudaStream_t st,
                  bool want_stats, bbrt::TraceArgs& A) {
    A = bbrt::TraceArgs();
    A.origins = d_o;
    A.dirs = d_d;
    A.n = n;
    A.max_bounces = max_bounces;
    A.cull = s->host.cfg.cull;
    if (out_dev) {
        A.record = out_dev->record_bounces;
        A.status = out_dev->status;
        A.bounce_count = out_dev->bounce_count;
        A.exit_dir = out_dev->exit_dir;
        A.end_point = out_dev->end_point;
        A.hit_object = out_dev->hit_object;
        A.hit_point = out_dev->hit_point;
        A.hit_uv = out_dev->hit_uv;
        A.err_object = out_dev->err_object;
        A.err_value = out_dev->err_value;
        A.ray_work = out_dev->ray_work;
    }
    if (A.record < 0) return fail(BBRT_ERR_ARG, "bbrt_trace: record_bounces < 0");
    A.hit_counts = hit_counts;
    A.count_from = count_from;
    A.stats = want_stats ? static_cast<long long*>(s->stats.p) : nullptr;
    A.work_counter = static_cast<unsigned long long*>(s->work.p);
    A.samples = s->rec_samples;
    A.sample_count = s->rec_count;
    A.sample_cap_pos = s->rec_cap_pos;
    A.sample_cap_neg = s->rec_cap_neg;
    A.ray_member = s->ray_member;
    if (want_stats) BBRT_CUDA(cudaMemsetAsync(s->stats.p, 0, sizeof(long long) * bbrt::ST_COUNT, st));
    BBRT_CUDA(cudaMemsetAsync(s->work.p, 0, sizeof(unsigned long long), st));
    if (learned_trace(s)) {
        BBRT_CUDA(cudaMemsetAsync(s->guess.err.p, 0, sizeof(int), st));
        A.off_patch_miss = 1;
    }
    s->timing = want_stats || s->time_kernels;
    s->kev_used = 0;
    s->kspans.clear();
    s->rounds = 0;
    s->launches = 0;
    BBRT_CUDA(cudaEventRecord(s->ev[0], st));
    return BBRT_OK;
}

// Records the call's end event and queues the statistics readback.
int complete_trace(bbrt_scene* s, cudaStream_t st, bool want_stats, long long* host_stats, float* kernel_ms) {
    BBRT_CUDA(cudaEventRecord(s->ev[1], st));
    if (want_stats) {
        BBRT_CUDA(cudaMemcpyAsync(host_stats, s->stats.p, sizeof(long long) * bbrt::ST_COUNT,
                                  cudaMemcpyDeviceToHost, st));
    }
    if (kernel_ms) {
        BBRT_CUDA(cudaEventSynchronize(s->ev[1]));
        BBRT_CUDA(cudaEventElapsedTime(kernel_ms, s->ev[0], s->ev[1]));
    }
    return BBRT_OK;
}

// Launches the trace kernel on device arrays.  hit_counts (device, may be
// null) receives per-object counts for bounces with index >= count_from.
int run_trace_device(bbrt_scene* s, const double* d_o, const double* d_d, long long n, int max_bounces,
                     const bbrt_trace_out* out_dev, unsigned long long* hit_counts, int count_from,
                     cudaStream_t st, bool want_stats, long long* host_stats, float* kernel_ms) {
    bbrt::TraceArgs A;
    int rc = prepare_trace(s, d_o, d_d, n, max_bounces, out_dev, hit_counts, count_from, st, want_stats, A);
    if (rc) return rc;
    GraphLaunch graph;
    if (n < scene_tuning(s).wave_min_rays) {
        BBRT_CUDA(timed(s, K_TAIL, st, [&] { return bbrt::launch_trace(s->dev, A, st, s->sm_count); }));
    } else {
        rc = run_wavefront(s, A, st, graph);
        if (rc) return rc;
    }
    rc = complete_trace(s, st, want_stats, host_stats, kernel_ms);
    if (!rc && graph.on) {
        // a graph-launched trace: one host wait, for its device-side bounds
        BBRT_CUDA(cudaEventSynchronize(s->ev[1]));
        rc = check_wave_graph(s, graph);
    }
    if (!rc && n >= scene_tuning(s).wave_min_rays) rc = check_guess_waits(s, st);
    return rc;
}

}  // namespace

extern "C" {

BBRT_API const char* bbrt_version(void) { return "bbrt-b200 0.1 (sm_100a)"; }

BBRT_API const char* bbrt_last_error(void) { return g_error.c_str(); }

BBRT_API void bbrt_config_init(bbrt_config* c) {
    if (!c) return;
    c->coarse_grid_n = 100;
    c->newton_max_iters = 20;
    c->newton_tol = 1e-3;
    c->leaf_threshold = 4;
    c->self_intersect_eps_factor = 1e-9;
    c->sagitta_clearance_factor = 5.0;
    c->backface_tol = 1e-9;
    c->precision = BBRT_PREC_FP64;
    c->guess = BBRT_GUESS_TRIANGLE;
    c->cull = 1;
    c->setup_on_device = -1;
}

BBRT_API int bbrt_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
    return n;
}

BBRT_API int bbrt_patch_file_read(const char* path, bbrt_patch_file* out) {
    if (!path || !out) return fail(BBRT_ERR_ARG, "bbrt_patch_file_read: NULL argument");
    std::memset(out, 0, sizeof *out);
    auto* d = new (std::nothrow) bbrt::PatchFileData();
    if (!d) return fail(BBRT_ERR_NOMEM, "bbrt_patch_file_read: out of memory");
    try {
        bbrt::read_patch_file(path, *d);
    } catch (const std::runtime_error& e) {
        delete d;
        const std::string m = e.what();
        return fail(m.find("cannot open") != std::string::npos ? BBRT_ERR_IO : BBRT_ERR_FORMAT, m);
    }
    out->desc = bbrt::patch_desc_of(*d);
    out->mask = d->mask.data();
    out->dS = d->f[9].data();
    for (int k = 0; k < 4; ++k) out->edge_flags[k] = d->edge_flags[k];
    out->storage_ = d;
    return BBRT_OK;
}

BBRT_API void bbrt_patch_file_free(bbrt_patch_file* f) {
    if (!f) return;
    delete static_cast<bbrt::PatchFileData*>(f->storage_);
    std::memset(f, 0, sizeof *f);
}

BBRT_API int bbrt_scene_create(const bbrt_object_desc* objects, int n_objects, const bbrt_config* cfg,
                               bbrt_scene_t* out) {
    return create_scene(objects, n_objects, cfg, out);
}

BBRT_API int bbrt_scene_create_from_dir(const char* directory, const bbrt_config* cfg, bbrt_scene_t* out) {
    namespace fs = std::filesystem;
    if (!directory || !out) return fail(BBRT_ERR_ARG, "bbrt_scene_create_from_dir: NULL argument");
    std::vector<fs::path> files;
    try {
        if (!fs::exists(directory) || !fs::is_directory(directory))
            return fail(BBRT_ERR_IO, std::string("RayTracingDriver: not a directory: ") + directory);
        for (const auto& entry : fs::directory_iterator(directory))
            if (entry.is_regular_file() && entry.path().extension() == ".txt") files.push_back(entry.path());
    } catch (const fs::filesystem_error& e) {
        return fail(BBRT_ERR_IO, e.what());
    }
    std::sort(files.begin(), files.end());
    if (files.empty())
        return fail(BBRT_ERR_IO, std::string("RayTracingDriver: no *.txt patch files found in: ") + directory);
    std::vector<std::string> paths;
    for (const auto& f : files) paths.push_back(f.string());
    return create_from_files(paths, cfg, out);
}

BBRT_API int bbrt_scene_create_from_range(const char* directory, const char* file_prefix, int first, int last,
                                          const bbrt_config* cfg, bbrt_scene_t* out) {
    if (!directory || !file_prefix || !out) return fail(BBRT_ERR_ARG, "bbrt_scene_create_from_range: NULL argument");
    if (last < first)
        return fail(BBRT_ERR_ARG, "RayTracingDriver: empty patch index range [" + std::to_string(first) + ", " +
                                      std::to_string(last) + "]");
    std::vector<std::string> paths;
    for (int i = first; i <= last; ++i) paths.push_back(std::string(directory) + file_prefix + std::to_string(i) + ".txt");
    return create_from_files(paths, cfg, out);
}

BBRT_API void bbrt_scene_destroy(bbrt_scene_t s) { delete s; }

BBRT_API int bbrt_scene_upload(bbrt_scene_t s) {
    if (!s) return fail(BBRT_ERR_ARG, "bbrt_scene_upload: NULL scene");
    std::lock_guard<std::mutex> g(s->mu);
    return ensure_uploaded(s);
}

BBRT_API int bbrt_scene_info_get(bbrt_scene_t s, bbrt_scene_info* out) {
    if (!s || !out) return fail(BBRT_ERR_ARG, "bbrt_scene_info_get: NULL argument");
    out->n_objects = s->host.n_objects;
    out->n_nodes = static_cast<int>(s->host.nodes.size());
    out->max_depth = s->host.max_depth;
    out->scene_diagonal = s->host.scene_diagonal;
    out->max_patch_sagitta = s->host.max_patch_sagitta;
    out->device_bytes = s->device_bytes;
    out->setup_on_device = s->setup_on_device ? 1 : 0;
    return BBRT_OK;
}

BBRT_API int bbrt_object_info_get(bbrt_scene_t s, int k, bbrt_object_info* out) {
    if (!s || !out) return fail(BBRT_ERR_ARG, "bbrt_object_info_get: NULL argument");
    if (k < 0 || k >= s->host.n_objects) return fail(BBRT_ERR_ARG, "bbrt_object_info_get: object out of range");
    const bbrt::HostScene& H = s->host;
    out->kind = H.kind[k];
    out->zone_id = H.zone[k];
    for (int a = 0; a < 3; ++a) {
        out->box_min[a] = H.box[6 * k + a];
        out->box_max[a] = H.box[6 * k + 3 + a];
        out->centroid[a] = H.centroid[3 * k + a];
    }
    out->padding = H.padding[k];
    return BBRT_OK;
}

BBRT_API int bbrt_patch_coarse_grid(bbrt_scene_t s, int k, int* n, double* u, double* v, double* xyz,
                                    double* sag, double* nrm) {
    if (!s) return fail(BBRT_ERR_ARG, "bbrt_patch_coarse_grid: NULL scene");
    const bbrt::HostScene& H = s->host;
    if (k < 0 || k >= H.n_objects || H.kind[k] != BBRT_OBJ_PATCH)
        return fail(BBRT_ERR_ARG, "bbrt_patch_coarse_grid: not a patch object");
    const int q = H.sub[k], cn = H.coarse_n, nc = cn - 1;
    if (n) *n = cn;
    if (u) std::memcpy(u, H.coarse_uv.data(), sizeof(double) * cn);
    if (v) std::memcpy(v, H.coarse_uv.data(), sizeof(double) * cn);
    const size_t per_xyz = 3 * static_cast<size_t>(cn) * cn, per_cell = 4 * static_cast<size_t>(nc) * nc;
    std::vector<double> dev_cell;
    const double* cc = nullptr;
    if (s->setup_on_device) {
        // the set-up lives on the GPU only
        std::lock_guard<std::mutex> g(s->mu);
        if (xyz) BBRT_CUDA(cudaMemcpy(xyz, s->dev.c_xyz + per_xyz * q, sizeof(double) * per_xyz, cudaMemcpyDeviceToHost));
        if (sag || nrm) {
            dev_cell.resize(per_cell);
            BBRT_CUDA(cudaMemcpy(dev_cell.data(), s->dev.c_cell + per_cell * q, sizeof(double) * per_cell,
                                 cudaMemcpyDeviceToHost));
            cc = dev_cell.data();
        }
    } else {
        if (xyz) std::memcpy(xyz, &H.c_xyz[per_xyz * q], sizeof(double) * per_xyz);
        cc = &H.c_cell[per_cell * q];
    }
    if (cc) for (int c = 0; c < nc * nc; ++c) {
        if (sag) sag[c] = cc[4 * c + 3];
        if (nrm) for (int a = 0; a < 3; ++a) nrm[3 * c + a] = cc[4 * c + a];
    }
    return BBRT_OK;
}

BBRT_API int bbrt_scene_setup_get(bbrt_scene_t s, int what, void* out, long long* count) {
    if (!s || !count) return fail(BBRT_ERR_ARG, "bbrt_scene_setup_get: NULL argument");
    const bbrt::HostScene& H = s->host;
    const bbrt::CullTables& Cu = s->cull;
    const long long P = H.n_patches, cn = H.coarse_n, nc = cn - 1;
    const long long nb = Cu.enabled ? Cu.n_blocks_side : 0;
    long long need = 0;
    size_t elem = sizeof(double);
    const void* host_src = nullptr;
    const void* dev_src = nullptr;
    double cull[11];
    switch (what) {
        case BBRT_SETUP_COARSE:
            need = P * cn * cn * 3;
            host_src = H.c_xyz.data();
            dev_src = s->dev.c_xyz;
            break;
        case BBRT_SETUP_CELLS:
            need = P * nc * nc * 4;
            host_src = H.c_cell.data();
            dev_src = s->dev.c_cell;
            break;
        case BBRT_SETUP_CELL_BOXES:
            need = Cu.enabled ? P * nc * nc * 6 : 0;
            elem = sizeof(float);
            host_src = Cu.cell_box.data();
            dev_src = s->dev.c_cell_box;
            break;
        case BBRT_SETUP_BLOCK_BOXES:
            need = P * nb * nb * 6;
            elem = sizeof(float);
            host_src = Cu.block_box.data();
            dev_src = s->dev.c_block_box;
            break;
        case BBRT_SETUP_CULL:
            need = 11;
            cull[0] = Cu.enabled ? 1.0 : 0.0;
            cull[1] = Cu.block_cells;
            cull[2] = static_cast<double>(nb);
            cull[3] = Cu.a; cull[4] = Cu.h; cull[5] = Cu.b; cull[6] = Cu.coord; cull[7] = Cu.radius;
            for (int a = 0; a < 3; ++a) cull[8 + a] = Cu.center[a];
            host_src = cull;
            dev_src = nullptr;
            break;
        default:
            return fail(BBRT_ERR_ARG, "bbrt_scene_setup_get: unknown array");
    }
    if (!out) {
        *count = need;
        return BBRT_OK;
    }
    if (*count != need) return fail(BBRT_ERR_ARG, "bbrt_scene_setup_get: count must be " + std::to_string(need));
    if (need == 0) return BBRT_OK;
    if (s->setup_on_device && dev_src) {
        std::lock_guard<std::mutex> g(s->mu);
        BBRT_CUDA(cudaMemcpy(out, dev_src, elem * static_cast<size_t>(need), cudaMemcpyDeviceToHost));
    } else {
        std::memcpy(out, host_src, elem * static_cast<size_t>(need));
    }
    return BBRT_OK;
}

BBRT_API int bbrt_self_intersect_epsilon(bbrt_scene_t s, int k, double* eps) {
    if (!s || !eps) return fail(BBRT_ERR_ARG, "bbrt_self_intersect_epsilon: NULL argument");
    const bbrt::HostScene& H = s->host;
    if (k >= H.n_objects) return fail(BBRT_ERR_ARG, "bbrt_self_intersect_epsilon: object out of range");
    const double pad = (k >= 0) ? H.padding[k] : H.max_patch_sagitta;
    const double a = H.cfg.self_intersect_eps_factor * H.scene_diagonal, b = H.cfg.sagitta_clearance_factor * pad;
    *eps = (a < b) ? b : a;
    return BBRT_OK;
}

BBRT_API int bbrt_intersect(bbrt_scene_t s, const double* origins, const double* dirs, long long n, int mode,
                            int object, int flags, bbrt_hit* out, void* stream) {
    if (!s || (n > 0 && (!origins || !dirs || !out))) return fail(BBRT_ERR_ARG, "bbrt_intersect: NULL argument");
    if (n < 0) return fail(BBRT_ERR_ARG, "bbrt_intersect: n < 0");
    if (mode < BBRT_QUERY_BVH || mode > BBRT_QUERY_OBJECT) return fail(BBRT_ERR_ARG, "bbrt_intersect: bad mode");
    if (mode == BBRT_QUERY_OBJECT && (object < 0 || object >= s->host.n_objects))
        return fail(BBRT_ERR_ARG, "bbrt_intersect: object out of range");
    std::lock_guard<std::mutex> g(s->mu);
    int rc = ensure_uploaded(s);
    if (rc) return rc;
    if (n == 0) return BBRT_OK;
    cudaStream_t st = pick_stream(s, stream);
    bbrt::QueryArgs Q;
    Q.n = n;
    Q.mode = mode;
    Q.object = object;
    Q.cull = s->host.cfg.cull;
    if (flags & BBRT_DEVICE_PTRS) {
        Q.origins = origins;
        Q.dirs = dirs;
        Q.out = out;
        BBRT_CUDA(bbrt::launch_query(s->dev, Q, st));
        return BBRT_OK;
    }
    const size_t vb = sizeof(double) * 3 * static_cast<size_t>(n);
    BBRT_CUDA(s->in_o.ensure(vb));
    BBRT_CUDA(s->in_d.ensure(vb));
    BBRT_CUDA(s->hits.ensure(sizeof(bbrt_hit) * static_cast<size_t>(n)));
    BBRT_CUDA(cudaMemcpyAsync(s->in_o.p, origins, vb, cudaMemcpyHostToDevice, st));
    BBRT_CUDA(cudaMemcpyAsync(s->in_d.p, dirs, vb, cudaMemcpyHostToDevice, st));
    Q.origins = static_cast<const double*>(s->in_o.p);
    Q.dirs = static_cast<const double*>(s->in_d.p);
    Q.out = s->hits.p;
    BBRT_CUDA(bbrt::launch_query(s->dev, Q, st));
    BBRT_CUDA(cudaMemcpyAsync(out, s->hits.p, sizeof(bbrt_hit) * static_cast<size_t>(n), cudaMemcpyDeviceToHost, st));
    BBRT_CUDA(cudaStreamSynchronize(st));
    return BBRT_OK;
}

BBRT_API int bbrt_trace(bbrt_scene_t s, const double* origins, const double* dirs, long long n, int max_bounces,
                        int flags, const bbrt_trace_out* out, bbrt_trace_stats* stats, void* stream) {
    if (!s) return fail(BBRT_ERR_ARG, "bbrt_trace: NULL scene");
    if (n < 0) return fail(BBRT_ERR_ARG, "bbrt_trace: n < 0");
    if (n > 0 && (!origins || !dirs)) return fail(BBRT_ERR_ARG, "bbrt_trace: NULL rays");
    if (max_bounces < 0) return fail(BBRT_ERR_ARG, "bbrt_trace: max_bounces < 0");
    if (out && out->record_bounces < 0) return fail(BBRT_ERR_ARG, "bbrt_trace: record_bounces < 0");
    std::lock_guard<std::mutex> g(s->mu);
    int rc = ensure_uploaded(s);
    if (rc) return rc;
    cudaStream_t st = pick_stream(s, stream);
    long long hs[bbrt::ST_COUNT] = { 0 };
    float kms = 0.0f;
    if (n == 0) {
        if (stats) fill_stats(s, hs, 0, 0.0f, 0.0f, stats);
        return BBRT_OK;
    }
    const bool counters = stats != nullptr && !(flags & BBRT_TIMES_ONLY);
    if (flags & BBRT_DEVICE_PTRS) {
        s->time_kernels = stats != nullptr;
        rc = run_trace_device(s, origins, dirs, n, max_bounces, out, nullptr, 1, st, counters, hs,
                              stats ? &kms : nullptr);
        s->time_kernels = false;
        if (rc) return rc;
        if (stats) {
            BBRT_CUDA(cudaStreamSynchronize(st));
            fill_stats(s, hs, n, kms, kms, stats);
        }
        return BBRT_OK;
    }
    // host arrays: stage through the scene's device buffers
    const size_t N = static_cast<size_t>(n), K = out ? static_cast<size_t>(out->record_bounces) : 0;
    BBRT_CUDA(cudaEventRecord(s->ev[2], st));
    BBRT_CUDA(s->in_o.ensure(sizeof(double) * 3 * N));
    BBRT_CUDA(s->in_d.ensure(sizeof(double) * 3 * N));
    BBRT_CUDA(cudaMemcpyAsync(s->in_o.p, origins, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, st));
    BBRT_CUDA(cudaMemcpyAsync(s->in_d.p, dirs, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, st));
    bbrt_trace_out dev{};
    struct Map { void* host; DevBuf* buf; size_t bytes; };
    std::vector<Map> maps;
    auto bind = [&](auto* host_ptr, DevBuf& b, size_t bytes, auto*& dev_field) -> int {
        using T = std::remove_pointer_t<std::remove_reference_t<decltype(dev_field)>>;
        if (!host_ptr || bytes == 0) { dev_field = nullptr; return BBRT_OK; }
        BBRT_CUDA(b.ensure(bytes));
        dev_field = static_cast<T*>(b.p);
        maps.push_back({ static_cast<void*>(host_ptr), &b, bytes });
        return BBRT_OK;
    };
    if (out) {
        dev.record_bounces = out->record_bounces;
        if ((rc = bind(out->status, s->o_status, sizeof(int) * N, dev.status))) return rc;
        if ((rc = bind(out->bounce_count, s->o_bounce, sizeof(int) * N, dev.bounce_count))) return rc;
        if ((rc = bind(out->exit_dir, s->o_dir, sizeof(double) * 3 * N, dev.exit_dir))) return rc;
        if ((rc = bind(out->end_point, s->o_end, sizeof(double) * 3 * N, dev.end_point))) return rc;
        if ((rc = bind(out->hit_object, s->o_hobj, sizeof(int) * N * K, dev.hit_object))) return rc;
        if ((rc = bind(out->hit_point, s->o_hpt, sizeof(double) * 3 * N * K, dev.hit_point))) return rc;
        if ((rc = bind(out->hit_uv, s->o_huv, sizeof(double) * 2 * N * K, dev.hit_uv))) return rc;
        if ((rc = bind(out->err_object, s->o_eobj, sizeof(int) * N, dev.err_object))) return rc;
        if ((rc = bind(out->err_value, s->o_eval, sizeof(double) * 2 * N, dev.err_value))) return rc;
        if ((rc = bind(out->ray_work, s->o_work, sizeof(long long) * 4 * N, dev.ray_work))) return rc;
    }
    s->time_kernels = stats != nullptr;
    rc = run_trace_device(s, static_cast<const double*>(s->in_o.p), static_cast<const double*>(s->in_d.p), n,
                          max_bounces, out ? &dev : nullptr, nullptr, 1, st, counters, hs, nullptr);
    s->time_kernels = false;
    if (rc) return rc;
    for (const Map& m : maps)
        BBRT_CUDA(cudaMemcpyAsync(m.host, m.buf->p, m.bytes, cudaMemcpyDeviceToHost, st));
    BBRT_CUDA(cudaEventRecord(s->ev[3], st));
    BBRT_CUDA(cudaStreamSynchronize(st));
    if (stats) {
        float tot = 0.0f;
        BBRT_CUDA(cudaEventElapsedTime(&kms, s->ev[0], s->ev[1]));
        BBRT_CUDA(cudaEventElapsedTime(&tot, s->ev[2], s->ev[3]));
        fill_stats(s, hs, n, kms, tot, stats);
    }
    return BBRT_OK;
}

BBRT_API int bbrt_plane_source(bbrt_scene_t s, const double c0[3], const double c1[3], const double dir[3], int nx,
                               int ny, int max_bounces, int count_direct_hit, long long* hit_counts,
                               bbrt_trace_stats* stats, void* stream) {
    if (!s || !c0 || !c1 || !dir || !hit_counts) return fail(BBRT_ERR_ARG, "bbrt_plane_source: NULL argument");
    if (nx < 1 || ny < 1) return fail(BBRT_ERR_ARG, "PlaneSourceDriver::run: nx and ny must both be >= 1");
    const double dl2 = dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2];
    if (dl2 < 1e-300) return fail(BBRT_ERR_ARG, "PlaneSourceDriver::run: direction has zero length");
    if (max_bounces < 0) return fail(BBRT_ERR_ARG, "bbrt_plane_source: max_bounces < 0");
    // build_plane_grid (PlaneSourceDriver.hpp:190-243)
    const double scale = std::max({ 1.0, std::fabs(c0[0]), std::fabs(c0[1]), std::fabs(c0[2]), std::fabs(c1[0]),
                                    std::fabs(c1[1]), std::fabs(c1[2]) });
    const double tol = 1e-9 * scale;
    int constant_axis = -1, matches = 0;
    for (int a = 0; a < 3; ++a)
        if (std::fabs(c0[a] - c1[a]) < tol) { constant_axis = a; ++matches; }
    if (matches != 1)
        return fail(BBRT_ERR_ARG,
                    "PlaneSourceDriver: corner0 and corner1 must agree in exactly one coordinate to define an "
                    "axis-aligned plane (got " + std::to_string(matches) + " matching coordinates)");
    int aa = -1, ab = -1;
    for (int a = 0; a < 3; ++a) {
        if (a == constant_axis) continue;
        if (aa < 0) aa = a; else ab = a;
    }
    const size_t N = static_cast<size_t>(nx) * ny;
    std::vector<double> src(3 * N), dirs(3 * N);
    std::vector<double> ga(nx), gb(ny);
    for (int i = 0; i < nx; ++i) ga[i] = (nx == 1) ? c0[aa] : c0[aa] + (c1[aa] - c0[aa]) * static_cast<double>(i) / (nx - 1);
    for (int j = 0; j < ny; ++j) gb[j] = (ny == 1) ? c0[ab] : c0[ab] + (c1[ab] - c0[ab]) * static_cast<double>(j) / (ny - 1);
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) {
            double* p = &src[3 * (static_cast<size_t>(i) * ny + j)];
            p[constant_axis] = c0[constant_axis];
            p[aa] = ga[i];
            p[ab] = gb[j];
        }
    for (size_t k = 0; k < N; ++k) { dirs[3 * k] = dir[0]; dirs[3 * k + 1] = dir[1]; dirs[3 * k + 2] = dir[2]; }
    std::lock_guard<std::mutex> g(s->mu);
    int rc = ensure_uploaded(s);
    if (rc) return rc;
    cudaStream_t st = pick_stream(s, stream);
    BBRT_CUDA(s->in_o.ensure(sizeof(double) * 3 * N));
    BBRT_CUDA(s->in_d.ensure(sizeof(double) * 3 * N));
    BBRT_CUDA(s->counts.ensure(sizeof(unsigned long long) * s->host.n_objects));
    BBRT_CUDA(cudaMemcpyAsync(s->in_o.p, src.data(), sizeof(double) * 3 * N, cudaMemcpyHostToDevice, st));
    BBRT_CUDA(cudaMemcpyAsync(s->in_d.p, dirs.data(), sizeof(double) * 3 * N, cudaMemcpyHostToDevice, st));
    BBRT_CUDA(cudaMemsetAsync(s->counts.p, 0, sizeof(unsigned long long) * s->host.n_objects, st));
    long long hs[bbrt::ST_COUNT] = { 0 };
    float kms = 0.0f;
    rc = run_trace_device(s, static_cast<const double*>(s->in_o.p), static_cast<const double*>(s->in_d.p),
                          static_cast<long long>(N), max_bounces, nullptr,
                          static_cast<unsigned long long*>(s->counts.p), count_direct_hit ? 0 : 1, st,
                          stats != nullptr, hs, stats ? &kms : nullptr);
    if (rc) return rc;
    std::vector<unsigned long long> c(s->host.n_objects);
    BBRT_CUDA(cudaMemcpyAsync(c.data(), s->counts.p, sizeof(unsigned long long) * c.size(), cudaMemcpyDeviceToHost, st));
    BBRT_CUDA(cudaStreamSynchronize(st));
    for (size_t k = 0; k < c.size(); ++k) hit_counts[k] = static_cast<long long>(c[k]);
    if (stats) fill_stats(s, hs, static_cast<long long>(N), kms, kms, stats);
    return BBRT_OK;
}

BBRT_API int bbrt_patch_sample_grid(const bbrt_patch_desc* p, int n, double* xyz, double* normal, double* dxdu) {
    if (!p || !xyz || !normal || !dxdu) return fail(BBRT_ERR_ARG, "bbrt_patch_sample_grid: NULL argument");
    if (n < 1) return fail(BBRT_ERR_ARG, "bbrt_patch_sample_grid: n must be >= 1");
    if (p->imax < 1 || p->jmax < 1) return fail(BBRT_ERR_ARG, "bbrt_patch_sample_grid: empty patch");
    bbrt::sample_grid(*p, n, xyz, normal, dxdu);
    return BBRT_OK;
}

// BounceMapDriver::run's validation (BounceMapDriver.hpp:103-117).
static int check_bounce_map_args(int grid_n, int theta_n, int phi_n, double cone_angle_deg) {
    if (grid_n < 2) return fail(BBRT_ERR_ARG, "BounceMapDriver::run: position_grid_n must be >= 2");
    if (theta_n < 1 || phi_n < 1) return fail(BBRT_ERR_ARG, "BounceMapDriver::run: theta_n and phi_n must both be >= 1");
    if (!(cone_angle_deg > 0.0) || cone_angle_deg > 180.0)
        return fail(BBRT_ERR_ARG, "BounceMapDriver::run: cone_angle_deg must be in (0, 180]");
    return BBRT_OK;
}

// Bounce-map launch rays on the host, in the reference's arithmetic
// (BounceMapDriver.hpp:119-237, build_tangent_frame :499-519).  Ray r is
// ((p * grid_n^2 + k) * theta_n + ti) * phi_n + pj for sample patch p, grid
// point k, polar index ti and azimuth index pj.  With idx == NULL all rays
// are written in that order (n must be their count); otherwise ray idx[i]
// goes to slot i.
// Direction tables of the sweep: mu[theta_n], sin(theta)[theta_n],
// cos(phi)[phi_n], sin(phi)[phi_n], in that order (host libm, as the reference).
static std::vector<double> bounce_trig(int theta_n, int phi_n, double cone_angle_deg) {
    const double kTwoPi = 6.283185307179586476925286766559;
    const double cos_max = std::cos(cone_angle_deg / 2.0 * kTwoPi / 360.0);
    std::vector<double> tab(2 * static_cast<size_t>(theta_n) + 2 * static_cast<size_t>(phi_n));
    double* mu = tab.data();
    double* sth = mu + theta_n;
    double* cphi = sth + theta_n;
    double* sphi = cphi + phi_n;
    for (int ti = 0; ti < theta_n; ++ti) {
        mu[ti] = cos_max + (static_cast<double>(ti) + 0.5) / static_cast<double>(theta_n) * (1.0 - cos_max);
        sth[ti] = std::sqrt(std::max(0.0, 1.0 - mu[ti] * mu[ti]));
    }
    for (int pj = 0; pj < phi_n; ++pj) {
        const double phi = (static_cast<double>(pj) + 0.5) * kTwoPi / static_cast<double>(phi_n);
        cphi[pj] = std::cos(phi);
        sphi[pj] = std::sin(phi);
    }
    return tab;
}

// Launch origin and frame (origin, t1, t2, n: 12 doubles) of every grid point
// of one sample patch, written to f[12 * per].
static void bounce_frame(const bbrt_scene* s, const bbrt_patch_desc& sample, int grid_n, double* f) {
    const long long per = static_cast<long long>(grid_n) * grid_n;
    bbrt::HostScene one;
    bbrt_object_desc od{};
    od.kind = BBRT_OBJ_PATCH;
    od.patch = &sample;
    bbrt::build_host_scene(&od, 1, s->host.cfg, one);
    const double a = s->host.cfg.self_intersect_eps_factor * s->host.scene_diagonal;
    const double b = s->host.cfg.sagitta_clearance_factor * one.padding[0];
    const double eps = (a < b) ? b : a;
    std::vector<double> xyz(3 * per), nrm(3 * per), du(3 * per);
    bbrt::sample_grid(sample, grid_n, xyz.data(), nrm.data(), du.data());
    for (long long k = 0; k < per; ++k) {
        const double* P = &xyz[3 * k];
        double n0 = nrm[3 * k], n1 = nrm[3 * k + 1], n2 = nrm[3 * k + 2];
        const double nl = std::sqrt(n0 * n0 + n1 * n1 + n2 * n2);
        n0 /= nl; n1 /= nl; n2 /= nl;
        const double d0 = du[3 * k], d1 = du[3 * k + 1], d2 = du[3 * k + 2];
        const double du2 = d0 * d0 + d1 * d1 + d2 * d2, dn = d0 * n0 + d1 * n1 + d2 * n2;
        const double q0 = d0 - dn * n0, q1 = d1 - dn * n1, q2 = d2 - dn * n2;
        const double qq = q0 * q0 + q1 * q1 + q2 * q2;
        double* F = f + 12 * k;
        double* t1 = F + 3;
        double* t2 = F + 6;
        if (qq > 1e-6 * 1e-6 * du2) {
            const double l = std::sqrt(q0 * q0 + q1 * q1 + q2 * q2);
            t1[0] = q0 / l; t1[1] = q1 / l; t1[2] = q2 / l;
        } else {
            double ax[3] = { 0, 0, 0 };
            if (std::fabs(n0) <= std::fabs(n1) && std::fabs(n0) <= std::fabs(n2)) ax[0] = 1.0;
            else if (std::fabs(n1) <= std::fabs(n2)) ax[1] = 1.0;
            else ax[2] = 1.0;
            const double c0v = n1 * ax[2] - n2 * ax[1], c1v = n2 * ax[0] - n0 * ax[2], c2v = n0 * ax[1] - n1 * ax[0];
            const double l = std::sqrt(c0v * c0v + c1v * c1v + c2v * c2v);
            t1[0] = c0v / l; t1[1] = c1v / l; t1[2] = c2v / l;
        }
        t2[0] = n1 * t1[2] - n2 * t1[1];
        t2[1] = n2 * t1[0] - n0 * t1[2];
        t2[2] = n0 * t1[1] - n1 * t1[0];
        F[0] = P[0] + n0 * eps; F[1] = P[1] + n1 * eps; F[2] = P[2] + n2 * eps;
        F[9] = n0; F[10] = n1; F[11] = n2;
    }
}

// Bounce-map launch rays on the host, in the reference's arithmetic
// (BounceMapDriver.hpp:119-237, build_tangent_frame :499-519).  Ray r is
// ((p * grid_n^2 + k) * theta_n + ti) * phi_n + pj for sample patch p, grid
// point k, polar index ti and azimuth index pj.  With idx == NULL all rays
// are written in that order (n must be their count); otherwise ray idx[i]
// goes to slot i.  (bbrt_bounce_map itself builds the rays on the device
// from the same frames and tables, k_bounce_rays.)
static void gen_bounce_rays(const bbrt_scene* s, const bbrt_patch_desc* samples, int n_sample, int grid_n, int theta_n,
                            int phi_n, double cone_angle_deg, const long long* idx, long long n, double* org,
                            double* dir) {
    const long long per = static_cast<long long>(grid_n) * grid_n, dirs_per = static_cast<long long>(theta_n) * phi_n;
    const std::vector<double> tab = bounce_trig(theta_n, phi_n, cone_angle_deg);
    const double* mu = tab.data();
    const double* sth = mu + theta_n;
    const double* cphi = sth + theta_n;
    const double* sphi = cphi + phi_n;
    // per sample patch, built on first use
    std::vector<std::vector<double>> frames(n_sample);
    auto frame_of = [&](int p) -> const std::vector<double>& {
        std::vector<double>& f = frames[p];
        if (f.empty()) {
            f.resize(12 * per);
            bounce_frame(s, samples[p], grid_n, f.data());
        }
        return f;
    };
    for (long long i = 0; i < n; ++i) {
        const long long r = idx ? idx[i] : i;
        const long long q = r / dirs_per, dk = r % dirs_per;
        const int p = static_cast<int>(q / per);
        const long long k = q % per;
        const int ti = static_cast<int>(dk / phi_n), pj = static_cast<int>(dk % phi_n);
        const double* F = &frame_of(p)[12 * k];
        const double *t1 = F + 3, *t2 = F + 6;
        const double n0 = F[9], n1 = F[10], n2 = F[11];
        org[3 * i] = F[0]; org[3 * i + 1] = F[1]; org[3 * i + 2] = F[2];
        const double st_ = sth[ti], m = mu[ti], cp = cphi[pj], sp = sphi[pj];
        dir[3 * i] = t1[0] * st_ * cp + t2[0] * st_ * sp + n0 * m;
        dir[3 * i + 1] = t1[1] * st_ * cp + t2[1] * st_ * sp + n1 * m;
        dir[3 * i + 2] = t1[2] * st_ * cp + t2[2] * st_ * sp + n2 * m;
    }
}

BBRT_API int bbrt_bounce_map_rays(bbrt_scene_t s, const bbrt_patch_desc* samples, int n_sample, int grid_n,
                                  int theta_n, int phi_n, double cone_angle_deg, const long long* ray_index,
                                  long long n, double* origins, double* dirs) {
    if (!s || !samples || !origins || !dirs) return fail(BBRT_ERR_ARG, "bbrt_bounce_map_rays: NULL argument");
    int rc = check_bounce_map_args(grid_n, theta_n, phi_n, cone_angle_deg);
    if (rc) return rc;
    if (n_sample < 1) return fail(BBRT_ERR_ARG, "bbrt_bounce_map_rays: no sample patches");
    const long long total = static_cast<long long>(n_sample) * grid_n * grid_n * theta_n * phi_n;
    if (n < 0 || (!ray_index && n != total))
        return fail(BBRT_ERR_ARG, "bbrt_bounce_map_rays: n must be the ray count (" + std::to_string(total) +
                                      ") when ray_index is NULL");
    if (ray_index)
        for (long long i = 0; i < n; ++i)
            if (ray_index[i] < 0 || ray_index[i] >= total)
                return fail(BBRT_ERR_ARG, "bbrt_bounce_map_rays: ray_index[" + std::to_string(i) + "] out of range");
    try {
        gen_bounce_rays(s, samples, n_sample, grid_n, theta_n, phi_n, cone_angle_deg, ray_index, n, origins, dirs);
    } catch (const std::exception& e) {
        return fail(BBRT_ERR_ARG, e.what());
    }
    return BBRT_OK;
}

BBRT_API int bbrt_bounce_map(bbrt_scene_t s, const bbrt_patch_desc* samples, int n_sample, int grid_n, int theta_n,
                             int phi_n, double cone_angle_deg, int max_bounces, int* max_out, int* err_out,
                             int* best_out, bbrt_trace_stats* stats, void* stream) {
    if (!s || !samples || !max_out || !err_out) return fail(BBRT_ERR_ARG, "bbrt_bounce_map: NULL argument");
    int rc0 = check_bounce_map_args(grid_n, theta_n, phi_n, cone_angle_deg);
    if (rc0) return rc0;
    if (n_sample < 1) return fail(BBRT_ERR_ARG, "bbrt_bounce_map: no sample patches");
    if (max_bounces < 0) return fail(BBRT_ERR_ARG, "bbrt_bounce_map: max_bounces < 0");
    const long long per = static_cast<long long>(grid_n) * grid_n, dirs_per = static_cast<long long>(theta_n) * phi_n;
    const long long points = static_cast<long long>(n_sample) * per;
    const long long N = points * dirs_per;
    // Host: the grid frames of the sample patches and the direction tables
    // (libm sin / cos, as the reference); device: every launch ray, the
    // trace, and the per-point reduction.
    std::vector<double> frames(12 * static_cast<size_t>(points));
    std::vector<double> tab;
    try {
        for (int p = 0; p < n_sample; ++p) bounce_frame(s, samples[p], grid_n, frames.data() + 12 * p * per);
        tab = bounce_trig(theta_n, phi_n, cone_angle_deg);
    } catch (const std::exception& e) {
        return fail(BBRT_ERR_ARG, e.what());
    }
    std::lock_guard<std::mutex> g(s->mu);
    int rc = ensure_uploaded(s);
    if (rc) return rc;
    cudaStream_t st = pick_stream(s, stream);
    const size_t fb = sizeof(double) * frames.size(), tb = sizeof(double) * tab.size();
    BBRT_CUDA(s->in_o.ensure(sizeof(double) * 3 * N));
    BBRT_CUDA(s->in_d.ensure(sizeof(double) * 3 * N));
    BBRT_CUDA(s->o_status.ensure(sizeof(int) * N));
    BBRT_CUDA(s->o_bounce.ensure(sizeof(int) * N));
    BBRT_CUDA(s->hits.ensure(fb + tb + 3 * sizeof(int) * static_cast<size_t>(points)));
    double* dframes = static_cast<double*>(s->hits.p);
    double* dtab = dframes + frames.size();
    int* dmax = reinterpret_cast<int*>(dtab + tab.size());
    int* derr = dmax + points;
    int* dbest = derr + points;
    BBRT_CUDA(cudaMemcpyAsync(dframes, frames.data(), fb, cudaMemcpyHostToDevice, st));
    BBRT_CUDA(cudaMemcpyAsync(dtab, tab.data(), tb, cudaMemcpyHostToDevice, st));
    double* dorg = static_cast<double*>(s->in_o.p);
    double* ddir = static_cast<double*>(s->in_d.p);
    BBRT_CUDA(bbrt::launch_bounce_rays(dframes, dtab, theta_n, phi_n, N, dorg, ddir, st));
    bbrt_trace_out o{};
    o.status = static_cast<int*>(s->o_status.p);
    o.bounce_count = static_cast<int*>(s->o_bounce.p);
    long long hs[bbrt::ST_COUNT] = { 0 };
    float kms = 0.0f;
    rc = run_trace_device(s, dorg, ddir, N, max_bounces, &o, nullptr, 1, st, stats != nullptr, hs,
                          stats ? &kms : nullptr);
    if (rc) return rc;
    BBRT_CUDA(bbrt::launch_bounce_reduce(o.status, o.bounce_count, points, static_cast<int>(dirs_per), dmax, derr,
                                         dbest, st));
    BBRT_CUDA(cudaMemcpyAsync(max_out, dmax, sizeof(int) * points, cudaMemcpyDeviceToHost, st));
    BBRT_CUDA(cudaMemcpyAsync(err_out, derr, sizeof(int) * points, cudaMemcpyDeviceToHost, st));
    if (best_out) BBRT_CUDA(cudaMemcpyAsync(best_out, dbest, sizeof(int) * points, cudaMemcpyDeviceToHost, st));
    BBRT_CUDA(cudaStreamSynchronize(st));
    if (stats) fill_stats(s, hs, N, kms, kms, stats);
    return BBRT_OK;
}

// Allocation-free trace: scratch in the library's static device array (see
// include/bbrt.h).  No cudaMalloc / cudaFree / event or stream creation here.
BBRT_API int bbrt_trace_noalloc(bbrt_scene_t s, const double* origins, const double* dirs, long long n,
                                int max_bounces, const bbrt_trace_out* out, long long* hit_counts,
                                int count_from, bbrt_trace_stats* stats, void* stream) {
    if (!s) return fail(BBRT_ERR_ARG, "bbrt_trace_noalloc: NULL scene");
    if (n < 0) return fail(BBRT_ERR_ARG, "bbrt_trace_noalloc: n < 0");
    if (n > 0 && (!origins || !dirs)) return fail(BBRT_ERR_ARG, "bbrt_trace_noalloc: NULL rays");
    if (max_bounces < 0) return fail(BBRT_ERR_ARG, "bbrt_trace_noalloc: max_bounces < 0");
    if (out && out->record_bounces < 0) return fail(BBRT_ERR_ARG, "bbrt_trace_noalloc: record_bounces < 0");
    if (hit_counts && s->host.n_objects > BBRT_NOALLOC_MAX_OBJECTS)
        return fail(BBRT_ERR_ARG, "bbrt_trace_noalloc: hit counts need a scene of at most " +
                                      std::to_string(BBRT_NOALLOC_MAX_OBJECTS) + " objects (this one has " +
                                      std::to_string(s->host.n_objects) + ")");
    std::lock_guard<std::mutex> g(s->mu);
    if (!s->uploaded)
        return fail(BBRT_ERR_STATE, "bbrt_trace_noalloc: the scene is not on the device yet (bbrt_scene_upload)");
    int dev = -1;
    BBRT_CUDA(cudaGetDevice(&dev));
    if (dev != s->device)
        return fail(BBRT_ERR_STATE, "bbrt_trace_noalloc: the current device is not the scene's device");
    cudaStream_t st = pick_stream(s, stream);
    long long hs[bbrt::ST_COUNT] = { 0 };
    s->kspans.clear();   // no per-kernel timing here (keeps capacity: no allocation)
    s->rounds = 0;
    s->launches = n > 0 ? 1 : 0;
    if (n > 0) {
        bbrt::TraceArgs A;
        A.origins = origins;
        A.dirs = dirs;
        A.n = n;
        A.max_bounces = max_bounces;
        A.cull = s->host.cfg.cull;
        if (out) {
            A.record = out->record_bounces;
            A.status = out->status;
            A.bounce_count = out->bounce_count;
            A.exit_dir = out->exit_dir;
            A.end_point = out->end_point;
            A.hit_object = out->hit_object;
            A.hit_point = out->hit_point;
            A.hit_uv = out->hit_uv;
            A.err_object = out->err_object;
            A.err_value = out->err_value;
            A.ray_work = out->ray_work;
        }
        A.count_from = count_from;
        BBRT_CUDA(bbrt::launch_trace_noalloc(s->dev, A, hit_counts != nullptr, hit_counts, stats ? hs : nullptr, st,
                                             s->sm_count));
    } else if (hit_counts) {
        BBRT_CUDA(cudaMemsetAsync(hit_counts, 0, sizeof(long long) * s->host.n_objects, st));
    }
    if (stats) fill_stats(s, hs, n, 0.0f, 0.0f, stats);
    return BBRT_OK;
}

}  // extern "C"

// Tensor-core layout self-check (diagnostic): four staged forms of one product.
BBRT_API int bbrt_umma_check(const uint16_t* a, const uint16_t* b, float* d) {
    if (!a || !b || !d) return fail(BBRT_ERR_ARG, "bbrt_umma_check: NULL argument");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0)
        return fail(BBRT_ERR_CUDA, "bbrt: no CUDA device available (the trace path has no CPU fallback)");
    uint16_t *da = nullptr, *db = nullptr;
    float* dd = nullptr;
    int* de = nullptr;
    const size_t nab = 128 * 64 * sizeof(uint16_t), nd = 4 * 128 * 128 * sizeof(float);
    auto cleanup = [&]() { cudaFree(da); cudaFree(db); cudaFree(dd); cudaFree(de); };
    if (cudaMalloc(&da, nab) != cudaSuccess || cudaMalloc(&db, nab) != cudaSuccess ||
        cudaMalloc(&dd, nd) != cudaSuccess || cudaMalloc(&de, sizeof(int)) != cudaSuccess) {
        cleanup();
        return fail(BBRT_ERR_CUDA, "bbrt_umma_check: cudaMalloc failed");
    }
    int herr = 0;
    cudaMemcpy(da, a, nab, cudaMemcpyHostToDevice);
    cudaMemcpy(db, b, nab, cudaMemcpyHostToDevice);
    cudaMemset(dd, 0, nd);
    cudaMemset(de, 0, sizeof(int));
    const int rc = bbrt::launch_umma_check(da, db, dd, de, nullptr);
    cudaError_t e = cudaDeviceSynchronize();
    if (rc == 0 && e == cudaSuccess) {
        cudaMemcpy(d, dd, nd, cudaMemcpyDeviceToHost);
        cudaMemcpy(&herr, de, sizeof(int), cudaMemcpyDeviceToHost);
    }
    cleanup();
    if (rc != 0 || e != cudaSuccess)
        return fail(BBRT_ERR_CUDA, std::string("bbrt_umma_check: ") + cudaGetErrorString(rc ? cudaError_t(rc) : e));
    if (herr) return fail(BBRT_ERR_KERNEL, "bbrt_umma_check: an MMA completion wait timed out");
    return BBRT_OK;
}

BBRT_API int bbrt_node_test_check(const double* o, const double* d, const double* best_t, long long n,
                                  const double* boxes, int* out) {
    if (n < 0 || (n > 0 && (!o || !d || !best_t || !boxes || !out)))
        return fail(BBRT_ERR_ARG, "bbrt_node_test_check: NULL argument or negative count");
    if (n == 0) return BBRT_OK;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0)
        return fail(BBRT_ERR_CUDA, "bbrt: no CUDA device available (the trace path has no CPU fallback)");
    bbrt::DScene S;
    node_bounds(boxes, static_cast<size_t>(6 * n), S);
    const size_t n3 = sizeof(double) * 3 * n, n1 = sizeof(double) * n, n6 = sizeof(double) * 6 * n,
                 no = sizeof(int) * 2 * n;
    DevBuf bo, bd, bb, bx, bout;
    if (bo.ensure(n3) || bd.ensure(n3) || bb.ensure(n1) || bx.ensure(n6) || bout.ensure(no))
        return fail(BBRT_ERR_CUDA, "bbrt_node_test_check: cudaMalloc failed");
    cudaError_t e = cudaMemcpy(bo.p, o, n3, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(bd.p, d, n3, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(bb.p, best_t, n1, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(bx.p, boxes, n6, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = bbrt::launch_node_check(S, static_cast<const double*>(bo.p), static_cast<const double*>(bd.p),
                                    static_cast<const double*>(bb.p), n, static_cast<const double*>(bx.p),
                                    static_cast<int*>(bout.p), nullptr);
    if (e == cudaSuccess) e = cudaMemcpy(out, bout.p, no, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return fail(BBRT_ERR_CUDA, std::string("bbrt_node_test_check: ") + cudaGetErrorString(e));
    return BBRT_OK;
}

// ---- arithmetic modes and the learned guess --------------------------------

BBRT_API int bbrt_scene_set_modes(bbrt_scene_t s, int precision, int guess) {
    if (!s) return fail(BBRT_ERR_ARG, "bbrt_scene_set_modes: NULL scene");
    if (precision != BBRT_PREC_FP64 && precision != BBRT_PREC_SPLIT)
        return fail(BBRT_ERR_ARG, "bbrt_scene_set_modes: unknown precision");
    if (guess != BBRT_GUESS_TRIANGLE && guess != BBRT_GUESS_LEARNED)
        return fail(BBRT_ERR_ARG, "bbrt_scene_set_modes: unknown guess");
    std::lock_guard<std::mutex> g(s->mu);
    s->host.cfg.precision = precision;
    s->host.cfg.guess = guess;
    s->dev.precision = precision;
    return BBRT_OK;
}

BBRT_API void bbrt_guess_train_config_init(bbrt_guess_train_config* c) {
    if (!c) return;
    c->epochs = 8;
    c->batch = 65536;
    c->lr = 1e-3f;
    c->max_positive = 4LL << 20;
    c->max_negative = 1LL << 20;
    c->seed = 1;
    c->min_logit = 0.0;
    c->t_window = 0.5;
}

BBRT_API long long bbrt_guess_param_count(bbrt_scene_t s) {
    if (!s) return 0;
    return bbrt::oE + static_cast<long long>(bbrt::kEmb) * s->host.n_patches;
}

namespace {

// Scaled-uniform weights, zero biases, N(0, 0.1) embeddings; the padded
// inputs (>= 41) and outputs (>= 4) start, and stay, at zero.
std::vector<float> init_network(long long n_params, unsigned long long seed) {
    std::vector<float> P(static_cast<size_t>(n_params), 0.0f);
    std::mt19937_64 rng(seed);
    auto fill = [&](int off, int rows, int cols, int used_rows, int used_cols, int fan_in) {
        const double lim = std::sqrt(6.0 / (fan_in + rows));
        std::uniform_real_distribution<double> U(-lim, lim);
        for (int o = 0; o < rows; ++o)
            for (int i = 0; i < cols; ++i)
                P[off + o * cols + i] = (o < used_rows && i < used_cols) ? static_cast<float>(U(rng)) : 0.0f;
    };
    fill(bbrt::oW0, bbrt::kH, bbrt::kIn, bbrt::kH, bbrt::kGeo + bbrt::kEmb, bbrt::kGeo + bbrt::kEmb);
    fill(bbrt::oW1, bbrt::kH, bbrt::kH, bbrt::kH, bbrt::kH, bbrt::kH);
    fill(bbrt::oW2, bbrt::kH, bbrt::kH, bbrt::kH, bbrt::kH, bbrt::kH);
    fill(bbrt::oW3, bbrt::kOut, bbrt::kH, 4, bbrt::kH, bbrt::kH);
    std::normal_distribution<double> N(0.0, 0.1);
    for (long long k = bbrt::oE; k < n_params; ++k) P[k] = static_cast<float>(N(rng));
    return P;
}

// Allocates the network buffers of a scene for n_params parameters.
int guess_alloc(bbrt_scene* s, long long n_params) {
    const size_t fb = sizeof(float) * static_cast<size_t>(n_params);
    BBRT_CUDA(s->guess.P.ensure(fb));
    BBRT_CUDA(s->guess.G.ensure(fb));
    BBRT_CUDA(s->guess.m1.ensure(fb));
    BBRT_CUDA(s->guess.m2.ensure(fb));
    BBRT_CUDA(s->guess.image.ensure(bbrt::kImageBytes));
    BBRT_CUDA(s->guess.err.ensure(sizeof(int)));
    return BBRT_OK;
}

int guess_err_check(bbrt_scene* s, cudaStream_t st) {
    int e = 0;
    BBRT_CUDA(cudaMemcpyAsync(&e, s->guess.err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    BBRT_CUDA(cudaStreamSynchronize(st));
    if (e) return fail(BBRT_ERR_KERNEL, "bbrt_guess: a tensor-core completion wait timed out");
    return BBRT_OK;
}

}  // namespace

BBRT_API int bbrt_guess_params(bbrt_scene_t s, float* params, long long n, int set) {
    if (!s || !params) return fail(BBRT_ERR_ARG, "bbrt_guess_params: NULL argument");
    const long long np = bbrt_guess_param_count(s);
    if (n != np) return fail(BBRT_ERR_ARG, "bbrt_guess_params: n must be " + std::to_string(np));
    std::lock_guard<std::mutex> g(s->mu);
    int rc = ensure_uploaded(s);
    if (rc) return rc;
    cudaStream_t st = s->stream;
    if (!set) {
        if (!s->guess.trained) return fail(BBRT_ERR_STATE, "bbrt_guess_params: the scene has no trained network");
        BBRT_CUDA(cudaMemcpyAsync(params, s->guess.P.p, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
        BBRT_CUDA(cudaStreamSynchronize(st));
        return BBRT_OK;
    }
    if ((rc = guess_alloc(s, np))) return rc;
    BBRT_CUDA(cudaMemcpyAsync(s->guess.P.p, params, sizeof(float) * n, cudaMemcpyHostToDevice, st));
    BBRT_CUDA(cudaMemsetAsync(s->guess.m1.p, 0, sizeof(float) * n, st));
    BBRT_CUDA(cudaMemsetAsync(s->guess.m2.p, 0, sizeof(float) * n, st));
    BBRT_CUDA(bbrt::mlp_pack(static_cast<const float*>(s->guess.P.p), static_cast<uint8_t*>(s->guess.image.p), st));
    BBRT_CUDA(cudaStreamSynchronize(st));
    s->guess.trained = true;
    return BBRT_OK;
}

namespace {
int guess_train_core(bbrt_scene* s, const double* d_o, const double* d_d, long long n, int max_bounces,
                     const bbrt_guess_train_config& cfg, bbrt_guess_train_report* rep, cudaStream_t st);
}  // namespace

BBRT_API int bbrt_guess_train(bbrt_scene_t s, const double* origins, const double* dirs, long long n, int max_bounces,
                              const bbrt_guess_train_config* cfg_in, bbrt_guess_train_report* rep, void* stream) {
    if (!s || !origins || !dirs) return fail(BBRT_ERR_ARG, "bbrt_guess_train: NULL argument");
    if (n <= 0) return fail(BBRT_ERR_ARG, "bbrt_guess_train: no rays");
    if (max_bounces < 0) return fail(BBRT_ERR_ARG, "bbrt_guess_train: max_bounces < 0");
    bbrt_guess_train_config cfg;
    bbrt_guess_train_config_init(&cfg);
    if (cfg_in) cfg = *cfg_in;
    if (cfg.epochs < 1 || cfg.batch < 128 || cfg.max_positive < 1 || cfg.max_negative < 0 || !(cfg.lr > 0.0f))
        return fail(BBRT_ERR_ARG, "bbrt_guess_train: bad training configuration");
    std::lock_guard<std::mutex> g(s->mu);
    int rc = ensure_uploaded(s);
    if (rc) return rc;
    if (s->host.n_patches == 0) return fail(BBRT_ERR_ARG, "bbrt_guess_train: the scene has no patches");
    cudaStream_t st = pick_stream(s, stream);
    BBRT_CUDA(s->in_o.ensure(sizeof(double) * 3 * n));
    BBRT_CUDA(s->in_d.ensure(sizeof(double) * 3 * n));
    BBRT_CUDA(cudaMemcpyAsync(s->in_o.p, origins, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, st));
    BBRT_CUDA(cudaMemcpyAsync(s->in_d.p, dirs, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, st));
    return guess_train_core(s, static_cast<const double*>(s->in_o.p), static_cast<const double*>(s->in_d.p), n,
                            max_bounces, cfg, rep, st);
}

namespace {

// The training of bbrt_guess_train on device rays (scene locked and on the
// device): samples from a plain FP64 trace of the rays, then Adam epochs.
int guess_train_core(bbrt_scene* s, const double* d_o, const double* d_d, long long n, int max_bounces,
                     const bbrt_guess_train_config& cfg, bbrt_guess_train_report* rep, cudaStream_t st) {
    int rc = BBRT_OK;
    // ---- 1. samples from a plain FP64 trace of the rays
    const long long cap_p = cfg.max_positive, cap_n = cfg.max_negative;
    DevBuf samples, counters, rows;
    BBRT_CUDA(samples.ensure(sizeof(bbrt::GuessSample) * static_cast<size_t>(cap_p + cap_n)));
    BBRT_CUDA(counters.ensure(2 * sizeof(unsigned long long)));
    BBRT_CUDA(cudaMemsetAsync(counters.p, 0, 2 * sizeof(unsigned long long), st));
    const int save_prec = s->dev.precision, save_guess = s->host.cfg.guess;
    s->dev.precision = BBRT_PREC_FP64;
    s->host.cfg.guess = BBRT_GUESS_TRIANGLE;
    s->rec_samples = static_cast<bbrt::GuessSample*>(samples.p);
    s->rec_count = static_cast<unsigned long long*>(counters.p);
    s->rec_cap_pos = cap_p;
    s->rec_cap_neg = cap_n;
    float collect_ms = 0.0f;
    rc = run_trace_device(s, d_o, d_d, n, max_bounces, nullptr, nullptr, 1, st, false, nullptr, &collect_ms);
    s->rec_samples = nullptr;
    s->rec_count = nullptr;
    s->dev.precision = save_prec;
    s->host.cfg.guess = save_guess;
    if (rc) return rc;
    unsigned long long cnt[2] = { 0, 0 };
    BBRT_CUDA(cudaMemcpyAsync(cnt, counters.p, sizeof cnt, cudaMemcpyDeviceToHost, st));
    BBRT_CUDA(cudaStreamSynchronize(st));
    const long long npos = std::min<long long>(static_cast<long long>(cnt[1]), cap_p);
    const long long nneg = std::min<long long>(static_cast<long long>(cnt[0]), cap_n);
    const long long N = npos + nneg;
    if (npos == 0) return fail(BBRT_ERR_STATE, "bbrt_guess_train: the rays produced no Newton solves to learn from");
    // ---- 2. training rows
    const size_t rb = static_cast<size_t>(N) * (bbrt::kGeo * 4 + 4 + 3 * 4 + 4 + 4);
    BBRT_CUDA(rows.ensure(rb));
    float* feat = static_cast<float*>(rows.p);
    int* pid = reinterpret_cast<int*>(feat + N * bbrt::kGeo);
    float* tgt = reinterpret_cast<float*>(pid + N);
    float* lbl = tgt + 3 * N;
    int* idx = reinterpret_cast<int*>(lbl + N);
    const bbrt::GuessSample* S0 = static_cast<const bbrt::GuessSample*>(samples.p);
    BBRT_CUDA(bbrt::mlp_make_rows(S0, npos, s->guess.frame, feat, pid, tgt, lbl, st));
    BBRT_CUDA(bbrt::mlp_make_rows(S0 + cap_p, nneg, s->guess.frame, feat + npos * bbrt::kGeo, pid + npos,
                                  tgt + 3 * npos, lbl + npos, st));
    // ---- 3. network
    const long long np = bbrt_guess_param_count(s);
    if ((rc = guess_alloc(s, np))) return rc;
    {
        const std::vector<float> P0 = init_network(np, cfg.seed);
        BBRT_CUDA(cudaMemcpyAsync(s->guess.P.p, P0.data(), sizeof(float) * np, cudaMemcpyHostToDevice, st));
        BBRT_CUDA(cudaStreamSynchronize(st));
    }
    BBRT_CUDA(cudaMemsetAsync(s->guess.m1.p, 0, sizeof(float) * np, st));
    BBRT_CUDA(cudaMemsetAsync(s->guess.m2.p, 0, sizeof(float) * np, st));
    BBRT_CUDA(cudaMemsetAsync(s->guess.G.p, 0, sizeof(float) * np, st));
    BBRT_CUDA(cudaMemsetAsync(s->guess.err.p, 0, sizeof(int), st));
    BBRT_CUDA(bbrt::mlp_pack(static_cast<const float*>(s->guess.P.p), static_cast<uint8_t*>(s->guess.image.p), st));
    // ---- 4. epochs of shuffled batches
    const int B = static_cast<int>(std::min<long long>(cfg.batch, N));
    const long long per_epoch = (N + B - 1) / B;
    const long long steps = per_epoch * cfg.epochs;
    BBRT_CUDA(s->guess.loss.ensure(sizeof(float) * static_cast<size_t>(steps)));
    BBRT_CUDA(cudaMemsetAsync(s->guess.loss.p, 0, sizeof(float) * steps, st));
    std::vector<int> perm(static_cast<size_t>(N));
    std::iota(perm.begin(), perm.end(), 0);
    std::mt19937_64 rng(cfg.seed ^ 0x9E3779B97F4A7C15ULL);
    BBRT_CUDA(cudaEventRecord(s->ev[0], st));
    bbrt::MlpNet net = guess_net(s);
    long long step = 0;
    for (int ep = 0; ep < cfg.epochs; ++ep) {
        std::shuffle(perm.begin(), perm.end(), rng);
        BBRT_CUDA(cudaMemcpyAsync(idx, perm.data(), sizeof(int) * N, cudaMemcpyHostToDevice, st));
        for (long long b0 = 0; b0 < N; b0 += B, ++step) {
            bbrt::MlpBatch bt;
            bt.feat = feat;
            bt.pid = pid;
            bt.tgt = tgt;
            bt.lbl = lbl;
            bt.idx = idx + b0;
            bt.B = static_cast<int>(std::min<long long>(B, N - b0));
            bt.inv_b = 1.0f / static_cast<float>(bt.B);
            net.loss = static_cast<float*>(s->guess.loss.p) + step;
            BBRT_CUDA(bbrt::mlp_train_batch(bt, net, st));
            BBRT_CUDA(bbrt::mlp_adam(net, static_cast<float*>(s->guess.m1.p), static_cast<float*>(s->guess.m2.p), np,
                                     cfg.lr, static_cast<int>(step + 1), st));
            BBRT_CUDA(cudaMemsetAsync(s->guess.G.p, 0, sizeof(float) * np, st));
            BBRT_CUDA(bbrt::mlp_pack(static_cast<const float*>(s->guess.P.p), static_cast<uint8_t*>(s->guess.image.p), st));
        }
        // the host copy of the permutation must outlive its upload
        BBRT_CUDA(cudaStreamSynchronize(st));
    }
    BBRT_CUDA(cudaEventRecord(s->ev[1], st));
    if ((rc = guess_err_check(s, st))) return rc;
    float train_ms = 0.0f;
    BBRT_CUDA(cudaEventElapsedTime(&train_ms, s->ev[0], s->ev[1]));
    std::vector<float> losses(static_cast<size_t>(steps));
    BBRT_CUDA(cudaMemcpy(losses.data(), s->guess.loss.p, sizeof(float) * steps, cudaMemcpyDeviceToHost));
    s->guess.trained = true;
    s->guess.steps = steps;
    s->guess.min_logit = cfg.min_logit;
    s->guess.t_window = cfg.t_window;
    if (rep) {
        std::memset(rep, 0, sizeof *rep);
        rep->positives = npos;
        rep->negatives = nneg;
        rep->steps = steps;
        double f = 0.0, l = 0.0;
        for (long long k = 0; k < per_epoch; ++k) {
            f += losses[k];
            l += losses[steps - per_epoch + k];
        }
        rep->first_loss = f / per_epoch;
        rep->last_loss = l / per_epoch;
        rep->collect_ms = collect_ms;
        rep->train_ms = train_ms;
    }
    return BBRT_OK;
}

// Standalone network buffers for the check entry points.
struct CheckNet {
    std::vector<void*> bufs;
    ~CheckNet() {
        for (void* p : bufs) cudaFree(p);
    }
    template <class T>
    T* alloc(size_t count) {
        void* p = nullptr;
        if (cudaMalloc(&p, sizeof(T) * (count ? count : 1)) != cudaSuccess) return nullptr;
        bufs.push_back(p);
        return static_cast<T*>(p);
    }
};

}  // namespace

BBRT_API int bbrt_mlp_check(const float* params, int n_patches, const float* feat, const int* patch,
                            const float* target, const float* label, int rows, float* loss, float* out,
                            float* grads) {
    if (!params || !feat || !patch || !target || !label || !loss || !out || !grads || rows < 1 || n_patches < 1)
        return fail(BBRT_ERR_ARG, "bbrt_mlp_check: bad argument");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0)
        return fail(BBRT_ERR_CUDA, "bbrt: no CUDA device available (the trace path has no CPU fallback)");
    for (int r = 0; r < rows; ++r)
        if (patch[r] < 0 || patch[r] >= n_patches) return fail(BBRT_ERR_ARG, "bbrt_mlp_check: patch index out of range");
    const long long np = bbrt::oE + static_cast<long long>(bbrt::kEmb) * n_patches;
    CheckNet c;
    float* P = c.alloc<float>(np);
    float* G = c.alloc<float>(np);
    uint8_t* image = c.alloc<uint8_t>(bbrt::kImageBytes);
    float* dfeat = c.alloc<float>(static_cast<size_t>(rows) * bbrt::kGeo);
    int* dpid = c.alloc<int>(rows);
    float* dtgt = c.alloc<float>(3 * static_cast<size_t>(rows));
    float* dlbl = c.alloc<float>(rows);
    float* dloss = c.alloc<float>(1);
    float* dout = c.alloc<float>(4 * static_cast<size_t>(rows));
    int* derr = c.alloc<int>(1);
    if (!P || !G || !image || !dfeat || !dpid || !dtgt || !dlbl || !dloss || !dout || !derr)
        return fail(BBRT_ERR_NOMEM, "bbrt_mlp_check: cudaMalloc failed");
    BBRT_CUDA(cudaMemcpy(P, params, sizeof(float) * np, cudaMemcpyHostToDevice));
    BBRT_CUDA(cudaMemset(G, 0, sizeof(float) * np));
    BBRT_CUDA(cudaMemcpy(dfeat, feat, sizeof(float) * rows * bbrt::kGeo, cudaMemcpyHostToDevice));
    BBRT_CUDA(cudaMemcpy(dpid, patch, sizeof(int) * rows, cudaMemcpyHostToDevice));
    BBRT_CUDA(cudaMemcpy(dtgt, target, sizeof(float) * 3 * rows, cudaMemcpyHostToDevice));
    BBRT_CUDA(cudaMemcpy(dlbl, label, sizeof(float) * rows, cudaMemcpyHostToDevice));
    BBRT_CUDA(cudaMemset(dloss, 0, sizeof(float)));
    BBRT_CUDA(cudaMemset(derr, 0, sizeof(int)));
    BBRT_CUDA(bbrt::mlp_pack(P, image, nullptr));
    bbrt::MlpNet net;
    net.image = image;
    net.P = P;
    net.G = G;
    net.loss = dloss;
    net.out = dout;
    net.err = derr;
    bbrt::MlpBatch bt;
    bt.feat = dfeat;
    bt.pid = dpid;
    bt.tgt = dtgt;
    bt.lbl = dlbl;
    bt.idx = nullptr;
    bt.B = rows;
    bt.inv_b = 1.0f / static_cast<float>(rows);
    BBRT_CUDA(bbrt::mlp_train_batch(bt, net, nullptr));
    BBRT_CUDA(cudaDeviceSynchronize());
    int herr = 0;
    BBRT_CUDA(cudaMemcpy(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost));
    if (herr) return fail(BBRT_ERR_KERNEL, "bbrt_mlp_check: a tensor-core completion wait timed out");
    std::vector<float> gdev(static_cast<size_t>(np));
    BBRT_CUDA(cudaMemcpy(gdev.data(), G, sizeof(float) * np, cudaMemcpyDeviceToHost));
    BBRT_CUDA(cudaMemcpy(loss, dloss, sizeof(float), cudaMemcpyDeviceToHost));
    BBRT_CUDA(cudaMemcpy(out, dout, sizeof(float) * 4 * rows, cudaMemcpyDeviceToHost));
    for (long long p = 0; p < np; ++p) grads[p] = gdev[static_cast<size_t>(bbrt::grad_index(p))];
    return BBRT_OK;
}

BBRT_API int bbrt_mlp_infer_check(const float* params, int n_patches, const float* feat, const int* patch, int rows,
                                  double* out) {
    if (!params || !feat || !patch || !out || rows < 1 || n_patches < 1)
        return fail(BBRT_ERR_ARG, "bbrt_mlp_infer_check: bad argument");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0)
        return fail(BBRT_ERR_CUDA, "bbrt: no CUDA device available (the trace path has no CPU fallback)");
    for (int r = 0; r < rows; ++r)
        if (patch[r] < 0 || patch[r] >= n_patches)
            return fail(BBRT_ERR_ARG, "bbrt_mlp_infer_check: patch index out of range");
    const long long np = bbrt::oE + static_cast<long long>(bbrt::kEmb) * n_patches;
    CheckNet c;
    float* P = c.alloc<float>(np);
    uint8_t* image = c.alloc<uint8_t>(bbrt::kImageBytes);
    float* dfeat = c.alloc<float>(static_cast<size_t>(rows) * bbrt::kGeo);
    int* dpid = c.alloc<int>(rows);
    double* dout = c.alloc<double>(4 * static_cast<size_t>(rows));
    int* derr = c.alloc<int>(1);
    if (!P || !image || !dfeat || !dpid || !dout || !derr) return fail(BBRT_ERR_NOMEM, "bbrt_mlp_infer_check: cudaMalloc failed");
    BBRT_CUDA(cudaMemcpy(P, params, sizeof(float) * np, cudaMemcpyHostToDevice));
    BBRT_CUDA(cudaMemcpy(dfeat, feat, sizeof(float) * rows * bbrt::kGeo, cudaMemcpyHostToDevice));
    BBRT_CUDA(cudaMemcpy(dpid, patch, sizeof(int) * rows, cudaMemcpyHostToDevice));
    BBRT_CUDA(cudaMemset(derr, 0, sizeof(int)));
    BBRT_CUDA(bbrt::mlp_pack(P, image, nullptr));
    bbrt::MlpNet net;
    net.image = image;
    net.P = P;
    net.G = nullptr;
    net.loss = nullptr;
    net.out = nullptr;
    net.err = derr;
    BBRT_CUDA(bbrt::mlp_infer_features(dfeat, dpid, rows, net, dout, nullptr));
    BBRT_CUDA(cudaDeviceSynchronize());
    int herr = 0;
    BBRT_CUDA(cudaMemcpy(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost));
    if (herr) return fail(BBRT_ERR_KERNEL, "bbrt_mlp_infer_check: a tensor-core completion wait timed out");
    BBRT_CUDA(cudaMemcpy(out, dout, sizeof(double) * 4 * rows, cudaMemcpyDeviceToHost));
    return BBRT_OK;
}

// ---- launch schedule and its autotuner -------------------------------------

BBRT_API int bbrt_scene_get_tuning(bbrt_scene_t s, bbrt_tuning* out) {
    if (!s || !out) return fail(BBRT_ERR_ARG, "bbrt_scene_get_tuning: NULL argument");
    std::lock_guard<std::mutex> g(s->mu);
    *out = scene_tuning(s);
    return BBRT_OK;
}

BBRT_API int bbrt_scene_set_tuning(bbrt_scene_t s, const bbrt_tuning* t) {
    if (!s || !t) return fail(BBRT_ERR_ARG, "bbrt_scene_set_tuning: NULL argument");
    if (t->advance_shape < 0 || t->advance_shape > 6) return fail(BBRT_ERR_ARG, "bbrt_scene_set_tuning: advance_shape must be 0..6");
    if (t->wave_tail < 0 || t->wave_min_rays < 0) return fail(BBRT_ERR_ARG, "bbrt_scene_set_tuning: negative size");
    if (t->graph_rounds != 0 && t->graph_rounds != 1) return fail(BBRT_ERR_ARG, "bbrt_scene_set_tuning: graph_rounds must be 0 or 1");
    if (t->watchdog_cycles < 0 || t->mma_wait_cycles < 0)
        return fail(BBRT_ERR_ARG, "bbrt_scene_set_tuning: negative wait bound");
    std::lock_guard<std::mutex> g(s->mu);
    s->tune = *t;
    s->tune_set = true;
    return BBRT_OK;
}

BBRT_API int bbrt_scene_autotune(bbrt_scene_t s, const double* origins, const double* dirs, long long n, int max_bounces,
                                 int trials, bbrt_tuning* best, double* best_ms, void* stream) {
    if (!s || !origins || !dirs) return fail(BBRT_ERR_ARG, "bbrt_scene_autotune: NULL argument");
    if (n <= 0 || max_bounces < 0 || trials < 1) return fail(BBRT_ERR_ARG, "bbrt_scene_autotune: bad size");
    std::lock_guard<std::mutex> g(s->mu);
    int rc = ensure_uploaded(s);
    if (rc) return rc;
    cudaStream_t st = pick_stream(s, stream);
    BBRT_CUDA(s->in_o.ensure(sizeof(double) * 3 * n));
    BBRT_CUDA(s->in_d.ensure(sizeof(double) * 3 * n));
    BBRT_CUDA(cudaMemcpyAsync(s->in_o.p, origins, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, st));
    BBRT_CUDA(cudaMemcpyAsync(s->in_d.p, dirs, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, st));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    BBRT_CUDA(cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return fail(BBRT_ERR_CUDA, "bbrt_scene_autotune: cudaEventCreate failed");
    }
    auto time_one = [&](const bbrt_tuning& t, double& ms) -> int {
        s->tune = t;
        s->tune_set = true;
        double total = 0.0;
        for (int k = 0; k <= trials; ++k) {
            BBRT_CUDA(cudaEventRecord(e0, st));
            const int r = run_trace_device(s, static_cast<const double*>(s->in_o.p), static_cast<const double*>(s->in_d.p),
                                           n, max_bounces, nullptr, nullptr, 1, st, false, nullptr, nullptr);
            if (r) return r;
            BBRT_CUDA(cudaEventRecord(e1, st));
            BBRT_CUDA(cudaEventSynchronize(e1));
            float el = 0.0f;
            BBRT_CUDA(cudaEventElapsedTime(&el, e0, e1));
            if (k > 0) total += el;
        }
        ms = total / trials;
        return BBRT_OK;
    };
    bbrt_tuning cur = scene_tuning(s);
    double cur_ms = 0.0;
    rc = time_one(cur, cur_ms);
    // coordinate descent: launch shape, then tail size
    const int shapes[] = { 3, 6, 1, 0 };
    for (int sh : shapes) {
        if (rc || sh == cur.advance_shape) continue;
        bbrt_tuning c = cur;
        c.advance_shape = sh;
        double ms = 0.0;
        rc = time_one(c, ms);
        if (!rc && ms < cur_ms) { cur = c; cur_ms = ms; }
    }
    const long long tails[] = { 0, 1024, 4096, 8192, 16384, 32768, 65536 };
    for (long long tl : tails) {
        if (rc || tl == cur.wave_tail) continue;
        bbrt_tuning c = cur;
        c.wave_tail = tl;
        double ms = 0.0;
        rc = time_one(c, ms);
        if (!rc && ms < cur_ms) { cur = c; cur_ms = ms; }
    }
    if (!rc) {   // graph-launched rounds or host-driven ones
        bbrt_tuning c = cur;
        c.graph_rounds = cur.graph_rounds ? 0 : 1;
        double ms = 0.0;
        rc = time_one(c, ms);
        if (!rc && ms < cur_ms) { cur = c; cur_ms = ms; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    s->tune = cur;
    s->tune_set = true;
    if (rc) return rc;
    if (best) *best = cur;
    if (best_ms) *best_ms = cur_ms;
    return BBRT_OK;
}

// ---- several scenes together -----------------------------------------------

BBRT_API int bbrt_trace_batch(const bbrt_scene_t* scenes, int n_scenes, const double* const* origins,
                              const double* const* dirs, const long long* n, int max_bounces,
                              const bbrt_trace_out* outs, bbrt_trace_stats* stats, double* batch_ms) {
    if (!scenes || !origins || !dirs || !n || n_scenes < 1) return fail(BBRT_ERR_ARG, "bbrt_trace_batch: bad argument");
    if (max_bounces < 0) return fail(BBRT_ERR_ARG, "bbrt_trace_batch: max_bounces < 0");
    std::vector<bbrt_scene*> order;
    for (int k = 0; k < n_scenes; ++k) {
        if (!scenes[k]) return fail(BBRT_ERR_ARG, "bbrt_trace_batch: NULL scene");
        if (n[k] < 0 || (n[k] > 0 && (!origins[k] || !dirs[k])))
            return fail(BBRT_ERR_ARG, "bbrt_trace_batch: bad rays of scene " + std::to_string(k));
        order.push_back(scenes[k]);
    }
    std::sort(order.begin(), order.end());
    if (std::adjacent_find(order.begin(), order.end()) != order.end())
        return fail(BBRT_ERR_ARG, "bbrt_trace_batch: a scene appears twice in the batch");
    std::vector<std::unique_lock<std::mutex>> locks;
    for (bbrt_scene* sc : order) locks.emplace_back(sc->mu);   // address order: no lock cycles
    for (int k = 0; k < n_scenes; ++k) {
        const int rc = ensure_uploaded(scenes[k]);
        if (rc) return rc;
    }
    // One device timeline for the whole batch: every scene's stream waits on
    // a start event, and the end event waits on every scene's stream.
    cudaStream_t bs = scenes[0]->stream;
    cudaEvent_t start = nullptr, end = nullptr;
    BBRT_CUDA(cudaEventCreate(&start));
    if (cudaEventCreate(&end) != cudaSuccess) {
        cudaEventDestroy(start);
        return fail(BBRT_ERR_CUDA, "bbrt_trace_batch: cudaEventCreate failed");
    }
    auto cleanup = [&]() { cudaEventDestroy(start); cudaEventDestroy(end); };
    const bool want = stats != nullptr;
    std::vector<WaveRun> runs(n_scenes);
    std::vector<std::vector<long long>> hs(n_scenes, std::vector<long long>(bbrt::ST_COUNT, 0));
    int rc = BBRT_OK;
    if (cudaEventRecord(start, bs) != cudaSuccess) rc = fail(BBRT_ERR_CUDA, "bbrt_trace_batch: cudaEventRecord failed");
    for (int k = 0; k < n_scenes && !rc; ++k) {
        bbrt_scene* s = scenes[k];
        if (s->stream != bs && cudaStreamWaitEvent(s->stream, start, 0) != cudaSuccess) {
            rc = fail(BBRT_ERR_CUDA, "bbrt_trace_batch: cudaStreamWaitEvent failed");
            break;
        }
        bbrt::TraceArgs A;
        rc = prepare_trace(s, origins[k], dirs[k], n[k], max_bounces, outs ? &outs[k] : nullptr, nullptr, 1, s->stream,
                           want, A);
        if (rc) break;
        if (n[k] < scene_tuning(s).wave_min_rays) {
            if (n[k] > 0) {
                const cudaError_t e = timed(s, K_TAIL, s->stream, [&] { return bbrt::launch_trace(s->dev, A, s->stream, s->sm_count); });
                if (e != cudaSuccess) rc = fail(BBRT_ERR_CUDA, std::string("bbrt_trace_batch: ") + cudaGetErrorString(e));
            }
            runs[k].s = s;
            runs[k].done = true;
        } else {
            rc = runs[k].begin(s, A, s->stream);
        }
    }
    // rounds of all scenes together: one wait per round for the whole batch
    bool active = true;
    while (!rc && active) {
        active = false;
        for (int k = 0; k < n_scenes && !rc; ++k) {
            if (runs[k].done) continue;
            if (cudaStreamSynchronize(scenes[k]->stream) != cudaSuccess) {
                rc = fail(BBRT_ERR_CUDA, "bbrt_trace_batch: stream synchronisation failed");
                break;
            }
            rc = runs[k].step();
            if (!runs[k].done) active = true;
        }
    }
    for (int k = 0; k < n_scenes && !rc; ++k) {
        if (runs[k].s && n[k] >= scene_tuning(scenes[k]).wave_min_rays) rc = runs[k].finish();
        if (!rc) rc = complete_trace(scenes[k], scenes[k]->stream, want, hs[k].data(), nullptr);
        if (!rc && scenes[k]->stream != bs) {
            cudaEvent_t e = scenes[k]->ev[1];
            if (cudaStreamWaitEvent(bs, e, 0) != cudaSuccess) rc = fail(BBRT_ERR_CUDA, "bbrt_trace_batch: cudaStreamWaitEvent failed");
        }
    }
    if (!rc && cudaEventRecord(end, bs) != cudaSuccess) rc = fail(BBRT_ERR_CUDA, "bbrt_trace_batch: cudaEventRecord failed");
    if (!rc && cudaEventSynchronize(end) != cudaSuccess) rc = fail(BBRT_ERR_CUDA, "bbrt_trace_batch: synchronisation failed");
    for (int k = 0; k < n_scenes && !rc; ++k)
        if (cudaStreamSynchronize(scenes[k]->stream) != cudaSuccess) rc = fail(BBRT_ERR_CUDA, "bbrt_trace_batch: synchronisation failed");
    for (int k = 0; k < n_scenes && !rc; ++k)
        if (runs[k].graph.on) rc = check_wave_graph(scenes[k], runs[k].graph);
    for (int k = 0; k < n_scenes && !rc; ++k)
        if (n[k] >= scene_tuning(scenes[k]).wave_min_rays) rc = check_guess_waits(scenes[k], scenes[k]->stream);
    if (!rc && batch_ms) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, start, end);
        *batch_ms = ms;
    }
    if (!rc && stats) {
        std::memset(stats, 0, sizeof *stats);
        for (int k = 0; k < n_scenes; ++k) {
            bbrt_trace_stats one;
            float kms = 0.0f;
            cudaEventElapsedTime(&kms, scenes[k]->ev[0], scenes[k]->ev[1]);
            fill_stats(scenes[k], hs[k].data(), n[k], kms, kms, &one);
            stats->rays += one.rays;
            stats->bounces += one.bounces;
            stats->queries += one.queries;
            stats->node_tests += one.node_tests;
            stats->patch_tests += one.patch_tests;
            stats->cell_tests += one.cell_tests;
            stats->tri_tests += one.tri_tests;
            stats->newton_iters += one.newton_iters;
            stats->newton_iters_fp32 += one.newton_iters_fp32;
            for (int q = 0; q < BBRT_RAY_STATUS_COUNT; ++q) stats->status_hist[q] += one.status_hist[q];
            stats->rounds += one.rounds;
            stats->launches += one.launches;
            stats->tail_rays += one.tail_rays;
            stats->guess_used += one.guess_used;
            stats->guess_fallback += one.guess_fallback;
            stats->off_patch += one.off_patch;
            stats->node_tests_fp64 += one.node_tests_fp64;
        }
        if (batch_ms) stats->kernel_ms = stats->total_ms = *batch_ms;
    }
    cleanup();
    return rc;
}

// ---- several scenes as one trace (scene set) --------------------------------
//
// A set copies its members' device arrays side by side into one scene: the
// objects, patch tables, coarse grids, cell data and cull boxes are
// concatenated (member m's object k becomes object obj_off[m] + k), and the
// BVH trees form one forest renumbered breadth-first across all trees, so
// that the top levels of every member land in the shared-memory node copy
// the trace kernels stage.  Each ray carries its member: its query starts at
// the member's root and uses the member's scale and cull constants.  Every
// per-object computation is the member's own, so the results equal a trace
// of each member alone, bit for bit.

struct bbrt_scene_set {
    bbrt_scene merged;
    int n_members = 0;
    std::vector<int> obj_off;              // [M + 1]
    std::vector<long long> patch_off;      // [M + 1]
    std::vector<bbrt::MemberIO> io;        // per-call member table (host copy of io_dev)
    DevBuf io_dev, ray_member, set_o, set_d, o_status, o_bounce, o_dir, o_end, o_hobj, o_hpt, o_huv, o_eobj,
        o_eval, o_work;
    cudaEvent_t ev[2] = { nullptr, nullptr };
    ~bbrt_scene_set() {
        for (DevBuf* b : { &io_dev, &ray_member, &set_o, &set_d, &o_status, &o_bounce, &o_dir, &o_end, &o_hobj,
                           &o_hpt, &o_huv, &o_eobj, &o_eval, &o_work })
            b->release();
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
    }
};

namespace {

// Device arrays of several members joined into one (device-to-device copies;
// a member without the array contributes zeros).
template <class T>
int join_device(bbrt_scene& S, const std::vector<std::pair<const T*, size_t>>& parts, const T*& dst) {
    size_t total = 0;
    for (const auto& pr : parts) total += pr.second;
    T* p = nullptr;
    int rc = S.alloc(total, p);
    if (rc) return rc;
    size_t at = 0;
    for (const auto& pr : parts) {
        if (pr.second) {
            if (pr.first) BBRT_CUDA(cudaMemcpyAsync(p + at, pr.first, sizeof(T) * pr.second, cudaMemcpyDeviceToDevice, S.stream));
            else BBRT_CUDA(cudaMemsetAsync(p + at, 0, sizeof(T) * pr.second, S.stream));
        }
        at += pr.second;
    }
    dst = p;
    return BBRT_OK;
}

int build_scene_set(const std::vector<bbrt_scene*>& mem, bbrt_scene_set* set) {
    const int M = static_cast<int>(mem.size());
    const bbrt::HostScene& H0 = mem[0]->host;
    for (bbrt_scene* m : mem) {
        const bbrt::HostScene& H = m->host;
        const bbrt_config &a = H.cfg, &b = H0.cfg;
        if (H.coarse_n != H0.coarse_n || a.newton_max_iters != b.newton_max_iters || a.newton_tol != b.newton_tol ||
            a.self_intersect_eps_factor != b.self_intersect_eps_factor ||
            a.sagitta_clearance_factor != b.sagitta_clearance_factor || a.backface_tol != b.backface_tol ||
            a.cull != b.cull || m->dev.precision != mem[0]->dev.precision || m->device != mem[0]->device)
            return fail(BBRT_ERR_ARG, "bbrt_scene_set_create: the member scenes must share the coarse grid size, "
                                      "the Newton and epsilon constants, culling, precision and device");
    }
    bbrt_scene& S = set->merged;
    int dev = -1;
    BBRT_CUDA(cudaGetDevice(&dev));
    if (dev != mem[0]->device) return fail(BBRT_ERR_STATE, "bbrt_scene_set_create: the current device is not the scenes' device");
    int rc = ensure_device(&S);
    if (rc) return rc;
    bbrt::HostScene& HM = S.host;
    HM.cfg = H0.cfg;
    HM.cfg.guess = BBRT_GUESS_TRIANGLE;
    HM.coarse_n = H0.coarse_n;
    HM.coarse_uv = H0.coarse_uv;
    std::vector<long long> obj_off(M + 1, 0), patch_off(M + 1, 0), tri_off(M + 1, 0), leaf_off(M + 1, 0),
        node_off(M + 1, 0), ntab_off(M + 1, 0), ftab_off(M + 1, 0);
    for (int m = 0; m < M; ++m) {
        const bbrt::HostScene& H = mem[m]->host;
        obj_off[m + 1] = obj_off[m] + H.n_objects;
        patch_off[m + 1] = patch_off[m] + H.n_patches;
        tri_off[m + 1] = tri_off[m] + static_cast<long long>(H.tri.size() / 9);
        leaf_off[m + 1] = leaf_off[m] + static_cast<long long>(H.leaf_objects.size());
        node_off[m + 1] = node_off[m] + static_cast<long long>(H.nodes.size());
        ntab_off[m + 1] = ntab_off[m] + static_cast<long long>(H.p_nodes.size());
        ftab_off[m + 1] = ftab_off[m] + static_cast<long long>(H.p_fields.size());
    }
    if (obj_off[M] > (1LL << 30) || node_off[M] >= (1LL << 24))
        return fail(BBRT_ERR_UNSUPPORTED, "bbrt_scene_set_create: too many objects or BVH nodes in the set");
    HM.n_objects = static_cast<int>(obj_off[M]);
    HM.n_patches = static_cast<int>(patch_off[M]);
    set->obj_off.assign(obj_off.begin(), obj_off.end());
    set->patch_off = patch_off;
    std::vector<int> pdims;
    for (int m = 0; m < M; ++m) {
        const bbrt::HostScene& H = mem[m]->host;
        for (int k = 0; k < H.n_objects; ++k) {
            HM.kind.push_back(H.kind[k]);
            HM.sub.push_back(H.sub[k] + static_cast<int>(H.kind[k] == BBRT_OBJ_PATCH ? patch_off[m] : tri_off[m]));
            HM.padding.push_back(H.padding[k]);
        }
        for (int q = 0; q < H.n_patches; ++q) {
            HM.p_imax.push_back(H.p_imax[q]);
            HM.p_jmax.push_back(H.p_jmax[q]);
            HM.p_node_off.push_back(H.p_node_off[q] + ntab_off[m]);
            HM.p_field_off.push_back(H.p_field_off[q] + ftab_off[m]);
            pdims.push_back(H.p_imax[q]);
            pdims.push_back(H.p_jmax[q]);
        }
        for (int o : H.leaf_objects) HM.leaf_objects.push_back(o + static_cast<int>(obj_off[m]));
    }
    // the forest, breadth-first across all trees (children explicit)
    const size_t NN = static_cast<size_t>(node_off[M]);
    std::vector<std::pair<int, int>> order;
    order.reserve(NN);
    std::vector<std::vector<int>> newid(M);
    for (int m = 0; m < M; ++m) {
        newid[m].assign(mem[m]->host.nodes.size(), -1);
        if (!mem[m]->host.nodes.empty()) order.push_back({ m, 0 });
    }
    for (size_t h = 0; h < order.size(); ++h) {
        const int m = order[h].first, idx = order[h].second;
        newid[m][idx] = static_cast<int>(h);
        const bbrt::BvhNode& nd = mem[m]->host.nodes[idx];
        if (nd.right >= 0) {
            order.push_back({ m, idx + 1 });
            order.push_back({ m, nd.right });
        }
    }
    std::vector<double> nbox(6 * NN);
    std::vector<int> nlink(4 * NN), roots(M, 0);
    std::vector<double> params(static_cast<size_t>(M) * bbrt::kMemberParams, 0.0);
    for (size_t h = 0; h < order.size(); ++h) {
        const int m = order[h].first, idx = order[h].second;
        const bbrt::BvhNode& nd = mem[m]->host.nodes[idx];
        std::memcpy(&nbox[6 * h], nd.box, sizeof(double) * 6);
        if (nd.right >= 0) {
            nlink[4 * h] = newid[m][idx + 1];
            nlink[4 * h + 1] = newid[m][nd.right];
            nlink[4 * h + 2] = 0;
            nlink[4 * h + 3] = nd.axis;
        } else {
            nlink[4 * h] = nd.start + static_cast<int>(leaf_off[m]);
            nlink[4 * h + 1] = -1;
            nlink[4 * h + 2] = nd.count;
            nlink[4 * h + 3] = 0;
        }
    }
    bbrt::DScene& D = S.dev;
    S.member_sphere.assign(4 * static_cast<size_t>(M), 0.0);
    double diag_max = 0.0, sag_max = 0.0;
    int cull_block_cells = 4, cull_blocks = 0;
    for (int m = 0; m < M; ++m) {
        const bbrt_scene* ms = mem[m];
        roots[m] = newid[m].empty() ? 0 : newid[m][0];
        double* pr = &params[static_cast<size_t>(m) * bbrt::kMemberParams];
        pr[0] = ms->host.scene_diagonal;
        pr[1] = ms->cull.enabled ? 1.0 : 0.0;
        pr[2] = ms->cull.a; pr[3] = ms->cull.h; pr[4] = ms->cull.b; pr[5] = ms->cull.coord; pr[6] = ms->cull.radius;
        for (int a = 0; a < 3; ++a) pr[7 + a] = ms->cull.center[a];
        for (int a = 0; a < 3; ++a) S.member_sphere[4 * m + a] = ms->cull.center[a];
        S.member_sphere[4 * m + 3] = ms->cull.radius > 0.0 ? ms->cull.radius : ms->host.scene_diagonal;
        diag_max = std::max(diag_max, ms->host.scene_diagonal);
        sag_max = std::max(sag_max, ms->host.max_patch_sagitta);
        if (ms->cull.enabled) {
            cull_block_cells = ms->cull.block_cells;
            cull_blocks = ms->cull.n_blocks_side;
        }
        D.max_nodes = std::max(D.max_nodes, ms->dev.max_nodes);
    }
    HM.scene_diagonal = diag_max;
    HM.max_patch_sagitta = sag_max;
    D.n_objects = HM.n_objects;
    D.n_nodes = static_cast<int>(NN);
    D.coarse_n = HM.coarse_n;
    D.newton_max_iters = H0.cfg.newton_max_iters;
    D.newton_tol = H0.cfg.newton_tol;
    D.scene_diagonal = diag_max;
    D.max_patch_sagitta = sag_max;
    D.eps_factor = H0.cfg.self_intersect_eps_factor;
    D.sag_factor = H0.cfg.sagitta_clearance_factor;
    D.backface_tol = H0.cfg.backface_tol;
    D.precision = mem[0]->dev.precision;
    D.smem_nodes = static_cast<int>(std::min<size_t>(NN, 3400));
    D.block_cells = cull_block_cells;
    D.n_blocks_side = cull_blocks;
    D.cull_enabled = 0;   // per member (m_param); a ray without a member never occurs in a set
    D.n_members = M;
    if ((rc = upload_node_tables(&S, nbox, nlink))) return rc;
    if ((rc = S.upload(HM.leaf_objects, D.leaf_objects))) return rc;
    if ((rc = S.upload(HM.kind, D.obj_kind))) return rc;
    if ((rc = S.upload(HM.sub, D.obj_sub))) return rc;
    if ((rc = S.upload(HM.padding, D.obj_pad))) return rc;
    if ((rc = S.upload(pdims, D.p_dims))) return rc;
    if ((rc = S.upload(HM.p_node_off, D.p_node_off))) return rc;
    if ((rc = S.upload(HM.p_field_off, D.p_field_off))) return rc;
    if ((rc = S.upload(HM.coarse_uv, D.coarse_uv))) return rc;
    if ((rc = S.upload(roots, D.m_root))) return rc;
    if ((rc = S.upload(params, D.m_param))) return rc;
    {
        // the learned guess's patch frames, member after member
        std::vector<double> fr;
        for (int m = 0; m < M; ++m) {
            const std::vector<double> f = patch_frames(mem[m]->host);
            fr.insert(fr.end(), f.begin(), f.end());
        }
        if ((rc = S.upload(fr, S.guess.frame))) return rc;
    }
    const int cn = HM.coarse_n, nc = cn - 1;
    std::vector<std::pair<const double*, size_t>> pn, pf, cx, cc, tr;
    std::vector<std::pair<const float*, size_t>> pn32, pf32, cb, bb;
    for (int m = 0; m < M; ++m) {
        const bbrt_scene* ms = mem[m];
        const bbrt::DScene& Dm = ms->dev;
        const size_t P = static_cast<size_t>(ms->host.n_patches);
        pn.push_back({ Dm.p_nodes, ms->host.p_nodes.size() });
        pf.push_back({ Dm.p_fields, ms->host.p_fields.size() });
        pn32.push_back({ Dm.p_nodes32, ms->host.p_nodes.size() });
        pf32.push_back({ Dm.p_fields32, ms->host.p_fields.size() });
        cx.push_back({ Dm.c_xyz, P * 3 * cn * cn });
        cc.push_back({ Dm.c_cell, P * 4 * nc * nc });
        tr.push_back({ Dm.tri, ms->host.tri.size() });
        const bool on = ms->cull.enabled;
        cb.push_back({ on ? Dm.c_cell_box : nullptr, cull_blocks ? P * 6 * nc * nc : 0 });
        bb.push_back({ on ? Dm.c_block_box : nullptr, cull_blocks ? P * 6 * cull_blocks * cull_blocks : 0 });
    }
    if ((rc = join_device(S, pn, D.p_nodes))) return rc;
    if ((rc = join_device(S, pf, D.p_fields))) return rc;
    if ((rc = join_device(S, pn32, D.p_nodes32))) return rc;
    if ((rc = join_device(S, pf32, D.p_fields32))) return rc;
    if ((rc = join_device(S, cx, D.c_xyz))) return rc;
    if ((rc = join_device(S, cc, D.c_cell))) return rc;
    if ((rc = join_device(S, tr, D.tri))) return rc;
    if (cull_blocks) {
        if ((rc = join_device(S, cb, D.c_cell_box))) return rc;
        if ((rc = join_device(S, bb, D.c_block_box))) return rc;
    }
    BBRT_CUDA(cudaStreamSynchronize(S.stream));
    BBRT_CUDA(S.stats.ensure(sizeof(long long) * bbrt::ST_COUNT));
    BBRT_CUDA(S.work.ensure(sizeof(unsigned long long)));
    S.tables_uploaded = true;
    S.setup_on_device = true;
    S.uploaded = true;
    set->n_members = M;
    BBRT_CUDA(cudaEventCreate(&set->ev[0]));
    BBRT_CUDA(cudaEventCreate(&set->ev[1]));
    return BBRT_OK;
}

}  // namespace

extern "C" {

BBRT_API int bbrt_scene_set_create(const bbrt_scene_t* scenes, int n_scenes, bbrt_scene_set_t* out) {
    if (!out) return fail(BBRT_ERR_ARG, "bbrt_scene_set_create: out is NULL");
    *out = nullptr;
    if (!scenes || n_scenes < 1) return fail(BBRT_ERR_ARG, "bbrt_scene_set_create: no scenes");
    std::vector<bbrt_scene*> mem(scenes, scenes + n_scenes), sorted;
    for (bbrt_scene* m : mem)
        if (!m) return fail(BBRT_ERR_ARG, "bbrt_scene_set_create: NULL scene");
    sorted = mem;
    std::sort(sorted.begin(), sorted.end());
    if (std::adjacent_find(sorted.begin(), sorted.end()) != sorted.end())
        return fail(BBRT_ERR_ARG, "bbrt_scene_set_create: a scene appears twice in the set");
    std::vector<std::unique_lock<std::mutex>> locks;
    for (bbrt_scene* m : sorted) locks.emplace_back(m->mu);   // address order: no lock cycles
    for (bbrt_scene* m : mem) {
        const int rc = ensure_uploaded(m);
        if (rc) return rc;
    }
    std::unique_ptr<bbrt_scene_set> set(new bbrt_scene_set());
    int rc = BBRT_OK;
    try {
        rc = build_scene_set(mem, set.get());
    } catch (const std::bad_alloc&) {
        return fail(BBRT_ERR_NOMEM, "bbrt_scene_set_create: out of host memory");
    }
    if (rc) return rc;
    *out = set.release();
    return BBRT_OK;
}

BBRT_API void bbrt_scene_set_destroy(bbrt_scene_set_t set) { delete set; }

BBRT_API int bbrt_scene_set_configure(bbrt_scene_set_t set, int precision, int guess, const bbrt_tuning* tuning) {
    if (!set) return fail(BBRT_ERR_ARG, "bbrt_scene_set_configure: NULL set");
    if (precision != BBRT_PREC_FP64 && precision != BBRT_PREC_SPLIT)
        return fail(BBRT_ERR_ARG, "bbrt_scene_set_configure: unknown precision");
    if (guess != BBRT_GUESS_TRIANGLE && guess != BBRT_GUESS_LEARNED)
        return fail(BBRT_ERR_ARG, "bbrt_scene_set_configure: unknown guess");
    if (tuning) {
        const int rc = bbrt_scene_set_tuning(&set->merged, tuning);
        if (rc) return rc;
    }
    std::lock_guard<std::mutex> g(set->merged.mu);
    if (guess == BBRT_GUESS_LEARNED && !set->merged.guess.trained)
        return fail(BBRT_ERR_STATE, "bbrt_scene_set_configure: the set has no trained network (bbrt_scene_set_guess_train)");
    set->merged.host.cfg.precision = precision;
    set->merged.dev.precision = precision;
    set->merged.host.cfg.guess = guess;
    return BBRT_OK;
}

BBRT_API int bbrt_scene_set_guess_train(bbrt_scene_set_t set, const double* const* origins, const double* const* dirs,
                                        const long long* n, int max_bounces, const bbrt_guess_train_config* cfg_in,
                                        bbrt_guess_train_report* rep) {
    if (!set || !origins || !dirs || !n) return fail(BBRT_ERR_ARG, "bbrt_scene_set_guess_train: NULL argument");
    if (max_bounces < 0) return fail(BBRT_ERR_ARG, "bbrt_scene_set_guess_train: max_bounces < 0");
    bbrt_guess_train_config cfg;
    bbrt_guess_train_config_init(&cfg);
    if (cfg_in) cfg = *cfg_in;
    if (cfg.epochs < 1 || cfg.batch < 128 || cfg.max_positive < 1 || cfg.max_negative < 0 || !(cfg.lr > 0.0f))
        return fail(BBRT_ERR_ARG, "bbrt_scene_set_guess_train: bad training configuration");
    const int M = set->n_members;
    std::vector<long long> off(M + 1, 0);
    for (int m = 0; m < M; ++m) {
        if (n[m] < 0 || (n[m] > 0 && (!origins[m] || !dirs[m])))
            return fail(BBRT_ERR_ARG, "bbrt_scene_set_guess_train: bad rays of member " + std::to_string(m));
        off[m + 1] = off[m] + n[m];
    }
    const long long N = off[M];
    if (N <= 0) return fail(BBRT_ERR_ARG, "bbrt_scene_set_guess_train: no rays");
    if (N >= (1LL << 31)) return fail(BBRT_ERR_UNSUPPORTED, "bbrt_scene_set_guess_train: more than 2^31 - 1 rays");
    bbrt_scene* s = &set->merged;
    std::lock_guard<std::mutex> g(s->mu);
    cudaStream_t st = s->stream;
    BBRT_CUDA(set->set_o.ensure(sizeof(double) * 3 * static_cast<size_t>(N)));
    BBRT_CUDA(set->set_d.ensure(sizeof(double) * 3 * static_cast<size_t>(N)));
    BBRT_CUDA(set->ray_member.ensure(sizeof(int) * static_cast<size_t>(N)));
    double* so = static_cast<double*>(set->set_o.p);
    double* sd = static_cast<double*>(set->set_d.p);
    set->io.assign(M, bbrt::MemberIO());
    for (int m = 0; m < M; ++m) {
        set->io[m].off = off[m];
        set->io[m].n = n[m];
        set->io[m].obj_off = set->obj_off[m];
        if (n[m] == 0) continue;
        BBRT_CUDA(cudaMemcpyAsync(so + 3 * off[m], origins[m], sizeof(double) * 3 * n[m], cudaMemcpyHostToDevice, st));
        BBRT_CUDA(cudaMemcpyAsync(sd + 3 * off[m], dirs[m], sizeof(double) * 3 * n[m], cudaMemcpyHostToDevice, st));
    }
    BBRT_CUDA(set->io_dev.ensure(sizeof(bbrt::MemberIO) * M));
    BBRT_CUDA(cudaMemcpyAsync(set->io_dev.p, set->io.data(), sizeof(bbrt::MemberIO) * M, cudaMemcpyHostToDevice, st));
    bbrt::SetIO io;
    io.m = static_cast<const bbrt::MemberIO*>(set->io_dev.p);
    io.n_members = M;
    io.n = N;
    io.ray_member = static_cast<int*>(set->ray_member.p);
    BBRT_CUDA(bbrt::set_members(io, st));
    BBRT_CUDA(cudaStreamSynchronize(st));   // the host copies of the rays and the table outlive the uploads
    s->member_rays = off;
    s->ray_member = io.ray_member;
    const int rc = guess_train_core(s, so, sd, N, max_bounces, cfg, rep, st);
    s->member_rays.clear();
    s->ray_member = nullptr;
    return rc;
}

BBRT_API int bbrt_scene_set_guess_export(bbrt_scene_set_t set, int member, bbrt_scene_t scene) {
    if (!set || !scene) return fail(BBRT_ERR_ARG, "bbrt_scene_set_guess_export: NULL argument");
    if (member < 0 || member >= set->n_members) return fail(BBRT_ERR_ARG, "bbrt_scene_set_guess_export: no such member");
    const long long np_member = set->patch_off[member + 1] - set->patch_off[member];
    if (scene->host.n_patches != np_member)
        return fail(BBRT_ERR_ARG, "bbrt_scene_set_guess_export: the scene's patch count is not the member's");
    std::vector<float> P;
    {
        bbrt_scene* s = &set->merged;
        std::lock_guard<std::mutex> g(s->mu);
        if (!s->guess.trained) return fail(BBRT_ERR_STATE, "bbrt_scene_set_guess_export: the set has no trained network");
        P.resize(static_cast<size_t>(bbrt::oE + bbrt::kEmb * np_member));
        BBRT_CUDA(cudaMemcpy(P.data(), s->guess.P.p, sizeof(float) * bbrt::oE, cudaMemcpyDeviceToHost));
        BBRT_CUDA(cudaMemcpy(P.data() + bbrt::oE,
                             static_cast<const float*>(s->guess.P.p) + bbrt::oE + bbrt::kEmb * set->patch_off[member],
                             sizeof(float) * bbrt::kEmb * np_member, cudaMemcpyDeviceToHost));
    }
    const int rc = bbrt_guess_params(scene, P.data(), static_cast<long long>(P.size()), 1);
    if (rc) return rc;
    std::lock_guard<std::mutex> g(scene->mu);
    scene->guess.min_logit = set->merged.guess.min_logit;
    scene->guess.t_window = set->merged.guess.t_window;
    return BBRT_OK;
}

BBRT_API int bbrt_trace_set(bbrt_scene_set_t set, const double* const* origins, const double* const* dirs,
                            const long long* n, int max_bounces, const bbrt_trace_out* outs,
                            bbrt_trace_stats* stats, double* set_ms, void* stream) {
    if (!set || !origins || !dirs || !n) return fail(BBRT_ERR_ARG, "bbrt_trace_set: NULL argument");
    if (max_bounces < 0) return fail(BBRT_ERR_ARG, "bbrt_trace_set: max_bounces < 0");
    const int M = set->n_members;
    std::vector<long long> off(M + 1, 0);
    for (int m = 0; m < M; ++m) {
        if (n[m] < 0 || (n[m] > 0 && (!origins[m] || !dirs[m])))
            return fail(BBRT_ERR_ARG, "bbrt_trace_set: bad rays of member " + std::to_string(m));
        off[m + 1] = off[m] + n[m];
    }
    const long long N = off[M];
    if (N >= (1LL << 31)) return fail(BBRT_ERR_UNSUPPORTED, "bbrt_trace_set: more than 2^31 - 1 rays");
    // the outputs' shape comes from the first member with rays (members without
    // rays may leave theirs empty)
    int first = 0;
    while (first < M - 1 && n[first] == 0) ++first;
    const int K = outs ? outs[first].record_bounces : 0;
    if (K < 0) return fail(BBRT_ERR_ARG, "bbrt_trace_set: record_bounces < 0");
    auto same_shape = [&](const bbrt_trace_out& a, const bbrt_trace_out& b) {
        return a.record_bounces == b.record_bounces && !a.status == !b.status && !a.bounce_count == !b.bounce_count &&
               !a.exit_dir == !b.exit_dir && !a.end_point == !b.end_point && !a.hit_object == !b.hit_object &&
               !a.hit_point == !b.hit_point && !a.hit_uv == !b.hit_uv && !a.err_object == !b.err_object &&
               !a.err_value == !b.err_value && !a.ray_work == !b.ray_work;
    };
    if (outs)
        for (int m = 0; m < M; ++m)
            if (n[m] > 0 && !same_shape(outs[first], outs[m]))
                return fail(BBRT_ERR_ARG, "bbrt_trace_set: every member must ask for the same outputs and record length");
    bbrt_scene* s = &set->merged;
    std::lock_guard<std::mutex> g(s->mu);
    cudaStream_t st = pick_stream(s, stream);
    long long hs[bbrt::ST_COUNT] = { 0 };
    if (N == 0) {
        if (stats) fill_stats(s, hs, 0, 0.0f, 0.0f, stats);
        if (set_ms) *set_ms = 0.0;
        return BBRT_OK;
    }
    const size_t NS = static_cast<size_t>(N), KS = static_cast<size_t>(K);
    BBRT_CUDA(set->set_o.ensure(sizeof(double) * 3 * NS));
    BBRT_CUDA(set->set_d.ensure(sizeof(double) * 3 * NS));
    BBRT_CUDA(set->ray_member.ensure(sizeof(int) * NS));
    bbrt_trace_out dev{};
    bbrt::SetIO io;
    if (outs) {
        const bbrt_trace_out& o0 = outs[first];
        dev.record_bounces = K;
        auto bind = [&](const void* want, DevBuf& b, size_t bytes, auto*& field, auto*& io_field) -> int {
            using T = std::remove_pointer_t<std::remove_reference_t<decltype(field)>>;
            if (!want || bytes == 0) return BBRT_OK;
            BBRT_CUDA(b.ensure(bytes));
            field = static_cast<T*>(b.p);
            io_field = static_cast<T*>(b.p);
            return BBRT_OK;
        };
        int rc;
        if ((rc = bind(o0.status, set->o_status, sizeof(int) * NS, dev.status, io.status))) return rc;
        if ((rc = bind(o0.bounce_count, set->o_bounce, sizeof(int) * NS, dev.bounce_count, io.bounce_count))) return rc;
        if ((rc = bind(o0.exit_dir, set->o_dir, sizeof(double) * 3 * NS, dev.exit_dir, io.exit_dir))) return rc;
        if ((rc = bind(o0.end_point, set->o_end, sizeof(double) * 3 * NS, dev.end_point, io.end_point))) return rc;
        if ((rc = bind(o0.hit_object, set->o_hobj, sizeof(int) * NS * KS, dev.hit_object, io.hit_object))) return rc;
        if ((rc = bind(o0.hit_point, set->o_hpt, sizeof(double) * 3 * NS * KS, dev.hit_point, io.hit_point))) return rc;
        if ((rc = bind(o0.hit_uv, set->o_huv, sizeof(double) * 2 * NS * KS, dev.hit_uv, io.hit_uv))) return rc;
        if ((rc = bind(o0.err_object, set->o_eobj, sizeof(int) * NS, dev.err_object, io.err_object))) return rc;
        if ((rc = bind(o0.err_value, set->o_eval, sizeof(double) * 2 * NS, dev.err_value, io.err_value))) return rc;
        if ((rc = bind(o0.ray_work, set->o_work, sizeof(long long) * 4 * NS, dev.ray_work, io.ray_work))) return rc;
    }
    set->io.assign(M, bbrt::MemberIO());
    for (int m = 0; m < M; ++m) {
        bbrt::MemberIO& x = set->io[m];
        x.o = origins[m];
        x.d = dirs[m];
        x.off = off[m];
        x.n = n[m];
        x.obj_off = set->obj_off[m];
        if (outs) {
            const bbrt_trace_out& om = outs[m];
            x.status = om.status; x.bounce_count = om.bounce_count; x.exit_dir = om.exit_dir;
            x.end_point = om.end_point; x.hit_object = om.hit_object; x.hit_point = om.hit_point;
            x.hit_uv = om.hit_uv; x.err_object = om.err_object; x.err_value = om.err_value;
            x.ray_work = om.ray_work;
        }
    }
    BBRT_CUDA(set->io_dev.ensure(sizeof(bbrt::MemberIO) * M));
    BBRT_CUDA(cudaEventRecord(set->ev[0], st));
    BBRT_CUDA(cudaMemcpyAsync(set->io_dev.p, set->io.data(), sizeof(bbrt::MemberIO) * M, cudaMemcpyHostToDevice, st));
    io.m = static_cast<const bbrt::MemberIO*>(set->io_dev.p);
    io.n_members = M;
    io.n = N;
    io.K = K;
    io.o = static_cast<double*>(set->set_o.p);
    io.d = static_cast<double*>(set->set_d.p);
    io.ray_member = static_cast<int*>(set->ray_member.p);
    BBRT_CUDA(bbrt::set_gather(io, st));
    s->member_rays = off;
    s->ray_member = io.ray_member;
    float kms = 0.0f;
    int rc = run_trace_device(s, io.o, io.d, N, max_bounces, outs ? &dev : nullptr, nullptr, 1, st, stats != nullptr,
                              hs, stats ? &kms : nullptr);
    s->member_rays.clear();
    s->ray_member = nullptr;
    if (rc) return rc;
    if (outs) BBRT_CUDA(bbrt::set_scatter(io, st));
    BBRT_CUDA(cudaEventRecord(set->ev[1], st));
    BBRT_CUDA(cudaEventSynchronize(set->ev[1]));
    float tot = 0.0f;
    BBRT_CUDA(cudaEventElapsedTime(&tot, set->ev[0], set->ev[1]));
    if (set_ms) *set_ms = tot;
    if (stats) fill_stats(s, hs, N, kms, tot, stats);
    return BBRT_OK;
}

}  // extern "C"
