// Reference oracle harness — TEST INFRASTRUCTURE ONLY.
//
// Compiles the reference's own headers (manuelarturosantana/BillardBallRayTracing3D,
// include/*.hpp) into oracle/_ref/libbbrt_ref.so and exposes a small C API
// so tests and the CPU-baseline leg of bench.py can run the reference's
// unmodified algorithms on generated scenes:
//   * RayTracingDriver::trace_ray under `#pragma omp parallel for
//     schedule(dynamic)`, the loop PlaneSourceDriver.hpp:96-99 uses;
//   * PlaneSourceDriver::run and BounceMapDriver::run as they are;
//   * BVH::intersect vs brute_force_intersect over Triangle objects
//     (the shape of tests/Triangle_Intersect.cpp).
//
// The only change to the reference is made by oracle/build_ref.sh on a
// throw-away copy of its headers: the three `static constexpr` trace
// constants of SurfacePatch (SurfacePatch.hpp:117,121,122) become
// `static inline` so ref_set_constants() can set a workload's coarse-grid
// size and Newton tolerance.  Their initial values stay the reference's.
//
// Nothing in the product links or loads this file.

// Standard headers first, so the access override below only reaches the
// reference's own classes.
#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <complex>
#include <cstddef>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <functional>
#include <iostream>
#include <limits>
#include <memory>
#include <optional>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>
#include <sys/resource.h>
#include <sys/time.h>
#include <unistd.h>
#include <omp.h>

#define private public
#include "RayTracingDriver.hpp"
#include "PlaneSourceDriver.hpp"
#include "BounceMapDriver.hpp"
#include "ScatObjects/Triangle.hpp"
#include "BVH.hpp"
#include "BruteForce.hpp"
#undef private

namespace {

thread_local std::string g_err;

// Per-ray status codes, identical to include/bbrt.h's BBRT_RAY_* values.
enum { ESCAPED = 0, MAX_BOUNCES = 1, NEWTON_SINGULAR = 2, NEWTON_NOCONV = 3,
       NEWTON_DOMAIN = 4, WENT_INSIDE = 5, BAD_DIR = 6, UNKNOWN_ERROR = 99 };

int classify_error(const std::string& msg) {
    if (msg.find("singular Jacobian") != std::string::npos) return NEWTON_SINGULAR;
    if (msg.find("failed to converge") != std::string::npos) return NEWTON_NOCONV;
    if (msg.find("outside the patch") != std::string::npos) return NEWTON_DOMAIN;
    if (msg.find("back face") != std::string::npos) return WENT_INSIDE;
    if (msg.find("zero-length direction") != std::string::npos) return BAD_DIR;
    return UNKNOWN_ERROR;
}

long long zone_in_message(const std::string& msg) {
    const auto k = msg.find("zoneID ");
    if (k == std::string::npos) return -1;
    return std::atoll(msg.c_str() + k + 7);
}

int status_code(const RayTracingDriver::RayPath& p) {
    switch (p.status) {
        case RayTracingDriver::RayPath::Status::Escaped: return ESCAPED;
        case RayTracingDriver::RayPath::Status::Trapped: return MAX_BOUNCES;
        default: return classify_error(p.error_message);
    }
}

}  // namespace

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

void ref_set_constants(int coarse_n, int newton_max_iters, double newton_tol) {
    SurfacePatch::kCoarseGridSize = coarse_n;
    SurfacePatch::kNewtonMaxIters = newton_max_iters;
    SurfacePatch::kNewtonTol = newton_tol;
}

void* ref_open(const char* dir) {
    try {
        return new RayTracingDriver(std::string(dir));
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

void ref_close(void* h) { delete static_cast<RayTracingDriver*>(h); }

int ref_info(void* h, long long* n_patches, double* scene_diag, double* max_sagitta) {
    auto* d = static_cast<RayTracingDriver*>(h);
    *n_patches = static_cast<long long>(d->patches().size());
    *scene_diag = d->scene_diagonal_;
    *max_sagitta = d->max_patch_sagitta_;
    return 0;
}

long long ref_zone_id(void* h, int idx) {
    auto* d = static_cast<RayTracingDriver*>(h);
    return d->patches()[static_cast<size_t>(idx)]->data().zoneID;
}

// Set-up values of one patch: box (min,max), centroid, max sagitta, coarse
// grid n, and optionally the coarse grid xyz[n*n*3], sagitta[(n-1)^2],
// normals[(n-1)^2*3].
int ref_patch_setup(void* h, int idx, double* box6, double* centroid3, double* max_sag, int* n,
                    double* coarse_xyz, double* sagitta, double* normals) {
    auto* d = static_cast<RayTracingDriver*>(h);
    const SurfacePatch& p = *d->patches()[static_cast<size_t>(idx)];
    const AABB& b = p.bounding_box();
    box6[0] = b.min.x; box6[1] = b.min.y; box6[2] = b.min.z;
    box6[3] = b.max.x; box6[4] = b.max.y; box6[5] = b.max.z;
    centroid3[0] = p.centroid().x; centroid3[1] = p.centroid().y; centroid3[2] = p.centroid().z;
    *max_sag = p.max_sagitta();
    const auto& g = p.coarse_grid();
    *n = g.n;
    if (coarse_xyz) {
        for (int k = 0; k < g.n * g.n; ++k) {
            coarse_xyz[3 * k] = g.x[k]; coarse_xyz[3 * k + 1] = g.y[k]; coarse_xyz[3 * k + 2] = g.z[k];
        }
    }
    if (sagitta) for (size_t k = 0; k < g.cell_sagitta.size(); ++k) sagitta[k] = g.cell_sagitta[k];
    if (normals) {
        for (size_t k = 0; k < g.cell_normal.size(); ++k) {
            normals[3 * k] = g.cell_normal[k].x;
            normals[3 * k + 1] = g.cell_normal[k].y;
            normals[3 * k + 2] = g.cell_normal[k].z;
        }
    }
    return 0;
}

// trace_ray for n rays under OpenMP (schedule(dynamic), as PlaneSourceDriver.hpp:96).
// K = number of hits recorded per ray.  err_zone[i] = zoneID quoted by an
// Error message (-1 if none).  *seconds = wall time of the parallel loop.
int ref_trace(void* h, long long n, const double* o, const double* dirs, int max_bounces,
              int nthreads, int K, int* status, int* bounce_count, double* exit_dir,
              double* end_point, int* hit_obj, double* hit_pts, long long* err_zone,
              double* seconds) {
    auto* drv = static_cast<RayTracingDriver*>(h);
    if (nthreads > 0) omp_set_num_threads(nthreads);
    const double t0 = omp_get_wtime();
    #pragma omp parallel for schedule(dynamic)
    for (long long i = 0; i < n; ++i) {
        const Vec3 src{ o[3 * i], o[3 * i + 1], o[3 * i + 2] };
        const Vec3 dir{ dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2] };
        const RayTracingDriver::RayPath path = drv->trace_ray(src, dir, max_bounces);
        if (status) status[i] = status_code(path);
        if (bounce_count) bounce_count[i] = path.bounce_count;
        if (err_zone) err_zone[i] = path.status == RayTracingDriver::RayPath::Status::Error
                                        ? zone_in_message(path.error_message) : -1;
        const Vec3& last = path.points.back();
        if (end_point) { end_point[3 * i] = last.x; end_point[3 * i + 1] = last.y; end_point[3 * i + 2] = last.z; }
        if (exit_dir) {
            double ex = 0, ey = 0, ez = 0;
            if (path.status == RayTracingDriver::RayPath::Status::Escaped && path.points.size() >= 2) {
                const Vec3& prev = path.points[path.points.size() - 2];
                const Vec3 e = vec_normalize(vec_sub(last, prev));
                ex = e.x; ey = e.y; ez = e.z;
            }
            exit_dir[3 * i] = ex; exit_dir[3 * i + 1] = ey; exit_dir[3 * i + 2] = ez;
        }
        for (int k = 0; k < K; ++k) {
            const bool have = k < path.bounce_count;
            if (hit_obj) hit_obj[i * K + k] = have ? static_cast<int>(drv->patch_index_of(path.hit_objects[k])) : -1;
            if (hit_pts) {
                const Vec3 p = have ? path.points[k + 1] : Vec3{ 0, 0, 0 };
                hit_pts[(i * K + k) * 3] = p.x; hit_pts[(i * K + k) * 3 + 1] = p.y; hit_pts[(i * K + k) * 3 + 2] = p.z;
            }
        }
    }
    if (seconds) *seconds = omp_get_wtime() - t0;
    return 0;
}

// One BVH::intersect per ray (no bounce).  status: 0 hit/miss, else the
// Newton error code the query threw.  obj = patch index or -1.
int ref_intersect(void* h, long long n, const double* o, const double* dirs,
                  double* t, double* point, double* normal, int* obj, int* status) {
    auto* drv = static_cast<RayTracingDriver*>(h);
    for (long long i = 0; i < n; ++i) {
        Ray ray{ { o[3 * i], o[3 * i + 1], o[3 * i + 2] }, { dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2] } };
        status[i] = 0; obj[i] = -1; t[i] = 0;
        try {
            auto hit = drv->bvh_->intersect(ray);
            if (hit) {
                t[i] = hit->t;
                point[3 * i] = hit->point.x; point[3 * i + 1] = hit->point.y; point[3 * i + 2] = hit->point.z;
                normal[3 * i] = hit->normal.x; normal[3 * i + 1] = hit->normal.y; normal[3 * i + 2] = hit->normal.z;
                obj[i] = static_cast<int>(drv->patch_index_of(hit->object));
            }
        } catch (const std::exception& e) {
            status[i] = classify_error(e.what());
        }
    }
    return 0;
}

// PlaneSourceDriver(dir).run(...) as is; counts[n_patches] in sorted-file order.
int ref_plane_source(const char* dir, const double* c0, const double* c1, const double* d,
                     int nx, int ny, int max_bounces, int count_direct_hit, int nthreads,
                     long long* counts, double* seconds) {
    try {
        if (nthreads > 0) omp_set_num_threads(nthreads);
        PlaneSourceDriver ps{ std::string(dir) };
        const double t0 = omp_get_wtime();
        ps.run({ c0[0], c0[1], c0[2] }, { c1[0], c1[1], c1[2] }, { d[0], d[1], d[2] }, nx, ny,
               max_bounces, count_direct_hit != 0);
        if (seconds) *seconds = omp_get_wtime() - t0;
        for (size_t k = 0; k < ps.hit_count_.size(); ++k) counts[k] = ps.hit_count_[k];
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// BounceMapDriver(dir, prefix, first, last).run(...) as is.  Outputs are
// [n_sampled * grid_n * grid_n] in sampled-patch order.
int ref_bounce_map(const char* dir, const char* prefix, int first, int last, int grid_n,
                   int theta_n, int phi_n, double cone_deg, int max_bounces, int nthreads,
                   int* max_b, int* errors, double* seconds) {
    try {
        if (nthreads > 0) omp_set_num_threads(nthreads);
        BounceMapDriver bm{ std::string(dir), std::string(prefix), first, last };
        std::streambuf* old = std::cout.rdbuf(nullptr);   // silence the progress bar
        const double t0 = omp_get_wtime();
        bm.run(grid_n, theta_n, phi_n, cone_deg, max_bounces, false);
        if (seconds) *seconds = omp_get_wtime() - t0;
        std::cout.rdbuf(old);
        size_t w = 0;
        for (size_t p = 0; p < bm.patch_max_bounces_.size(); ++p) {
            for (size_t k = 0; k < bm.patch_max_bounces_[p].size(); ++k, ++w) {
                max_b[w] = bm.patch_max_bounces_[p][k];
                errors[w] = bm.patch_error_counts_[p][k];
            }
        }
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// BVH(objects, leaf_threshold).intersect vs brute_force_intersect over
// Triangle objects (tests/Triangle_Intersect.cpp:11-50 shape).
int ref_triangle_queries(int n_tris, const double* tris, int leaf_threshold, long long n_rays,
                         const double* o, const double* dirs, double* bvh_t, int* bvh_obj,
                         double* brute_t, int* brute_obj) {
    std::vector<Triangle> store;
    store.reserve(static_cast<size_t>(n_tris));
    for (int k = 0; k < n_tris; ++k) {
        const double* v = tris + 9 * k;
        store.emplace_back(Vec3{ v[0], v[1], v[2] }, Vec3{ v[3], v[4], v[5] }, Vec3{ v[6], v[7], v[8] });
    }
    std::vector<const ScatObject*> objects;
    for (auto& t : store) objects.push_back(&t);
    BVH bvh(objects, leaf_threshold);
    for (long long i = 0; i < n_rays; ++i) {
        Ray ray{ { o[3 * i], o[3 * i + 1], o[3 * i + 2] }, { dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2] } };
        auto hb = bvh.intersect(ray);
        auto hf = brute_force_intersect(ray, objects);
        bvh_t[i] = hb ? hb->t : -1.0;
        bvh_obj[i] = hb ? static_cast<int>(static_cast<const Triangle*>(hb->object) - store.data()) : -1;
        brute_t[i] = hf ? hf->t : -1.0;
        brute_obj[i] = hf ? 0 : -1;   // brute_force_intersect does not tag Hit::object
    }
    return 0;
}

}  // extern "C"
