// Drop-in for the reference's include/RayTracingDriver.hpp
// (RayTracingDriver.hpp:68-425): load a directory of IFGF-RP patches, build
// one BVH, bounce rays specularly until they escape, reach the bounce cap
// or fail, and write the paths as VTK.
//
// Same constructors, RayPath, set_rays/run/paths/patches/patch_index_of/
// trace_ray/self_intersect_epsilon/write_vtk and exception texts.  The
// trace itself runs on the GPU: run() traces all configured rays in batched
// bbrt_trace calls (one per chunk of rays) and rebuilds every RayPath from
// the recorded hits; trace_ray() is the one-ray form (concurrent calls from
// several threads are traced together as one batch).  trace_rays() is the
// batch form for callers with their own rays.
#pragma once

#include <algorithm>
#include <cmath>
#include <condition_variable>
#include <exception>
#include <filesystem>
#include <fstream>
#include <memory>
#include <mutex>
#include <optional>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "BVH.hpp"
#include "ScatObject.hpp"
#include "ScatObjects/SurfacePatch.hpp"

class RayTracingDriver {
public:
    // One traced ray's outcome (RayTracingDriver.hpp:70-89).
    struct RayPath {
        enum class Status { Escaped, Trapped, Error };
        std::vector<Vec3> points;   // source, each hit point, then (Escaped) the tail point
        Status status = Status::Trapped;
        int bounce_count = 0;
        std::string error_message;  // only when status == Error
        std::vector<const ScatObject*> hit_objects;   // hit_objects[k] produced points[k+1]
    };

    // Every regular "*.txt" file in the directory, in sorted path order.
    explicit RayTracingDriver(const std::string& patch_directory) {
        namespace fs = std::filesystem;
        if (!fs::exists(patch_directory) || !fs::is_directory(patch_directory))
            throw std::runtime_error("RayTracingDriver: not a directory: " + patch_directory);
        std::vector<fs::path> files;
        for (const auto& e : fs::directory_iterator(patch_directory))
            if (e.is_regular_file() && e.path().extension() == ".txt") files.push_back(e.path());
        std::sort(files.begin(), files.end());
        if (files.empty())
            throw std::runtime_error("RayTracingDriver: no *.txt patch files found in: " + patch_directory);
        std::vector<std::string> paths;
        for (const auto& f : files) paths.push_back(f.string());
        load(paths);
    }

    // "<directory><file_prefix><i>.txt" for i in [first, last], 1-based.
    RayTracingDriver(const std::string& directory, const std::string& file_prefix, int first_index_1based,
                     int last_index_1based) {
        if (last_index_1based < first_index_1based)
            throw std::invalid_argument("RayTracingDriver: empty patch index range [" +
                                        std::to_string(first_index_1based) + ", " +
                                        std::to_string(last_index_1based) + "]");
        std::vector<std::string> paths;
        for (int i = first_index_1based; i <= last_index_1based; ++i)
            paths.push_back(directory + file_prefix + std::to_string(i) + ".txt");
        load(paths);
    }

    RayTracingDriver(const RayTracingDriver&) = delete;
    RayTracingDriver& operator=(const RayTracingDriver&) = delete;

    void set_rays(std::vector<Vec3> sources, std::vector<Vec3> directions) {
        if (sources.size() != directions.size())
            throw std::invalid_argument(
                "RayTracingDriver::set_rays: sources and directions must be the same length (paired 1:1) — got " +
                std::to_string(sources.size()) + " sources and " + std::to_string(directions.size()) + " directions");
        for (size_t i = 0; i < directions.size(); ++i) {
            const Vec3& d = directions[i];
            if (d.x * d.x + d.y * d.y + d.z * d.z < 1e-300)
                throw std::invalid_argument("RayTracingDriver::set_rays: direction " + std::to_string(i) +
                                            " has zero length");
        }
        sources_ = std::move(sources);
        directions_ = std::move(directions);
    }

    void run(int max_bounces = 50) { paths_ = trace_rays(sources_, directions_, max_bounces); }

    const std::vector<RayPath>& paths() const { return paths_; }
    const std::vector<std::unique_ptr<SurfacePatch>>& patches() const { return patches_; }

    long long patch_index_of(const ScatObject* object) const {
        auto it = index_of_.find(object);
        return it == index_of_.end() ? -1 : static_cast<long long>(it->second);
    }

    // RayTracingDriver::trace_ray (RayTracingDriver.hpp:172-242) for one ray.
    //
    // The reference's drivers call this from many OpenMP threads at once
    // (PlaneSourceDriver.hpp:96-99, BounceMapDriver.hpp:153-237); one GPU
    // launch per ray would serialise them.  Concurrent calls are therefore
    // combined: a caller queues its ray, and whichever caller finds no batch
    // in flight takes every queued ray with the same max_bounces and traces
    // them as one batch while the others wait (and queue the next batch).  A
    // single-threaded caller still gets one launch per ray: loops that own
    // their rays should call trace_rays() or run().  The result of every ray
    // is the one trace_rays() gives it; an exception is rethrown in every
    // caller of the failed batch.
    RayPath trace_ray(const Vec3& origin, const Vec3& direction, int max_bounces) const {
        Combiner::Slot slot;
        slot.origin = origin;
        slot.direction = direction;
        slot.max_bounces = max_bounces;
        std::unique_lock<std::mutex> lk(comb_.mu);
        comb_.queue.push_back(&slot);
        while (!slot.done) {
            if (comb_.busy) {
                comb_.cv.wait(lk);
                continue;
            }
            comb_.busy = true;
            std::vector<Combiner::Slot*> batch;
            std::vector<Combiner::Slot*> rest;
            const int mb = comb_.queue.front()->max_bounces;
            for (Combiner::Slot* q : comb_.queue) (q->max_bounces == mb ? batch : rest).push_back(q);
            comb_.queue.swap(rest);
            lk.unlock();
            std::vector<Vec3> os, ds;
            os.reserve(batch.size());
            ds.reserve(batch.size());
            for (const Combiner::Slot* q : batch) {
                os.push_back(q->origin);
                ds.push_back(q->direction);
            }
            std::vector<RayPath> res;
            std::exception_ptr err;
            try {
                res = trace_rays(os, ds, mb);
            } catch (...) {
                err = std::current_exception();
            }
            lk.lock();
            for (size_t k = 0; k < batch.size(); ++k) {
                if (err) batch[k]->error = err;
                else batch[k]->path = std::move(res[k]);
                batch[k]->done = true;
            }
            comb_.busy = false;
            comb_.cv.notify_all();
        }
        lk.unlock();
        if (slot.error) std::rethrow_exception(slot.error);
        return std::move(slot.path);
    }

    // trace_ray for every (origins[i], directions[i]), on the GPU in chunks.
    std::vector<RayPath> trace_rays(const std::vector<Vec3>& origins, const std::vector<Vec3>& directions,
                                    int max_bounces) const {
        if (origins.size() != directions.size())
            throw std::invalid_argument("RayTracingDriver::trace_rays: origins and directions differ in length");
        const long long n = static_cast<long long>(origins.size());
        std::vector<RayPath> out(static_cast<size_t>(n));
        const int K = std::max(max_bounces, 0);
        const long long chunk = std::max<long long>(4096, (1LL << 23) / std::max(K, 1));
        for (long long c0 = 0; c0 < n; c0 += chunk) trace_chunk(origins, directions, c0, std::min(n, c0 + chunk), K, out);
        return out;
    }

    // RayTracingDriver::self_intersect_epsilon (RayTracingDriver.hpp:260-265).
    double self_intersect_epsilon(const ScatObject* leaving_object = nullptr) const {
        const double pad = leaving_object ? leaving_object->self_intersect_padding() : max_patch_sagitta_;
        return std::max(kSelfIntersectEpsilonFactor * scene_diagonal_, kSagittaClearanceFactor * pad);
    }

    // Legacy ASCII VTK PolyData, one 2-point LINE per bounce leg with
    // RayID / BounceIndex cell scalars (RayTracingDriver.hpp:270-310).
    void write_vtk(const std::string& filename) const {
        std::ofstream out(filename);
        if (!out.is_open())
            throw std::runtime_error("RayTracingDriver::write_vtk: cannot open output file: " + filename);
        size_t n_points = 0, n_legs = 0;
        for (const RayPath& p : paths_) {
            n_points += p.points.size();
            n_legs += p.points.empty() ? 0 : p.points.size() - 1;
        }
        out << "# vtk DataFile Version 3.0\nBilliard-ball ray traces\nASCII\nDATASET POLYDATA\n";
        out << "POINTS " << n_points << " double\n";
        for (const RayPath& p : paths_)
            for (const Vec3& v : p.points) out << v.x << ' ' << v.y << ' ' << v.z << '\n';
        out << "LINES " << n_legs << ' ' << n_legs * 3 << '\n';
        size_t base = 0;
        for (const RayPath& p : paths_) {
            for (size_t k = 0; k + 1 < p.points.size(); ++k) out << "2 " << base + k << ' ' << base + k + 1 << '\n';
            base += p.points.size();
        }
        out << "CELL_DATA " << n_legs << '\n';
        out << "SCALARS RayID int 1\nLOOKUP_TABLE default\n";
        for (size_t r = 0; r < paths_.size(); ++r)
            for (size_t k = 0; k + 1 < paths_[r].points.size(); ++k) out << r << '\n';
        out << "SCALARS BounceIndex int 1\nLOOKUP_TABLE default\n";
        for (const RayPath& p : paths_)
            for (size_t k = 0; k + 1 < p.points.size(); ++k) out << k << '\n';
    }

    const BVH& bvh() const { return *bvh_; }
    double scene_diagonal() const { return scene_diagonal_; }

private:
    std::vector<std::unique_ptr<SurfacePatch>> patches_;
    std::unique_ptr<BVH> bvh_;
    double scene_diagonal_ = 0.0;
    double max_patch_sagitta_ = 0.0;
    std::vector<Vec3> sources_, directions_;
    std::vector<RayPath> paths_;
    std::unordered_map<const ScatObject*, size_t> index_of_;

    // Rays of concurrent trace_ray() calls waiting to be traced together.
    struct Combiner {
        struct Slot {
            Vec3 origin, direction;
            int max_bounces = 0;
            bool done = false;
            RayPath path;
            std::exception_ptr error;
        };
        std::mutex mu;
        std::condition_variable cv;
        std::vector<Slot*> queue;
        bool busy = false;   // a batch is being traced
    };
    mutable Combiner comb_;

    static constexpr double kSelfIntersectEpsilonFactor = 1e-9;   // RayTracingDriver.hpp:328
    static constexpr double kSagittaClearanceFactor = 5.0;        // RayTracingDriver.hpp:337
    static constexpr double kBackfaceHitTol = 1e-9;               // RayTracingDriver.hpp:344

    // Reads every file, builds one scene (host set-up and BVH once, in file
    // order) and gives each SurfacePatch its object of that scene.
    void load(const std::vector<std::string>& paths) {
        std::vector<SurfacePatch::Data> data;
        data.reserve(paths.size());
        for (const auto& p : paths) data.push_back(SurfacePatch::load(p));
        std::vector<bbrt_patch_desc> pd(data.size());
        std::vector<bbrt_object_desc> od(data.size());
        for (size_t i = 0; i < data.size(); ++i) {
            pd[i] = describe(data[i]);
            od[i] = bbrt_object_desc{};
            od[i].kind = BBRT_OBJ_PATCH;
            od[i].patch = &pd[i];
        }
        bbrt_config cfg = SurfacePatch::config();
        cfg.self_intersect_eps_factor = kSelfIntersectEpsilonFactor;
        cfg.sagitta_clearance_factor = kSagittaClearanceFactor;
        cfg.backface_tol = kBackfaceHitTol;
        auto scene = std::make_shared<bbrt_detail::SceneHandle>();
        bbrt_detail::check(bbrt_scene_create(od.data(), static_cast<int>(od.size()), &cfg, &scene->h),
                           "RayTracingDriver");
        std::vector<const ScatObject*> objs;
        for (size_t i = 0; i < data.size(); ++i) {
            patches_.push_back(std::make_unique<SurfacePatch>(std::move(data[i]), scene, static_cast<int>(i)));
            objs.push_back(patches_.back().get());
            index_of_[patches_.back().get()] = i;
        }
        bvh_ = std::make_unique<BVH>(std::move(objs), scene);
        const bbrt_scene_info info = bvh_->info();
        scene_diagonal_ = info.scene_diagonal;
        max_patch_sagitta_ = info.max_patch_sagitta;
    }

    static bbrt_patch_desc describe(const SurfacePatch::Data& d) {
        bbrt_patch_desc p{};
        p.imax = d.imax; p.jmax = d.jmax; p.kmax = d.kmax; p.zone_id = d.zoneID;
        p.u_nodes = d.uNodes.data(); p.v_nodes = d.vNodes.data();
        p.x = d.x.data(); p.y = d.y.data(); p.z = d.z.data();
        p.dxdu = d.dxdu.data(); p.dydu = d.dydu.data(); p.dzdu = d.dzdu.data();
        p.dxdv = d.dxdv.data(); p.dydv = d.dydv.data(); p.dzdv = d.dzdv.data();
        p.nu_x = d.nuX.data(); p.nu_y = d.nuY.data(); p.nu_z = d.nuZ.data();
        return p;
    }

    // The reference's error_message for a failed ray (RayTracingDriver.hpp:177-228).
    std::string error_text(int status, int err_object, const double* ev) const {
        switch (status) {
            case BBRT_RAY_BAD_DIR: return "RayTracingDriver::trace_ray: zero-length direction";
            case BBRT_RAY_WENT_INSIDE:
                return "RayTracingDriver::trace_ray: hit back face of patch (dot(dir, normal) > 0) — ray likely "
                       "tunneled through a triangulation gap";
            default: {
                const long long zone = err_object >= 0 ? bvh_->zone_of(err_object) : -1;
                return bbrt_detail::newton_message(status, zone, ev, SurfacePatch::kNewtonMaxIters);
            }
        }
    }

    void trace_chunk(const std::vector<Vec3>& origins, const std::vector<Vec3>& directions, long long a, long long b,
                     int K, std::vector<RayPath>& out) const {
        const long long n = b - a;
        std::vector<double> o(3 * n), d(3 * n), endp(3 * n), ev(2 * n), hp(3 * n * K);
        std::vector<int> st(n), bc(n), eo(n), ho(n * K);
        for (long long i = 0; i < n; ++i) {
            const Vec3& O = origins[a + i];
            const Vec3& D = directions[a + i];
            o[3 * i] = O.x; o[3 * i + 1] = O.y; o[3 * i + 2] = O.z;
            d[3 * i] = D.x; d[3 * i + 1] = D.y; d[3 * i + 2] = D.z;
        }
        bbrt_trace_out t{};
        t.status = st.data();
        t.bounce_count = bc.data();
        t.end_point = endp.data();
        t.record_bounces = K;
        t.hit_object = K ? ho.data() : nullptr;
        t.hit_point = K ? hp.data() : nullptr;
        t.err_object = eo.data();
        t.err_value = ev.data();
        bbrt_detail::check(bbrt_trace(bvh_->scene(), o.data(), d.data(), n, K, 0, &t, nullptr, nullptr),
                           "RayTracingDriver::trace_ray");
        const auto& objs = bvh_->objects();
        for (long long i = 0; i < n; ++i) {
            RayPath& p = out[static_cast<size_t>(a + i)];
            p.points.assign(1, origins[a + i]);
            p.bounce_count = bc[i];
            for (int k = 0; k < bc[i]; ++k) {
                const double* q = &hp[3 * (i * K + k)];
                p.points.push_back({ q[0], q[1], q[2] });
                p.hit_objects.push_back(objs[static_cast<size_t>(ho[i * K + k])]);
            }
            if (st[i] == BBRT_RAY_ESCAPED) {
                p.status = RayPath::Status::Escaped;
                p.points.push_back({ endp[3 * i], endp[3 * i + 1], endp[3 * i + 2] });
            } else if (st[i] == BBRT_RAY_MAX_BOUNCES) {
                p.status = RayPath::Status::Trapped;
            } else {
                p.status = RayPath::Status::Error;
                p.error_message = error_text(st[i], eo[i], &ev[2 * i]);
            }
        }
    }
};
