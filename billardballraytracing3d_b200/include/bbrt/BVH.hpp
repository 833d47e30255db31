// Drop-in for the reference's include/BVH.hpp (ray_box :14-32, union_box
// :34-43, class BVH :65-190): a bounding-volume hierarchy over ScatObjects
// whose intersect() runs on the GPU.
//
// The constructor describes every object to libbbrt_cuda.so, which builds
// the same median-split tree as the reference (same objects in the same
// order, so the same std::nth_element partitions) and keeps it on the
// device.  intersect(ray) is BVH::intersect for one ray; intersect(rays) is
// the batch form, one GPU launch for all rays.  A patch's Newton failure
// throws the reference's std::runtime_error; the batch form reports it per
// ray instead (BatchHit::error).
#pragma once

#include <algorithm>
#include <cstdint>
#include <limits>
#include <memory>
#include <optional>
#include <string>
#include <utility>
#include <vector>

#include "ScatObject.hpp"
#include "ScatObjects/SurfacePatch.hpp"

// Slab test with a precomputed inverse direction (host helper).
inline bool ray_box(const Vec3& origin, const double inv_dir[3], const AABB& box, double& tmin_out) {
    const double o[3] = { origin.x, origin.y, origin.z };
    const double lo[3] = { box.min.x, box.min.y, box.min.z };
    const double hi[3] = { box.max.x, box.max.y, box.max.z };
    double t0 = -std::numeric_limits<double>::infinity();
    double t1 = std::numeric_limits<double>::infinity();
    for (int a = 0; a < 3; ++a) {
        double ta = (lo[a] - o[a]) * inv_dir[a];
        double tb = (hi[a] - o[a]) * inv_dir[a];
        if (inv_dir[a] < 0.0) std::swap(ta, tb);
        t0 = std::max(t0, ta);
        t1 = std::min(t1, tb);
        if (t1 < t0) return false;
    }
    tmin_out = t0;
    return t1 >= std::max(t0, 0.0);
}

inline AABB union_box(const AABB& a, const AABB& b) {
    AABB u;
    u.min = { std::min(a.min.x, b.min.x), std::min(a.min.y, b.min.y), std::min(a.min.z, b.min.z) };
    u.max = { std::max(a.max.x, b.max.x), std::max(a.max.y, b.max.y), std::max(a.max.z, b.max.z) };
    return u;
}

class BVH {
public:
    // One ray's answer from the batch form.
    struct BatchHit {
        std::optional<Hit> hit;
        std::string error;   // non-empty when the reference would have thrown
    };

    explicit BVH(std::vector<const ScatObject*> objects, int leaf_threshold = 4)
        : objects_(std::move(objects)) {
        if (objects_.empty()) throw std::invalid_argument("BVH: no objects");
        std::vector<bbrt_patch_desc> storage(objects_.size());
        std::vector<bbrt_object_desc> descs(objects_.size());
        for (size_t i = 0; i < objects_.size(); ++i) descs[i] = objects_[i]->device_desc(&storage[i]);
        bbrt_config cfg = SurfacePatch::config();
        cfg.leaf_threshold = leaf_threshold;
        scene_ = std::make_shared<bbrt_detail::SceneHandle>();
        bbrt_detail::check(bbrt_scene_create(descs.data(), static_cast<int>(descs.size()), &cfg, &scene_->h), "BVH");
        read_zones();
    }

    // A BVH over an existing scene whose object i is objects[i] (the tree
    // the scene was built with).
    BVH(std::vector<const ScatObject*> objects, std::shared_ptr<bbrt_detail::SceneHandle> scene)
        : objects_(std::move(objects)), scene_(std::move(scene)) {
        bbrt_scene_info s = info();
        if (s.n_objects != static_cast<int>(objects_.size()))
            throw std::invalid_argument("BVH: the scene holds " + std::to_string(s.n_objects) + " objects, not " +
                                        std::to_string(objects_.size()));
        read_zones();
    }

    // BVH::intersect (BVH.hpp:75-128) for one ray.
    std::optional<Hit> intersect(const Ray& ray) const {
        BatchHit b = intersect_one(ray);
        if (!b.error.empty()) throw std::runtime_error(b.error);
        return b.hit;
    }

    // The batch form: every ray in one device call.
    std::vector<BatchHit> intersect(const std::vector<Ray>& rays) const {
        const size_t n = rays.size();
        std::vector<double> o(3 * n), d(3 * n);
        for (size_t i = 0; i < n; ++i) {
            o[3 * i] = rays[i].origin.x; o[3 * i + 1] = rays[i].origin.y; o[3 * i + 2] = rays[i].origin.z;
            d[3 * i] = rays[i].dir.x; d[3 * i + 1] = rays[i].dir.y; d[3 * i + 2] = rays[i].dir.z;
        }
        std::vector<bbrt_hit> h(n);
        bbrt_detail::check(bbrt_intersect(scene_->h, o.data(), d.data(), static_cast<long long>(n), BBRT_QUERY_BVH, 0,
                                          0, h.data(), nullptr),
                           "BVH::intersect");
        std::vector<BatchHit> out(n);
        for (size_t i = 0; i < n; ++i) out[i] = to_batch(h[i]);
        return out;
    }

    bbrt_scene_t scene() const { return scene_->h; }
    const std::vector<const ScatObject*>& objects() const { return objects_; }

    bbrt_scene_info info() const {
        bbrt_scene_info s;
        bbrt_detail::check(bbrt_scene_info_get(scene_->h, &s), "BVH");
        return s;
    }

    // zoneID of object i (-1 for a triangle), as the library holds it.
    long long zone_of(int i) const { return zone_[static_cast<size_t>(i)]; }

private:
    std::vector<const ScatObject*> objects_;
    std::vector<long long> zone_;
    std::shared_ptr<bbrt_detail::SceneHandle> scene_;

    void read_zones() {
        zone_.resize(objects_.size());
        for (size_t i = 0; i < objects_.size(); ++i) {
            bbrt_object_info info;
            bbrt_detail::check(bbrt_object_info_get(scene_->h, static_cast<int>(i), &info), "BVH");
            zone_[i] = info.zone_id;
        }
    }

    BatchHit intersect_one(const Ray& ray) const {
        const double o[3] = { ray.origin.x, ray.origin.y, ray.origin.z };
        const double d[3] = { ray.dir.x, ray.dir.y, ray.dir.z };
        bbrt_hit h;
        bbrt_detail::check(bbrt_intersect(scene_->h, o, d, 1, BBRT_QUERY_BVH, 0, 0, &h, nullptr), "BVH::intersect");
        return to_batch(h);
    }

    BatchHit to_batch(const bbrt_hit& h) const {
        BatchHit b;
        if (h.status) {
            const long long zone = h.err_object >= 0 ? zone_[static_cast<size_t>(h.err_object)] : -1;
            b.error = bbrt_detail::newton_message(h.status, zone, h.err_value, SurfacePatch::kNewtonMaxIters);
            return b;
        }
        if (h.object < 0) return b;
        Hit hit;
        hit.t = h.t;
        hit.point = { h.point[0], h.point[1], h.point[2] };
        hit.normal = { h.normal[0], h.normal[1], h.normal[2] };
        hit.object = objects_[static_cast<size_t>(h.object)];
        b.hit = hit;
        return b;
    }
};
