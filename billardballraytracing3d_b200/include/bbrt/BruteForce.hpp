// Drop-in for the reference's include/BruteForce.hpp (BruteForce.hpp:7-16):
// the no-tree ground truth, every object tested, closest hit kept.
//
// brute_force_intersect(ray, objects) keeps the reference's call: each
// object's intersect() (on the GPU) in list order, the first Newton failure
// thrown.  BruteForce is the batch form over a device scene: every ray
// against every object in one launch (bbrt_intersect, BBRT_QUERY_BRUTE).
#pragma once

#include <memory>
#include <optional>
#include <vector>

#include "BVH.hpp"
#include "ScatObject.hpp"

inline std::optional<Hit> brute_force_intersect(const Ray& ray, const std::vector<const ScatObject*>& objects) {
    std::optional<Hit> best;
    for (const ScatObject* obj : objects) {
        std::optional<Hit> h = obj->intersect(ray);
        if (h && (!best || h->t < best->t)) best = h;
    }
    return best;
}

class BruteForce {
public:
    explicit BruteForce(std::vector<const ScatObject*> objects) : bvh_(std::move(objects)) {}

    // Per ray: the closest hit over every object (Hit::object set), or the
    // first Newton failure's message in list order.
    std::vector<BVH::BatchHit> intersect(const std::vector<Ray>& rays) const {
        const size_t n = rays.size();
        std::vector<double> o(3 * n), d(3 * n);
        for (size_t i = 0; i < n; ++i) {
            o[3 * i] = rays[i].origin.x; o[3 * i + 1] = rays[i].origin.y; o[3 * i + 2] = rays[i].origin.z;
            d[3 * i] = rays[i].dir.x; d[3 * i + 1] = rays[i].dir.y; d[3 * i + 2] = rays[i].dir.z;
        }
        std::vector<bbrt_hit> h(n);
        bbrt_detail::check(bbrt_intersect(bvh_.scene(), o.data(), d.data(), static_cast<long long>(n),
                                          BBRT_QUERY_BRUTE, 0, 0, h.data(), nullptr),
                           "BruteForce::intersect");
        std::vector<BVH::BatchHit> out(n);
        const auto& objs = bvh_.objects();
        for (size_t i = 0; i < n; ++i) {
            if (h[i].status) {
                const ScatObject* bad = h[i].err_object >= 0 ? objs[static_cast<size_t>(h[i].err_object)] : nullptr;
                const auto* patch = dynamic_cast<const SurfacePatch*>(bad);
                out[i].error = bbrt_detail::newton_message(h[i].status, patch ? patch->data().zoneID : -1,
                                                           h[i].err_value, SurfacePatch::kNewtonMaxIters);
                continue;
            }
            if (h[i].object < 0) continue;
            Hit hit;
            hit.t = h[i].t;
            hit.point = { h[i].point[0], h[i].point[1], h[i].point[2] };
            hit.normal = { h[i].normal[0], h[i].normal[1], h[i].normal[2] };
            hit.object = objs[static_cast<size_t>(h[i].object)];
            out[i].hit = hit;
        }
        return out;
    }

private:
    BVH bvh_;
};
