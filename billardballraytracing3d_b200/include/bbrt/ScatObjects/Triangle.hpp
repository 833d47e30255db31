// Drop-in for the reference's include/ScatObjects/Triangle.hpp (Triangle.hpp:9-32):
// a flat triangle ScatObject whose intersect() runs Moller-Trumbore on the GPU.
#pragma once

#include <memory>
#include <optional>

#include "../ScatObject.hpp"

class Triangle : public ScatObject {
public:
    Triangle(Vec3 v0, Vec3 v1, Vec3 v2) : v0_(v0), v1_(v1), v2_(v2) {
        bbrt_object_desc d = device_desc(nullptr);
        bbrt_config cfg;
        bbrt_config_init(&cfg);
        scene_ = std::make_shared<bbrt_detail::SceneHandle>();
        bbrt_detail::check(bbrt_scene_create(&d, 1, &cfg, &scene_->h), "Triangle");
        bbrt_object_info info;
        bbrt_detail::check(bbrt_object_info_get(scene_->h, 0, &info), "Triangle");
        box_.min = { info.box_min[0], info.box_min[1], info.box_min[2] };
        box_.max = { info.box_max[0], info.box_max[1], info.box_max[2] };
        centroid_ = { info.centroid[0], info.centroid[1], info.centroid[2] };
    }

    std::optional<Hit> intersect(const Ray& ray) const override {
        const double o[3] = { ray.origin.x, ray.origin.y, ray.origin.z };
        const double d[3] = { ray.dir.x, ray.dir.y, ray.dir.z };
        bbrt_hit h;
        bbrt_detail::check(bbrt_intersect(scene_->h, o, d, 1, BBRT_QUERY_OBJECT, 0, 0, &h, nullptr),
                           "Triangle::intersect");
        if (h.object < 0) return std::nullopt;
        Hit hit;
        hit.t = h.t;
        hit.point = { h.point[0], h.point[1], h.point[2] };
        hit.normal = { h.normal[0], h.normal[1], h.normal[2] };
        return hit;
    }

    bbrt_object_desc device_desc(bbrt_patch_desc*) const override {
        bbrt_object_desc d{};
        d.kind = BBRT_OBJ_TRIANGLE;
        const double v[9] = { v0_.x, v0_.y, v0_.z, v1_.x, v1_.y, v1_.z, v2_.x, v2_.y, v2_.z };
        for (int k = 0; k < 9; ++k) d.tri[k] = v[k];
        return d;
    }

private:
    Vec3 v0_, v1_, v2_;
    std::shared_ptr<bbrt_detail::SceneHandle> scene_;
};
