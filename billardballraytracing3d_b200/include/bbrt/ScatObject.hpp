// Drop-in for the reference's include/ScatObject.hpp (Vec3, Ray, AABB, Hit,
// ScatObject; ScatObject.hpp:10-89), backed by libbbrt_cuda.so.
//
// The types keep the reference's names and members.  What changes is where
// intersect() runs: on the GPU, through the C ABI of bbrt.h.  Only the two
// concrete object kinds the device path implements exist (SurfacePatch,
// Triangle); a BVH over any other ScatObject subclass throws
// std::invalid_argument, because user virtual code cannot run on the device.
#pragma once

#include <limits>
#include <optional>
#include <stdexcept>
#include <string>

#include "bbrt.h"

struct Vec3 {
    double x, y, z;
};

struct Ray {
    Vec3 origin;
    Vec3 dir;
};

struct AABB {
    Vec3 min{ std::numeric_limits<double>::infinity(), std::numeric_limits<double>::infinity(),
              std::numeric_limits<double>::infinity() };
    Vec3 max{ -std::numeric_limits<double>::infinity(), -std::numeric_limits<double>::infinity(),
              -std::numeric_limits<double>::infinity() };
};

class ScatObject;

// What an intersection reports (ScatObject.hpp:34-47).
struct Hit {
    double t;
    Vec3 point;
    Vec3 normal;
    const ScatObject* object = nullptr;
};

namespace bbrt_detail {

// A failed library call as the reference's exception: std::invalid_argument
// for a bad argument, std::runtime_error otherwise.  The library's messages
// are the reference's own texts where the reference has one.
inline void check(int rc, const char* what) {
    if (rc == BBRT_OK) return;
    const char* last = bbrt_last_error();
    const std::string msg = (last && *last) ? std::string(last) : std::string(what) + ": failed";
    if (rc == BBRT_ERR_ARG) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}

// The reference's exception text for a per-ray Newton failure
// (SurfacePatch.hpp:618-646), rebuilt from the status code, the failing
// patch's zoneID and the value the reference quotes.
inline std::string newton_message(int status, long long zone, const double ev[2], int max_iters) {
    switch (status) {
        case BBRT_RAY_NEWTON_SINGULAR:
            return "SurfacePatch::intersect: singular Jacobian during Newton refinement (zoneID " +
                   std::to_string(zone) + "), likely a grazing ray";
        case BBRT_RAY_NEWTON_NOCONV:
            return "SurfacePatch::intersect: Newton refinement failed to converge in " + std::to_string(max_iters) +
                   " iterations (zoneID " + std::to_string(zone) + "), final step norm " + std::to_string(ev[0]);
        case BBRT_RAY_NEWTON_DOMAIN:
            return "SurfacePatch::intersect: Newton refinement converged outside the patch domain (u=" +
                   std::to_string(ev[0]) + ", v=" + std::to_string(ev[1]) + ", zoneID " + std::to_string(zone) + ")";
        case BBRT_RAY_STACK_OVERFLOW:
            return "BVH::intersect: traversal stack exceeded 64 entries";
        default:
            return "bbrt: ray failed with status " + std::to_string(status);
    }
}

// Owns one device scene (bbrt_scene_destroy on destruction).
struct SceneHandle {
    bbrt_scene_t h = nullptr;
    SceneHandle() = default;
    SceneHandle(const SceneHandle&) = delete;
    SceneHandle& operator=(const SceneHandle&) = delete;
    ~SceneHandle() { if (h) bbrt_scene_destroy(h); }
};

}  // namespace bbrt_detail

// Anything the BVH can hold (ScatObject.hpp:55-89).
class ScatObject {
public:
    virtual ~ScatObject() = default;

    const AABB& bounding_box() const { return box_; }
    const Vec3& centroid() const { return centroid_; }

    // Does this ray hit me, and where.  Runs on the GPU; throws the
    // reference's std::runtime_error when a patch's Newton refinement fails.
    virtual std::optional<Hit> intersect(const Ray& ray) const = 0;

    virtual double self_intersect_padding() const { return 0.0; }

    // The object's description for a device scene.  A patch writes its
    // bbrt_patch_desc into *storage, which must outlive the returned value.
    // Other ScatObject subclasses have no device form: their virtual
    // intersect() cannot run on the GPU, so a BVH over them is refused.
    virtual bbrt_object_desc device_desc(bbrt_patch_desc* storage) const {
        (void)storage;
        throw std::invalid_argument(
            "BVH: only SurfacePatch and Triangle objects can be traced on the device");
    }

protected:
    AABB box_;
    Vec3 centroid_;
};
