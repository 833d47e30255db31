// The reference's BVH-vs-brute-force check on four triangles
// (tests/Triangle_Intersect.cpp), against the C++ mirror headers: the same
// scene and rays, both answers from the GPU, compared with each other and
// with the known t of each ray.  Exit status = number of failures.
#include <cmath>
#include <iostream>
#include <vector>

#include "BVH.hpp"
#include "BruteForce.hpp"
#include "ScatObjects/Triangle.hpp"

namespace {

struct Case {
    Ray ray;
    const char* what;
    double t;   // expected t, or < 0 for a miss
};

bool same_t(double a, double b) { return std::fabs(a - b) < 1e-9; }

}  // namespace

int main() {
    std::vector<Triangle> tris;
    tris.emplace_back(Vec3{ 0, 0, 0 }, Vec3{ 1, 0, 0 }, Vec3{ 0, 1, 0 });
    tris.emplace_back(Vec3{ 10, 0, 0 }, Vec3{ 11, 0, 0 }, Vec3{ 10, 1, 0 });
    tris.emplace_back(Vec3{ 0, 0, 5 }, Vec3{ 1, 0, 5 }, Vec3{ 0, 1, 5 });
    tris.emplace_back(Vec3{ -5, 0, 0 }, Vec3{ -4, 0, 0 }, Vec3{ -5, 1, 0 });
    std::vector<const ScatObject*> objects;
    for (const Triangle& t : tris) objects.push_back(&t);

    BVH bvh(objects, /*leaf_threshold=*/1);
    const std::vector<Case> cases = {
        { { { 0.2, 0.2, -1 }, { 0, 0, 1 } }, "near triangle, t=1", 1.0 },
        { { { 10.2, 0.2, -1 }, { 0, 0, 1 } }, "far triangle, t=1", 1.0 },
        { { { 100, 100, -1 }, { 0, 0, 1 } }, "miss", -1.0 },
        { { { 0.2, 0.2, 10 }, { 0, 0, -1 } }, "z=5 triangle before z=0, t=5", 5.0 },
    };

    int failures = 0;
    std::vector<Ray> batch;
    for (const Case& c : cases) {
        const auto a = bvh.intersect(c.ray);
        const auto b = brute_force_intersect(c.ray, objects);
        bool ok = a.has_value() == b.has_value() && a.has_value() == (c.t >= 0.0);
        if (ok && a) ok = same_t(a->t, b->t) && same_t(a->t, c.t) && a->object != nullptr;
        std::cout << c.what << ": " << (ok ? "PASS" : "FAIL") << " (bvh t=" << (a ? a->t : -1)
                  << ", brute t=" << (b ? b->t : -1) << ")\n";
        failures += ok ? 0 : 1;
        batch.push_back(c.ray);
    }

    // The batch forms agree with the one-ray form.
    const auto many = bvh.intersect(batch);
    BruteForce brute(objects);
    const auto many_brute = brute.intersect(batch);
    for (size_t i = 0; i < cases.size(); ++i) {
        const bool hit = cases[i].t >= 0.0;
        bool ok = many[i].error.empty() && many_brute[i].error.empty() && many[i].hit.has_value() == hit &&
                  many_brute[i].hit.has_value() == hit;
        if (ok && hit)
            ok = same_t(many[i].hit->t, cases[i].t) && same_t(many_brute[i].hit->t, cases[i].t) &&
                 many[i].hit->object == many_brute[i].hit->object;
        if (!ok) {
            std::cout << "batch ray " << i << ": FAIL\n";
            ++failures;
        }
    }

    // Box and centroid of a triangle, as Triangle.hpp:11-24 defines them.
    const Triangle& t0 = tris[0];
    if (!(t0.bounding_box().min.x == 0 && t0.bounding_box().max.x == 1 && t0.bounding_box().max.z == 0 &&
          same_t(t0.centroid().x, 1.0 / 3.0))) {
        std::cout << "triangle box/centroid: FAIL\n";
        ++failures;
    }

    std::cout << (failures == 0 ? "\nAll tests passed.\n" : "\nSome tests FAILED.\n");
    return failures;
}
