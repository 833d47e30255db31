// Drop-in for the reference's include/PlaneSourceDriver.hpp
// (PlaneSourceDriver.hpp:64-244): a grid of sources on an axis-aligned
// rectangle, all fired in one direction; per patch, how many recorded
// bounces landed on it.
//
// run() is one bbrt_plane_source call: the source grid, the trace and the
// per-patch counting (device atomics) all happen in the library, so no
// RayPath is built on the host.
#pragma once

#include <fstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "RayTracingDriver.hpp"

class PlaneSourceDriver {
public:
    explicit PlaneSourceDriver(const std::string& patch_directory) : driver_(patch_directory) {}

    // PlaneSourceDriver::run (PlaneSourceDriver.hpp:79-109).  Throws
    // std::invalid_argument for nx or ny < 1, a zero direction, or corners
    // that do not span an axis-aligned rectangle.
    void run(const Vec3& corner0, const Vec3& corner1, const Vec3& direction, int nx, int ny, int max_bounces = 50,
             bool count_direct_hit = false) {
        const double c0[3] = { corner0.x, corner0.y, corner0.z };
        const double c1[3] = { corner1.x, corner1.y, corner1.z };
        const double dir[3] = { direction.x, direction.y, direction.z };
        std::vector<long long> counts(driver_.patches().size(), 0);
        bbrt_detail::check(bbrt_plane_source(driver_.bvh().scene(), c0, c1, dir, nx, ny, max_bounces < 0 ? 0 : max_bounces,
                                             count_direct_hit ? 1 : 0, counts.data(), nullptr, nullptr),
                           "PlaneSourceDriver::run");
        hit_count_ = std::move(counts);
    }

    // Every patch's node grid as triangles with a per-point HitCount
    // (PlaneSourceDriver.hpp:118-181).
    void write_vtk(const std::string& filename) const {
        if (hit_count_.empty()) throw std::runtime_error("PlaneSourceDriver::write_vtk: no data — call run() first");
        const auto& patches = driver_.patches();
        std::ofstream out(filename);
        if (!out.is_open())
            throw std::runtime_error("PlaneSourceDriver::write_vtk: cannot open output file: " + filename);
        size_t n_points = 0, n_tris = 0;
        for (const auto& p : patches) {
            const auto& d = p->data();
            n_points += static_cast<size_t>(d.imax) * d.jmax;
            n_tris += 2 * static_cast<size_t>(d.imax > 0 ? d.imax - 1 : 0) * (d.jmax > 0 ? d.jmax - 1 : 0);
        }
        out << "# vtk DataFile Version 3.0\nPlane-source patch hit counts\nASCII\nDATASET POLYDATA\n";
        out << "POINTS " << n_points << " double\n";
        for (const auto& p : patches) {
            const auto& d = p->data();
            for (int k = 0; k < d.imax * d.jmax; ++k) out << d.x[k] << ' ' << d.y[k] << ' ' << d.z[k] << '\n';
        }
        out << "POLYGONS " << n_tris << ' ' << n_tris * 4 << '\n';
        long long base = 0;
        for (const auto& p : patches) {
            const int I = p->data().imax, J = p->data().jmax;
            for (int i = 0; i + 1 < I; ++i)
                for (int j = 0; j + 1 < J; ++j) {
                    const long long a = base + i * J + j, b = base + (i + 1) * J + j;
                    out << "3 " << a << ' ' << b << ' ' << b + 1 << '\n';
                    out << "3 " << a << ' ' << b + 1 << ' ' << a + 1 << '\n';
                }
            base += static_cast<long long>(I) * J;
        }
        out << "POINT_DATA " << n_points << '\n';
        out << "SCALARS HitCount long 1\nLOOKUP_TABLE default\n";
        for (size_t p = 0; p < patches.size(); ++p) {
            const auto& d = patches[p]->data();
            for (int k = 0; k < d.imax * d.jmax; ++k) out << hit_count_[p] << '\n';
        }
    }

    const RayTracingDriver& driver() const { return driver_; }

    // Per patch (patches() order), the counts of the last run().
    const std::vector<long long>& hit_counts() const { return hit_count_; }

private:
    RayTracingDriver driver_;
    std::vector<long long> hit_count_;
};
