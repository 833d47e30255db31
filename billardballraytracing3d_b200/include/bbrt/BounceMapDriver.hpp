// Drop-in for the reference's include/BounceMapDriver.hpp
// (BounceMapDriver.hpp:71-520): from an n x n grid of points on each sampled
// patch, sweep a cone of directions about the surface normal, trace them
// through the whole scene and keep, per point, the largest bounce count and
// the number of failed directions.
//
// run() is one bbrt_bounce_map call (every ray of every point in one GPU
// trace).  With capture_best_rays the library reports, per point, which
// direction first reached the maximum; those rays are regenerated
// (bbrt_bounce_map_rays) and traced once more with their paths recorded,
// which gives the same RayPath the reference keeps.  The progress bar is
// printed once, complete, when the trace returns.
#pragma once

#include <algorithm>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "RayTracingDriver.hpp"
#include "ScatObjects/SurfacePatch.hpp"

class BounceMapDriver {
public:
    BounceMapDriver(const std::string& patch_directory, const std::string& file_prefix, int first_index_1based,
                    int last_index_1based)
        : driver_(patch_directory), first_index_1based_(first_index_1based) {
        if (last_index_1based < first_index_1based)
            throw std::invalid_argument("BounceMapDriver: empty patch index range [" +
                                        std::to_string(first_index_1based) + ", " +
                                        std::to_string(last_index_1based) + "]");
        for (int i = first_index_1based; i <= last_index_1based; ++i)
            sample_patches_.push_back(
                std::make_unique<SurfacePatch>(patch_directory + file_prefix + std::to_string(i) + ".txt"));
    }

    // BounceMapDriver::run (BounceMapDriver.hpp:103-259).
    void run(int position_grid_n, int theta_n, int phi_n, double cone_angle_deg = 180.0, int max_bounces = 50,
             bool capture_best_rays = false) {
        const int P = static_cast<int>(sample_patches_.size());
        std::vector<bbrt_patch_desc> descs(P);
        for (int p = 0; p < P; ++p) descs[p] = sample_patches_[p]->desc();
        const long long per = static_cast<long long>(position_grid_n) * position_grid_n;
        const long long points = per * P;
        std::vector<int> mb(static_cast<size_t>(std::max<long long>(points, 1))), er(mb.size()), best(mb.size());
        bbrt_detail::check(bbrt_bounce_map(driver_.bvh().scene(), descs.data(), P, position_grid_n, theta_n, phi_n,
                                           cone_angle_deg, max_bounces < 0 ? 0 : max_bounces, mb.data(), er.data(),
                                           best.data(), nullptr, nullptr),
                           "BounceMapDriver::run");
        capture_best_rays_ = capture_best_rays;
        patch_grids_.assign(P, SurfacePatch::SampledGrid{});
        patch_max_bounces_.assign(P, {});
        patch_error_counts_.assign(P, {});
        patch_best_paths_.clear();
        for (int p = 0; p < P; ++p) {
            patch_grids_[p] = sample_patches_[p]->sample_grid(position_grid_n);
            patch_max_bounces_[p].assign(mb.begin() + p * per, mb.begin() + (p + 1) * per);
            patch_error_counts_[p].assign(er.begin() + p * per, er.begin() + (p + 1) * per);
        }
        if (capture_best_rays_) {
            patch_best_paths_.assign(P, std::vector<RayTracingDriver::RayPath>(static_cast<size_t>(per)));
            std::vector<long long> idx, slot;
            const long long dirs = static_cast<long long>(theta_n) * phi_n;
            for (long long q = 0; q < points; ++q)
                if (best[q] >= 0) {
                    idx.push_back(q * dirs + best[q]);
                    slot.push_back(q);
                }
            if (!idx.empty()) {
                const long long n = static_cast<long long>(idx.size());
                std::vector<double> o(3 * n), d(3 * n);
                bbrt_detail::check(bbrt_bounce_map_rays(driver_.bvh().scene(), descs.data(), P, position_grid_n, theta_n,
                                                        phi_n, cone_angle_deg, idx.data(), n, o.data(), d.data()),
                                   "BounceMapDriver::run");
                std::vector<Vec3> org(n), dir(n);
                for (long long i = 0; i < n; ++i) {
                    org[i] = { o[3 * i], o[3 * i + 1], o[3 * i + 2] };
                    dir[i] = { d[3 * i], d[3 * i + 1], d[3 * i + 2] };
                }
                std::vector<RayTracingDriver::RayPath> paths = driver_.trace_rays(org, dir, max_bounces);
                for (long long i = 0; i < n; ++i)
                    patch_best_paths_[slot[i] / per][slot[i] % per] = std::move(paths[i]);
            }
        }
        print_progress(points, points);
        std::cout << '\n';
    }

    // Every sampled grid as triangles with MaxBounces / ErrorCount point
    // scalars (BounceMapDriver.hpp:272-337).
    void write_vtk(const std::string& filename) const {
        if (patch_grids_.empty()) throw std::runtime_error("BounceMapDriver::write_vtk: no data — call run() first");
        std::ofstream out(filename);
        if (!out.is_open())
            throw std::runtime_error("BounceMapDriver::write_vtk: cannot open output file: " + filename);
        size_t n_points = 0, n_tris = 0;
        for (const auto& g : patch_grids_) {
            n_points += static_cast<size_t>(g.n) * g.n;
            n_tris += 2 * static_cast<size_t>(g.n - 1) * (g.n - 1);
        }
        out << "# vtk DataFile Version 3.0\nBilliard-ball bounce map\nASCII\nDATASET POLYDATA\n";
        out << "POINTS " << n_points << " double\n";
        for (const auto& g : patch_grids_)
            for (int k = 0; k < g.n * g.n; ++k) out << g.x[k] << ' ' << g.y[k] << ' ' << g.z[k] << '\n';
        out << "POLYGONS " << n_tris << ' ' << n_tris * 4 << '\n';
        long long base = 0;
        for (const auto& g : patch_grids_) {
            for (int i = 0; i + 1 < g.n; ++i)
                for (int j = 0; j + 1 < g.n; ++j) {
                    const long long a = base + i * g.n + j, b = base + (i + 1) * g.n + j;
                    out << "3 " << a << ' ' << b << ' ' << b + 1 << '\n';
                    out << "3 " << a << ' ' << b + 1 << ' ' << a + 1 << '\n';
                }
            base += static_cast<long long>(g.n) * g.n;
        }
        out << "POINT_DATA " << n_points << '\n';
        out << "SCALARS MaxBounces int 1\nLOOKUP_TABLE default\n";
        for (const auto& v : patch_max_bounces_)
            for (int b : v) out << b << '\n';
        out << "SCALARS ErrorCount int 1\nLOOKUP_TABLE default\n";
        for (const auto& v : patch_error_counts_)
            for (int e : v) out << e << '\n';
    }

    // One file per sampled patch: the best ray of every grid point as line
    // legs with PointID / BounceIndex cell scalars (BounceMapDriver.hpp:350-430).
    void write_best_ray_vtks(const std::string& output_directory,
                             const std::string& file_prefix = "best_rays_patch_") const {
        if (!capture_best_rays_)
            throw std::runtime_error(
                "BounceMapDriver::write_best_ray_vtks: best rays weren't captured — call run(..., "
                "/*capture_best_rays=*/true) first");
        if (patch_best_paths_.empty())
            throw std::runtime_error("BounceMapDriver::write_best_ray_vtks: no data — call run() first");
        std::filesystem::create_directories(output_directory);
        for (size_t p = 0; p < patch_best_paths_.size(); ++p) {
            const auto& paths = patch_best_paths_[p];
            const std::string filename = output_directory + "/" + file_prefix +
                                         std::to_string(first_index_1based_ + static_cast<int>(p)) + ".vtk";
            std::ofstream out(filename);
            if (!out.is_open())
                throw std::runtime_error("BounceMapDriver::write_best_ray_vtks: cannot open output file: " + filename);
            size_t n_points = 0, n_legs = 0;
            for (const auto& r : paths) {
                n_points += r.points.size();
                n_legs += r.points.empty() ? 0 : r.points.size() - 1;
            }
            out << "# vtk DataFile Version 3.0\nBest bounce ray per grid point\nASCII\nDATASET POLYDATA\n";
            out << "POINTS " << n_points << " double\n";
            for (const auto& r : paths)
                for (const Vec3& v : r.points) out << v.x << ' ' << v.y << ' ' << v.z << '\n';
            out << "LINES " << n_legs << ' ' << n_legs * 3 << '\n';
            size_t base = 0;
            for (const auto& r : paths) {
                for (size_t k = 0; k + 1 < r.points.size(); ++k) out << "2 " << base + k << ' ' << base + k + 1 << '\n';
                base += r.points.size();
            }
            out << "CELL_DATA " << n_legs << '\n';
            out << "SCALARS PointID int 1\nLOOKUP_TABLE default\n";
            for (size_t q = 0; q < paths.size(); ++q)
                for (size_t k = 0; k + 1 < paths[q].points.size(); ++k) out << q << '\n';
            out << "SCALARS BounceIndex int 1\nLOOKUP_TABLE default\n";
            for (const auto& r : paths)
                for (size_t k = 0; k + 1 < r.points.size(); ++k) out << k << '\n';
        }
    }

    const RayTracingDriver& driver() const { return driver_; }

    // Per sampled patch: the grid, and per grid point the max bounce count
    // and error count of the last run().
    const std::vector<SurfacePatch::SampledGrid>& grids() const { return patch_grids_; }
    const std::vector<std::vector<int>>& max_bounces() const { return patch_max_bounces_; }
    const std::vector<std::vector<int>>& error_counts() const { return patch_error_counts_; }
    const std::vector<std::vector<RayTracingDriver::RayPath>>& best_paths() const { return patch_best_paths_; }

private:
    RayTracingDriver driver_;
    std::vector<std::unique_ptr<SurfacePatch>> sample_patches_;
    int first_index_1based_ = 1;
    std::vector<SurfacePatch::SampledGrid> patch_grids_;
    std::vector<std::vector<int>> patch_max_bounces_;
    std::vector<std::vector<int>> patch_error_counts_;
    bool capture_best_rays_ = false;
    std::vector<std::vector<RayTracingDriver::RayPath>> patch_best_paths_;

    static void print_progress(long long done, long long total) {
        const int width = 30;
        const double frac = total > 0 ? static_cast<double>(done) / static_cast<double>(total) : 1.0;
        const int filled = static_cast<int>(frac * width);
        std::cout << "\rBounce map [" << std::string(filled, '#') << std::string(width - filled, '-') << "] "
                  << static_cast<int>(frac * 100.0) << "% (" << done << '/' << total << " points)" << std::flush;
    }
};
