// Runs the three drivers of the C++ mirror headers the way the reference's
// example programs do (src/main.cpp, tests/PlaneSource_Example.cpp,
// tests/BounceMap_Example.cpp) and writes what they produced as text, for
// the Python tests to compare with the oracle.
//
//   drivers trace <patch_dir> <rays.bin> <max_bounces> <out_prefix>
//   drivers plane <patch_dir> c0x c0y c0z c1x c1y c1z dx dy dz nx ny max_bounces count_direct <out_prefix>
//   drivers bmap  <patch_dir> <file_prefix> <first> <last> grid theta phi cone max_bounces <out_prefix>
//
// rays.bin: int64 n, then n origins (3 doubles each), then n directions.
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <string>
#include <thread>
#include <vector>

#include "BounceMapDriver.hpp"
#include "PlaneSourceDriver.hpp"
#include "RayTracingDriver.hpp"

namespace {

void dump_paths(const RayTracingDriver& drv, const std::vector<RayTracingDriver::RayPath>& paths,
                const std::string& file) {
    std::ofstream out(file);
    out << std::setprecision(17);
    for (const auto& p : paths) {
        out << "R " << static_cast<int>(p.status) << ' ' << p.bounce_count << ' ' << p.points.size() << '\n';
        for (const Vec3& v : p.points) out << "P " << v.x << ' ' << v.y << ' ' << v.z << '\n';
        out << "H";
        for (const ScatObject* o : p.hit_objects) out << ' ' << drv.patch_index_of(o);
        out << "\nE " << p.error_message << '\n';
    }
}

int run_trace(char** a) {
    std::ifstream in(a[1], std::ios::binary);
    long long n = 0;
    in.read(reinterpret_cast<char*>(&n), sizeof n);
    std::vector<double> o(3 * n), d(3 * n);
    in.read(reinterpret_cast<char*>(o.data()), sizeof(double) * 3 * n);
    in.read(reinterpret_cast<char*>(d.data()), sizeof(double) * 3 * n);
    if (!in) throw std::runtime_error("drivers: short rays file");
    std::vector<Vec3> src(n), dir(n);
    for (long long i = 0; i < n; ++i) {
        src[i] = { o[3 * i], o[3 * i + 1], o[3 * i + 2] };
        dir[i] = { d[3 * i], d[3 * i + 1], d[3 * i + 2] };
    }
    RayTracingDriver drv(a[0]);
    drv.set_rays(src, dir);
    drv.run(std::atoi(a[2]));
    const std::string prefix = a[3];
    dump_paths(drv, drv.paths(), prefix + "paths.txt");
    drv.write_vtk(prefix + "traces.vtk");
    // The one-ray form gives the same path as the batch.
    const long long m = std::min<long long>(n, 8);
    std::vector<RayTracingDriver::RayPath> one;
    for (long long i = 0; i < m; ++i) one.push_back(drv.trace_ray(src[i], dir[i], std::atoi(a[2])));
    dump_paths(drv, one, prefix + "paths_one.txt");
    // Many threads calling trace_ray at once (the reference's OpenMP loop,
    // PlaneSourceDriver.hpp:96-99): their rays are combined into batches,
    // and every ray still gets its own path.
    {
        std::vector<RayTracingDriver::RayPath> par(static_cast<size_t>(n));
        const int maxb = std::atoi(a[2]);
        std::vector<std::thread> pool;
        std::atomic<long long> next{ 0 };
        for (int t = 0; t < 8; ++t)
            pool.emplace_back([&] {
                for (long long i = next++; i < n; i = next++) par[static_cast<size_t>(i)] = drv.trace_ray(src[i], dir[i], maxb);
            });
        for (auto& th : pool) th.join();
        dump_paths(drv, par, prefix + "paths_threads.txt");
    }
    std::ofstream info(prefix + "info.txt");
    info << std::setprecision(17) << drv.patches().size() << ' ' << drv.self_intersect_epsilon() << ' '
         << drv.self_intersect_epsilon(drv.patches().front().get()) << '\n';
    return 0;
}

int run_plane(char** a) {
    const Vec3 c0{ std::atof(a[1]), std::atof(a[2]), std::atof(a[3]) };
    const Vec3 c1{ std::atof(a[4]), std::atof(a[5]), std::atof(a[6]) };
    const Vec3 dir{ std::atof(a[7]), std::atof(a[8]), std::atof(a[9]) };
    PlaneSourceDriver drv(a[0]);
    drv.run(c0, c1, dir, std::atoi(a[10]), std::atoi(a[11]), std::atoi(a[12]), std::atoi(a[13]) != 0);
    const std::string prefix = a[14];
    std::ofstream out(prefix + "plane_counts.txt");
    for (long long c : drv.hit_counts()) out << c << '\n';
    drv.write_vtk(prefix + "plane.vtk");
    return 0;
}

int run_bmap(char** a) {
    BounceMapDriver drv(a[0], a[1], std::atoi(a[2]), std::atoi(a[3]));
    drv.run(std::atoi(a[4]), std::atoi(a[5]), std::atoi(a[6]), std::atof(a[7]), std::atoi(a[8]), true);
    const std::string prefix = a[9];
    std::ofstream out(prefix + "bmap.txt");
    for (size_t p = 0; p < drv.max_bounces().size(); ++p)
        for (size_t k = 0; k < drv.max_bounces()[p].size(); ++k)
            out << drv.max_bounces()[p][k] << ' ' << drv.error_counts()[p][k] << '\n';
    std::vector<RayTracingDriver::RayPath> best;
    for (const auto& v : drv.best_paths()) best.insert(best.end(), v.begin(), v.end());
    dump_paths(drv.driver(), best, prefix + "bmap_best.txt");
    drv.write_vtk(prefix + "bmap.vtk");
    drv.write_best_ray_vtks(prefix + "best_rays");
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    try {
        const std::string cmd = argc > 1 ? argv[1] : "";
        if (cmd == "trace" && argc == 6) return run_trace(argv + 2);
        if (cmd == "plane" && argc == 17) return run_plane(argv + 2);
        if (cmd == "bmap" && argc == 12) return run_bmap(argv + 2);
        std::cerr << "usage: drivers trace|plane|bmap ...\n";
        return 2;
    } catch (const std::exception& e) {
        std::cerr << "Fatal error: " << e.what() << "\n";
        return 1;
    }
}
