// The drivers' exceptions for bad arguments and misuse, one line each:
// "<case>|<exception type>|<what()>", with the patch directory written as
// <dir>.  Uses only the reference's own API, so the same file compiled
// against the reference's headers (tests/golden/make_driver_errors.sh)
// gives the golden output this one is compared with.
//
//   driver_errors <patch_dir/> <sample_prefix>
//
// <patch_dir/><sample_prefix>1.txt must be a patch file.
#include <iostream>
#include <stdexcept>
#include <string>

#include "BounceMapDriver.hpp"
#include "PlaneSourceDriver.hpp"
#include "RayTracingDriver.hpp"

namespace {

std::string dir;

std::string scrub(std::string s) {
    for (size_t at; !dir.empty() && (at = s.find(dir)) != std::string::npos;) s.replace(at, dir.size(), "<dir>");
    return s;
}

template <class Fn>
void report(const char* label, Fn&& fn) {
    try {
        fn();
        std::cout << label << "|none|\n";
    } catch (const std::invalid_argument& e) {
        std::cout << label << "|invalid_argument|" << scrub(e.what()) << '\n';
    } catch (const std::runtime_error& e) {
        std::cout << label << "|runtime_error|" << scrub(e.what()) << '\n';
    }
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 3) {
        std::cerr << "usage: driver_errors <patch_dir/> <sample_prefix>\n";
        return 2;
    }
    dir = argv[1];
    const std::string sample = argv[2];
    RayTracingDriver drv(dir);
    report("set_rays_len", [&] { drv.set_rays({ { 0, 0, 0 } }, {}); });
    report("set_rays_zero", [&] { drv.set_rays({ { 0, 0, 0 }, { 1, 1, 1 } }, { { 1, 0, 0 }, { 0, 0, 0 } }); });
    report("trace_zero", [&] {
        const auto p = drv.trace_ray({ 0, 0, 0 }, { 0, 0, 0 }, 5);
        throw std::runtime_error(std::to_string(static_cast<int>(p.status)) + ":" +
                                 std::to_string(p.points.size()) + ":" + p.error_message);
    });
    report("not_dir", [&] { RayTracingDriver bad(dir + "no_such_dir"); });
    report("range", [&] { RayTracingDriver bad(dir, sample, 3, 2); });
    report("vtk_path", [&] { drv.write_vtk(dir + "no_such_dir/x.vtk"); });
    PlaneSourceDriver ps(dir);
    report("plane_vtk_first", [&] { ps.write_vtk("/dev/null"); });
    report("plane_n", [&] { ps.run({ 0, 0, 0 }, { 0, 1, 1 }, { 1, 0, 0 }, 0, 3); });
    report("plane_dir", [&] { ps.run({ 0, 0, 0 }, { 0, 1, 1 }, { 0, 0, 0 }, 3, 3); });
    report("plane_axis3", [&] { ps.run({ 0, 0, 0 }, { 1, 1, 1 }, { 1, 0, 0 }, 3, 3); });
    report("plane_axis2", [&] { ps.run({ 0, 0, 0 }, { 0, 0, 1 }, { 1, 0, 0 }, 3, 3); });
    BounceMapDriver bm(dir, sample, 1, 1);
    report("bmap_range", [&] { BounceMapDriver bad(dir, sample, 2, 1); });
    report("bmap_vtk_first", [&] { bm.write_vtk("/dev/null"); });
    report("bmap_best_first", [&] { bm.write_best_ray_vtks(dir + "unused_best_rays"); });
    report("bmap_grid", [&] { bm.run(1, 2, 2); });
    report("bmap_dirs", [&] { bm.run(2, 0, 2); });
    report("bmap_cone0", [&] { bm.run(2, 2, 2, 0.0); });
    report("bmap_cone", [&] { bm.run(2, 2, 2, 190.0); });
    return 0;
}
