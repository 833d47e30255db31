// Drop-in for the reference's include/ScatObjects/SurfacePatch.hpp
// (SurfacePatch.hpp:52-661): one curved Lagrange patch read from an IFGF-RP
// ".txt" file.  Loading, set-up (centroid, box, coarse grid, cell padding)
// and intersect() go through libbbrt_cuda.so; intersect() runs stage 1 and
// Newton on the GPU.
//
// One difference in kind: the trace constants are `static inline` members
// here (the reference has `static constexpr`), so a program can set the
// coarse-grid size and Newton tolerance before building patches.  Their
// initial values are the reference's.
#pragma once

#include <array>
#include <memory>
#include <optional>
#include <string>
#include <vector>

#include "../ScatObject.hpp"

class SurfacePatch : public ScatObject {
public:
    // SurfacePatch::Data (SurfacePatch.hpp:59-89)
    struct Data {
        int imax = 0, jmax = 0, kmax = 0;
        long long zoneID = 0;
        std::vector<double> uNodes, vNodes, uWeights, vWeights;
        std::vector<double> x, y, z;
        std::vector<int> mask;
        std::vector<double> dxdu, dydu, dzdu, dxdv, dydv, dzdv;
        std::vector<double> dS;
        std::vector<double> nuX, nuY, nuZ;
        std::array<int, 4> edge_flags{ { 0, 0, 0, 0 } };
        long long point_count() const { return static_cast<long long>(imax) * jmax * kmax; }
    };

    // SurfacePatch::CoarseGrid (SurfacePatch.hpp:95-115)
    struct CoarseGrid {
        int n = 0;
        std::vector<double> u, v;
        std::vector<double> x, y, z;
        std::vector<double> cell_sagitta;
        std::vector<Vec3> cell_normal;
        Vec3 point(int i, int j) const { const int k = i * n + j; return { x[k], y[k], z[k] }; }
        int cell_index(int i, int j) const { return i * (n - 1) + j; }
    };

    // SurfacePatch::SampledGrid (SurfacePatch.hpp:167-197)
    struct SampledGrid {
        int n = 0;
        std::vector<double> u, v;
        std::vector<double> x, y, z;
        std::vector<double> nx, ny, nz;
        std::vector<double> dxdu, dydu, dzdu;
        Vec3 point(int i, int j) const { const int k = i * n + j; return { x[k], y[k], z[k] }; }
        Vec3 normal(int i, int j) const { const int k = i * n + j; return { nx[k], ny[k], nz[k] }; }
        Vec3 tangent_u(int i, int j) const { const int k = i * n + j; return { dxdu[k], dydu[k], dzdu[k] }; }
    };

    static inline int kCoarseGridSize = 100;   // SurfacePatch.hpp:117
    static inline int kNewtonMaxIters = 20;    // SurfacePatch.hpp:121
    static inline double kNewtonTol = 1e-3;    // SurfacePatch.hpp:122

    // The constants above as a bbrt_config (what a BVH over patches uses).
    static bbrt_config config() {
        bbrt_config c;
        bbrt_config_init(&c);
        c.coarse_grid_n = kCoarseGridSize;
        c.newton_max_iters = kNewtonMaxIters;
        c.newton_tol = kNewtonTol;
        return c;
    }

    explicit SurfacePatch(const std::string& path) : data_(load(path)) {
        bbrt_patch_desc pd;
        bbrt_object_desc o = device_desc(&pd);
        const bbrt_config cfg = config();
        auto scene = std::make_shared<bbrt_detail::SceneHandle>();
        bbrt_detail::check(bbrt_scene_create(&o, 1, &cfg, &scene->h), "SurfacePatch");
        attach(std::move(scene), 0);
    }

    // A patch that is object `index` of an existing scene built from this
    // same data (what RayTracingDriver does for every file it loads, so the
    // host set-up runs once per patch).
    SurfacePatch(Data data, std::shared_ptr<bbrt_detail::SceneHandle> scene, int index) : data_(std::move(data)) {
        attach(std::move(scene), index);
    }

    // SurfacePatch::load_patch_file (SurfacePatch.hpp:313-371), parsed by the library.
    static Data load(const std::string& path) {
        bbrt_patch_file f;
        bbrt_detail::check(bbrt_patch_file_read(path.c_str(), &f), "SurfacePatch");
        Data d;
        copy_data(f, d);
        bbrt_patch_file_free(&f);
        return d;
    }

    // IFGF-RP naming: files on disk are 1-based (SurfacePatch.hpp:135-139).
    SurfacePatch(const std::string& directory, const std::string& file_prefix, long long index)
        : SurfacePatch(directory + file_prefix + std::to_string(index + 1) + ".txt") {}

    const Data& data() const { return data_; }
    const CoarseGrid& coarse_grid() const { return coarse_; }
    double max_sagitta() const { return max_sagitta_; }
    double self_intersect_padding() const override { return max_sagitta_; }

    SampledGrid sample_grid(int n) const {
        SampledGrid g;
        g.n = n;
        g.u.resize(n);
        g.v.resize(n);
        for (int i = 0; i < n; ++i) {
            const double t = (n == 1) ? 0.0 : -1.0 + 2.0 * static_cast<double>(i) / (n - 1);
            g.u[i] = t;
            g.v[i] = t;
        }
        const size_t nn = static_cast<size_t>(n) * n;
        std::vector<double> xyz(3 * nn), nrm(3 * nn), du(3 * nn);
        const bbrt_patch_desc d = desc();
        bbrt_detail::check(bbrt_patch_sample_grid(&d, n, xyz.data(), nrm.data(), du.data()), "SurfacePatch::sample_grid");
        for (auto* v : { &g.x, &g.y, &g.z, &g.nx, &g.ny, &g.nz, &g.dxdu, &g.dydu, &g.dzdu }) v->resize(nn);
        for (size_t k = 0; k < nn; ++k) {
            g.x[k] = xyz[3 * k]; g.y[k] = xyz[3 * k + 1]; g.z[k] = xyz[3 * k + 2];
            g.nx[k] = nrm[3 * k]; g.ny[k] = nrm[3 * k + 1]; g.nz[k] = nrm[3 * k + 2];
            g.dxdu[k] = du[3 * k]; g.dydu[k] = du[3 * k + 1]; g.dzdu[k] = du[3 * k + 2];
        }
        return g;
    }

    // SurfacePatch::intersect (SurfacePatch.hpp:253-303), on the GPU.
    std::optional<Hit> intersect(const Ray& ray) const override {
        const double o[3] = { ray.origin.x, ray.origin.y, ray.origin.z };
        const double d[3] = { ray.dir.x, ray.dir.y, ray.dir.z };
        bbrt_hit h;
        bbrt_detail::check(bbrt_intersect(scene_->h, o, d, 1, BBRT_QUERY_OBJECT, index_, 0, &h, nullptr),
                           "SurfacePatch::intersect");
        if (h.status) throw std::runtime_error(bbrt_detail::newton_message(h.status, data_.zoneID, h.err_value,
                                                                            kNewtonMaxIters));
        if (h.object < 0) return std::nullopt;
        Hit hit;
        hit.t = h.t;
        hit.point = { h.point[0], h.point[1], h.point[2] };
        hit.normal = { h.normal[0], h.normal[1], h.normal[2] };
        return hit;
    }

    bbrt_patch_desc desc() const {
        bbrt_patch_desc d{};
        d.imax = data_.imax; d.jmax = data_.jmax; d.kmax = data_.kmax; d.zone_id = data_.zoneID;
        d.u_nodes = data_.uNodes.data(); d.v_nodes = data_.vNodes.data();
        d.x = data_.x.data(); d.y = data_.y.data(); d.z = data_.z.data();
        d.dxdu = data_.dxdu.data(); d.dydu = data_.dydu.data(); d.dzdu = data_.dzdu.data();
        d.dxdv = data_.dxdv.data(); d.dydv = data_.dydv.data(); d.dzdv = data_.dzdv.data();
        d.nu_x = data_.nuX.data(); d.nu_y = data_.nuY.data(); d.nu_z = data_.nuZ.data();
        return d;
    }

    bbrt_object_desc device_desc(bbrt_patch_desc* storage) const override {
        *storage = desc();
        bbrt_object_desc o{};
        o.kind = BBRT_OBJ_PATCH;
        o.patch = storage;
        return o;
    }

private:
    Data data_;
    CoarseGrid coarse_;
    double max_sagitta_ = 0.0;
    std::shared_ptr<bbrt_detail::SceneHandle> scene_;
    int index_ = 0;

    static void copy_data(const bbrt_patch_file& f, Data& out) {
        const bbrt_patch_desc& d = f.desc;
        out.imax = d.imax; out.jmax = d.jmax; out.kmax = d.kmax; out.zoneID = d.zone_id;
        const size_t n = static_cast<size_t>(d.imax) * d.jmax * d.kmax;
        out.uNodes.assign(d.u_nodes, d.u_nodes + d.imax);
        out.vNodes.assign(d.v_nodes, d.v_nodes + d.jmax);
        auto cp = [n](std::vector<double>& v, const double* p) { v.assign(p, p + n); };
        cp(out.x, d.x); cp(out.y, d.y); cp(out.z, d.z);
        cp(out.dxdu, d.dxdu); cp(out.dydu, d.dydu); cp(out.dzdu, d.dzdu);
        cp(out.dxdv, d.dxdv); cp(out.dydv, d.dydv); cp(out.dzdv, d.dzdv);
        cp(out.dS, f.dS);
        cp(out.nuX, d.nu_x); cp(out.nuY, d.nu_y); cp(out.nuZ, d.nu_z);
        out.mask.assign(f.mask, f.mask + n);
        for (int k = 0; k < 4; ++k) out.edge_flags[k] = f.edge_flags[k];
        out.uWeights = bary(out.uNodes);   // barycentric_weights, PatchInterpolation.hpp:25-52
        out.vWeights = bary(out.vNodes);
    }

    static std::vector<double> bary(const std::vector<double>& x) {
        std::vector<double> w(x.size());
        for (size_t j = 0; j < x.size(); ++j) {
            double p = 1.0;
            for (size_t i = 0; i < x.size(); ++i)
                if (i != j) p *= (x[j] - x[i]);
            w[j] = 1.0 / p;
        }
        return w;
    }

    // Centroid, box, coarse grid and padding from the library's host set-up
    // of object `index` of `scene`.
    void attach(std::shared_ptr<bbrt_detail::SceneHandle> scene, int index) {
        scene_ = std::move(scene);
        index_ = index;
        bbrt_object_info info;
        bbrt_detail::check(bbrt_object_info_get(scene_->h, index_, &info), "SurfacePatch");
        box_.min = { info.box_min[0], info.box_min[1], info.box_min[2] };
        box_.max = { info.box_max[0], info.box_max[1], info.box_max[2] };
        centroid_ = { info.centroid[0], info.centroid[1], info.centroid[2] };
        max_sagitta_ = info.padding;
        int n = 0;
        bbrt_detail::check(bbrt_patch_coarse_grid(scene_->h, index_, &n, nullptr, nullptr, nullptr, nullptr, nullptr),
                           "SurfacePatch");
        coarse_.n = n;
        coarse_.u.resize(n);
        coarse_.v.resize(n);
        std::vector<double> xyz(3 * static_cast<size_t>(n) * n), nrm(3 * static_cast<size_t>(n - 1) * (n - 1));
        coarse_.cell_sagitta.resize(static_cast<size_t>(n - 1) * (n - 1));
        bbrt_detail::check(bbrt_patch_coarse_grid(scene_->h, index_, &n, coarse_.u.data(), coarse_.v.data(), xyz.data(),
                                                  coarse_.cell_sagitta.data(), nrm.data()),
                           "SurfacePatch");
        const size_t nn = static_cast<size_t>(n) * n;
        coarse_.x.resize(nn); coarse_.y.resize(nn); coarse_.z.resize(nn);
        for (size_t k = 0; k < nn; ++k) { coarse_.x[k] = xyz[3 * k]; coarse_.y[k] = xyz[3 * k + 1]; coarse_.z[k] = xyz[3 * k + 2]; }
        coarse_.cell_normal.resize(coarse_.cell_sagitta.size());
        for (size_t k = 0; k < coarse_.cell_normal.size(); ++k)
            coarse_.cell_normal[k] = { nrm[3 * k], nrm[3 * k + 1], nrm[3 * k + 2] };
    }
};
