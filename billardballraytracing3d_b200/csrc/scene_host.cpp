// Host scene compiler: object set-up, BVH build, flattening.
//
// Reference counterparts (manuelarturosantana/BillardBallRayTracing3D):
//   SurfacePatch constructor          include/ScatObjects/SurfacePatch.hpp:125-131
//     compute_centroid_and_box        :380-407
//     compute_coarse_grid             :416-436  (lagrange_interpolation_2D,
//                                                Utils/PatchInterpolation.hpp:54-159)
//     compute_cell_padding            :446-492  (lagrange_basis_1d :518-538,
//                                                eval_scalar_field :542-555)
//   Triangle constructor              include/ScatObjects/Triangle.hpp:11-24
//   BVH::build                        include/BVH.hpp:136-189
//   RayTracingDriver::compute_scene_scale   include/RayTracingDriver.hpp:386-396
//
// Every value the GPU reads in a decision (coarse vertices, cell normals and
// sagittas, boxes) must equal the reference's to the last bit, so each
// formula keeps the reference's operand order; this file must be compiled
// without floating-point contraction (-ffp-contract=off).  The two matrix
// products of the coarse-grid interpolation use MKL's cblas_dgemm in the
// reference; here they are plain loops summing over k left to right, the
// order of the oracle's dgemm stand-in (oracle/shim/mkl.h).
#include "scene_host.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>
#include <limits>
#include <stdexcept>

namespace bbrt {
namespace {

constexpr double kEqualTol = 1.0e-12;   // EQUAL_TOL, Utils/PatchInterpolation.hpp:21

// Barycentric weights 1 / prod_{i != j} (x_j - x_i), product taken over i ascending.
std::vector<double> bary_weights(const double* x, int n) {
    std::vector<double> w(n);
    for (int j = 0; j < n; ++j) {
        double p = 1.0;
        for (int i = 0; i < n; ++i)
            if (i != j) p *= (x[j] - x[i]);
        w[j] = 1.0 / p;
    }
    return w;
}

// First-form Lagrange row for evaluation point t: w_j / (t - x_j) and the
// scale prod_j (t - x_j); a node within kEqualTol gives a one-hot row and
// scale 1.  (Both axes of lagrange_interpolation_2D use this.)
void first_form_row(const double* x, const double* w, int n, double t, double* row, double& scale) {
    double prod = 1.0;
    int hit = -1;
    for (int j = 0; j < n; ++j) {
        const double diff = t - x[j];
        if (std::abs(diff) < kEqualTol) { hit = j; break; }
        row[j] = w[j] / diff;
        prod *= diff;
    }
    if (hit >= 0) {
        for (int j = 0; j < n; ++j) row[j] = 0.0;
        row[hit] = 1.0;
        scale = 1.0;
    } else {
        scale = prod;
    }
}

// Second-form basis at t (normalised by the sum of the w_j / (t - x_j)).
void second_form_basis(const double* x, const double* w, int n, double t, double* b) {
    for (int i = 0; i < n; ++i) b[i] = 0.0;
    for (int i = 0; i < n; ++i)
        if (std::fabs(t - x[i]) < kEqualTol) { b[i] = 1.0; return; }
    double denom = 0.0;
    for (int i = 0; i < n; ++i) {
        const double li = w[i] / (t - x[i]);
        b[i] = li;
        denom += li;
    }
    for (int i = 0; i < n; ++i) b[i] /= denom;
}

// sum_i bu_i * (sum_j bv_j f_ij), rows with bu_i == 0 skipped.
double tensor_eval(const double* f, int imax, int jmax, const double* bu, const double* bv) {
    double sum = 0.0;
    for (int i = 0; i < imax; ++i) {
        const double li = bu[i];
        if (li == 0.0) continue;
        const double* r = f + static_cast<size_t>(i) * jmax;
        double rs = 0.0;
        for (int j = 0; j < jmax; ++j) rs += bv[j] * r[j];
        sum += li * rs;
    }
    return sum;
}

// Tensor-product interpolation of f (imax x jmax) at the grid tu[P] x tv[Q].
void interp_grid(const double* un, const double* uw, int imax, const double* vn, const double* vw, int jmax,
                 const double* f, const std::vector<double>& tu, const std::vector<double>& tv, double* out) {
    const int P = static_cast<int>(tu.size()), Q = static_cast<int>(tv.size());
    std::vector<double> ru(static_cast<size_t>(P) * imax, 0.0), rv(static_cast<size_t>(Q) * jmax, 0.0);
    std::vector<double> su(P), sv(Q);
    for (int i = 0; i < P; ++i) first_form_row(un, uw, imax, tu[i], &ru[static_cast<size_t>(i) * imax], su[i]);
    for (int i = 0; i < Q; ++i) first_form_row(vn, vw, jmax, tv[i], &rv[static_cast<size_t>(i) * jmax], sv[i]);
    // partial[i][m] = sum_k ru[i][k] f[k][m];  out[i][q] = sum_m partial[i][m] rv[q][m]
    std::vector<double> partial(static_cast<size_t>(P) * jmax);
    for (int i = 0; i < P; ++i)
        for (int m = 0; m < jmax; ++m) {
            double s = 0.0;
            for (int k = 0; k < imax; ++k) s += ru[static_cast<size_t>(i) * imax + k] * f[static_cast<size_t>(k) * jmax + m];
            partial[static_cast<size_t>(i) * jmax + m] = 1.0 * s;
        }
    for (int i = 0; i < P; ++i)
        for (int q = 0; q < Q; ++q) {
            double s = 0.0;
            for (int m = 0; m < jmax; ++m)
                s += partial[static_cast<size_t>(i) * jmax + m] * rv[static_cast<size_t>(q) * jmax + m];
            out[static_cast<size_t>(i) * Q + q] = (1.0 * s) * (su[i] * sv[q]);
        }
}

inline double dmin(double a, double b) { return (b < a) ? b : a; }   // std::min(a, b)
inline double dmax(double a, double b) { return (a < b) ? b : a; }   // std::max(a, b)

struct PatchSetup {
    double box[6];
    double centroid[3];
    double max_sag;
};

// One patch's flat tables: nodes un[I] vn[J] and their barycentric weights
// uw[I] vw[J]; the kFields values of every node (i, j), node-major.
void copy_patch_tables(const bbrt_patch_desc& d, double* nodes, double* fields) {
    const int I = d.imax, J = d.jmax;
    const size_t nn = static_cast<size_t>(I) * J;
    std::memcpy(nodes, d.u_nodes, sizeof(double) * I);
    std::memcpy(nodes + I, d.v_nodes, sizeof(double) * J);
    const std::vector<double> uw = bary_weights(d.u_nodes, I), vw = bary_weights(d.v_nodes, J);
    std::memcpy(nodes + I + J, uw.data(), sizeof(double) * I);
    std::memcpy(nodes + 2 * I + J, vw.data(), sizeof(double) * J);
    const double* src[kFields] = { d.x, d.y, d.z, d.dxdu, d.dydu, d.dzdu, d.dxdv, d.dydv, d.dzdv,
                                   d.nu_x, d.nu_y, d.nu_z };
    for (size_t q = 0; q < nn; ++q)
        for (int k = 0; k < kFields; ++k) fields[q * kFields + k] = src[k][q];
}

// One patch: the centroid/box, the coarse grid and the per-cell padding.
PatchSetup setup_patch(const bbrt_patch_desc& d, int cn, const std::vector<double>& cuv, double* cxyz, double* ccell) {
    const int I = d.imax, J = d.jmax;
    const size_t nn = static_cast<size_t>(I) * J;
    const std::vector<double> uw = bary_weights(d.u_nodes, I), vw = bary_weights(d.v_nodes, J);
    const double* src[kFields] = { d.x, d.y, d.z, d.dxdu, d.dydu, d.dzdu, d.dxdv, d.dydv, d.dzdv,
                                   d.nu_x, d.nu_y, d.nu_z };

    PatchSetup s;
    // centroid = mean of the nodes; box = node AABB (later inflated)
    double sx = 0.0, sy = 0.0, sz = 0.0;
    double lo[3] = { std::numeric_limits<double>::infinity(), std::numeric_limits<double>::infinity(),
                     std::numeric_limits<double>::infinity() };
    double hi[3] = { -lo[0], -lo[1], -lo[2] };
    for (size_t i = 0; i < nn; ++i) {
        const double p[3] = { d.x[i], d.y[i], d.z[i] };
        sx += p[0]; sy += p[1]; sz += p[2];
        for (int a = 0; a < 3; ++a) { lo[a] = dmin(lo[a], p[a]); hi[a] = dmax(hi[a], p[a]); }
    }
    const double inv_n = 1.0 / static_cast<double>(nn);
    s.centroid[0] = sx * inv_n; s.centroid[1] = sy * inv_n; s.centroid[2] = sz * inv_n;

    // coarse grid vertices, stored xyz-interleaved
    const size_t cnn = static_cast<size_t>(cn) * cn;
    std::vector<double> g(3 * cnn);
    for (int c = 0; c < 3; ++c)
        interp_grid(d.u_nodes, uw.data(), I, d.v_nodes, vw.data(), J, src[c], cuv, cuv, &g[c * cnn]);
    for (size_t k = 0; k < cnn; ++k)
        for (int c = 0; c < 3; ++c) cxyz[3 * k + c] = g[c * cnn + k];

    // per-cell sagitta at the parameter midpoint and the unit normal there
    double bu[kMaxNodes], bv[kMaxNodes];
    double ms = 0.0;
    for (int i = 0; i + 1 < cn; ++i) {
        for (int j = 0; j + 1 < cn; ++j) {
            const double um = 0.5 * (cuv[i] + cuv[i + 1]);
            const double vm = 0.5 * (cuv[j] + cuv[j + 1]);
            second_form_basis(d.u_nodes, uw.data(), I, um, bu);
            second_form_basis(d.v_nodes, vw.data(), J, vm, bv);
            double mid[3], nrm[3];
            for (int c = 0; c < 3; ++c) mid[c] = tensor_eval(src[c], I, J, bu, bv);
            for (int c = 0; c < 3; ++c) nrm[c] = tensor_eval(src[9 + c], I, J, bu, bv);
            const double nl = std::sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
            const size_t k00 = static_cast<size_t>(i) * cn + j, k10 = k00 + cn, k01 = k00 + 1, k11 = k00 + cn + 1;
            double df[3];
            for (int c = 0; c < 3; ++c) {
                const double bil = 0.25 * (g[c * cnn + k00] + g[c * cnn + k10] + g[c * cnn + k01] + g[c * cnn + k11]);
                df[c] = mid[c] - bil;
            }
            const double sag = std::sqrt(df[0] * df[0] + df[1] * df[1] + df[2] * df[2]);
            double* cell = ccell + 4 * (static_cast<size_t>(i) * (cn - 1) + j);
            cell[0] = nrm[0] / nl; cell[1] = nrm[1] / nl; cell[2] = nrm[2] / nl;
            cell[3] = sag;
            ms = dmax(ms, sag);
        }
    }
    for (int a = 0; a < 3; ++a) { s.box[a] = lo[a] - ms; s.box[3 + a] = hi[a] + ms; }
    s.max_sag = ms;
    return s;
}

// Median-split BVH over object indices (BVH.hpp:136-189): node box = union of
// the object boxes; a range of at most leaf_threshold objects is a leaf;
// otherwise split at size/2 with std::nth_element on the centroid coordinate
// of the widest centroid spread (first widest axis wins), left child stored
// right after its parent.
class BvhBuilder {
public:
    BvhBuilder(const HostScene& s, std::vector<BvhNode>& nodes, std::vector<int>& leaves, int leaf_threshold)
        : s_(s), nodes_(nodes), leaves_(leaves), leaf_threshold_(leaf_threshold) {}

    int build(std::vector<int> ids, int depth) {
        max_depth = std::max(max_depth, depth);
        const int me = static_cast<int>(nodes_.size());
        nodes_.emplace_back();
        double b[6];
        std::memcpy(b, &s_.box[6 * ids.front()], sizeof b);
        for (size_t k = 1; k < ids.size(); ++k) {
            const double* o = &s_.box[6 * ids[k]];
            for (int a = 0; a < 3; ++a) { b[a] = dmin(b[a], o[a]); b[3 + a] = dmax(b[3 + a], o[3 + a]); }
        }
        if (static_cast<int>(ids.size()) <= leaf_threshold_) {
            BvhNode& nd = nodes_[me];
            std::memcpy(nd.box, b, sizeof b);
            nd.right = -1;
            nd.start = static_cast<int>(leaves_.size());
            nd.count = static_cast<int>(ids.size());
            nd.axis = 0;
            leaves_.insert(leaves_.end(), ids.begin(), ids.end());
            return me;
        }
        double clo[3], chi[3];
        for (int a = 0; a < 3; ++a) clo[a] = chi[a] = s_.centroid[3 * ids.front() + a];
        for (int id : ids)
            for (int a = 0; a < 3; ++a) {
                const double c = s_.centroid[3 * id + a];
                clo[a] = dmin(clo[a], c);
                chi[a] = dmax(chi[a], c);
            }
        const double spread[3] = { chi[0] - clo[0], chi[1] - clo[1], chi[2] - clo[2] };
        const int axis = static_cast<int>(std::max_element(spread, spread + 3) - spread);
        const auto mid = ids.begin() + ids.size() / 2;
        const double* cen = s_.centroid.data();
        std::nth_element(ids.begin(), mid, ids.end(),
                         [cen, axis](int a, int c) { return cen[3 * a + axis] < cen[3 * c + axis]; });
        std::vector<int> left(ids.begin(), mid), right(mid, ids.end());
        ids.clear();
        ids.shrink_to_fit();
        build(std::move(left), depth + 1);
        const int r = build(std::move(right), depth + 1);
        BvhNode& nd = nodes_[me];
        std::memcpy(nd.box, b, sizeof b);
        nd.right = r;
        nd.start = 0;
        nd.count = 0;
        nd.axis = axis;
        return me;
    }

    int max_depth = 0;

private:
    const HostScene& s_;
    std::vector<BvhNode>& nodes_;
    std::vector<int>& leaves_;
    int leaf_threshold_;
};

}  // namespace

void build_host_tables(const bbrt_object_desc* objects, int n_objects, const bbrt_config& cfg, HostScene& S) {
    if (n_objects <= 0 || objects == nullptr) throw std::invalid_argument("bbrt: a scene needs at least one object");
    if (cfg.coarse_grid_n < 2) throw std::invalid_argument("bbrt: coarse_grid_n must be >= 2");
    if (cfg.leaf_threshold < 1) throw std::invalid_argument("bbrt: leaf_threshold must be >= 1");
    if (cfg.newton_max_iters < 1) throw std::invalid_argument("bbrt: newton_max_iters must be >= 1");
    S = HostScene();
    S.cfg = cfg;
    S.n_objects = n_objects;
    S.kind.resize(n_objects);
    S.sub.resize(n_objects);
    S.zone.resize(n_objects);
    S.box.resize(6 * static_cast<size_t>(n_objects));
    S.centroid.resize(3 * static_cast<size_t>(n_objects));
    S.padding.resize(n_objects);
    const int cn = cfg.coarse_grid_n;
    S.coarse_n = cn;
    S.coarse_uv.resize(cn);
    for (int i = 0; i < cn; ++i) S.coarse_uv[i] = (cn == 1) ? 0.0 : -1.0 + 2.0 * static_cast<double>(i) / (cn - 1);

    // tables and offsets
    std::vector<int> patch_obj;
    long long node_total = 0, field_total = 0;
    for (int k = 0; k < n_objects; ++k) {
        const bbrt_object_desc& o = objects[k];
        S.kind[k] = o.kind;
        if (o.kind == BBRT_OBJ_PATCH) {
            const bbrt_patch_desc* p = o.patch;
            if (!p) throw std::invalid_argument("bbrt: patch object without a descriptor");
            if (static_cast<long long>(p->imax) * p->jmax * p->kmax == 0)
                throw std::runtime_error("SurfacePatch: patch has no points");
            if (p->kmax != 1) throw std::invalid_argument("bbrt: only surface patches (kmax == 1) are supported");
            if (p->imax < 1 || p->jmax < 1 || p->imax > kMaxNodes || p->jmax > kMaxNodes)
                throw std::invalid_argument("bbrt: patch node counts must be in [1, 16]");
            if (!p->u_nodes || !p->v_nodes || !p->x || !p->y || !p->z || !p->dxdu || !p->dydu || !p->dzdu ||
                !p->dxdv || !p->dydv || !p->dzdv || !p->nu_x || !p->nu_y || !p->nu_z)
                throw std::invalid_argument("bbrt: patch descriptor with a null field");
            S.sub[k] = S.n_patches++;
            S.zone[k] = p->zone_id;
            S.p_imax.push_back(p->imax);
            S.p_jmax.push_back(p->jmax);
            S.p_node_off.push_back(node_total);
            S.p_field_off.push_back(field_total);
            node_total += 2LL * (p->imax + p->jmax);
            field_total += static_cast<long long>(kFields) * p->imax * p->jmax;
            patch_obj.push_back(k);
        } else if (o.kind == BBRT_OBJ_TRIANGLE) {
            S.sub[k] = static_cast<int>(S.tri.size() / 9);
            S.zone[k] = k;
            S.tri.insert(S.tri.end(), o.tri, o.tri + 9);
        } else {
            throw std::invalid_argument("bbrt: unknown object kind");
        }
    }
    S.p_nodes.resize(static_cast<size_t>(node_total));
    S.p_fields.resize(static_cast<size_t>(field_total));
    S.patch_obj = patch_obj;
    // node tables (nodes and barycentric weights) and node-major fields
    #pragma omp parallel for schedule(dynamic, 64)
    for (int q = 0; q < S.n_patches; ++q)
        copy_patch_tables(*objects[patch_obj[q]].patch, &S.p_nodes[S.p_node_off[q]], &S.p_fields[S.p_field_off[q]]);
    // triangles: exact AABB, centroid (a+b+c)/3, no padding
    for (int k = 0; k < n_objects; ++k) {
        if (S.kind[k] != BBRT_OBJ_TRIANGLE) continue;
        const double* v = objects[k].tri;
        for (int a = 0; a < 3; ++a) {
            S.box[6 * k + a] = std::min({ v[a], v[3 + a], v[6 + a] });
            S.box[6 * k + 3 + a] = std::max({ v[a], v[3 + a], v[6 + a] });
            S.centroid[3 * k + a] = (v[a] + v[3 + a] + v[6 + a]) / 3.0;
        }
        S.padding[k] = 0.0;
    }
}

void setup_patches_host(const bbrt_object_desc* objects, HostScene& S) {
    const int cn = S.coarse_n;
    const size_t per_xyz = 3 * static_cast<size_t>(cn) * cn, per_cell = 4 * static_cast<size_t>(cn - 1) * (cn - 1);
    S.c_xyz.resize(per_xyz * S.n_patches);
    S.c_cell.resize(per_cell * S.n_patches);
    // patch set-up, in parallel over patches
    #pragma omp parallel for schedule(dynamic, 16)
    for (int q = 0; q < S.n_patches; ++q) {
        const int k = S.patch_obj[q];
        const PatchSetup ps = setup_patch(*objects[k].patch, cn, S.coarse_uv, &S.c_xyz[per_xyz * q],
                                          &S.c_cell[per_cell * q]);
        std::memcpy(&S.box[6 * static_cast<size_t>(k)], ps.box, sizeof ps.box);
        std::memcpy(&S.centroid[3 * static_cast<size_t>(k)], ps.centroid, sizeof ps.centroid);
        S.padding[k] = ps.max_sag;
    }
}

void finish_host_scene(HostScene& S) {
    const int n_objects = S.n_objects;
    // BVH
    std::vector<int> ids(n_objects);
    for (int k = 0; k < n_objects; ++k) ids[k] = k;
    S.nodes.reserve(2 * static_cast<size_t>(n_objects));
    S.leaf_objects.reserve(n_objects);
    BvhBuilder bb(S, S.nodes, S.leaf_objects, S.cfg.leaf_threshold);
    bb.build(std::move(ids), 0);
    S.max_depth = bb.max_depth;

    // scene scale: diagonal of the union of all boxes, max sagitta
    double lo[3], hi[3];
    for (int a = 0; a < 3; ++a) { lo[a] = S.box[a]; hi[a] = S.box[3 + a]; }
    double ms = 0.0;
    for (int k = 0; k < n_objects; ++k) {
        for (int a = 0; a < 3; ++a) { lo[a] = dmin(lo[a], S.box[6 * k + a]); hi[a] = dmax(hi[a], S.box[6 * k + 3 + a]); }
        ms = dmax(ms, S.padding[k]);
    }
    const double dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
    S.scene_diagonal = std::sqrt(dx * dx + dy * dy + dz * dz);
    S.max_patch_sagitta = ms;
}

void build_host_scene(const bbrt_object_desc* objects, int n_objects, const bbrt_config& cfg, HostScene& S) {
    build_host_tables(objects, n_objects, cfg, S);
    setup_patches_host(objects, S);
    finish_host_scene(S);
}

void sample_grid(const bbrt_patch_desc& d, int n, double* xyz, double* normal, double* dxdu) {
    const int I = d.imax, J = d.jmax;
    std::vector<double> t(n);
    for (int i = 0; i < n; ++i) t[i] = (n == 1) ? 0.0 : -1.0 + 2.0 * static_cast<double>(i) / (n - 1);
    const std::vector<double> uw = bary_weights(d.u_nodes, I), vw = bary_weights(d.v_nodes, J);
    const size_t nn = static_cast<size_t>(n) * n;
    const double* src[9] = { d.x, d.y, d.z, d.nu_x, d.nu_y, d.nu_z, d.dxdu, d.dydu, d.dzdu };
    std::vector<double> g(9 * nn);
    for (int c = 0; c < 9; ++c) interp_grid(d.u_nodes, uw.data(), I, d.v_nodes, vw.data(), J, src[c], t, t, &g[c * nn]);
    for (size_t k = 0; k < nn; ++k) {
        const double nx = g[3 * nn + k], ny = g[4 * nn + k], nz = g[5 * nn + k];
        const double len = std::sqrt(nx * nx + ny * ny + nz * nz);
        xyz[3 * k] = g[k]; xyz[3 * k + 1] = g[nn + k]; xyz[3 * k + 2] = g[2 * nn + k];
        normal[3 * k] = nx / len; normal[3 * k + 1] = ny / len; normal[3 * k + 2] = nz / len;
        dxdu[3 * k] = g[6 * nn + k]; dxdu[3 * k + 1] = g[7 * nn + k]; dxdu[3 * k + 2] = g[8 * nn + k];
    }
}

void read_patch_file(const std::string& path, PatchFileData& d) {
    std::ifstream fin(path);
    if (!fin.is_open()) throw std::runtime_error("SurfacePatch: cannot open patch file: " + path);
    fin >> d.imax >> d.jmax >> d.kmax >> d.zone;
    if (!fin) throw std::runtime_error("SurfacePatch: bad header in patch file: " + path);
    const long long n = static_cast<long long>(d.imax) * d.jmax * d.kmax;
    if (d.imax < 0 || d.jmax < 0 || d.kmax < 0 || n > (1LL << 28))
        throw std::runtime_error("SurfacePatch: bad header in patch file: " + path);
    auto rd = [&](std::vector<double>& v, long long count) {
        v.resize(static_cast<size_t>(count));
        for (long long i = 0; i < count; ++i) fin >> v[static_cast<size_t>(i)];
    };
    rd(d.un, d.imax);
    rd(d.vn, d.jmax);
    rd(d.f[0], n); rd(d.f[1], n); rd(d.f[2], n);
    d.mask.resize(static_cast<size_t>(n));
    for (long long i = 0; i < n; ++i) fin >> d.mask[static_cast<size_t>(i)];
    for (int k = 3; k < 13; ++k) rd(d.f[k], n);
    if (!fin) throw std::runtime_error("SurfacePatch: truncated patch file: " + path);
    fin >> std::ws;
    if (!fin.eof()) {
        if (!(fin >> d.edge_flags[0] >> d.edge_flags[1] >> d.edge_flags[2] >> d.edge_flags[3]))
            throw std::runtime_error("SurfacePatch: malformed sharp-edge data in patch file: " + path);
    }
}

bbrt_patch_desc patch_desc_of(const PatchFileData& d) {
    bbrt_patch_desc p{};
    p.imax = d.imax; p.jmax = d.jmax; p.kmax = d.kmax; p.zone_id = d.zone;
    p.u_nodes = d.un.data(); p.v_nodes = d.vn.data();
    p.x = d.f[0].data(); p.y = d.f[1].data(); p.z = d.f[2].data();
    p.dxdu = d.f[3].data(); p.dydu = d.f[4].data(); p.dzdu = d.f[5].data();
    p.dxdv = d.f[6].data(); p.dydv = d.f[7].data(); p.dzdv = d.f[8].data();
    // f[9] is dS
    p.nu_x = d.f[10].data(); p.nu_y = d.f[11].data(); p.nu_z = d.f[12].data();
    return p;
}

}  // namespace bbrt

namespace bbrt {
namespace {

// Largest float <= x and smallest float >= x (outward rounding of box bounds).
inline float float_down(double x) {
    float f = static_cast<float>(x);
    if (static_cast<double>(f) > x) f = std::nextafter(f, -std::numeric_limits<float>::infinity());
    return f;
}
inline float float_up(double x) {
    float f = static_cast<float>(x);
    if (static_cast<double>(f) < x) f = std::nextafter(f, std::numeric_limits<float>::infinity());
    return f;
}

}  // namespace

// Cull tables.  A cell box is the AABB of the twelve offset corners the six
// stage-1 triangles of that cell are built from, computed with the same
// expression p + normal * (sign * sagitta) the device evaluates; a block box
// is the union of its cells' boxes.  The per-ray inflation constants bound
// how far outside its triangle a Moller-Trumbore hit can be accepted in FP64
// (|det| >= 1e-9 bounds the error amplification: a barycentric error of at
// most ~16 eps h (|o - v0| + 2h) / 1e-9 per coordinate, with h the longest
// triangle edge) plus the FP32 slab test's own rounding.  Culling is turned
// off where that bound stops being small (very large triangles, non-finite
// or huge coordinates), so it can only skip work, never change a result.
void build_cull_tables(const HostScene& S, CullTables& C) {
    C = CullTables();
    if (S.n_patches == 0 || !S.cfg.cull) return;
    const int n = S.coarse_n, nc = n - 1;
    const int B = std::max(4, static_cast<int>(std::ceil(std::sqrt(static_cast<double>(nc)))));
    const int NB = (nc + B - 1) / B;
    C.block_cells = B;
    C.n_blocks_side = NB;
    C.cell_box.assign(static_cast<size_t>(S.n_patches) * nc * nc * 6, 0.0f);
    C.block_box.assign(static_cast<size_t>(S.n_patches) * NB * NB * 6, 0.0f);
    const size_t per_xyz = 3 * static_cast<size_t>(n) * n, per_cell = 4 * static_cast<size_t>(nc) * nc;
    double hmax = 0.0, cmax = 0.0;
    bool finite = true;
    #pragma omp parallel for schedule(dynamic, 16) reduction(max : hmax, cmax) reduction(&& : finite)
    for (int q = 0; q < S.n_patches; ++q) {
        const double* X = &S.c_xyz[per_xyz * q];
        const double* CC = &S.c_cell[per_cell * q];
        float* cb = &C.cell_box[static_cast<size_t>(q) * nc * nc * 6];
        float* bb = &C.block_box[static_cast<size_t>(q) * NB * NB * 6];
        for (int k = 0; k < NB * NB; ++k) {
            for (int a = 0; a < 3; ++a) {
                bb[6 * k + a] = std::numeric_limits<float>::infinity();
                bb[6 * k + 3 + a] = -std::numeric_limits<float>::infinity();
            }
        }
        for (int i = 0; i < nc; ++i) {
            for (int j = 0; j < nc; ++j) {
                const double* p[4] = { X + 3 * (i * n + j), X + 3 * ((i + 1) * n + j), X + 3 * (i * n + j + 1),
                                       X + 3 * ((i + 1) * n + j + 1) };   // p00 p10 p01 p11
                const double* c = CC + 4 * (i * nc + j);
                double lo[3] = { std::numeric_limits<double>::infinity(), std::numeric_limits<double>::infinity(),
                                 std::numeric_limits<double>::infinity() };
                double hi[3] = { -lo[0], -lo[1], -lo[2] };
                for (int k = 0; k < 3; ++k) {
                    const double sg = (k == 0) ? 0.0 : ((k == 1) ? 1.0 : -1.0);
                    const double dd = sg * c[3];
                    double qv[4][3];
                    for (int r = 0; r < 4; ++r)
                        for (int a = 0; a < 3; ++a) {
                            qv[r][a] = p[r][a] + c[a] * dd;
                            lo[a] = std::min(lo[a], qv[r][a]);
                            hi[a] = std::max(hi[a], qv[r][a]);
                            finite = finite && std::isfinite(qv[r][a]);
                            cmax = std::max(cmax, std::fabs(qv[r][a]));
                        }
                    // edge lengths Moller-Trumbore sees: q10-q00, q11-q00, q01-q00
                    const int ends[3] = { 1, 3, 2 };
                    for (int e : ends) {
                        const double dx = qv[e][0] - qv[0][0], dy = qv[e][1] - qv[0][1], dz = qv[e][2] - qv[0][2];
                        hmax = std::max(hmax, std::sqrt(dx * dx + dy * dy + dz * dz));
                    }
                }
                float* box = cb + 6 * (i * nc + j);
                float* blk = bb + 6 * ((i / B) * NB + (j / B));
                for (int a = 0; a < 3; ++a) {
                    box[a] = float_down(lo[a]);
                    box[3 + a] = float_up(hi[a]);
                    blk[a] = std::min(blk[a], box[a]);
                    blk[3 + a] = std::max(blk[3 + a], box[3 + a]);
                }
            }
        }
    }
    cull_constants(S, hmax, cmax, finite, C);
}

void cull_constants(const HostScene& S, double hmax, double cmax, bool finite, CullTables& C) {
    C.enabled = false;
    const double eps64 = std::ldexp(1.0, -53), eps32 = std::ldexp(1.0, -24);
    if (!finite || cmax > 1e15 || 16.0 * eps64 * hmax * hmax > 1e-11) return;   // bound not small: no culling
    double lo[3], hi[3];
    for (int a = 0; a < 3; ++a) { lo[a] = S.box[a]; hi[a] = S.box[3 + a]; }
    for (int k = 0; k < S.n_objects; ++k)
        for (int a = 0; a < 3; ++a) { lo[a] = std::min(lo[a], S.box[6 * k + a]); hi[a] = std::max(hi[a], S.box[6 * k + 3 + a]); }
    double r2 = 0.0;
    for (int a = 0; a < 3; ++a) {
        C.center[a] = 0.5 * (lo[a] + hi[a]);
        r2 += (hi[a] - lo[a]) * (hi[a] - lo[a]);
    }
    C.radius = 0.5 * std::sqrt(r2) * (1.0 + 1e-12) + 1e-300;
    C.h = hmax;
    C.a = 256.0 * eps64 * hmax * hmax / 1e-9;
    C.b = 32.0 * eps32;
    C.coord = std::sqrt(C.center[0] * C.center[0] + C.center[1] * C.center[1] + C.center[2] * C.center[2]) + C.radius;
    C.enabled = true;
}

}  // namespace bbrt
