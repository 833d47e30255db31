// bbrt oracle — TEST INFRASTRUCTURE ONLY.
//
// A CPU restatement, in plain C++17, of the reference's multi-bounce
// specular trace loop (manuelarturosantana/BillardBallRayTracing3D; paths
// below are relative to that project).  It is the checker the GPU path is
// compared against in tests/, in __graft_entry__.smoke() and in the
// cpu_baseline leg of bench.py, and nothing else: the product never links,
// loads or calls it.
//
// It follows the reference operation by operation (same association order
// of every sum and product, same comparisons, same NaN behaviour of
// std::min/std::max, no FMA), so on the same inputs it is bit-identical to
// the reference's x86-64 build.  That claim is pinned by tests against the
// reference itself (oracle/_ref, built by oracle/build_ref.sh) and against
// committed fixtures generated from it (tests/golden/).
//
// Instead of exceptions, Newton failures and trace errors come back as the
// status codes of include/bbrt.h (BBRT_RAY_*); the reference throws
// std::runtime_error and trace_ray turns that into RayPath::Status::Error.
//
// Third-party arithmetic: the coarse grid uses cblas_dgemm (MKL, not
// available here).  This file restates the published dgemm semantic with
// the summation order of oracle/shim/mkl.h (left-to-right over k).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <vector>
#include <omp.h>

#include "../include/bbrt.h"

namespace oracle {

struct V3 { double x, y, z; };

// MollerTrumbore.hpp:13-27
static inline V3 sub(const V3& a, const V3& b) { return { a.x - b.x, a.y - b.y, a.z - b.z }; }
static inline V3 cross(const V3& a, const V3& b) {
    return { a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x };
}
static inline double dot(const V3& a, const V3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline V3 normalize(const V3& v) {
    const double len = std::sqrt(dot(v, v));
    return { v.x / len, v.y / len, v.z / len };
}

struct Box { V3 mn{ INFINITY, INFINITY, INFINITY }, mx{ -INFINITY, -INFINITY, -INFINITY }; };

struct Hit {
    double t = 0;
    V3 p{ 0, 0, 0 }, n{ 0, 0, 0 };
    double u = 0, v = 0;
    int obj = -1;
};

// Outcome of one object's intersect(): miss, hit, or a thrown error.
struct Result {
    bool hit = false;
    Hit h;
    int err = 0;          // BBRT_RAY_NEWTON_* when the reference would throw
    double err_val[2] = { 0, 0 };
};

// moller_trumbore, MollerTrumbore.hpp:32-64 (eps = 1e-9).  Only t and the
// barycentrics are returned: the reference's Hit point/normal of a stage-1
// triangle hit are never read.
static inline bool moller_trumbore(const V3& o, const V3& d, const V3& v0, const V3& v1, const V3& v2,
                                   double& t_out, double& u_out, double& v_out) {
    const double eps = 1e-9;
    const V3 e1 = sub(v1, v0);
    const V3 e2 = sub(v2, v0);
    const V3 pvec = cross(d, e2);
    const double det = dot(e1, pvec);
    if (std::fabs(det) < eps) return false;
    const double inv_det = 1.0 / det;
    const V3 tvec = sub(o, v0);
    const double u = dot(tvec, pvec) * inv_det;
    if (u < 0.0 || u > 1.0) return false;
    const V3 qvec = cross(tvec, e1);
    const double v = dot(d, qvec) * inv_det;
    if (v < 0.0 || u + v > 1.0) return false;
    const double t = dot(e2, qvec) * inv_det;
    if (t < eps) return false;
    t_out = t; u_out = u; v_out = v;
    return true;
}

// barycentric_weights, PatchInterpolation.hpp:25-52
static std::vector<double> barycentric_weights(const std::vector<double>& nodes) {
    const int N = static_cast<int>(nodes.size());
    std::vector<double> w(N, 1.0);
    for (int j = 0; j < N; ++j) {
        double p = 1.0;
        for (int i = 0; i < N; ++i)
            if (i != j) p *= (nodes[j] - nodes[i]);
        w[j] = 1.0 / p;
    }
    return w;
}

// Row-major C = A*op(B) with the shim's order (oracle/shim/mkl.h), alpha=1, beta=0.
static void gemm_nn(int P, int M, int N, const double* A, const double* B, double* C) {
    for (int i = 0; i < P; ++i)
        for (int j = 0; j < M; ++j) {
            double s = 0.0;
            for (int k = 0; k < N; ++k) s += A[i * N + k] * B[k * M + j];
            C[i * M + j] = 1.0 * s;
        }
}
static void gemm_nt(int P, int Q, int M, const double* A, const double* B, double* C) {
    for (int i = 0; i < P; ++i)
        for (int j = 0; j < Q; ++j) {
            double s = 0.0;
            for (int k = 0; k < M; ++k) s += A[i * M + k] * B[j * M + k];
            C[i * Q + j] = 1.0 * s;
        }
}

// lagrange_interpolation_2D, PatchInterpolation.hpp:54-159 (EQUAL_TOL 1e-12, :21)
static void lagrange_2d(const std::vector<double>& xn, const std::vector<double>& yn,
                        const std::vector<double>& xw, const std::vector<double>& yw,
                        const double* f, const std::vector<double>& x, const std::vector<double>& y,
                        double* out) {
    const double EQ = 1.0e-12;
    const int N = static_cast<int>(xn.size()), M = static_cast<int>(yn.size());
    const int P = static_cast<int>(x.size()), Q = static_cast<int>(y.size());
    std::vector<double> lx(P, 1.0), ly(Q, 1.0), vx(static_cast<size_t>(P) * N), vy(static_cast<size_t>(M) * Q);
    for (int i = 0; i < P; ++i) {
        double prod = 1.0; int eq = -1;
        for (int j = 0; j < N; ++j) {
            const double diff = x[i] - xn[j];
            if (std::abs(diff) < EQ) { eq = j; break; }
            vx[i * N + j] = xw[j] / diff;
            prod *= diff;
        }
        if (eq != -1) {
            std::fill(vx.begin() + i * N, vx.begin() + (i + 1) * N, 0.0);
            vx[i * N + eq] = 1.0; lx[i] = 1.0;
        } else {
            lx[i] = prod;
        }
    }
    for (int i = 0; i < Q; ++i) {
        double prod = 1.0; int eq = -1;
        for (int j = 0; j < M; ++j) {
            const double diff = y[i] - yn[j];
            if (std::abs(diff) < EQ) { eq = j; break; }
            vy[i * M + j] = yw[j] / diff;
            prod *= diff;
        }
        if (eq != -1) {
            std::fill(vy.begin() + i * M, vy.begin() + (i + 1) * M, 0.0);
            vy[i * M + eq] = 1.0; ly[i] = 1.0;
        } else {
            ly[i] = prod;
        }
    }
    std::vector<double> mp(static_cast<size_t>(P) * M);
    gemm_nn(P, M, N, vx.data(), f, mp.data());
    gemm_nt(P, Q, M, mp.data(), vy.data(), out);
    for (int i = 0; i < P; ++i)
        for (int j = 0; j < Q; ++j) out[i * Q + j] *= lx[i] * ly[j];
}

// lagrange_basis_1d, SurfacePatch.hpp:518-538
static void basis_1d(const std::vector<double>& nodes, const std::vector<double>& w, double x, double* b) {
    const double EQ = 1.0e-12;
    const int N = static_cast<int>(nodes.size());
    for (int i = 0; i < N; ++i) b[i] = 0.0;
    for (int i = 0; i < N; ++i)
        if (std::fabs(x - nodes[i]) < EQ) { b[i] = 1.0; return; }
    double denom = 0.0;
    for (int i = 0; i < N; ++i) {
        const double li = w[i] / (x - nodes[i]);
        b[i] = li;
        denom += li;
    }
    for (int i = 0; i < N; ++i) b[i] /= denom;
}

// solve3x3, SurfacePatch.hpp:559-579
static bool solve3x3(const double J[3][3], const V3& b, double x[3]) {
    const double a11 = J[0][0], a12 = J[0][1], a13 = J[0][2];
    const double a21 = J[1][0], a22 = J[1][1], a23 = J[1][2];
    const double a31 = J[2][0], a32 = J[2][1], a33 = J[2][2];
    const double det = a11 * (a22 * a33 - a23 * a32) - a12 * (a21 * a33 - a23 * a31) + a13 * (a21 * a32 - a22 * a31);
    if (std::fabs(det) < 1e-14) return false;
    const double bx = b.x, by = b.y, bz = b.z;
    const double d0 = bx * (a22 * a33 - a23 * a32) - a12 * (by * a33 - a23 * bz) + a13 * (by * a32 - a22 * bz);
    const double d1 = a11 * (by * a33 - a23 * bz) - bx * (a21 * a33 - a23 * a31) + a13 * (a21 * bz - by * a31);
    const double d2 = a11 * (a22 * bz - by * a32) - a12 * (a21 * bz - by * a31) + bx * (a21 * a32 - a22 * a31);
    x[0] = d0 / det; x[1] = d1 / det; x[2] = d2 / det;
    return true;
}

struct Config {
    int coarse_n = 100, newton_max_iters = 20, leaf_threshold = 4;
    double newton_tol = 1e-3, eps_factor = 1e-9, sag_factor = 5.0, backface_tol = 1e-9;
};

struct Object {
    int kind = BBRT_OBJ_PATCH;
    long long zone = 0;
    Box box;
    V3 centroid{ 0, 0, 0 };
    double max_sag = 0.0;
    // patch data (SurfacePatch::Data, SurfacePatch.hpp:59-89)
    int imax = 0, jmax = 0;
    std::vector<double> un, vn, uw, vw;
    std::vector<double> f[12];   // x y z dxdu dydu dzdu dxdv dydv dzdv nuX nuY nuZ
    // coarse grid (SurfacePatch.hpp:95-115)
    int n = 0;
    std::vector<double> cu, cv, cx, cy, cz, sag;
    std::vector<V3> cn;
    // triangle (ScatObjects/Triangle.hpp)
    V3 tv[3];

    V3 cpoint(int i, int j) const { const int k = i * n + j; return { cx[k], cy[k], cz[k] }; }

    // eval_scalar_field, SurfacePatch.hpp:542-555
    double eval(const double* lu, const double* lv, int field) const {
        const std::vector<double>& F = f[field];
        double sum = 0.0;
        for (int i = 0; i < imax; ++i) {
            const double li = lu[i];
            if (li == 0.0) continue;
            const double* row = &F[static_cast<size_t>(i) * jmax];
            double rs = 0.0;
            for (int j = 0; j < jmax; ++j) rs += lv[j] * row[j];
            sum += li * rs;
        }
        return sum;
    }
};

// SurfacePatch set-up: constructor SurfacePatch.hpp:125-131.
static void setup_patch(Object& P, const bbrt_patch_desc& d, const Config& cfg) {
    P.kind = BBRT_OBJ_PATCH;
    P.zone = d.zone_id;
    P.imax = d.imax; P.jmax = d.jmax;
    const long long n = static_cast<long long>(d.imax) * d.jmax;
    P.un.assign(d.u_nodes, d.u_nodes + d.imax);
    P.vn.assign(d.v_nodes, d.v_nodes + d.jmax);
    P.uw = barycentric_weights(P.un);            // :335-336
    P.vw = barycentric_weights(P.vn);
    const double* src[12] = { d.x, d.y, d.z, d.dxdu, d.dydu, d.dzdu, d.dxdv, d.dydv, d.dzdv, d.nu_x, d.nu_y, d.nu_z };
    for (int k = 0; k < 12; ++k) P.f[k].assign(src[k], src[k] + n);

    // compute_centroid_and_box, :380-407
    double sx = 0, sy = 0, sz = 0;
    Box b;
    for (long long i = 0; i < n; ++i) {
        const double px = P.f[0][i], py = P.f[1][i], pz = P.f[2][i];
        sx += px; sy += py; sz += pz;
        b.mn.x = std::min(b.mn.x, px); b.mn.y = std::min(b.mn.y, py); b.mn.z = std::min(b.mn.z, pz);
        b.mx.x = std::max(b.mx.x, px); b.mx.y = std::max(b.mx.y, py); b.mx.z = std::max(b.mx.z, pz);
    }
    const double inv_n = 1.0 / static_cast<double>(n);
    P.centroid = { sx * inv_n, sy * inv_n, sz * inv_n };
    P.box = b;

    // compute_coarse_grid, :416-436
    const int cn = cfg.coarse_n;
    P.n = cn;
    P.cu.resize(cn); P.cv.resize(cn);
    for (int i = 0; i < cn; ++i) {
        const double t = (cn == 1) ? 0.0 : -1.0 + 2.0 * static_cast<double>(i) / (cn - 1);
        P.cu[i] = t; P.cv[i] = t;
    }
    P.cx.resize(static_cast<size_t>(cn) * cn); P.cy.resize(P.cx.size()); P.cz.resize(P.cx.size());
    lagrange_2d(P.un, P.vn, P.uw, P.vw, P.f[0].data(), P.cu, P.cv, P.cx.data());
    lagrange_2d(P.un, P.vn, P.uw, P.vw, P.f[1].data(), P.cu, P.cv, P.cy.data());
    lagrange_2d(P.un, P.vn, P.uw, P.vw, P.f[2].data(), P.cu, P.cv, P.cz.data());

    // compute_cell_padding, :446-492
    const int cells = (cn - 1) * (cn - 1);
    P.sag.assign(cells, 0.0);
    P.cn.assign(cells, V3{ 0, 0, 0 });
    std::vector<double> lu(P.imax), lv(P.jmax);
    double ms = 0.0;
    for (int i = 0; i + 1 < cn; ++i)
        for (int j = 0; j + 1 < cn; ++j) {
            const double um = 0.5 * (P.cu[i] + P.cu[i + 1]);
            const double vm = 0.5 * (P.cv[j] + P.cv[j + 1]);
            basis_1d(P.un, P.uw, um, lu.data());
            basis_1d(P.vn, P.vw, vm, lv.data());
            const V3 tm{ P.eval(lu.data(), lv.data(), 0), P.eval(lu.data(), lv.data(), 1), P.eval(lu.data(), lv.data(), 2) };
            const V3 nm = normalize({ P.eval(lu.data(), lv.data(), 9), P.eval(lu.data(), lv.data(), 10),
                                      P.eval(lu.data(), lv.data(), 11) });
            const V3 p00 = P.cpoint(i, j), p10 = P.cpoint(i + 1, j), p01 = P.cpoint(i, j + 1), p11 = P.cpoint(i + 1, j + 1);
            const V3 bm{ 0.25 * (p00.x + p10.x + p01.x + p11.x), 0.25 * (p00.y + p10.y + p01.y + p11.y),
                         0.25 * (p00.z + p10.z + p01.z + p11.z) };
            const V3 df = sub(tm, bm);
            const double s = std::sqrt(dot(df, df));
            const int idx = i * (cn - 1) + j;
            P.sag[idx] = s;
            P.cn[idx] = nm;
            ms = std::max(ms, s);
        }
    P.box.mn.x -= ms; P.box.mn.y -= ms; P.box.mn.z -= ms;
    P.box.mx.x += ms; P.box.mx.y += ms; P.box.mx.z += ms;
    P.max_sag = ms;
}

// Triangle constructor, ScatObjects/Triangle.hpp:11-24
static void setup_triangle(Object& T, const double* v) {
    T.kind = BBRT_OBJ_TRIANGLE;
    T.tv[0] = { v[0], v[1], v[2] }; T.tv[1] = { v[3], v[4], v[5] }; T.tv[2] = { v[6], v[7], v[8] };
    const V3 &a = T.tv[0], &b = T.tv[1], &c = T.tv[2];
    T.box.mn = { std::min({ a.x, b.x, c.x }), std::min({ a.y, b.y, c.y }), std::min({ a.z, b.z, c.z }) };
    T.box.mx = { std::max({ a.x, b.x, c.x }), std::max({ a.y, b.y, c.y }), std::max({ a.z, b.z, c.z }) };
    T.centroid = { (a.x + b.x + c.x) / 3.0, (a.y + b.y + c.y) / 3.0, (a.z + b.z + c.z) / 3.0 };
    T.max_sag = 0.0;   // ScatObject::self_intersect_padding default, ScatObject.hpp:81
}

// newton_refine, SurfacePatch.hpp:593-660
static Result newton_refine(const Object& P, const V3& o, const V3& d, double u0, double v0, double t0,
                            const Config& cfg, long long* iters) {
    Result r;
    double u = u0, v = v0, t = t0;
    std::vector<double> lu(P.imax), lv(P.jmax);
    double step = std::numeric_limits<double>::infinity();
    for (int it = 0; it < cfg.newton_max_iters; ++it) {
        if (iters) ++*iters;
        basis_1d(P.un, P.uw, u, lu.data());
        basis_1d(P.vn, P.vw, v, lv.data());
        const V3 X{ P.eval(lu.data(), lv.data(), 0), P.eval(lu.data(), lv.data(), 1), P.eval(lu.data(), lv.data(), 2) };
        const V3 Xu{ P.eval(lu.data(), lv.data(), 3), P.eval(lu.data(), lv.data(), 4), P.eval(lu.data(), lv.data(), 5) };
        const V3 Xv{ P.eval(lu.data(), lv.data(), 6), P.eval(lu.data(), lv.data(), 7), P.eval(lu.data(), lv.data(), 8) };
        const V3 R{ o.x + t * d.x, o.y + t * d.y, o.z + t * d.z };
        const V3 F = sub(X, R);
        const double J[3][3] = { { Xu.x, Xv.x, -d.x }, { Xu.y, Xv.y, -d.y }, { Xu.z, Xv.z, -d.z } };
        double dl[3];
        if (!solve3x3(J, F, dl)) { r.err = BBRT_RAY_NEWTON_SINGULAR; return r; }
        u -= dl[0]; v -= dl[1]; t -= dl[2];
        step = std::sqrt(dl[0] * dl[0] + dl[1] * dl[1] + dl[2] * dl[2]);
        if (step < cfg.newton_tol) break;
    }
    if (step >= cfg.newton_tol) { r.err = BBRT_RAY_NEWTON_NOCONV; r.err_val[0] = step; return r; }
    const double tol = 1e-6;
    if (u < -1.0 - tol || u > 1.0 + tol || v < -1.0 - tol || v > 1.0 + tol) {
        r.err = BBRT_RAY_NEWTON_DOMAIN; r.err_val[0] = u; r.err_val[1] = v; return r;
    }
    basis_1d(P.un, P.uw, u, lu.data());
    basis_1d(P.vn, P.vw, v, lv.data());
    r.hit = true;
    r.h.t = t;
    r.h.p = { P.eval(lu.data(), lv.data(), 0), P.eval(lu.data(), lv.data(), 1), P.eval(lu.data(), lv.data(), 2) };
    r.h.n = normalize({ P.eval(lu.data(), lv.data(), 9), P.eval(lu.data(), lv.data(), 10), P.eval(lu.data(), lv.data(), 11) });
    r.h.u = u; r.h.v = v;
    return r;
}

struct Counters { long long patch_tests = 0, tri_tests = 0, newton_iters = 0, node_tests = 0; };

// SurfacePatch::intersect, SurfacePatch.hpp:253-303 (stage 1 brute force,
// triangle_uv_centroid :499-510, then newton_refine).
static Result patch_intersect(const Object& P, const V3& o, const V3& d, const Config& cfg, Counters* c) {
    Result r;
    const int n = P.n;
    bool have = false;
    double best_t = 0;
    int bi = -1, bj = -1;
    bool second = false;
    if (c) ++c->patch_tests;
    for (int i = 0; i + 1 < n; ++i)
        for (int j = 0; j + 1 < n; ++j) {
            const V3 p00 = P.cpoint(i, j), p10 = P.cpoint(i + 1, j), p01 = P.cpoint(i, j + 1), p11 = P.cpoint(i + 1, j + 1);
            const int idx = i * (n - 1) + j;
            const double s = P.sag[idx];
            const V3& cn = P.cn[idx];
            const double signs[3] = { 0.0, 1.0, -1.0 };
            for (int k = 0; k < 3; ++k) {
                const double dd = signs[k] * s;
                const V3 q00{ p00.x + cn.x * dd, p00.y + cn.y * dd, p00.z + cn.z * dd };
                const V3 q10{ p10.x + cn.x * dd, p10.y + cn.y * dd, p10.z + cn.z * dd };
                const V3 q01{ p01.x + cn.x * dd, p01.y + cn.y * dd, p01.z + cn.z * dd };
                const V3 q11{ p11.x + cn.x * dd, p11.y + cn.y * dd, p11.z + cn.z * dd };
                double t, bu, bv;
                if (c) c->tri_tests += 2;
                if (moller_trumbore(o, d, q00, q10, q11, t, bu, bv) && (!have || t < best_t)) {
                    have = true; best_t = t; bi = i; bj = j; second = false;
                }
                if (moller_trumbore(o, d, q00, q11, q01, t, bu, bv) && (!have || t < best_t)) {
                    have = true; best_t = t; bi = i; bj = j; second = true;
                }
            }
        }
    if (!have) return r;
    double u0, v0;
    const double ui = P.cu[bi], ui1 = P.cu[bi + 1], vj = P.cv[bj], vj1 = P.cv[bj + 1];
    if (!second) { u0 = (ui + ui1 + ui1) / 3.0; v0 = (vj + vj + vj1) / 3.0; }
    else         { u0 = (ui + ui + ui1) / 3.0; v0 = (vj + vj1 + vj1) / 3.0; }
    return newton_refine(P, o, d, u0, v0, best_t, cfg, c ? &c->newton_iters : nullptr);
}

// Triangle::intersect, ScatObjects/Triangle.hpp:26-28 -> moller_trumbore,
// whose Hit carries point o + t d and normal normalize(e1 x e2).
static Result triangle_intersect(const Object& T, const V3& o, const V3& d) {
    Result r;
    double t, u, v;
    if (!moller_trumbore(o, d, T.tv[0], T.tv[1], T.tv[2], t, u, v)) return r;
    r.hit = true;
    r.h.t = t;
    r.h.p = { o.x + t * d.x, o.y + t * d.y, o.z + t * d.z };
    r.h.n = normalize(cross(sub(T.tv[1], T.tv[0]), sub(T.tv[2], T.tv[0])));
    r.h.u = u; r.h.v = v;
    return r;
}

static Result object_intersect(const Object& ob, const V3& o, const V3& d, const Config& cfg, Counters* c) {
    return ob.kind == BBRT_OBJ_PATCH ? patch_intersect(ob, o, d, cfg, c) : triangle_intersect(ob, o, d);
}

// BVH, BVH.hpp:14-189
struct Node { Box box; int right = -1, start = 0, count = 0; int axis = 0; };

struct Scene {
    Config cfg;
    std::vector<Object> objs;
    std::vector<Node> nodes;
    std::vector<int> leaf_objs;
    double diag = 0.0, max_sag = 0.0;

    // union_box, BVH.hpp:39-48
    static Box unite(const Box& a, const Box& b) {
        Box r;
        r.mn = { std::min(a.mn.x, b.mn.x), std::min(a.mn.y, b.mn.y), std::min(a.mn.z, b.mn.z) };
        r.mx = { std::max(a.mx.x, b.mx.x), std::max(a.mx.y, b.mx.y), std::max(a.mx.z, b.mx.z) };
        return r;
    }

    // BVH::build, BVH.hpp:136-189
    int build(std::vector<int> ids) {
        const int me = static_cast<int>(nodes.size());
        nodes.emplace_back();
        Box box = objs[ids.front()].box;
        for (size_t i = 1; i < ids.size(); ++i) box = unite(box, objs[ids[i]].box);
        if (static_cast<int>(ids.size()) <= cfg.leaf_threshold) {
            nodes[me].box = box; nodes[me].right = -1;
            nodes[me].start = static_cast<int>(leaf_objs.size());
            nodes[me].count = static_cast<int>(ids.size());
            for (int id : ids) leaf_objs.push_back(id);
            return me;
        }
        V3 lo = objs[ids.front()].centroid, hi = lo;
        for (int id : ids) {
            const V3& c = objs[id].centroid;
            lo.x = std::min(lo.x, c.x); hi.x = std::max(hi.x, c.x);
            lo.y = std::min(lo.y, c.y); hi.y = std::max(hi.y, c.y);
            lo.z = std::min(lo.z, c.z); hi.z = std::max(hi.z, c.z);
        }
        const double spread[3] = { hi.x - lo.x, hi.y - lo.y, hi.z - lo.z };
        const int axis = static_cast<int>(std::max_element(spread, spread + 3) - spread);
        auto mid = ids.begin() + ids.size() / 2;
        std::nth_element(ids.begin(), mid, ids.end(), [&](int a, int b) {
            const V3& ca = objs[a].centroid; const V3& cb = objs[b].centroid;
            const double va = axis == 0 ? ca.x : axis == 1 ? ca.y : ca.z;
            const double vb = axis == 0 ? cb.x : axis == 1 ? cb.y : cb.z;
            return va < vb;
        });
        std::vector<int> L(ids.begin(), mid), R(mid, ids.end());
        ids.clear(); ids.shrink_to_fit();
        build(std::move(L));
        const int r = build(std::move(R));
        nodes[me].box = box; nodes[me].right = r; nodes[me].count = 0; nodes[me].axis = axis;
        return me;
    }

    // ray_box, BVH.hpp:14-37 (std::max/std::min NaN behaviour kept)
    static bool ray_box(const V3& o, const double inv[3], const Box& b, double best_t, double& tmin_out) {
        double tmin = -INFINITY, tmax = INFINITY;
        const double oo[3] = { o.x, o.y, o.z }, lo[3] = { b.mn.x, b.mn.y, b.mn.z }, hi[3] = { b.mx.x, b.mx.y, b.mx.z };
        for (int a = 0; a < 3; ++a) {
            double t1 = (lo[a] - oo[a]) * inv[a];
            double t2 = (hi[a] - oo[a]) * inv[a];
            if (inv[a] < 0.0) std::swap(t1, t2);
            tmin = std::max(tmin, t1);
            tmax = std::min(tmax, t2);
            if (tmax < tmin) return false;
        }
        if (tmin > best_t) return false;
        tmin_out = tmin;
        return tmax >= std::max(tmin, 0.0);
    }

    // BVH::intersect, BVH.hpp:75-128; a Newton failure of any tested patch
    // aborts the query (the reference's exception propagates out).
    Result bvh_intersect(const V3& o, const V3& d, Counters* c) const {
        const double inv[3] = { 1.0 / d.x, 1.0 / d.y, 1.0 / d.z };
        const bool neg[3] = { inv[0] < 0.0, inv[1] < 0.0, inv[2] < 0.0 };
        Result best;
        double best_t = INFINITY;
        int stack[64], sp = 0;
        stack[sp++] = 0;
        while (sp > 0) {
            const int idx = stack[--sp];
            const Node& nd = nodes[idx];
            double tmin;
            if (c) ++c->node_tests;
            if (!ray_box(o, inv, nd.box, best_t, tmin)) continue;
            if (nd.right < 0) {
                for (int i = 0; i < nd.count; ++i) {
                    const int id = leaf_objs[nd.start + i];
                    Result r = object_intersect(objs[id], o, d, cfg, c);
                    if (r.err) { r.h.obj = id; return r; }
                    if (r.hit && r.h.t < best_t) { best_t = r.h.t; best = r; best.h.obj = id; }
                }
                continue;
            }
            const int left = idx + 1, right = nd.right;
            if (neg[nd.axis]) { stack[sp++] = left; stack[sp++] = right; }
            else              { stack[sp++] = right; stack[sp++] = left; }
        }
        return best;
    }

    // brute_force_intersect, BruteForce.hpp:7-16 (Hit::object left untagged there;
    // the index is reported here for convenience)
    Result brute_intersect(const V3& o, const V3& d) const {
        Result best;
        for (size_t i = 0; i < objs.size(); ++i) {
            Result r = object_intersect(objs[i], o, d, cfg, nullptr);
            if (r.err) { r.h.obj = static_cast<int>(i); return r; }
            if (r.hit && (!best.hit || r.h.t < best.h.t)) { best = r; best.h.obj = static_cast<int>(i); }
        }
        return best;
    }

    // RayTracingDriver::self_intersect_epsilon, RayTracingDriver.hpp:260-265
    double eps_for(int obj) const {
        const double pad = obj >= 0 ? objs[obj].max_sag : max_sag;
        return std::max(cfg.eps_factor * diag, cfg.sag_factor * pad);
    }
};

struct TraceOut {
    int status = BBRT_RAY_MAX_BOUNCES, bounces = 0, err_obj = -1;
    double err_val[2] = { 0, 0 };
    V3 dir{ 0, 0, 0 }, end{ 0, 0, 0 };
};

// RayTracingDriver::trace_ray, RayTracingDriver.hpp:172-242 (reflect :405-408,
// normalize_dir :398-401).  rec(k, obj, point, u, v) receives every hit.
template <class Rec>
static TraceOut trace_ray(const Scene& S, const V3& origin, const V3& direction, int max_bounces,
                          Counters* c, Rec&& rec) {
    TraceOut out;
    out.end = origin;
    const double len2 = direction.x * direction.x + direction.y * direction.y + direction.z * direction.z;
    if (len2 < 1e-300) { out.status = BBRT_RAY_BAD_DIR; return out; }
    V3 o = origin;
    const double len = std::sqrt(direction.x * direction.x + direction.y * direction.y + direction.z * direction.z);
    V3 d{ direction.x / len, direction.y / len, direction.z / len };
    for (int b = 0; b < max_bounces; ++b) {
        Result h = S.bvh_intersect(o, d, c);
        if (h.err) {
            out.status = h.err; out.err_obj = h.h.obj;
            out.err_val[0] = h.err_val[0]; out.err_val[1] = h.err_val[1];
            out.dir = d;
            return out;
        }
        if (!h.hit) {
            out.status = BBRT_RAY_ESCAPED;
            out.end = { o.x + d.x * S.diag, o.y + d.y * S.diag, o.z + d.z * S.diag };
            out.dir = d;
            return out;
        }
        if (dot(d, h.h.n) > S.cfg.backface_tol) { out.status = BBRT_RAY_WENT_INSIDE; out.dir = d; return out; }
        rec(out.bounces, h.h.obj, h.h.p, h.h.u, h.h.v);
        out.bounces++;
        out.end = h.h.p;
        const double dn = d.x * h.h.n.x + d.y * h.h.n.y + d.z * h.h.n.z;
        d = { d.x - 2.0 * dn * h.h.n.x, d.y - 2.0 * dn * h.h.n.y, d.z - 2.0 * dn * h.h.n.z };
        const double eps = S.eps_for(h.h.obj);
        o = { h.h.p.x + d.x * eps, h.h.p.y + d.y * eps, h.h.p.z + d.z * eps };
    }
    out.status = BBRT_RAY_MAX_BOUNCES;
    out.dir = d;
    return out;
}

static Config to_cfg(const bbrt_config* c) {
    Config k;
    if (c) {
        k.coarse_n = c->coarse_grid_n; k.newton_max_iters = c->newton_max_iters; k.newton_tol = c->newton_tol;
        k.leaf_threshold = c->leaf_threshold; k.eps_factor = c->self_intersect_eps_factor;
        k.sag_factor = c->sagitta_clearance_factor; k.backface_tol = c->backface_tol;
    }
    return k;
}

}  // namespace oracle

using namespace oracle;

extern "C" {

// Builds a scene exactly as RayTracingDriver's constructor does:
// per-object set-up, BVH over the objects in the given order, scene scale
// (compute_scene_scale, RayTracingDriver.hpp:386-396).
void* oracle_scene_create(const bbrt_object_desc* descs, int n, const bbrt_config* cfg) {
    if (n <= 0) return nullptr;
    auto* S = new Scene();
    S->cfg = to_cfg(cfg);
    S->objs.resize(n);
    for (int k = 0; k < n; ++k) {
        if (descs[k].kind == BBRT_OBJ_PATCH) setup_patch(S->objs[k], *descs[k].patch, S->cfg);
        else setup_triangle(S->objs[k], descs[k].tri);
    }
    std::vector<int> ids(n);
    for (int k = 0; k < n; ++k) ids[k] = k;
    S->nodes.reserve(2 * n);
    S->build(std::move(ids));
    Box b = S->objs.front().box;
    for (const auto& o : S->objs) { b = Scene::unite(b, o.box); S->max_sag = std::max(S->max_sag, o.max_sag); }
    const double dx = b.mx.x - b.mn.x, dy = b.mx.y - b.mn.y, dz = b.mx.z - b.mn.z;
    S->diag = std::sqrt(dx * dx + dy * dy + dz * dz);
    return S;
}

void oracle_scene_destroy(void* s) { delete static_cast<Scene*>(s); }

int oracle_scene_info(void* s, int* n_nodes, double* diag, double* max_sag) {
    auto* S = static_cast<Scene*>(s);
    *n_nodes = static_cast<int>(S->nodes.size());
    *diag = S->diag;
    *max_sag = S->max_sag;
    return 0;
}

int oracle_object_setup(void* s, int idx, double* box6, double* centroid3, double* max_sag, int* n,
                        double* coarse_xyz, double* sagitta, double* normals) {
    auto* S = static_cast<Scene*>(s);
    const Object& P = S->objs[idx];
    box6[0] = P.box.mn.x; box6[1] = P.box.mn.y; box6[2] = P.box.mn.z;
    box6[3] = P.box.mx.x; box6[4] = P.box.mx.y; box6[5] = P.box.mx.z;
    centroid3[0] = P.centroid.x; centroid3[1] = P.centroid.y; centroid3[2] = P.centroid.z;
    *max_sag = P.max_sag;
    *n = P.n;
    if (P.kind != BBRT_OBJ_PATCH) return 0;
    if (coarse_xyz)
        for (int k = 0; k < P.n * P.n; ++k) {
            coarse_xyz[3 * k] = P.cx[k]; coarse_xyz[3 * k + 1] = P.cy[k]; coarse_xyz[3 * k + 2] = P.cz[k];
        }
    if (sagitta) for (size_t k = 0; k < P.sag.size(); ++k) sagitta[k] = P.sag[k];
    if (normals)
        for (size_t k = 0; k < P.cn.size(); ++k) {
            normals[3 * k] = P.cn[k].x; normals[3 * k + 1] = P.cn[k].y; normals[3 * k + 2] = P.cn[k].z;
        }
    return 0;
}

// BVH nodes as [box6, right, start, count, axis] for layout checks.
int oracle_bvh_nodes(void* s, double* boxes, int* links, int* leaf_objs) {
    auto* S = static_cast<Scene*>(s);
    for (size_t k = 0; k < S->nodes.size(); ++k) {
        const Node& nd = S->nodes[k];
        const double b[6] = { nd.box.mn.x, nd.box.mn.y, nd.box.mn.z, nd.box.mx.x, nd.box.mx.y, nd.box.mx.z };
        std::memcpy(boxes + 6 * k, b, sizeof b);
        links[4 * k] = nd.right; links[4 * k + 1] = nd.start; links[4 * k + 2] = nd.count; links[4 * k + 3] = nd.axis;
    }
    for (size_t k = 0; k < S->leaf_objs.size(); ++k) leaf_objs[k] = S->leaf_objs[k];
    return 0;
}

// One query per ray (no bounce): mode = BBRT_QUERY_BVH / BRUTE / OBJECT.
int oracle_intersect(void* s, long long n, const double* o, const double* d, int mode, int object,
                     bbrt_hit* out) {
    auto* S = static_cast<Scene*>(s);
    for (long long i = 0; i < n; ++i) {
        const V3 oo{ o[3 * i], o[3 * i + 1], o[3 * i + 2] }, dd{ d[3 * i], d[3 * i + 1], d[3 * i + 2] };
        Result r;
        if (mode == BBRT_QUERY_BVH) r = S->bvh_intersect(oo, dd, nullptr);
        else if (mode == BBRT_QUERY_BRUTE) r = S->brute_intersect(oo, dd);
        else { r = object_intersect(S->objs[object], oo, dd, S->cfg, nullptr); if (r.hit || r.err) r.h.obj = object; }
        bbrt_hit& h = out[i];
        std::memset(&h, 0, sizeof h);
        h.object = -1; h.err_object = -1;
        if (r.err) {
            h.status = r.err; h.err_object = r.h.obj; h.err_value[0] = r.err_val[0]; h.err_value[1] = r.err_val[1];
        } else if (r.hit) {
            h.t = r.h.t;
            h.point[0] = r.h.p.x; h.point[1] = r.h.p.y; h.point[2] = r.h.p.z;
            h.normal[0] = r.h.n.x; h.normal[1] = r.h.n.y; h.normal[2] = r.h.n.z;
            h.uv[0] = r.h.u; h.uv[1] = r.h.v;
            h.object = r.h.obj;
        }
    }
    return 0;
}

// trace_ray over n rays (OpenMP, schedule(dynamic)); outputs as bbrt_trace_out.
int oracle_trace(void* s, long long n, const double* o, const double* d, int max_bounces, int nthreads,
                 const bbrt_trace_out* out, bbrt_trace_stats* stats, double* seconds) {
    auto* S = static_cast<Scene*>(s);
    if (nthreads > 0) omp_set_num_threads(nthreads);
    const int K = out ? out->record_bounces : 0;
    long long bounces = 0, queries = 0, pt = 0, tt = 0, ni = 0, nt = 0;
    long long hist[BBRT_RAY_STATUS_COUNT] = { 0 };
    const double t0 = omp_get_wtime();
    #pragma omp parallel
    {
        long long lb = 0, lq = 0;
        long long lh[BBRT_RAY_STATUS_COUNT] = { 0 };
        Counters c;
        #pragma omp for schedule(dynamic, 64)
        for (long long i = 0; i < n; ++i) {
            const V3 oo{ o[3 * i], o[3 * i + 1], o[3 * i + 2] }, dd{ d[3 * i], d[3 * i + 1], d[3 * i + 2] };
            auto rec = [&](int k, int obj, const V3& p, double u, double v) {
                if (k >= K) return;
                if (out->hit_object) out->hit_object[i * K + k] = obj;
                if (out->hit_point) {
                    out->hit_point[(i * K + k) * 3] = p.x; out->hit_point[(i * K + k) * 3 + 1] = p.y;
                    out->hit_point[(i * K + k) * 3 + 2] = p.z;
                }
                if (out->hit_uv) { out->hit_uv[(i * K + k) * 2] = u; out->hit_uv[(i * K + k) * 2 + 1] = v; }
            };
            if (out && K > 0) {
                for (int k = 0; k < K; ++k) {
                    if (out->hit_object) out->hit_object[i * K + k] = -1;
                    if (out->hit_point) for (int q = 0; q < 3; ++q) out->hit_point[(i * K + k) * 3 + q] = 0.0;
                    if (out->hit_uv) for (int q = 0; q < 2; ++q) out->hit_uv[(i * K + k) * 2 + q] = 0.0;
                }
            }
            const TraceOut r = trace_ray(*S, oo, dd, max_bounces, &c, rec);
            lb += r.bounces;
            // every recorded bounce was one query; escapes, Newton failures and
            // back-face hits add the query that ended the ray
            lq += r.bounces + ((r.status == BBRT_RAY_BAD_DIR || r.status == BBRT_RAY_MAX_BOUNCES) ? 0 : 1);
            lh[r.status]++;
            if (out) {
                if (out->status) out->status[i] = r.status;
                if (out->bounce_count) out->bounce_count[i] = r.bounces;
                if (out->exit_dir) { out->exit_dir[3 * i] = r.dir.x; out->exit_dir[3 * i + 1] = r.dir.y; out->exit_dir[3 * i + 2] = r.dir.z; }
                if (out->end_point) { out->end_point[3 * i] = r.end.x; out->end_point[3 * i + 1] = r.end.y; out->end_point[3 * i + 2] = r.end.z; }
                if (out->err_object) out->err_object[i] = r.err_obj;
                if (out->err_value) { out->err_value[2 * i] = r.err_val[0]; out->err_value[2 * i + 1] = r.err_val[1]; }
            }
        }
        #pragma omp critical
        {
            bounces += lb; queries += lq; pt += c.patch_tests; tt += c.tri_tests; ni += c.newton_iters; nt += c.node_tests;
            for (int k = 0; k < BBRT_RAY_STATUS_COUNT; ++k) hist[k] += lh[k];
        }
    }
    const double secs = omp_get_wtime() - t0;
    if (seconds) *seconds = secs;
    if (stats) {
        std::memset(stats, 0, sizeof *stats);
        stats->rays = n; stats->bounces = bounces; stats->queries = queries;
        stats->patch_tests = pt; stats->tri_tests = tt; stats->newton_iters = ni; stats->node_tests = nt;
        for (int k = 0; k < BBRT_RAY_STATUS_COUNT; ++k) stats->status_hist[k] = hist[k];
        stats->total_ms = secs * 1e3;
    }
    return 0;
}

// PlaneSourceDriver::run's counting (PlaneSourceDriver.hpp:96-107) over
// given sources and one direction.
int oracle_plane_counts(void* s, long long n, const double* src, const double* dir, int max_bounces,
                        int count_direct_hit, long long* counts) {
    auto* S = static_cast<Scene*>(s);
    std::vector<long long> c(S->objs.size(), 0);
    #pragma omp parallel for schedule(dynamic, 64)
    for (long long i = 0; i < n; ++i) {
        const V3 oo{ src[3 * i], src[3 * i + 1], src[3 * i + 2] }, dd{ dir[0], dir[1], dir[2] };
        const size_t first = count_direct_hit ? 0 : 1;
        trace_ray(*S, oo, dd, max_bounces, nullptr, [&](int k, int obj, const V3&, double, double) {
            if (static_cast<size_t>(k) >= first) {
                #pragma omp atomic
                c[obj]++;
            }
        });
    }
    for (size_t k = 0; k < c.size(); ++k) counts[k] = c[k];
    return 0;
}

// SurfacePatch::sample_grid(n), SurfacePatch.hpp:199-242: xyz, unit normal, dX/du.
int oracle_sample_grid(const bbrt_patch_desc* d, int n, double* xyz, double* nrm, double* du) {
    Object P;
    Config cfg; cfg.coarse_n = 2;
    setup_patch(P, *d, cfg);
    std::vector<double> g(n);
    for (int i = 0; i < n; ++i) g[i] = (n == 1) ? 0.0 : -1.0 + 2.0 * static_cast<double>(i) / (n - 1);
    const size_t nn = static_cast<size_t>(n) * n;
    std::vector<double> F[9];
    const int fields[9] = { 0, 1, 2, 9, 10, 11, 3, 4, 5 };
    for (int k = 0; k < 9; ++k) {
        F[k].resize(nn);
        lagrange_2d(P.un, P.vn, P.uw, P.vw, P.f[fields[k]].data(), g, g, F[k].data());
    }
    for (size_t k = 0; k < nn; ++k) {
        const V3 nv = normalize({ F[3][k], F[4][k], F[5][k] });
        xyz[3 * k] = F[0][k]; xyz[3 * k + 1] = F[1][k]; xyz[3 * k + 2] = F[2][k];
        nrm[3 * k] = nv.x; nrm[3 * k + 1] = nv.y; nrm[3 * k + 2] = nv.z;
        du[3 * k] = F[6][k]; du[3 * k + 1] = F[7][k]; du[3 * k + 2] = F[8][k];
    }
    return 0;
}

// BounceMapDriver::run, BounceMapDriver.hpp:103-259, for sample patches given
// as descriptors (the reference loads them by file range).  eps per sample
// patch is the scene's self_intersect_epsilon of that patch's own padding.
}  // extern "C"

// Every launch ray of one sample patch, in BounceMapDriver::run's order
// (BounceMapDriver.hpp:119-237): fn(k, ti, pj, origin, dir) per grid point k
// and direction (ti, pj).
template <class Fn>
static void bounce_rays_of_patch(const Scene& S, const bbrt_patch_desc& sample, int grid_n, int theta_n, int phi_n,
                                 double cone_deg, Fn&& fn) {
    const double kTwoPi = 6.283185307179586476925286766559;
    const double half = cone_deg / 2.0;
    const double cos_max = std::cos(half * kTwoPi / 360.0);
    const long long per = static_cast<long long>(grid_n) * grid_n;
    Object P;
    setup_patch(P, sample, S.cfg);
    const double eps = std::max(S.cfg.eps_factor * S.diag, S.cfg.sag_factor * P.max_sag);
    std::vector<double> xyz(3 * per), nrm(3 * per), du(3 * per);
    oracle_sample_grid(&sample, grid_n, xyz.data(), nrm.data(), du.data());
    for (long long k = 0; k < per; ++k) {
        const V3 pt{ xyz[3 * k], xyz[3 * k + 1], xyz[3 * k + 2] };
        const V3 nv = normalize({ nrm[3 * k], nrm[3 * k + 1], nrm[3 * k + 2] });
        const V3 dv{ du[3 * k], du[3 * k + 1], du[3 * k + 2] };
        // build_tangent_frame, BounceMapDriver.hpp:499-519
        V3 t1, t2;
        const double du2 = dot(dv, dv), dn = dot(dv, nv);
        const V3 dp{ dv.x - dn * nv.x, dv.y - dn * nv.y, dv.z - dn * nv.z };
        const double dp2 = dot(dp, dp);
        const double rel = 1e-6;
        if (dp2 > rel * rel * du2) t1 = normalize(dp);
        else {
            const V3 a = (std::fabs(nv.x) <= std::fabs(nv.y) && std::fabs(nv.x) <= std::fabs(nv.z)) ? V3{ 1, 0, 0 }
                       : (std::fabs(nv.y) <= std::fabs(nv.z) ? V3{ 0, 1, 0 } : V3{ 0, 0, 1 });
            t1 = normalize(cross(nv, a));
        }
        t2 = cross(nv, t1);
        const V3 org{ pt.x + nv.x * eps, pt.y + nv.y * eps, pt.z + nv.z * eps };
        for (int ti = 0; ti < theta_n; ++ti) {
            const double mu = cos_max + (static_cast<double>(ti) + 0.5) / static_cast<double>(theta_n) * (1.0 - cos_max);
            const double st = std::sqrt(std::max(0.0, 1.0 - mu * mu));
            for (int pj = 0; pj < phi_n; ++pj) {
                const double phi = (static_cast<double>(pj) + 0.5) * kTwoPi / static_cast<double>(phi_n);
                const double cp = std::cos(phi), sp = std::sin(phi);
                const V3 dir{ t1.x * st * cp + t2.x * st * sp + nv.x * mu,
                              t1.y * st * cp + t2.y * st * sp + nv.y * mu,
                              t1.z * st * cp + t2.z * st * sp + nv.z * mu };
                fn(k, ti, pj, org, dir);
            }
        }
    }
}

extern "C" {

int oracle_bounce_map(void* s, const bbrt_patch_desc* samples, int n_sample, int grid_n, int theta_n,
                      int phi_n, double cone_deg, int max_bounces, int* max_b, int* errors, int* best_dir) {
    auto* S = static_cast<Scene*>(s);
    const long long per = static_cast<long long>(grid_n) * grid_n;
    #pragma omp parallel for schedule(dynamic)
    for (int p = 0; p < n_sample; ++p) {
        int best = 0, nerr = 0, bdir = -1;
        bounce_rays_of_patch(*S, samples[p], grid_n, theta_n, phi_n, cone_deg,
                             [&](long long k, int ti, int pj, const V3& org, const V3& dir) {
            if (ti == 0 && pj == 0) { best = 0; nerr = 0; bdir = -1; }
            const TraceOut r = trace_ray(*S, org, dir, max_bounces, nullptr,
                                         [](int, int, const V3&, double, double) {});
            if (r.status != BBRT_RAY_ESCAPED && r.status != BBRT_RAY_MAX_BOUNCES) ++nerr;
            else {
                if (bdir < 0 || r.bounces > best) bdir = ti * phi_n + pj;   // first maximum, :232-235
                best = std::max(best, r.bounces);
            }
            if (ti == theta_n - 1 && pj == phi_n - 1) {
                max_b[p * per + k] = best;
                errors[p * per + k] = nerr;
                if (best_dir) best_dir[p * per + k] = bdir;
            }
        });
    }
    return 0;
}

// The launch rays of oracle_bounce_map, all of them, ray r at
// ((p * grid_n^2 + k) * theta_n + ti) * phi_n + pj.
int oracle_bounce_map_rays(void* s, const bbrt_patch_desc* samples, int n_sample, int grid_n, int theta_n,
                           int phi_n, double cone_deg, double* origins, double* dirs) {
    auto* S = static_cast<Scene*>(s);
    const long long per = static_cast<long long>(grid_n) * grid_n;
    for (int p = 0; p < n_sample; ++p)
        bounce_rays_of_patch(*S, samples[p], grid_n, theta_n, phi_n, cone_deg,
                             [&](long long k, int ti, int pj, const V3& org, const V3& dir) {
            const long long r = ((p * per + k) * theta_n + ti) * phi_n + pj;
            origins[3 * r] = org.x; origins[3 * r + 1] = org.y; origins[3 * r + 2] = org.z;
            dirs[3 * r] = dir.x; dirs[3 * r + 1] = dir.y; dirs[3 * r + 2] = dir.z;
        });
    return 0;
}

}  // extern "C"
