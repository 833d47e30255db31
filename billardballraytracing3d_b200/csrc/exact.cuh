// Exact FP64 device primitives of the trace path.
//
// Each function reproduces one reference routine operation by operation:
// the same association of every sum and product, the same comparisons, and
// std::min/std::max's NaN behaviour written out as ternaries.  The
// translation unit that includes this header is compiled with -fmad=false,
// so no product is fused into an add: with IEEE division and sqrt the
// results are bit-identical to the reference's x86-64 (SSE2) build.
//
// Reference (manuelarturosantana/BillardBallRayTracing3D):
//   vec helpers, moller_trumbore     include/Utils/MollerTrumbore.hpp:13-64
//   ray_box                          include/BVH.hpp:14-37
//   lagrange_basis_1d                include/ScatObjects/SurfacePatch.hpp:518-538
//   eval_scalar_field                SurfacePatch.hpp:542-555
//   solve3x3                         SurfacePatch.hpp:559-579
//   newton_refine                    SurfacePatch.hpp:593-660
//   SurfacePatch::intersect stage 1  SurfacePatch.hpp:253-303, triangle_uv_centroid :499-510
#pragma once

#include <cuda_runtime.h>
#include <math_constants.h>

#include "dscene.h"

namespace bbrt {

struct V3 { double x, y, z; };

__device__ __forceinline__ V3 v3(double x, double y, double z) { V3 r; r.x = x; r.y = y; r.z = z; return r; }
__device__ __forceinline__ V3 vsub(const V3& a, const V3& b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ V3 vcross(const V3& a, const V3& b) {
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double vdot(const V3& a, const V3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 vnormalize(const V3& v) {
    const double len = sqrt(vdot(v, v));
    return v3(v.x / len, v.y / len, v.z / len);
}
// std::max(a, b) / std::min(a, b)
__device__ __forceinline__ double smax(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double smin(double a, double b) { return (b < a) ? b : a; }

__device__ __forceinline__ V3 load3(const double* p) { return v3(p[0], p[1], p[2]); }

// Moller-Trumbore with eps = 1e-9; returns the hit t.  Before the one FP64
// division it rejects, from the signs and magnitudes of a = tvec.pvec and
// det alone, every triangle whose u = fl(a * fl(1/det)) is certain to fall
// outside [0, 1]: opposite signs with |a| > 1e-290 |det| give u < 0 (no
// underflow to -0 possible), equal signs with |a| > |det| (1 + 1e-14) give
// u > 1 (the rounding of 1/det and of the product is at most 2^-52
// relative).  NaN or infinite operands fail both tests and take the exact
// path, so the outcome is always the reference's.
__device__ __forceinline__ bool mt_exact(const V3& o, const V3& d, const V3& v0, const V3& v1, const V3& v2,
                                         double& t_out) {
    const V3 e1 = vsub(v1, v0);
    const V3 e2 = vsub(v2, v0);
    const V3 pvec = vcross(d, e2);
    const double det = vdot(e1, pvec);
    if (fabs(det) < 1e-9) return false;
    const V3 tvec = vsub(o, v0);
    const double a = vdot(tvec, pvec);
    const double fa = fabs(a), fd = fabs(det);
    if ((a < 0.0) != (det < 0.0)) {
        if (fa > fd * 1e-290) return false;
    } else if (fa > fd * (1.0 + 1e-14)) {
        return false;
    }
    const double inv_det = 1.0 / det;
    const double u = a * inv_det;
    if (u < 0.0 || u > 1.0) return false;
    const V3 qvec = vcross(tvec, e1);
    const double v = vdot(d, qvec) * inv_det;
    if (v < 0.0 || u + v > 1.0) return false;
    const double t = vdot(e2, qvec) * inv_det;
    if (t < 1e-9) return false;
    t_out = t;
    return true;
}

// Plain Moller-Trumbore returning u, v too (Triangle objects).
__device__ __forceinline__ bool mt_full(const V3& o, const V3& d, const V3& v0, const V3& v1, const V3& v2,
                                        double& t_out, double& u_out, double& v_out) {
    const V3 e1 = vsub(v1, v0);
    const V3 e2 = vsub(v2, v0);
    const V3 pvec = vcross(d, e2);
    const double det = vdot(e1, pvec);
    if (fabs(det) < 1e-9) return false;
    const double inv_det = 1.0 / det;
    const V3 tvec = vsub(o, v0);
    const double u = vdot(tvec, pvec) * inv_det;
    if (u < 0.0 || u > 1.0) return false;
    const V3 qvec = vcross(tvec, e1);
    const double v = vdot(d, qvec) * inv_det;
    if (v < 0.0 || u + v > 1.0) return false;
    const double t = vdot(e2, qvec) * inv_det;
    if (t < 1e-9) return false;
    t_out = t; u_out = u; v_out = v;
    return true;
}

// Slab test of BVH.hpp:14-37 (tmin_out is never used by the caller there).
// Node boxes are 6 doubles on a 48-byte stride from a 16-byte aligned array
// (global memory checked at upload, shared copies declared aligned): read as
// three 16-byte loads.
__device__ __forceinline__ bool ray_box_exact(const V3& o, const double inv[3], const double* box, double best_t) {
    double tmin = -CUDART_INF, tmax = CUDART_INF;
    const double oo[3] = { o.x, o.y, o.z };
    const double2 b01 = *reinterpret_cast<const double2*>(box);
    const double2 b23 = *reinterpret_cast<const double2*>(box + 2);
    const double2 b45 = *reinterpret_cast<const double2*>(box + 4);
    const double bx[6] = { b01.x, b01.y, b23.x, b23.y, b45.x, b45.y };
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        double t1 = (bx[a] - oo[a]) * inv[a];
        double t2 = (bx[3 + a] - oo[a]) * inv[a];
        if (inv[a] < 0.0) { const double s = t1; t1 = t2; t2 = s; }
        tmin = smax(tmin, t1);
        tmax = smin(tmax, t2);
        if (tmax < tmin) return false;
    }
    if (tmin > best_t) return false;
    return tmax >= smax(tmin, 0.0);
}

// Largest node count per axis the device Newton solve handles.
constexpr int kDevMaxNodes = 16;

// Second-form barycentric basis at x over N nodes (one-hot within 1e-12 of a node).
__device__ __forceinline__ void basis_1d(const double* nodes, const double* w, int N, double x, double* b) {
    for (int i = 0; i < N; ++i) b[i] = 0.0;
    for (int i = 0; i < N; ++i)
        if (fabs(x - nodes[i]) < 1.0e-12) { b[i] = 1.0; return; }
    double denom = 0.0;
    for (int i = 0; i < N; ++i) {
        const double li = w[i] / (x - nodes[i]);
        b[i] = li;
        denom += li;
    }
    for (int i = 0; i < N; ++i) b[i] /= denom;
}

// Evaluates NF node-major fields (stride 12, starting at field `first`) at
// basis (bu, bv) in the reference's order: per row i a left-to-right sum
// over j, then the rows summed in i order, skipping rows whose bu_i is 0.
template <int NF>
__device__ __forceinline__ void eval_fields(const double* __restrict__ F, int I, int J, const double* bu,
                                            const double* bv, int first, double* out) {
#pragma unroll
    for (int f = 0; f < NF; ++f) out[f] = 0.0;
    for (int i = 0; i < I; ++i) {
        const double li = bu[i];
        if (li == 0.0) continue;
        double rs[NF];
#pragma unroll
        for (int f = 0; f < NF; ++f) rs[f] = 0.0;
        const double* row = F + static_cast<long long>(i) * J * 12 + first;
        for (int j = 0; j < J; ++j) {
            const double lj = bv[j];
#pragma unroll
            for (int f = 0; f < NF; ++f) rs[f] += lj * row[j * 12 + f];
        }
#pragma unroll
        for (int f = 0; f < NF; ++f) out[f] += li * rs[f];
    }
}

// eval_fields<9> from field 0, each node's fields 0-7 read as four 16-byte
// loads and field 8 alone (a node's 12 doubles start on a 16-byte boundary,
// checked at upload); the same values in the same order.
__device__ __forceinline__ void eval_fields9(const double* __restrict__ F, int I, int J, const double* bu,
                                             const double* bv, double* out) {
#pragma unroll
    for (int f = 0; f < 9; ++f) out[f] = 0.0;
    for (int i = 0; i < I; ++i) {
        const double li = bu[i];
        if (li == 0.0) continue;
        double rs[9];
#pragma unroll
        for (int f = 0; f < 9; ++f) rs[f] = 0.0;
        const double* row = F + static_cast<long long>(i) * J * 12;
        for (int j = 0; j < J; ++j) {
            const double lj = bv[j];
            const double2 f01 = *reinterpret_cast<const double2*>(row + j * 12);
            const double2 f23 = *reinterpret_cast<const double2*>(row + j * 12 + 2);
            const double2 f45 = *reinterpret_cast<const double2*>(row + j * 12 + 4);
            const double2 f67 = *reinterpret_cast<const double2*>(row + j * 12 + 6);
            const double f8 = row[j * 12 + 8];
            rs[0] += lj * f01.x;
            rs[1] += lj * f01.y;
            rs[2] += lj * f23.x;
            rs[3] += lj * f23.y;
            rs[4] += lj * f45.x;
            rs[5] += lj * f45.y;
            rs[6] += lj * f67.x;
            rs[7] += lj * f67.y;
            rs[8] += lj * f8;
        }
#pragma unroll
        for (int f = 0; f < 9; ++f) out[f] += li * rs[f];
    }
}

// basis_1d for a compile-time node count N, the values in registers: the
// same operations in the same order (first node within 1e-12 wins).
template <int N>
__device__ __forceinline__ void basis_1d_n(const double* nodes, const double* w, double x, double (&b)[N]) {
    int hit = -1;
#pragma unroll
    for (int i = 0; i < N; ++i)
        if (hit < 0 && fabs(x - nodes[i]) < 1.0e-12) hit = i;
    if (hit >= 0) {
#pragma unroll
        for (int i = 0; i < N; ++i) b[i] = (i == hit) ? 1.0 : 0.0;
        return;
    }
    double denom = 0.0;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        const double li = w[i] / (x - nodes[i]);
        b[i] = li;
        denom += li;
    }
#pragma unroll
    for (int i = 0; i < N; ++i) b[i] /= denom;
}

// eval_fields9 for rows of JN nodes: the row's basis values in registers and
// its loop unrolled, so a row's loads issue together instead of one node's
// at a time; the same sums in the same order.
template <int JN>
__device__ __forceinline__ void eval_fields9_n(const double* __restrict__ F, int I, const double* bu,
                                               const double (&bv)[JN], double* out) {
#pragma unroll
    for (int f = 0; f < 9; ++f) out[f] = 0.0;
    for (int i = 0; i < I; ++i) {
        const double li = bu[i];
        if (li == 0.0) continue;
        double rs[9];
#pragma unroll
        for (int f = 0; f < 9; ++f) rs[f] = 0.0;
        const double* row = F + static_cast<long long>(i) * JN * 12;
#pragma unroll
        for (int j = 0; j < JN; ++j) {
            const double lj = bv[j];
            const double2 f01 = *reinterpret_cast<const double2*>(row + j * 12);
            const double2 f23 = *reinterpret_cast<const double2*>(row + j * 12 + 2);
            const double2 f45 = *reinterpret_cast<const double2*>(row + j * 12 + 4);
            const double2 f67 = *reinterpret_cast<const double2*>(row + j * 12 + 6);
            const double f8 = row[j * 12 + 8];
            rs[0] += lj * f01.x;
            rs[1] += lj * f01.y;
            rs[2] += lj * f23.x;
            rs[3] += lj * f23.y;
            rs[4] += lj * f45.x;
            rs[5] += lj * f45.y;
            rs[6] += lj * f67.x;
            rs[7] += lj * f67.y;
            rs[8] += lj * f8;
        }
#pragma unroll
        for (int f = 0; f < 9; ++f) out[f] += li * rs[f];
    }
}

// Per-ray outcome of one object intersect: hit, miss, or a Newton failure.
struct QHit {
    double t;
    V3 p, n;
    double u, v;
    int obj;
    int err;          // 0 or BBRT_RAY_NEWTON_*
    double ev0, ev1;  // values the reference's error message quotes
};

// Newton on F(u,v,t) = X(u,v) - (o + t d) from (u0, v0, t0).  Returns
// 1 hit, or 0 with h.err set (singular / no convergence / out of domain).
// JN > 0: the patch has JN nodes per row (the v basis in registers, each
// row's loads together); JN = 0: any count.  The same arithmetic either way.
template <int JN>
__device__ __forceinline__ int newton_exact_j(const DScene& S, int pidx, const V3 o, const V3 d, double u, double v,
                                             double t, QHit& h, long long& iters) {
    const int I = S.p_dims[2 * pidx], J = S.p_dims[2 * pidx + 1];
    const double* un = S.p_nodes + S.p_node_off[pidx];
    const double* vn = un + I;
    const double* uw = vn + J;
    const double* vw = uw + I;
    const double* F = S.p_fields + S.p_field_off[pidx];
    double bu[kDevMaxNodes], bv[kDevMaxNodes];
    double step = CUDART_INF;
    for (int it = 0; it < S.newton_max_iters; ++it) {
        ++iters;
        basis_1d(un, uw, I, u, bu);
        double e[9];
        if constexpr (JN > 0) {
            double bvr[JN > 0 ? JN : 1];
            basis_1d_n<JN>(vn, vw, v, bvr);
            eval_fields9_n<JN>(F, I, bu, bvr, e);
        } else {
            basis_1d(vn, vw, J, v, bv);
            eval_fields9(F, I, J, bu, bv, e);
        }
        const V3 R = v3(o.x + t * d.x, o.y + t * d.y, o.z + t * d.z);
        const double Fx = e[0] - R.x, Fy = e[1] - R.y, Fz = e[2] - R.z;
        const double a11 = e[3], a12 = e[6], a13 = -d.x;
        const double a21 = e[4], a22 = e[7], a23 = -d.y;
        const double a31 = e[5], a32 = e[8], a33 = -d.z;
        const double det = a11 * (a22 * a33 - a23 * a32) - a12 * (a21 * a33 - a23 * a31) + a13 * (a21 * a32 - a22 * a31);
        if (fabs(det) < 1e-14) { h.err = 2; return 0; }   // BBRT_RAY_NEWTON_SINGULAR
        const double bx = Fx, by = Fy, bz = Fz;
        const double d0 = bx * (a22 * a33 - a23 * a32) - a12 * (by * a33 - a23 * bz) + a13 * (by * a32 - a22 * bz);
        const double d1 = a11 * (by * a33 - a23 * bz) - bx * (a21 * a33 - a23 * a31) + a13 * (a21 * bz - by * a31);
        const double d2 = a11 * (a22 * bz - by * a32) - a12 * (a21 * bz - by * a31) + bx * (a21 * a32 - a22 * a31);
        const double x0 = d0 / det, x1 = d1 / det, x2 = d2 / det;
        u -= x0;
        v -= x1;
        t -= x2;
        step = sqrt(x0 * x0 + x1 * x1 + x2 * x2);
        if (step < S.newton_tol) break;
    }
    if (step >= S.newton_tol) { h.err = 3; h.ev0 = step; return 0; }     // BBRT_RAY_NEWTON_NOCONV
    if (u < -1.0 - 1e-6 || u > 1.0 + 1e-6 || v < -1.0 - 1e-6 || v > 1.0 + 1e-6) {
        h.err = 4; h.ev0 = u; h.ev1 = v; return 0;                       // BBRT_RAY_NEWTON_DOMAIN
    }
    basis_1d(un, uw, I, u, bu);
    basis_1d(vn, vw, J, v, bv);
    double e[3], nn[3];
    eval_fields<3>(F, I, J, bu, bv, 0, e);
    eval_fields<3>(F, I, J, bu, bv, 9, nn);
    h.t = t;
    h.p = v3(e[0], e[1], e[2]);
    h.n = vnormalize(v3(nn[0], nn[1], nn[2]));
    h.u = u;
    h.v = v;
    return 1;
}

// Newton in the reference's arithmetic, with the fixed-row forms for the
// measured node counts (5 and 7 per row).
__device__ __forceinline__ int newton_exact(const DScene& S, int pidx, const V3 o, const V3 d, double u, double v,
                                         double t, QHit& h, long long& iters) {
    const int J = S.p_dims[2 * pidx + 1];
    if (J == 7) return newton_exact_j<7>(S, pidx, o, d, u, v, t, h, iters);
    if (J == 5) return newton_exact_j<5>(S, pidx, o, d, u, v, t, h, iters);
    return newton_exact_j<0>(S, pidx, o, d, u, v, t, h, iters);
}

// ---- FP32 Newton phase (precision split) -----------------------------------

constexpr int kFp32Iters = 8;          // FP32 iterations before giving up on the phase
constexpr float kFp32Residual = 1e-5f; // |F| at which the FP64 finish takes over

__device__ __forceinline__ void basis_1d_f(const float* nodes, const float* w, int N, float x, float* b) {
    for (int i = 0; i < N; ++i) b[i] = 0.0f;
    for (int i = 0; i < N; ++i)
        if (x == nodes[i]) { b[i] = 1.0f; return; }
    float denom = 0.0f;
    for (int i = 0; i < N; ++i) {
        const float li = w[i] / (x - nodes[i]);
        b[i] = li;
        denom += li;
    }
    const float inv = 1.0f / denom;
    for (int i = 0; i < N; ++i) b[i] *= inv;
}

// basis_1d_f for a compile-time node count N, the values in registers: the
// same operations in the same order.
template <int N>
__device__ __forceinline__ void basis_1d_f_n(const float* nodes, const float* w, float x, float (&b)[N]) {
    int hit = -1;
#pragma unroll
    for (int i = 0; i < N; ++i)
        if (hit < 0 && x == nodes[i]) hit = i;
    if (hit >= 0) {
#pragma unroll
        for (int i = 0; i < N; ++i) b[i] = (i == hit) ? 1.0f : 0.0f;
        return;
    }
    float denom = 0.0f;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        const float li = w[i] / (x - nodes[i]);
        b[i] = li;
        denom += li;
    }
    const float inv = 1.0f / denom;
#pragma unroll
    for (int i = 0; i < N; ++i) b[i] *= inv;
}

// Newton on F(u,v,t) in FP32 until |F| < kFp32Residual.  Returns true with
// the FP32 iterate in (u, v, t); false when it is singular, leaves the
// neighbourhood of the patch or does not get there in kFp32Iters steps.
// JN > 0: rows of JN nodes (v basis in registers, a row's loads together).
template <int JN>
__device__ __forceinline__ bool newton_fp32_j(const DScene& S, int pidx, const V3& o, const V3& d, double& u,
                                              double& v, double& t, long long& iters32) {
    const int I = S.p_dims[2 * pidx], J = S.p_dims[2 * pidx + 1];
    const float* un = S.p_nodes32 + S.p_node_off[pidx];
    const float* vn = un + I;
    const float* uw = vn + J;
    const float* vw = uw + I;
    const float* Fd = S.p_fields32 + S.p_field_off[pidx];
    const float ox = static_cast<float>(o.x), oy = static_cast<float>(o.y), oz = static_cast<float>(o.z);
    const float dx = static_cast<float>(d.x), dy = static_cast<float>(d.y), dz = static_cast<float>(d.z);
    float uf = static_cast<float>(u), vf = static_cast<float>(v), tf = static_cast<float>(t);
    float bu[kDevMaxNodes], bv[kDevMaxNodes];
    for (int it = 0; it < kFp32Iters; ++it) {
        ++iters32;
        basis_1d_f(un, uw, I, uf, bu);
        float bvr[JN > 0 ? JN : 1];
        if constexpr (JN > 0) basis_1d_f_n<JN>(vn, vw, vf, bvr);
        else basis_1d_f(vn, vw, J, vf, bv);
        float e[9];
        for (int f = 0; f < 9; ++f) e[f] = 0.0f;
        for (int i = 0; i < I; ++i) {
            const float li = bu[i];
            if (li == 0.0f) continue;
            float rs[9];
            for (int f = 0; f < 9; ++f) rs[f] = 0.0f;
            const float* row = Fd + static_cast<long long>(i) * (JN > 0 ? JN : J) * 12;
#pragma unroll
            for (int j = 0; j < (JN > 0 ? JN : J); ++j) {
                // a node's 12 floats start on a 16-byte boundary (checked at
                // upload): fields 0-7 as two 16-byte loads, field 8 alone
                const float4 fa = *reinterpret_cast<const float4*>(row + j * 12);
                const float4 fb = *reinterpret_cast<const float4*>(row + j * 12 + 4);
                const float f8 = row[j * 12 + 8];
                const float b = JN > 0 ? bvr[JN > 0 ? j : 0] : bv[j];
                rs[0] = fmaf(b, fa.x, rs[0]);
                rs[1] = fmaf(b, fa.y, rs[1]);
                rs[2] = fmaf(b, fa.z, rs[2]);
                rs[3] = fmaf(b, fa.w, rs[3]);
                rs[4] = fmaf(b, fb.x, rs[4]);
                rs[5] = fmaf(b, fb.y, rs[5]);
                rs[6] = fmaf(b, fb.z, rs[6]);
                rs[7] = fmaf(b, fb.w, rs[7]);
                rs[8] = fmaf(b, f8, rs[8]);
            }
            for (int f = 0; f < 9; ++f) e[f] = fmaf(li, rs[f], e[f]);
        }
        const float Fx = e[0] - fmaf(tf, dx, ox), Fy = e[1] - fmaf(tf, dy, oy), Fz = e[2] - fmaf(tf, dz, oz);
        if (fabsf(Fx) < kFp32Residual && fabsf(Fy) < kFp32Residual && fabsf(Fz) < kFp32Residual) {
            u = uf;
            v = vf;
            t = tf;
            return true;
        }
        const float a11 = e[3], a12 = e[6], a13 = -dx, a21 = e[4], a22 = e[7], a23 = -dy, a31 = e[5], a32 = e[8],
                    a33 = -dz;
        const float c1 = a22 * a33 - a23 * a32, c2 = a21 * a33 - a23 * a31, c3 = a21 * a32 - a22 * a31;
        const float det = a11 * c1 - a12 * c2 + a13 * c3;
        if (!(fabsf(det) > 1e-30f)) return false;
        const float id = 1.0f / det;
        const float x0 = (Fx * c1 - a12 * (Fy * a33 - a23 * Fz) + a13 * (Fy * a32 - a22 * Fz)) * id;
        const float x1 = (a11 * (Fy * a33 - a23 * Fz) - Fx * c2 + a13 * (a21 * Fz - Fy * a31)) * id;
        const float x2 = (a11 * (a22 * Fz - Fy * a32) - a12 * (a21 * Fz - Fy * a31) + Fx * c3) * id;
        uf -= x0;
        vf -= x1;
        tf -= x2;
        if (!(fabsf(uf) < 2.0f && fabsf(vf) < 2.0f) || !isfinite(tf)) return false;
    }
    return false;
}

__device__ __forceinline__ bool newton_fp32(const DScene& S, int pidx, const V3& o, const V3& d, double& u,
                                            double& v, double& t, long long& iters32) {
    const int J = S.p_dims[2 * pidx + 1];
    if (J == 7) return newton_fp32_j<7>(S, pidx, o, d, u, v, t, iters32);
    if (J == 5) return newton_fp32_j<5>(S, pidx, o, d, u, v, t, iters32);
    return newton_fp32_j<0>(S, pidx, o, d, u, v, t, iters32);
}

// The precision split: FP32 Newton to |F| < 1e-5 from (u, v, t), then the
// FP64 loop (the reference's step test and iteration cap) from that iterate.
// When the FP32 phase fails, the FP64 loop starts from (u, v, t) itself.
__device__ __forceinline__ int newton_split(const DScene& S, int pidx, const V3 o, const V3 d, double u, double v,
                                            double t, QHit& h, long long& iters, long long& iters32) {
    double uu = u, vv = v, tt = t;
    if (!newton_fp32(S, pidx, o, d, uu, vv, tt, iters32)) {
        uu = u;
        vv = v;
        tt = t;
    }
    return newton_exact(S, pidx, o, d, uu, vv, tt, h, iters);
}

}  // namespace bbrt
