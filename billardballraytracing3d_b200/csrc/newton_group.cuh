// Newton on a patch by a group of 8 lanes, with the reference's arithmetic.
//
// The per-thread solve (exact.cuh newton_exact) spends each iteration
// loading every node's fields of the patch, one dependent load after
// another.  Here lane g of the group owns node row g: it loads only that
// row and forms the row's partial sums over j in the reference's order;
// the rows are then combined, and the barycentric denominators summed, in
// the reference's order on every lane from shuffled values.  Every operation
// and its order is the per-thread solve's, so the result is bit-identical
// (this file is compiled, like the rest of the trace path, without fused
// multiply-adds).  Requires at most 8 nodes per patch axis.
//
// Reference (manuelarturosantana/BillardBallRayTracing3D):
//   lagrange_basis_1d  include/ScatObjects/SurfacePatch.hpp:518-538
//   eval_scalar_field  SurfacePatch.hpp:542-555
//   newton_refine      SurfacePatch.hpp:593-660
#pragma once

#include "exact.cuh"

namespace bbrt {

constexpr int kGroup = 8;

// A lane's place in its 8-lane group.
struct Grp {
    int g;           // lane within the group
    int base;        // first lane of the group within the warp
    unsigned mask;   // the group's lanes
};

__device__ __forceinline__ Grp make_grp() {
    Grp G;
    const int lane = threadIdx.x & 31;
    G.g = lane & (kGroup - 1);
    G.base = lane & ~(kGroup - 1);
    G.mask = 0xFFu << G.base;
    return G;
}

// basis_1d for node G.g (0 beyond N): one-hot at the first node within
// 1e-12, else w_g / (x - node_g) over the ordered sum of those terms.
__device__ __forceinline__ double grp_basis(const double* nodes, const double* w, int N, double x, const Grp& G) {
    const bool mine = G.g < N;
    const bool hit = mine && fabs(x - nodes[G.g]) < 1.0e-12;
    const unsigned hm = (__ballot_sync(G.mask, hit) >> G.base) & 0xFFu;
    if (hm) return (G.g == __ffs(hm) - 1) ? 1.0 : 0.0;
    const double li = mine ? w[G.g] / (x - nodes[G.g]) : 0.0;
    double denom = 0.0;
    for (int i = 0; i < N; ++i) denom += __shfl_sync(G.mask, li, G.base + i);
    return mine ? li / denom : 0.0;
}

// eval_fields<NF, FIRST>: lane g forms row g's sums over j (j in order),
// every lane then adds the rows in i order, skipping rows whose basis is 0.
// JN > 0: rows of JN nodes, the row loop unrolled so that its loads issue
// together (the same sums in the same order); JN = 0: any J.
template <int NF, int FIRST, int JN = 0>
__device__ __forceinline__ void grp_eval(const double* __restrict__ F, int I, int J, double bu, double bv,
                                         const Grp& G, double* out) {
    double rs[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) rs[f] = 0.0;
    const bool row = G.g < I && bu != 0.0;
    const int JJ = JN > 0 ? JN : J;
    const double* rp = F + static_cast<long long>(G.g < I ? G.g : 0) * JJ * 12 + FIRST;
#pragma unroll
    for (int j = 0; j < JJ; ++j) {
        const double lj = __shfl_sync(G.mask, bv, G.base + j);
        if (row) {
            if constexpr (NF == 9 && FIRST == 0) {
                // fields 0-7 as four 16-byte loads (a node's 12 doubles start
                // on a 16-byte boundary, checked at upload), field 8 alone
                const double2 f01 = *reinterpret_cast<const double2*>(rp + j * 12);
                const double2 f23 = *reinterpret_cast<const double2*>(rp + j * 12 + 2);
                const double2 f45 = *reinterpret_cast<const double2*>(rp + j * 12 + 4);
                const double2 f67 = *reinterpret_cast<const double2*>(rp + j * 12 + 6);
                rs[0] += lj * f01.x;
                rs[1] += lj * f01.y;
                rs[2] += lj * f23.x;
                rs[3] += lj * f23.y;
                rs[4] += lj * f45.x;
                rs[5] += lj * f45.y;
                rs[6] += lj * f67.x;
                rs[7] += lj * f67.y;
                rs[8] += lj * rp[j * 12 + 8];
            } else {
#pragma unroll
                for (int f = 0; f < NF; ++f) rs[f] += lj * rp[j * 12 + f];
            }
        }
    }
#pragma unroll
    for (int f = 0; f < NF; ++f) out[f] = 0.0;
    for (int i = 0; i < I; ++i) {
        const double li = __shfl_sync(G.mask, bu, G.base + i);
        if (li == 0.0) continue;   // uniform over the group
#pragma unroll
        for (int f = 0; f < NF; ++f) out[f] += li * __shfl_sync(G.mask, rs[f], G.base + i);
    }
}

// newton_exact by a group: every lane returns the same result.
template <int JN>
__device__ __forceinline__ int grp_newton_exact_j(const DScene& S, int pidx, const V3 o, const V3 d, double u,
                                                  double v, double t, QHit& h, long long& iters, const Grp& G) {
    const int I = S.p_dims[2 * pidx], J = S.p_dims[2 * pidx + 1];
    const double* un = S.p_nodes + S.p_node_off[pidx];
    const double* vn = un + I;
    const double* uw = vn + J;
    const double* vw = uw + I;
    const double* F = S.p_fields + S.p_field_off[pidx];
    double step = CUDART_INF;
    for (int it = 0; it < S.newton_max_iters; ++it) {
        ++iters;
        const double bu = grp_basis(un, uw, I, u, G);
        const double bv = grp_basis(vn, vw, J, v, G);
        double e[9];
        grp_eval<9, 0, JN>(F, I, J, bu, bv, G, e);
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
    const double bu = grp_basis(un, uw, I, u, G);
    const double bv = grp_basis(vn, vw, J, v, G);
    double e[3], nn[3];
    grp_eval<3, 0>(F, I, J, bu, bv, G, e);
    grp_eval<3, 9>(F, I, J, bu, bv, G, nn);
    h.t = t;
    h.p = v3(e[0], e[1], e[2]);
    h.n = vnormalize(v3(nn[0], nn[1], nn[2]));
    h.u = u;
    h.v = v;
    return 1;
}

// Dispatch to the fixed-row forms for 5 and 7 nodes per row.
__device__ __forceinline__ int grp_newton_exact(const DScene& S, int pidx, const V3 o, const V3 d, double u, double v,
                                                double t, QHit& h, long long& iters, const Grp& G) {
    const int J = S.p_dims[2 * pidx + 1];
    if (J == 7) return grp_newton_exact_j<7>(S, pidx, o, d, u, v, t, h, iters, G);
    if (J == 5) return grp_newton_exact_j<5>(S, pidx, o, d, u, v, t, h, iters, G);
    return grp_newton_exact_j<0>(S, pidx, o, d, u, v, t, h, iters, G);
}

// ---- FP32 phase of the precision split, by a group ---------------------------

__device__ __forceinline__ float grp_basis_f(const float* nodes, const float* w, int N, float x, const Grp& G) {
    const bool mine = G.g < N;
    const bool hit = mine && x == nodes[G.g];
    const unsigned hm = (__ballot_sync(G.mask, hit) >> G.base) & 0xFFu;
    if (hm) return (G.g == __ffs(hm) - 1) ? 1.0f : 0.0f;
    const float li = mine ? w[G.g] / (x - nodes[G.g]) : 0.0f;
    float denom = 0.0f;
    for (int i = 0; i < N; ++i) denom += __shfl_sync(G.mask, li, G.base + i);
    return mine ? li * (1.0f / denom) : 0.0f;
}

// newton_fp32 by a group (same stopping rules); every lane returns the same.
template <int JN>
__device__ __forceinline__ bool grp_newton_fp32_j(const DScene& S, int pidx, const V3& o, const V3& d, double& u,
                                                  double& v, double& t, long long& iters32, const Grp& G) {
    const int I = S.p_dims[2 * pidx], J = S.p_dims[2 * pidx + 1];
    const float* un = S.p_nodes32 + S.p_node_off[pidx];
    const float* vn = un + I;
    const float* uw = vn + J;
    const float* vw = uw + I;
    const float* Fd = S.p_fields32 + S.p_field_off[pidx];
    const float ox = static_cast<float>(o.x), oy = static_cast<float>(o.y), oz = static_cast<float>(o.z);
    const float dx = static_cast<float>(d.x), dy = static_cast<float>(d.y), dz = static_cast<float>(d.z);
    float uf = static_cast<float>(u), vf = static_cast<float>(v), tf = static_cast<float>(t);
    for (int it = 0; it < kFp32Iters; ++it) {
        ++iters32;
        const float bu = grp_basis_f(un, uw, I, uf, G);
        const float bv = grp_basis_f(vn, vw, J, vf, G);
        float rs[9];
        for (int f = 0; f < 9; ++f) rs[f] = 0.0f;
        const bool row = G.g < I && bu != 0.0f;
        const int JJ = JN > 0 ? JN : J;
        const float* rp = Fd + static_cast<long long>(G.g < I ? G.g : 0) * JJ * 12;
#pragma unroll
        for (int j = 0; j < JJ; ++j) {
            const float lj = __shfl_sync(G.mask, bv, G.base + j);
            if (row)
                for (int f = 0; f < 9; ++f) rs[f] = fmaf(lj, rp[j * 12 + f], rs[f]);
        }
        float e[9];
        for (int f = 0; f < 9; ++f) e[f] = 0.0f;
        for (int i = 0; i < I; ++i) {
            const float li = __shfl_sync(G.mask, bu, G.base + i);
            if (li == 0.0f) continue;
            for (int f = 0; f < 9; ++f) e[f] = fmaf(li, __shfl_sync(G.mask, rs[f], G.base + i), e[f]);
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

__device__ __forceinline__ bool grp_newton_fp32(const DScene& S, int pidx, const V3& o, const V3& d, double& u,
                                                double& v, double& t, long long& iters32, const Grp& G) {
    const int J = S.p_dims[2 * pidx + 1];
    if (J == 7) return grp_newton_fp32_j<7>(S, pidx, o, d, u, v, t, iters32, G);
    if (J == 5) return grp_newton_fp32_j<5>(S, pidx, o, d, u, v, t, iters32, G);
    return grp_newton_fp32_j<0>(S, pidx, o, d, u, v, t, iters32, G);
}

// Newton in the scene's precision mode, by a group.
__device__ __forceinline__ int grp_newton_mode(const DScene& S, int pidx, const V3& o, const V3& d, double u,
                                               double v, double t, QHit& h, long long& iters, long long& iters32,
                                               const Grp& G) {
    if (S.precision == BBRT_PREC_SPLIT) {
        double uu = u, vv = v, tt = t;
        if (!grp_newton_fp32(S, pidx, o, d, uu, vv, tt, iters32, G)) {
            uu = u;
            vv = v;
            tt = t;
        }
        return grp_newton_exact(S, pidx, o, d, uu, vv, tt, h, iters, G);
    }
    return grp_newton_exact(S, pidx, o, d, u, v, t, h, iters, G);
}

}  // namespace bbrt
