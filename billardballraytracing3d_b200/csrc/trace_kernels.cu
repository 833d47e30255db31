// Trace-path kernels for sm_100a: BVH query, SurfacePatch stage 1 + Newton,
// and the bounce loop with reflection and nudge, all in exact FP64.
//
// Compiled with -fmad=false: every FP64 decision equals the reference's
// (see exact.cuh).  Work distribution: one thread per ray, persistent
// blocks that pull 32-ray batches from a global counter, so warps whose rays
// finish early (escape on the first query) take new rays instead of idling
// while a long multi-bounce ray in another warp keeps bouncing.
//
// Reference (manuelarturosantana/BillardBallRayTracing3D):
//   RayTracingDriver::trace_ray   include/RayTracingDriver.hpp:172-242
//   BVH::intersect                include/BVH.hpp:75-128
//   SurfacePatch::intersect       include/ScatObjects/SurfacePatch.hpp:253-303
//   Triangle::intersect           include/ScatObjects/Triangle.hpp:26-28
//   brute_force_intersect         include/BruteForce.hpp:7-16
#include <cuda_runtime.h>
#include <math_constants.h>

#include <algorithm>
#include <mutex>

#include "../../include/bbrt.h"
#include "exact.cuh"
#include "guess.h"
#include "newton_group.cuh"

namespace bbrt {

// Work counters of the statistics, per thread (summed per warp at the end of
// a launch).  CountersT<false> holds nothing: a launch that collects no
// statistics (and no per-ray work profile) uses it, so the counting, its
// 64-bit registers and their spills compile away.
struct NoCount {
    __device__ __forceinline__ NoCount& operator++() { return *this; }
    __device__ __forceinline__ NoCount operator++(int) { return *this; }
    __device__ __forceinline__ NoCount& operator+=(long long) { return *this; }
    __device__ __forceinline__ operator long long() const { return 0; }
};

template <bool ON>
struct CountersT {
    static constexpr bool kOn = true;
    long long node_tests = 0, patch_tests = 0, cell_tests = 0, tri_tests = 0, newton_iters = 0;
    long long off_patch = 0;   // learned form: Newton roots outside their patch taken as misses
    long long node_f64 = 0;    // node tests the FP32 test left to the FP64 one
};
template <>
struct CountersT<false> {
    static constexpr bool kOn = false;
    NoCount node_tests, patch_tests, cell_tests, tri_tests, newton_iters, off_patch, node_f64;
};
using Counters = CountersT<true>;

// Per-ray data of the FP32 cull test (computed once per query).
struct CullRay {
    float ox, oy, oz, ix, iy, iz, delta;
};

__device__ __forceinline__ bool finite3(const V3& a) {
    return isfinite(a.x) && isfinite(a.y) && isfinite(a.z);
}

// Scene values of a ray's scene: the scene itself, or member m of a scene set.
__device__ __forceinline__ double scene_diag(const DScene& S, int m) {
    return m < 0 ? S.scene_diagonal : S.m_param[m * kMemberParams];
}
__device__ __forceinline__ int root_node(const DScene& S, int m) { return m < 0 ? 0 : S.m_root[m]; }

// The cull inflation bound is derived for |d| <= 1 (the trace loop always
// normalises d); single queries with longer or non-finite rays skip culling.
__device__ __forceinline__ bool cull_ok(const DScene& S, int m, int cull_flag, const V3& o, const V3& d) {
    const bool on = m < 0 ? S.cull_enabled != 0 : S.m_param[m * kMemberParams + 1] != 0.0;
    return cull_flag && on && finite3(o) && finite3(d) && d.x * d.x + d.y * d.y + d.z * d.z <= 1.0 + 1e-6;
}

__device__ __forceinline__ CullRay make_cull_ray(const DScene& S, int m, const V3& o, const V3& d) {
    CullRay c;
    double ca = S.cull_a, ch = S.cull_h, cb = S.cull_b, cc = S.cull_coord, cr = S.cull_radius;
    double c0 = S.cull_center[0], c1 = S.cull_center[1], c2 = S.cull_center[2];
    if (m >= 0) {
        const double* p = S.m_param + m * kMemberParams;
        ca = p[2]; ch = p[3]; cb = p[4]; cc = p[5]; cr = p[6]; c0 = p[7]; c1 = p[8]; c2 = p[9];
    }
    const double cx = o.x - c0, cy = o.y - c1, cz = o.z - c2;
    const double L = sqrt(cx * cx + cy * cy + cz * cz) + cr;
    const double on = sqrt(o.x * o.x + o.y * o.y + o.z * o.z);
    const double delta = ca * (L + ch) + cb * (L + on + cc);
    c.ox = static_cast<float>(o.x);
    c.oy = static_cast<float>(o.y);
    c.oz = static_cast<float>(o.z);
    c.ix = 1.0f / static_cast<float>(d.x);
    c.iy = 1.0f / static_cast<float>(d.y);
    c.iz = 1.0f / static_cast<float>(d.z);
    c.delta = __double2float_ru(delta * 1.0001);
    return c;
}

// FP32 slab test of the ray [0, inf) against a box inflated by c.delta.
// Conservative: a triangle inside the box that the exact FP64 test accepts
// always passes (the inflation bounds both roundings); only work is skipped.
// Boxes are 6 floats on a 24-byte stride from a 16-byte aligned array
// (checked at upload): read as three 8-byte loads.
__device__ __forceinline__ bool cull_box(const float* __restrict__ b, const CullRay& c) {
    const float2 b01 = *reinterpret_cast<const float2*>(b);
    const float2 b23 = *reinterpret_cast<const float2*>(b + 2);
    const float2 b45 = *reinterpret_cast<const float2*>(b + 4);
    float t1 = (b01.x - c.delta - c.ox) * c.ix, t2 = (b23.y + c.delta - c.ox) * c.ix;
    float tmin = fmaxf(0.0f, fminf(t1, t2)), tmax = fmaxf(t1, t2);
    t1 = (b01.y - c.delta - c.oy) * c.iy; t2 = (b45.x + c.delta - c.oy) * c.iy;
    tmin = fmaxf(tmin, fminf(t1, t2)); tmax = fminf(tmax, fmaxf(t1, t2));
    t1 = (b23.x - c.delta - c.oz) * c.iz; t2 = (b45.y + c.delta - c.oz) * c.iz;
    tmin = fmaxf(tmin, fminf(t1, t2)); tmax = fminf(tmax, fmaxf(t1, t2));
    return tmin <= tmax;
}

// FP32 BVH node test that reproduces ray_box_exact's decision or defers it.
//
// ray_box_exact(o, 1/d, box, best_t) passes exactly when, over the three
// axes, tmin = max(lo_a) <= tmax = min(hi_a), tmin <= best_t and tmax >= 0,
// where lo_a / hi_a are the FP64 slab times fl(fl(b - o) * fl(1/d)) of the
// near / far face (its early exit and swap give that; every t is finite for
// finite o and 1/d).  The same times in FP32 from b32 = fl32(b), o32 =
// fl32(o) and 1/fl32(d) (the cull ray's values), each face
// fl32(fl32(b32 - o32) * i32), differ from the FP64 ones by at most
// (5 * 2^-24 + 2 * 2^-53) (|b| + |o|) |1/d| plus underflow terms below 2^-120
// (roundings of b and o: 1, of d and the division: 2, of the subtraction and
// the product: 1 each, in units of 2^-24 (|b| + |o|) |1/d|); e
// (node_margin) bounds that with 2^-21 (B_a + |o32_a|) |i32_a| for the
// largest axis, B_a bounding every node coordinate on axis a.  So
// [tmin32 - e, tmin32 + e] holds the FP64 tmin and likewise tmax, and the
// test decides wherever the interval decides: 1 = passes, 0 = fails, -1 =
// undecided (run ray_box_exact).  Boxes are 6 floats (min xyz, max xyz) on a
// 24-byte stride, read as three 8-byte loads.
__device__ __forceinline__ int node_box_f32(const float* __restrict__ b, const CullRay& c, float e, double best_t) {
    const float2 b01 = *reinterpret_cast<const float2*>(b);
    const float2 b23 = *reinterpret_cast<const float2*>(b + 2);
    const float2 b45 = *reinterpret_cast<const float2*>(b + 4);
    float t1 = (b01.x - c.ox) * c.ix, t2 = (b23.y - c.ox) * c.ix;
    float tmin = fminf(t1, t2), tmax = fmaxf(t1, t2);
    t1 = (b01.y - c.oy) * c.iy; t2 = (b45.x - c.oy) * c.iy;
    tmin = fmaxf(tmin, fminf(t1, t2)); tmax = fminf(tmax, fmaxf(t1, t2));
    t1 = (b23.x - c.oz) * c.iz; t2 = (b45.y - c.oz) * c.iz;
    tmin = fmaxf(tmin, fminf(t1, t2)); tmax = fminf(tmax, fmaxf(t1, t2));
    const float lo_dn = __fsub_rd(tmin, e), lo_up = __fadd_ru(tmin, e);
    const float hi_dn = __fsub_rd(tmax, e), hi_up = __fadd_ru(tmax, e);
    if (lo_dn > hi_up || hi_up < 0.0f || static_cast<double>(lo_dn) > best_t) return 0;
    if (lo_up <= hi_dn && hi_dn >= 0.0f && static_cast<double>(lo_up) <= best_t) return 1;
    return -1;
}

// The margin e of node_box_f32 for a ray (false: the ray's FP32 values lie
// outside the range the bound covers, and its node tests stay FP64).  The
// limits keep every FP32 time below 2^81 and 1/d normal; the 2^-100 floor
// covers the underflow terms.
__device__ __forceinline__ bool node_margin(const DScene& S, const CullRay& c, float& e) {
    const float o[3] = { c.ox, c.oy, c.oz }, iv[3] = { c.ix, c.iy, c.iz };
    float m = 0x1p-100f;
    bool ok = S.node_f32_ok != 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float ai = fabsf(iv[a]), ao = fabsf(o[a]);
        ok = ok && ai >= 0x1p-40f && ai <= 0x1p40f && ao <= 0x1p40f;
        m = fmaxf(m, __fmul_ru(__fadd_ru(S.node_bound[a], ao), ai) * 0x1p-21f);
    }
    e = m;
    return ok;
}

// Stage-1 winner bookkeeping.  key = ((cell * 3 + sign) * 2 + triangle) is
// the position of a test in the reference's loop order (i, j, sign 0/+1/-1,
// triangle); the reference keeps the first strictly smaller t, i.e. the
// smallest (t, key) pair, which is what this keeps in any visiting order.
struct Stage1 {
    bool have = false;
    double t = 0.0;
    int key = 0;
    __device__ __forceinline__ void consider(double tc, int kc) {
        if (!have || tc < t || (tc == t && kc < key)) { have = true; t = tc; key = kc; }
    }
};

// The six Moller-Trumbore tests of coarse cell (i, j): signs 0, +1, -1 of
// the cell's sagitta along its normal, triangles (q00,q10,q11), (q00,q11,q01).
__device__ __forceinline__ void stage1_cell(const double* __restrict__ X, const double* __restrict__ CC, int n,
                                            int i, int j, const V3& o, const V3& d, Stage1& best) {
    const int nc = n - 1;
    const double* r0 = X + static_cast<long long>(i * n + j) * 3;
    const double* r1 = r0 + 3 * n;
    const V3 p00 = load3(r0), p01 = load3(r0 + 3), p10 = load3(r1), p11 = load3(r1 + 3);
    const double* c = CC + static_cast<long long>(i * nc + j) * 4;
    const V3 cn = v3(c[0], c[1], c[2]);
    const double s = c[3];
    const int base = (i * nc + j) * 6;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double sg = (k == 0) ? 0.0 : ((k == 1) ? 1.0 : -1.0);
        const double dd = sg * s;
        const V3 q00 = v3(p00.x + cn.x * dd, p00.y + cn.y * dd, p00.z + cn.z * dd);
        const V3 q10 = v3(p10.x + cn.x * dd, p10.y + cn.y * dd, p10.z + cn.z * dd);
        const V3 q01 = v3(p01.x + cn.x * dd, p01.y + cn.y * dd, p01.z + cn.z * dd);
        const V3 q11 = v3(p11.x + cn.x * dd, p11.y + cn.y * dd, p11.z + cn.z * dd);
        double t;
        if (mt_exact(o, d, q00, q10, q11, t)) best.consider(t, base + 2 * k);
        if (mt_exact(o, d, q00, q11, q01, t)) best.consider(t, base + 2 * k + 1);
    }
}

// SurfacePatch::intersect stage 1: the winning (t, key) over the coarse
// triangulation (all cells, or only cells whose inflated box the ray crosses).
template <class Ctr>
__device__ __forceinline__ Stage1 patch_stage1(const DScene& S, int pidx, const V3& o, const V3& d, bool use_cull,
                                               const CullRay& cr, Ctr& ctr) {
    const int n = S.coarse_n, nc = n - 1;
    const double* X = S.c_xyz + static_cast<long long>(pidx) * n * n * 3;
    const double* CC = S.c_cell + static_cast<long long>(pidx) * nc * nc * 4;
    Stage1 best;
    ++ctr.patch_tests;
    if (use_cull) {
        const int B = S.block_cells, NB = S.n_blocks_side;
        const float* BB = S.c_block_box + static_cast<long long>(pidx) * NB * NB * 6;
        const float* CB = S.c_cell_box + static_cast<long long>(pidx) * nc * nc * 6;
        for (int bi = 0; bi < NB; ++bi) {
            for (int bj = 0; bj < NB; ++bj) {
                ++ctr.cell_tests;
                if (!cull_box(BB + (bi * NB + bj) * 6, cr)) continue;
                const int i1 = min(nc, (bi + 1) * B), j1 = min(nc, (bj + 1) * B);
                for (int i = bi * B; i < i1; ++i) {
                    for (int j = bj * B; j < j1; ++j) {
                        ++ctr.cell_tests;
                        if (!cull_box(CB + (i * nc + j) * 6, cr)) continue;
                        ctr.tri_tests += 6;
                        stage1_cell(X, CC, n, i, j, o, d, best);
                    }
                }
            }
        }
    } else {
        for (int i = 0; i < nc; ++i)
            for (int j = 0; j < nc; ++j) stage1_cell(X, CC, n, i, j, o, d, best);
        ctr.tri_tests += 6LL * nc * nc;
    }
    return best;
}

// triangle_uv_centroid (SurfacePatch.hpp:499-510) of the stage-1 winner `key`.
__device__ __forceinline__ void key_to_uv(const DScene& S, int key, double& u0, double& v0) {
    const int nc = S.coarse_n - 1;
    const int cell = key / 6;
    const bool second = (key & 1) != 0;
    const int bi = cell / nc, bj = cell % nc;
    const double ui = S.coarse_uv[bi], ui1 = S.coarse_uv[bi + 1];
    const double vj = S.coarse_uv[bj], vj1 = S.coarse_uv[bj + 1];
    if (!second) { u0 = (ui + ui1 + ui1) / 3.0; v0 = (vj + vj + vj1) / 3.0; }
    else         { u0 = (ui + ui + ui1) / 3.0; v0 = (vj + vj1 + vj1) / 3.0; }
}

// SurfacePatch::intersect: stage 1, then Newton from the winning triangle's
// (u, v) centroid and its t.
template <class Ctr>
__device__ __forceinline__ int patch_intersect(const DScene& S, int pidx, const V3& o, const V3& d, bool use_cull,
                                               const CullRay& cr, QHit& h, Ctr& ctr) {
    const Stage1 best = patch_stage1(S, pidx, o, d, use_cull, cr, ctr);
    if (!best.have) return 0;
    double u0, v0;
    key_to_uv(S, best.key, u0, v0);
    long long it = 0;
    const int r = newton_exact(S, pidx, o, d, u0, v0, best.t, h, it);
    ctr.newton_iters += it;
    return r;
}

// Triangle::intersect (Triangle.hpp:26-28): Moller-Trumbore, point o + t d,
// normal normalize(e1 x e2).
template <class Ctr>
__device__ __forceinline__ int triangle_intersect(const DScene& S, int sub, const V3& o, const V3& d, QHit& h,
                                                  Ctr& ctr) {
    h.err = 0;
    h.ev0 = 0.0;
    h.ev1 = 0.0;
    const double* v = S.tri + static_cast<long long>(sub) * 9;
    const V3 v0 = load3(v), v1 = load3(v + 3), v2 = load3(v + 6);
    double t, u, w;
    ++ctr.tri_tests;
    if (!mt_full(o, d, v0, v1, v2, t, u, w)) return 0;
    h.t = t;
    h.p = v3(o.x + t * d.x, o.y + t * d.y, o.z + t * d.z);
    h.n = vnormalize(vcross(vsub(v1, v0), vsub(v2, v0)));
    h.u = u;
    h.v = w;
    return 1;
}

// ScatObject::intersect for object `obj`: 1 hit, 0 miss (h.err set on a
// Newton failure).
template <class Ctr>
__device__ __forceinline__ int object_intersect(const DScene& S, int obj, const V3& o, const V3& d, bool use_cull,
                                                const CullRay& cr, QHit& h, Ctr& ctr) {
    h.err = 0;
    h.ev0 = 0.0;
    h.ev1 = 0.0;
    const int sub = S.obj_sub[obj];
    if (S.obj_kind[obj] == BBRT_OBJ_PATCH) return patch_intersect(S, sub, o, d, use_cull, cr, h, ctr);
    return triangle_intersect(S, sub, o, d, h, ctr);
}

// BVH::intersect with a 64-entry stack.  Returns the closest hit (obj >= 0),
// a miss (obj < 0, err 0), or the first Newton failure met (err != 0).
// off_patch_miss (learned form): a Newton root outside its patch is a miss.
template <class Ctr>
__device__ QHit bvh_query(const DScene& S, const V3& o, const V3& d, int cull_flag, Ctr& ctr,
                          bool off_patch_miss = false, int member = -1) {
    QHit best;
    best.obj = -1;
    best.err = 0;
    best.t = CUDART_INF;
    const double inv[3] = { 1.0 / d.x, 1.0 / d.y, 1.0 / d.z };
    const bool neg[3] = { inv[0] < 0.0, inv[1] < 0.0, inv[2] < 0.0 };
    const bool use_cull = cull_ok(S, member, cull_flag, o, d);
    CullRay cr;
    if (use_cull) cr = make_cull_ray(S, member, o, d);
    double best_t = CUDART_INF;
    int stack[64];
    int sp = 0;
    stack[sp++] = root_node(S, member);
    while (sp > 0) {
        const int idx = stack[--sp];
        ++ctr.node_tests;
        if (!ray_box_exact(o, inv, S.node_box + 6LL * idx, best_t)) continue;
        const int* link = S.node_link + 4LL * idx;
        if (link[1] < 0) {
            const int start = link[0], count = link[2];
            for (int k = 0; k < count; ++k) {
                const int obj = S.leaf_objects[start + k];
                QHit h;
                const int r = object_intersect(S, obj, o, d, use_cull, cr, h, ctr);
                if (off_patch_miss && h.err == BBRT_RAY_NEWTON_DOMAIN) {
                    ++ctr.off_patch;
                    continue;
                }
                if (h.err) {
                    h.obj = obj;
                    return h;
                }
                if (r && h.t < best_t) {
                    best_t = h.t;
                    best = h;
                    best.obj = obj;
                }
            }
            continue;
        }
        if (sp + 2 > 64) {
            best.err = BBRT_RAY_STACK_OVERFLOW;
            best.obj = -1;
            return best;
        }
        const int left = link[0], right = link[1];
        if (neg[link[3]]) { stack[sp++] = left; stack[sp++] = right; }
        else              { stack[sp++] = right; stack[sp++] = left; }
    }
    return best;
}

__device__ __forceinline__ void warp_add(long long* dst, long long v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(reinterpret_cast<unsigned long long*>(dst), static_cast<unsigned long long>(v));
}

// ---- the bounce loop (RayTracingDriver::trace_ray) as per-ray state steps ----

// Registers of one ray between queries.
struct RayCtx {
    V3 o, d, end;
    int member;      // scene-set member of the ray, -1 for a single scene
    int bounces;
    int status;      // final status once set; -1 while the ray is running
    int err_obj;
    double ev0, ev1;
};

__device__ __forceinline__ void init_outputs(const TraceArgs& A, long long i) {
    if (A.ray_work) for (int k = 0; k < 4; ++k) A.ray_work[4 * i + k] = 0;
    const int K = A.record;
    for (int k = 0; k < K; ++k) {
        if (A.hit_object) A.hit_object[i * K + k] = -1;
        if (A.hit_point) { double* p = A.hit_point + (i * K + k) * 3; p[0] = 0.0; p[1] = 0.0; p[2] = 0.0; }
        if (A.hit_uv) { double* p = A.hit_uv + (i * K + k) * 2; p[0] = 0.0; p[1] = 0.0; }
    }
}

// Start of trace_ray: zero-length check, normalisation (RayTracingDriver.hpp:174-184).
__device__ __forceinline__ RayCtx start_ray(const TraceArgs& A, long long i) {
    RayCtx r;
    r.o = load3(A.origins + 3 * i);
    r.member = A.ray_member ? A.ray_member[i] : -1;
    const V3 dir_in = load3(A.dirs + 3 * i);
    r.end = r.o;
    r.d = v3(0.0, 0.0, 0.0);
    r.bounces = 0;
    r.status = -1;
    r.err_obj = -1;
    r.ev0 = r.ev1 = 0.0;
    const double len2 = dir_in.x * dir_in.x + dir_in.y * dir_in.y + dir_in.z * dir_in.z;
    if (len2 < 1e-300) {
        r.status = BBRT_RAY_BAD_DIR;
    } else {
        const double len = sqrt(dir_in.x * dir_in.x + dir_in.y * dir_in.y + dir_in.z * dir_in.z);
        r.d = v3(dir_in.x / len, dir_in.y / len, dir_in.z / len);
    }
    return r;
}

// One bounce of trace_ray given the query result h (RayTracingDriver.hpp:187-237).
// Returns true when the ray goes on to another query.
__device__ __forceinline__ bool step_ray(const DScene& S, const TraceArgs& A, long long i, RayCtx& r, const QHit& h,
                                        bool write = true) {
    if (h.err) {
        r.status = h.err;
        r.err_obj = h.obj;
        r.ev0 = h.ev0;
        r.ev1 = h.ev1;
        return false;
    }
    if (h.obj < 0) {
        r.status = BBRT_RAY_ESCAPED;
        const double diag = scene_diag(S, r.member);
        r.end = v3(r.o.x + r.d.x * diag, r.o.y + r.d.y * diag, r.o.z + r.d.z * diag);
        return false;
    }
    if (vdot(r.d, h.n) > S.backface_tol) { r.status = BBRT_RAY_WENT_INSIDE; return false; }
    const int K = A.record;
    if (write && r.bounces < K) {
        if (A.hit_object) A.hit_object[i * K + r.bounces] = h.obj;
        if (A.hit_point) { double* p = A.hit_point + (i * K + r.bounces) * 3; p[0] = h.p.x; p[1] = h.p.y; p[2] = h.p.z; }
        if (A.hit_uv) { double* p = A.hit_uv + (i * K + r.bounces) * 2; p[0] = h.u; p[1] = h.v; }
    }
    if (write && A.hit_counts && r.bounces >= A.count_from) atomicAdd(A.hit_counts + h.obj, 1ULL);
    ++r.bounces;
    r.end = h.p;
    const V3 d = r.d;
    const double dn = d.x * h.n.x + d.y * h.n.y + d.z * h.n.z;
    r.d = v3(d.x - 2.0 * dn * h.n.x, d.y - 2.0 * dn * h.n.y, d.z - 2.0 * dn * h.n.z);
    const double eps = smax(S.eps_factor * scene_diag(S, r.member), S.sag_factor * S.obj_pad[h.obj]);
    r.o = v3(h.p.x + r.d.x * eps, h.p.y + r.d.y * eps, h.p.z + r.d.z * eps);
    return true;
}

__device__ __forceinline__ void finish_ray(const TraceArgs& A, long long i, const RayCtx& r) {
    if (A.status) A.status[i] = r.status;
    if (A.bounce_count) A.bounce_count[i] = r.bounces;
    if (A.exit_dir) { double* p = A.exit_dir + 3 * i; p[0] = r.d.x; p[1] = r.d.y; p[2] = r.d.z; }
    if (A.end_point) { double* p = A.end_point + 3 * i; p[0] = r.end.x; p[1] = r.end.y; p[2] = r.end.z; }
    if (A.err_object) A.err_object[i] = r.err_obj;
    if (A.err_value) { A.err_value[2 * i] = r.ev0; A.err_value[2 * i + 1] = r.ev1; }
}

// Runs the bounce loop of one ray to the end with inline queries.
template <class Ctr>
__device__ __forceinline__ void run_ray(const DScene& S, const TraceArgs& A, long long i, RayCtx& r, Ctr& ctr,
                                        long long& queries) {
    while (r.status < 0) {
        if (r.bounces >= A.max_bounces) { r.status = BBRT_RAY_MAX_BOUNCES; break; }
        ++queries;
        const QHit h = bvh_query(S, r.o, r.d, A.cull, ctr, A.off_patch_miss != 0, r.member);
        if (!step_ray(S, A, i, r, h)) break;
    }
}

// Adds one thread's work counters for ray i to the optional per-ray profile
// (a ray is owned by one thread at a time, so no atomics are needed).
template <class Ctr>
__device__ __forceinline__ void add_ray_work(const TraceArgs& A, long long i, const Ctr& c) {
    if constexpr (!Ctr::kOn) return;
    if (!A.ray_work || i < 0) return;
    long long* w = A.ray_work + 4 * i;
    w[0] += c.node_tests;
    w[1] += c.cell_tests;
    w[2] += c.tri_tests;
    w[3] += c.newton_iters;
}

template <bool ON>
struct RayTallyT {
    long long bounces = 0, queries = 0;
    long long hist[BBRT_RAY_STATUS_COUNT] = { 0, 0, 0, 0, 0, 0, 0, 0 };
};
template <>
struct RayTallyT<false> {
    NoCount bounces, queries;
    NoCount hist[BBRT_RAY_STATUS_COUNT];
};
using RayTally = RayTallyT<true>;

template <class Ctr, class Tally>
__device__ __forceinline__ void flush_stats(const TraceArgs& A, const Ctr& ctr, const Tally& t, bool tail = false) {
    if constexpr (!Ctr::kOn) return;
    if (!A.stats) return;
    if (tail) {
        long long rays = 0;
#pragma unroll
        for (int k = 0; k < BBRT_RAY_STATUS_COUNT; ++k) rays += t.hist[k];
        warp_add(A.stats + ST_TAIL_NODE_TESTS, ctr.node_tests);
        warp_add(A.stats + ST_TAIL_CELL_TESTS, ctr.cell_tests);
        warp_add(A.stats + ST_TAIL_TRI_TESTS, ctr.tri_tests);
        warp_add(A.stats + ST_TAIL_NEWTON_ITERS, ctr.newton_iters);
        warp_add(A.stats + ST_TAIL_RAYS, rays);
    }
    warp_add(A.stats + ST_BOUNCES, t.bounces);
    warp_add(A.stats + ST_QUERIES, t.queries);
    warp_add(A.stats + ST_NODE_TESTS, ctr.node_tests);
    warp_add(A.stats + ST_PATCH_TESTS, ctr.patch_tests);
    warp_add(A.stats + ST_CELL_TESTS, ctr.cell_tests);
    warp_add(A.stats + ST_TRI_TESTS, ctr.tri_tests);
    warp_add(A.stats + ST_NEWTON_ITERS, ctr.newton_iters);
    warp_add(A.stats + ST_OFF_PATCH, ctr.off_patch);
    warp_add(A.stats + ST_NODE_F64, ctr.node_f64);
#pragma unroll
    for (int k = 0; k < BBRT_RAY_STATUS_COUNT; ++k) warp_add(A.stats + ST_HIST0 + k, t.hist[k]);
}

// Fused per-ray kernel (small batches): warps pull 32-ray batches until none are left.
__global__ void __launch_bounds__(128) k_trace(DScene S, TraceArgs A) {
    Counters ctr;
    RayTally tally;
    const int lane = threadIdx.x & 31;
    while (true) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(A.work_counter, 32ULL);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= static_cast<unsigned long long>(A.n)) break;
        const long long i = static_cast<long long>(base) + lane;
        if (i < A.n) {
            init_outputs(A, i);
            RayCtx r = start_ray(A, i);
            Counters c1;
            run_ray(S, A, i, r, c1, tally.queries);
            add_ray_work(A, i, c1);
            ctr.node_tests += c1.node_tests; ctr.patch_tests += c1.patch_tests; ctr.cell_tests += c1.cell_tests;
            ctr.tri_tests += c1.tri_tests; ctr.newton_iters += c1.newton_iters; ctr.off_patch += c1.off_patch;
            finish_ray(A, i, r);
            tally.bounces += r.bounces;
            tally.hist[r.status]++;
        }
    }
    flush_stats(A, ctr, tally, true);
}

// ---- wavefront form: advance rays until they need a Newton solve ----------

__device__ __forceinline__ void save_ray(const WaveArgs& W, long long i, const RayCtx& r, int nres) {
    double* o = W.o + 3 * i;
    double* d = W.d + 3 * i;
    double* e = W.end + 3 * i;
    o[0] = r.o.x; o[1] = r.o.y; o[2] = r.o.z;
    d[0] = r.d.x; d[1] = r.d.y; d[2] = r.d.z;
    e[0] = r.end.x; e[1] = r.end.y; e[2] = r.end.z;
    W.bounces[i] = r.bounces;
    W.nres[i] = nres;
}

__device__ __forceinline__ RayCtx load_ray(const TraceArgs& A, const WaveArgs& W, long long i, int& nres) {
    RayCtx r;
    r.member = A.ray_member ? A.ray_member[i] : -1;
    r.o = load3(W.o + 3 * i);
    r.d = load3(W.d + 3 * i);
    r.end = load3(W.end + 3 * i);
    r.bounces = W.bounces[i];
    r.status = -1;
    r.err_obj = -1;
    r.ev0 = r.ev1 = 0.0;
    nres = W.nres[i];
    return r;
}

// Warp-aggregated append: returns this lane's slot (or -1 when !want).
__device__ __forceinline__ long long warp_append(unsigned int* counter, bool want) {
    const unsigned mask = __ballot_sync(0xffffffffu, want);
    const int lane = threadIdx.x & 31;
    unsigned int base = 0;
    if (lane == 0 && mask) base = atomicAdd(counter, static_cast<unsigned int>(__popc(mask)));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (!want) return -1;
    return static_cast<long long>(base) + __popc(mask & ((1u << lane) - 1u));
}

// Appends one training sample (learned guess) when recording is on.
__device__ __forceinline__ void record_sample(const TraceArgs& A, int label, const V3& o, const V3& d, int pidx,
                                              double u, double v, double t) {
    const unsigned long long k = atomicAdd(A.sample_count + label, 1ULL);
    const long long cap = label ? A.sample_cap_pos : A.sample_cap_neg;
    if (static_cast<long long>(k) >= cap) return;
    GuessSample* s = A.samples + (label ? 0 : A.sample_cap_pos) + k;
    s->o[0] = o.x; s->o[1] = o.y; s->o[2] = o.z;
    s->d[0] = d.x; s->d[1] = d.y; s->d[2] = d.z;
    s->u = u; s->v = v; s->t = t;
    s->patch = pidx;
    s->label = label;
}

// One of the six Moller-Trumbore tests of cell (i, j): step = 2 * sign + triangle,
// sign order 0, +1, -1 of the sagitta along the cell normal, triangles
// (q00,q10,q11) then (q00,q11,q01) — the order and arithmetic of stage1_cell.
__device__ __forceinline__ void stage1_tri(const double* __restrict__ X, const double* __restrict__ CC, int n, int i,
                                           int j, int step, const V3& o, const V3& d, Stage1& best) {
    const int nc = n - 1;
    const double* r0 = X + static_cast<long long>(i * n + j) * 3;
    const double* r1 = r0 + 3 * n;
    // cell normal and sagitta: 4 doubles on a 32-byte stride (16-byte loads)
    const double* c = CC + static_cast<long long>(i * nc + j) * 4;
    const double2 c01 = *reinterpret_cast<const double2*>(c);
    const double2 c23 = *reinterpret_cast<const double2*>(c + 2);
    const V3 cn = v3(c01.x, c01.y, c23.x);
    const int k = step >> 1;
    const double sg = (k == 0) ? 0.0 : ((k == 1) ? 1.0 : -1.0);
    const double dd = sg * c23.y;
    const V3 p00 = load3(r0), p11 = load3(r1 + 3);
    const V3 pm = (step & 1) ? load3(r0 + 3) : load3(r1);   // p01 for the second triangle, p10 for the first
    const V3 q00 = v3(p00.x + cn.x * dd, p00.y + cn.y * dd, p00.z + cn.z * dd);
    const V3 q11 = v3(p11.x + cn.x * dd, p11.y + cn.y * dd, p11.z + cn.z * dd);
    const V3 qm = v3(pm.x + cn.x * dd, pm.y + cn.y * dd, pm.z + cn.z * dd);
    double t;
    const bool hit = (step & 1) ? mt_exact(o, d, q00, q11, qm, t) : mt_exact(o, d, q00, qm, q11, t);
    if (hit) best.consider(t, (i * nc + j) * 6 + step);
}

// ---- warp-cooperative stage 1 (used by k_advance and the warp-per-ray tail) ----

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ void warp_min_stage1(Stage1& s) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const int oh = __shfl_xor_sync(kFull, s.have ? 1 : 0, off);
        const double ot = __shfl_xor_sync(kFull, s.t, off);
        const int ok = __shfl_xor_sync(kFull, s.key, off);
        if (oh) s.consider(ot, ok);
    }
}

// Lane `lane` runs the `k`-th of the six triangle tests of each passing cell in
// `cm` (cells enumerated by the set bits of cm, offsets into (ci0, cj0) grid of
// width w), 32 tests at a time.
__device__ __forceinline__ void warp_cell_tris(const double* X, const double* CC, int n, unsigned cm, int base_i,
                                               int base_j, int w, int c0, const V3& o, const V3& d, int lane,
                                               Stage1& best) {
    const int total = __popc(cm) * 6;
    for (int p0 = 0; p0 < total; p0 += 32) {
        const int p = p0 + lane;
        if (p < total) {
            const int bit = __fns(cm, 0, p / 6 + 1);
            const int c = c0 + bit;
            stage1_tri(X, CC, n, base_i + c / w, base_j + c % w, p % 6, o, d, best);
        }
    }
}

template <class Ctr>
__device__ Stage1 warp_patch_stage1(const DScene& S, int pidx, const V3& o, const V3& d, bool use_cull,
                                    const CullRay& cr, int lane, Ctr& ctr) {
    const int n = S.coarse_n, nc = n - 1;
    const double* X = S.c_xyz + static_cast<long long>(pidx) * n * n * 3;
    const double* CC = S.c_cell + static_cast<long long>(pidx) * nc * nc * 4;
    Stage1 best;
    if (lane == 0) ++ctr.patch_tests;
    if (!(finite3(o) && finite3(d))) {
        // ordered loop on every lane (same result everywhere)
        CountersT<false> dummy;
        best = patch_stage1(S, pidx, o, d, false, cr, dummy);
        if (lane == 0) ctr.tri_tests += 6LL * nc * nc;
        return best;
    }
    if (use_cull) {
        const int B = S.block_cells, NB = S.n_blocks_side, NB2 = NB * NB;
        const float* BB = S.c_block_box + static_cast<long long>(pidx) * NB2 * 6;
        const float* CB = S.c_cell_box + static_cast<long long>(pidx) * nc * nc * 6;
        for (int b0 = 0; b0 < NB2; b0 += 32) {
            const int b = b0 + lane;
            unsigned bm = __ballot_sync(kFull, b < NB2 && cull_box(BB + b * 6, cr));
            if (lane == 0) ctr.cell_tests += min(32, NB2 - b0);
            while (bm) {
                const int bl = __ffs(bm) - 1;
                bm &= bm - 1;
                const int bi = (b0 + bl) / NB, bj = (b0 + bl) % NB;
                const int i0 = bi * B, j0 = bj * B;
                const int h = min(nc, i0 + B) - i0, w = min(nc, j0 + B) - j0;
                for (int c0 = 0; c0 < h * w; c0 += 32) {
                    const int c = c0 + lane;
                    const unsigned cm = __ballot_sync(kFull, c < h * w && cull_box(CB + ((i0 + c / w) * nc + j0 + c % w) * 6, cr));
                    if (lane == 0) { ctr.cell_tests += min(32, h * w - c0); ctr.tri_tests += 6 * __popc(cm); }
                    warp_cell_tris(X, CC, n, cm, i0, j0, w, c0, o, d, lane, best);
                }
            }
        }
    } else {
        const int total = nc * nc * 6;
        for (int p = lane; p < total; p += 32) stage1_tri(X, CC, n, (p / 6) / nc, (p / 6) % nc, p % 6, o, d, best);
        if (lane == 0) ctr.tri_tests += total;
    }
    warp_min_stage1(best);
    return best;
}

// Stage 1 of one patch by a group of WH lanes, 16 (a half-warp) or 8 (a
// quarter; lane hl of the group whose lanes are hmask, the first being
// hbase): warp_patch_stage1's block, cell and triangle tests over WH lanes,
// and the same (t, key) winner on every lane of the group.  With at most 16
// blocks per patch and 16 cells per block each level is one ballot for a
// half-warp (two for a quarter), so two halves take two patches, four
// quarters four, in about the time the whole warp takes one.  The group's
// test counts (uniform over it) go to c.
template <int WH, class Ctr>
__device__ Stage1 group_patch_stage1(const DScene& S, int pidx, const V3& o, const V3& d, bool use_cull,
                                     const CullRay& cr, int hl, unsigned hmask, int hbase, Ctr& c) {
    constexpr unsigned kGroupBits = (1u << WH) - 1u;
    const int n = S.coarse_n, nc = n - 1;
    const double* X = S.c_xyz + static_cast<long long>(pidx) * n * n * 3;
    const double* CC = S.c_cell + static_cast<long long>(pidx) * nc * nc * 4;
    Stage1 best;
    ++c.patch_tests;
    if (!(finite3(o) && finite3(d))) {
        CountersT<false> dummy;
        best = patch_stage1(S, pidx, o, d, false, cr, dummy);
        c.tri_tests += 6LL * nc * nc;
        return best;
    }
    if (use_cull) {
        const int B = S.block_cells, NB = S.n_blocks_side, NB2 = NB * NB;
        const float* BB = S.c_block_box + static_cast<long long>(pidx) * NB2 * 6;
        const float* CB = S.c_cell_box + static_cast<long long>(pidx) * nc * nc * 6;
        for (int b0 = 0; b0 < NB2; b0 += WH) {
            const int b = b0 + hl;
            unsigned bm = (__ballot_sync(hmask, b < NB2 && cull_box(BB + b * 6, cr)) >> hbase) & kGroupBits;
            c.cell_tests += min(WH, NB2 - b0);
            while (bm) {
                const int bl = __ffs(bm) - 1;
                bm &= bm - 1;
                const int bi = (b0 + bl) / NB, bj = (b0 + bl) % NB;
                const int i0 = bi * B, j0 = bj * B;
                const int h = min(nc, i0 + B) - i0, w = min(nc, j0 + B) - j0;
                for (int c0 = 0; c0 < h * w; c0 += WH) {
                    const int ce = c0 + hl;
                    const unsigned cm =
                        (__ballot_sync(hmask, ce < h * w && cull_box(CB + ((i0 + ce / w) * nc + j0 + ce % w) * 6, cr)) >>
                         hbase) & kGroupBits;
                    c.cell_tests += min(WH, h * w - c0);
                    c.tri_tests += 6 * __popc(cm);
                    const int total = __popc(cm) * 6;
                    for (int p0 = 0; p0 < total; p0 += WH) {
                        const int p = p0 + hl;
                        if (p < total) {
                            const int cell = c0 + __fns(cm, 0, p / 6 + 1);
                            stage1_tri(X, CC, n, i0 + cell / w, j0 + cell % w, p % 6, o, d, best);
                        }
                    }
                }
            }
        }
    } else {
        const int total = nc * nc * 6;
        for (int p = hl; p < total; p += WH) stage1_tri(X, CC, n, (p / 6) / nc, (p / 6) % nc, p % 6, o, d, best);
        c.tri_tests += total;
    }
#pragma unroll
    for (int off = WH / 2; off > 0; off >>= 1) {
        const int oh = __shfl_xor_sync(hmask, best.have ? 1 : 0, off);
        const double ot = __shfl_xor_sync(hmask, best.t, off);
        const int ok = __shfl_xor_sync(hmask, best.key, off);
        if (oh) best.consider(ot, ok);
    }
    return best;
}

// Advance-kernel modes.  The kernel is persistent: each lane owns one ray at
// a time and the body is one flat loop in which every iteration does one
// small unit of work for the lane's ray (one BVH node test, one leaf object,
// one block or cell box, one Moller-Trumbore test).  A lane whose ray
// suspends or finishes fetches the next runnable ray at once, so lanes stay
// busy and the warp reconverges every iteration instead of waiting on its
// slowest ray.
enum AdvMode {
    M_NODE = 0,      // pop and test a BVH node
    M_LEAF = 1,      // next object of the current leaf
    M_BLOCK = 2,     // next stage-1 block box
    M_CELL = 3,      // next cell box of the current block
    M_CELL_ALL = 4,  // next cell, culling off
    M_TRI = 5,       // next of the six triangle tests of a cell
    M_S1_DONE = 6,   // stage 1 of the current patch finished
    M_S1_WARP = 7,   // stage 1 of the current patch waits for the whole warp
    M_RESOLVE = 8,   // query finished: bounce, escape or error
    M_FINISH = 9,    // ray finished
    M_SUSPEND = 10,  // waiting for a Newton solve
    M_OVERFLOW = 11, // more solves than the resolved list holds
    M_IDLE = 12,     // lane has no ray
    M_DRAINED = 13   // no runnable ray left
};

struct AdvState {
    // query
    double inv[3];
    bool neg[3];
    bool use_cull;
    bool node32;     // node boxes tested in FP32 (node_box_f32) with margin e32
    float e32;
    CullRay cr;      // also the FP32 origin and 1/d of the FP32 node test
    double best_t;
    int best_ver;    // times best_t went down in this query, saturating at kStackAlways
    int best_obj;    // -1: no hit yet
    int best_e;      // resolved entry of the best patch hit, -1 for a triangle
    double tri_u, tri_v;
    int err, err_obj;
    double ev0, ev1;
    int sp;
    int leaf_start, leaf_count, leaf_k;
    // stage 1 of the current patch
    int obj, pidx, bi, bj, ci, cj, i1, j0, j1;
    int tci, tcj, tri, tri_ret;   // cell and step of the triangle tests
    Stage1 s1;
};

// Traversal stack entries of k_advance: node index in the low 24 bits, and
// in the top 8 the best_ver at which the node's box passed ray_box_exact when
// its parent pushed it.  A popped node whose tag equals the query's current
// best_ver passed with the same best_t, so it passes again; any other tag
// (kStackAlways: the root, resumed stacks, a saturated best_ver) re-tests the
// box with the current best_t — the reference's test at the reference's
// time, so the visit sequence is the reference's.
constexpr unsigned kStackAlways = 0xFFu;
constexpr unsigned kStackIdx = 0x00FFFFFFu;
__device__ __forceinline__ int stack_entry(int idx, unsigned ver) { return static_cast<int>((ver << 24) | static_cast<unsigned>(idx)); }

__device__ __forceinline__ void adv_start_query(const DScene& S, const TraceArgs& A, const WaveArgs& W,
                                                const RayCtx& r, AdvState& q, int* stack) {
    q.inv[0] = 1.0 / r.d.x;
    q.inv[1] = 1.0 / r.d.y;
    q.inv[2] = 1.0 / r.d.z;
    q.neg[0] = q.inv[0] < 0.0;
    q.neg[1] = q.inv[1] < 0.0;
    q.neg[2] = q.inv[2] < 0.0;
    q.use_cull = cull_ok(S, r.member, A.cull, r.o, r.d);
    q.node32 = W.node_f32 && finite3(r.o) && finite3(r.d);
    if (q.use_cull || q.node32) q.cr = make_cull_ray(S, r.member, r.o, r.d);
    if (q.node32) q.node32 = node_margin(S, q.cr, q.e32);
    q.best_t = CUDART_INF;
    q.best_ver = 0;
    q.best_obj = -1;
    q.best_e = -1;
    q.err = 0;
    q.err_obj = -1;
    q.ev0 = q.ev1 = 0.0;
    q.sp = 0;
    stack[q.sp++] = stack_entry(root_node(S, r.member), kStackAlways);
}

// One BVH node test of k_advance: in FP32 where the ray allows it and the
// FP32 interval decides (node_box_f32), else ray_box_exact, on FP64 boxes
// from the shared-memory copy when it holds them (n64 nodes; n32 FP32 boxes
// otherwise), else from global memory.
template <class Ctr>
__device__ __forceinline__ bool adv_node_pass(const DScene& S, const RayCtx& r, const AdvState& q, int idx,
                                              const double* sbox, const float* sbox32, int n64, int n32, Ctr& c) {
    int dec = -1;
    if (q.node32) dec = node_box_f32(idx < n32 ? sbox32 + 6 * idx : S.node_box32 + 6LL * idx, q.cr, q.e32, q.best_t);
    if (dec < 0) {
        if (q.node32) ++c.node_f64;
        dec = ray_box_exact(r.o, q.inv, idx < n64 ? sbox + 6 * idx : S.node_box + 6LL * idx, q.best_t);
    }
    return dec != 0;
}

// Keeps the traversal state of a query that suspends for a Newton solve
// (the lane stands at the leaf position of the patch being solved).
__device__ __forceinline__ void save_query(const WaveArgs& W, long long i, const AdvState& q, const int* stack) {
    int* qi = W.qs_int + i * kQsInt;
    if (!W.resume_queries || q.sp > kSaveStack) {
        qi[0] = -1;
        return;
    }
    qi[0] = q.sp;
    qi[1] = q.leaf_start;
    qi[2] = q.leaf_count;
    qi[3] = q.leaf_k;
    qi[4] = q.best_obj;
    qi[5] = q.best_e;
    double* qd = W.qs_dbl + i * 3;
    qd[0] = q.best_t;
    qd[1] = q.tri_u;
    qd[2] = q.tri_v;
    // saved entries re-test their boxes when popped after the resume
    int* st = W.qs_stack + i * kSaveStack;
    for (int k = 0; k < q.sp; ++k) st[k] = stack_entry(stack[k] & static_cast<int>(kStackIdx), kStackAlways);
}

// Resumes a suspended query where it stopped (false when none was saved).
// The visit sequence is the one a replay from the root would produce, whose
// already-solved patches come from the resolved list.
__device__ __forceinline__ bool resume_query(const DScene& S, const TraceArgs& A, const WaveArgs& W, long long i,
                                             const RayCtx& r, AdvState& q, int* stack) {
    if (!W.resume_queries) return false;
    const int* qi = W.qs_int + i * kQsInt;
    const int sp = qi[0];
    if (sp < 0) return false;
    adv_start_query(S, A, W, r, q, stack);
    q.sp = sp;
    q.leaf_start = qi[1];
    q.leaf_count = qi[2];
    q.leaf_k = qi[3];
    q.best_obj = qi[4];
    q.best_e = qi[5];
    const double* qd = W.qs_dbl + i * 3;
    q.best_t = qd[0];
    q.tri_u = qd[1];
    q.tri_v = qd[2];
    const int* st = W.qs_stack + i * kSaveStack;
    for (int k = 0; k < sp; ++k) stack[k] = st[k];
    return true;
}

// Advances runnable rays until each needs a Newton solve, overflows its
// resolved list, or finishes.  Persistent: lanes fetch rays from the
// runnable set until it is drained.

// NT threads per block, MINB blocks per SM requested from the register
// allocator (launch shape variants of the same body); CHILD: a node's
// children are tested with it (see the traversal stack tags); HALF: the
// warp's queued stage 1s are taken two at a time by half-warps (patches of at
// most 16 blocks of at most 16 cells).
template <int NT, int MINB, bool CHILD, int G, bool STATS>
__global__ void __launch_bounds__(NT, MINB) k_advance(DScene S, TraceArgs A, WaveArgs W) {
    CountersT<STATS> ctr, cray;
    RayTallyT<STATS> tally;
    NewtonRequest rq;
    rq.ray = -1;
    long long i = -1;
    int mode = M_IDLE;
    RayCtx r;
    int nres = 0;
    AdvState q;
    int stack[64];
    const int n = S.coarse_n, nc = n - 1, NB = S.n_blocks_side, B = S.block_cells;
    const int lane = threadIdx.x & 31;
    // The first S.smem_nodes BVH nodes (breadth-first order: the top levels)
    // are staged in shared memory for the whole launch: their FP64 boxes, or
    // with the FP32 node test their FP32 boxes (24 instead of 48 bytes a node),
    // and their links.
    extern __shared__ __align__(16) double smem_bvh[];
    const int n64 = W.node_f32 ? 0 : S.smem_nodes, n32 = W.node_f32 ? S.smem_nodes : 0;
    double* sbox = smem_bvh;
    float* sbox32 = reinterpret_cast<float*>(smem_bvh);
    int* slink = W.node_f32 ? reinterpret_cast<int*>(sbox32 + 6 * n32) : reinterpret_cast<int*>(sbox + 6 * n64);
    for (int k = threadIdx.x; k < 6 * n64; k += blockDim.x) sbox[k] = S.node_box[k];
    for (int k = threadIdx.x; k < 6 * n32; k += blockDim.x) sbox32[k] = S.node_box32[k];
    for (int k = threadIdx.x; k < 4 * S.smem_nodes; k += blockDim.x) slink[k] = S.node_link[k];
    __syncthreads();
    // Runnable rays of this round: the host's count, or (graph-launched
    // trace) the count the previous round's control kernel left on the device.
    const long long n_run = W.count_dev ? static_cast<long long>(*W.count_dev) : W.n_runnable;
    // Rays per warp: a lane owns a ray, and the warp takes its lanes' stage 1s
    // one (two) at a time, so a warp's share of a round is the sum of its
    // rays' stage-1 work.  In a round with fewer rays than the grid has lanes
    // (the late, small rounds) only the first ray_lanes lanes of each warp
    // take rays (the fewest, a power of two, that still cover the round), so
    // the round is spread over all the grid's warps instead of packed into a
    // few full ones; the other lanes only help with the stage 1s.
    int ray_lanes = 32;
    if (W.adapt_lanes) {
        const long long warps = static_cast<long long>(gridDim.x) * (blockDim.x >> 5);
        const long long per = (n_run + warps - 1) / warps;
        while (ray_lanes > 1 && ray_lanes / 2 >= per) ray_lanes >>= 1;
    }
    if (lane >= ray_lanes) mode = M_DRAINED;
    // Watchdog: a launch that runs far past any real trace (W.watchdog_cycles
    // of SM clock, about 17 s by default) records an error and ends instead
    // of holding the GPU; checked on the first iteration and every 1024th
    // after it.  Both exits of the loop are warp-uniform (this vote and the
    // drained vote at the end of the body).
    const long long t_start = clock64();
    unsigned int iter = 0;
    while (true) {
        if ((++iter & 1023u) == 1u && __any_sync(0xffffffffu, clock64() - t_start > W.watchdog_cycles)) {
            if ((threadIdx.x & 31) == 0) atomicOr(&W.counters[3], 1u);
            break;
        }
        // ---- one unit of work
        if (mode == M_NODE) {
            if (q.sp == 0) {
                mode = M_RESOLVE;
            } else {
                const int ent = stack[--q.sp];
                const int idx = ent & static_cast<int>(kStackIdx);
                const unsigned tag = static_cast<unsigned>(ent) >> 24;
                bool pass = true;
                if (tag == kStackAlways || tag != static_cast<unsigned>(q.best_ver)) {
                    ++cray.node_tests;
                    pass = adv_node_pass(S, r, q, idx, sbox, sbox32, n64, n32, ctr);
                }
                if (pass) {
                    const int* link = idx < S.smem_nodes ? slink + 4 * idx : S.node_link + 4LL * idx;
                    if (link[1] < 0) {
                        q.leaf_start = link[0];
                        q.leaf_count = link[2];
                        q.leaf_k = 0;
                        mode = M_LEAF;
                    } else if (q.sp + 2 > 64) {
                        q.err = BBRT_RAY_STACK_OVERFLOW;
                        q.err_obj = -1;
                        mode = M_RESOLVE;
                    } else if constexpr (!CHILD) {
                        // children tested when popped (tagged to re-test)
                        const int left = link[0], right = link[1];
                        const int el = stack_entry(left, kStackAlways), er = stack_entry(right, kStackAlways);
                        if (q.neg[link[3]]) { stack[q.sp++] = el; stack[q.sp++] = er; }
                        else                { stack[q.sp++] = er; stack[q.sp++] = el; }
                    } else {
                        // both children's boxes now (independent loads); a
                        // child that fails would fail when popped as well
                        const int left = link[0], right = link[1];
                        const bool pl = adv_node_pass(S, r, q, left, sbox, sbox32, n64, n32, ctr);
                        const bool pr = adv_node_pass(S, r, q, right, sbox, sbox32, n64, n32, ctr);
                        cray.node_tests += 2;
                        const unsigned v = static_cast<unsigned>(q.best_ver);
                        if (q.neg[link[3]]) {
                            if (pl) stack[q.sp++] = stack_entry(left, v);
                            if (pr) stack[q.sp++] = stack_entry(right, v);
                        } else {
                            if (pr) stack[q.sp++] = stack_entry(right, v);
                            if (pl) stack[q.sp++] = stack_entry(left, v);
                        }
                    }
                }
            }
        } else if (mode == M_LEAF) {
            if (q.leaf_k >= q.leaf_count) {
                mode = M_NODE;
            } else {
                const int obj = S.leaf_objects[q.leaf_start + q.leaf_k];
                if (S.obj_kind[obj] != BBRT_OBJ_PATCH) {
                    QHit h;
                    if (triangle_intersect(S, S.obj_sub[obj], r.o, r.d, h, cray) && h.t < q.best_t) {
                        q.best_t = h.t;
                        if (q.best_ver < static_cast<int>(kStackAlways)) ++q.best_ver;
                        q.best_obj = obj;
                        q.best_e = -1;
                        q.tri_u = h.u;
                        q.tri_v = h.v;
                    }
                    ++q.leaf_k;
                } else {
                    int e = -1;
                    for (int k = 0; k < nres; ++k)
                        if (W.res_obj[i * kResolved + k] == obj) { e = k; break; }
                    if (e >= 0) {
                        const long long ei = i * kResolved + e;
                        const int err = W.res_err[ei];
                        if (err) {
                            q.err = err;
                            q.err_obj = obj;
                            q.ev0 = W.res_data[ei * kResData + 9];
                            q.ev1 = W.res_data[ei * kResData + 10];
                            mode = M_RESOLVE;
                        } else {
                            const double t = W.res_data[ei * kResData];
                            if (t < q.best_t) {
                                q.best_t = t;
                                if (q.best_ver < static_cast<int>(kStackAlways)) ++q.best_ver;
                                q.best_obj = obj;
                                q.best_e = e;
                            }
                            ++q.leaf_k;
                        }
                    } else if (G > 1 || W.warp_stage1) {
                        // (instances with G > 1 run only with the warp-cooperative
                        // stage 1, so they carry no per-lane stage-1 modes)
                        q.obj = obj;
                        q.pidx = S.obj_sub[obj];
                        mode = M_S1_WARP;
                    } else {
                        q.obj = obj;
                        q.pidx = S.obj_sub[obj];
                        q.s1.have = false;
                        ++cray.patch_tests;
                        if (q.use_cull) {
                            q.bi = 0;
                            q.bj = 0;
                            mode = M_BLOCK;
                        } else {
                            q.ci = 0;
                            mode = M_CELL_ALL;
                        }
                    }
                }
            }
        } else if (G == 1 && mode == M_BLOCK) {
            if (q.bi >= NB) {
                mode = M_S1_DONE;
            } else {
                const float* bb = S.c_block_box + (static_cast<long long>(q.pidx) * NB * NB + q.bi * NB + q.bj) * 6;
                ++cray.cell_tests;
                const bool pass = cull_box(bb, q.cr);
                const int bi = q.bi, bj = q.bj;
                if (++q.bj == NB) { q.bj = 0; ++q.bi; }
                if (pass) {
                    q.ci = bi * B;
                    q.cj = bj * B;
                    q.j0 = q.cj;
                    q.i1 = min(nc, (bi + 1) * B);
                    q.j1 = min(nc, (bj + 1) * B);
                    mode = M_CELL;
                }
            }
        } else if (G == 1 && mode == M_CELL) {
            if (q.ci >= q.i1) {
                mode = M_BLOCK;
            } else {
                const int ci = q.ci, cj = q.cj;
                if (++q.cj == q.j1) { q.cj = q.j0; ++q.ci; }
                ++cray.cell_tests;
                const float* cb = S.c_cell_box + (static_cast<long long>(q.pidx) * nc * nc + ci * nc + cj) * 6;
                if (cull_box(cb, q.cr)) {
                    q.tci = ci;
                    q.tcj = cj;
                    q.tri = 0;
                    q.tri_ret = M_CELL;
                    mode = M_TRI;
                }
            }
        } else if (G == 1 && mode == M_CELL_ALL) {
            if (q.ci >= nc * nc) {
                mode = M_S1_DONE;
            } else {
                q.tci = q.ci / nc;
                q.tcj = q.ci % nc;
                ++q.ci;
                q.tri = 0;
                q.tri_ret = M_CELL_ALL;
                mode = M_TRI;
            }
        } else if (G == 1 && mode == M_TRI) {
            ++cray.tri_tests;
            stage1_tri(S.c_xyz + static_cast<long long>(q.pidx) * n * n * 3,
                       S.c_cell + static_cast<long long>(q.pidx) * nc * nc * 4, n, q.tci, q.tcj, q.tri, r.o, r.d, q.s1);
            if (++q.tri == 6) mode = q.tri_ret;
        } else if (mode == M_S1_DONE) {
            if (!q.s1.have) {
                if (A.samples) record_sample(A, 0, r.o, r.d, q.pidx, 0.0, 0.0, 0.0);
                ++q.leaf_k;
                mode = M_LEAF;
            } else if (nres >= kResolved) {
                mode = M_OVERFLOW;
            } else {
                W.res_obj[i * kResolved + nres] = q.obj;
                rq.ray = static_cast<int>(i);
                rq.entry = nres;
                rq.obj = q.obj;
                rq.key = q.s1.key;
                rq.t0 = q.s1.t;
                mode = M_SUSPEND;
            }
        } else if (mode == M_RESOLVE) {
            ++tally.queries;
            QHit h;
            h.err = q.err;
            h.obj = q.err ? q.err_obj : q.best_obj;
            h.ev0 = q.ev0;
            h.ev1 = q.ev1;
            if (!q.err && q.best_obj >= 0) {
                if (q.best_e >= 0) {
                    const double* rd = W.res_data + (i * kResolved + q.best_e) * kResData;
                    h.t = rd[0];
                    h.p = v3(rd[1], rd[2], rd[3]);
                    h.n = v3(rd[4], rd[5], rd[6]);
                    h.u = rd[7];
                    h.v = rd[8];
                } else {
                    const double* v = S.tri + static_cast<long long>(S.obj_sub[q.best_obj]) * 9;
                    const V3 v0 = load3(v), v1 = load3(v + 3), v2 = load3(v + 6);
                    h.t = q.best_t;
                    h.p = v3(r.o.x + h.t * r.d.x, r.o.y + h.t * r.d.y, r.o.z + h.t * r.d.z);
                    h.n = vnormalize(vcross(vsub(v1, v0), vsub(v2, v0)));
                    h.u = q.tri_u;
                    h.v = q.tri_v;
                }
            }
            nres = 0;
            if (!step_ray(S, A, i, r, h)) {
                mode = M_FINISH;
            } else if (r.bounces >= A.max_bounces) {
                r.status = BBRT_RAY_MAX_BOUNCES;
                mode = M_FINISH;
            } else {
                adv_start_query(S, A, W, r, q, stack);
                mode = M_NODE;
            }
        }
        // Stage 1 of every lane that reached a patch, one patch at a time with
        // all 32 lanes: the block, cell and triangle tests of the patch are
        // split over the lanes and the (t, key) minimum is taken over the warp
        // (the same winner as the lane's own ordered loop).
        // With G > 1 (patches of at most 16 blocks of at most 16 cells), G
        // patches at a time, one per group of 32 / G lanes; the instance keeps
        // the whole-warp path too and checks at run time (measured faster
        // than an instance without it).
        if (G > 1 && W.warp_stage1 && W.half_stage1 && S.n_blocks_side * S.n_blocks_side <= 16 &&
            S.block_cells * S.block_cells <= 16) {
            constexpr int WH = 32 / (G > 1 ? G : 2);
            unsigned pend = __ballot_sync(kFull, mode == M_S1_WARP);
            while (pend) {
                // this pass takes the first G waiting lanes; a group without
                // one repeats the first patch (its result is not used)
                const unsigned batch = pend;
#pragma unroll
                for (int g = 0; g < G; ++g) pend &= pend - 1;
                const int gg = lane / WH;
                const unsigned pos = __fns(batch, 0, gg + 1);
                const int src = pos < 32u ? static_cast<int>(pos) : __ffs(batch) - 1;
                V3 so, sd;
                so.x = __shfl_sync(kFull, r.o.x, src);
                so.y = __shfl_sync(kFull, r.o.y, src);
                so.z = __shfl_sync(kFull, r.o.z, src);
                sd.x = __shfl_sync(kFull, r.d.x, src);
                sd.y = __shfl_sync(kFull, r.d.y, src);
                sd.z = __shfl_sync(kFull, r.d.z, src);
                const int spidx = __shfl_sync(kFull, q.pidx, src);
                const bool scull = __shfl_sync(kFull, q.use_cull ? 1 : 0, src) != 0;
                CullRay scr;
                scr.ox = __shfl_sync(kFull, q.cr.ox, src);
                scr.oy = __shfl_sync(kFull, q.cr.oy, src);
                scr.oz = __shfl_sync(kFull, q.cr.oz, src);
                scr.ix = __shfl_sync(kFull, q.cr.ix, src);
                scr.iy = __shfl_sync(kFull, q.cr.iy, src);
                scr.iz = __shfl_sync(kFull, q.cr.iz, src);
                scr.delta = __shfl_sync(kFull, q.cr.delta, src);
                CountersT<STATS> c2;
                const Stage1 res = group_patch_stage1<WH>(S, spidx, so, sd, scull, scr, lane % WH,
                                                          ((1u << WH) - 1u) << (WH * gg), WH * gg, c2);
                __syncwarp();
#pragma unroll
                for (int hv = 0; hv < (G > 1 ? G : 2); ++hv) {
                    const int leader = WH * hv;
                    const int have = __shfl_sync(kFull, res.have ? 1 : 0, leader);
                    const double st = __shfl_sync(kFull, res.t, leader);
                    const int sk = __shfl_sync(kFull, res.key, leader);
                    long long pt = 0, ct = 0, tt = 0;
                    if constexpr (STATS) {
                        pt = __shfl_sync(kFull, c2.patch_tests, leader);
                        ct = __shfl_sync(kFull, c2.cell_tests, leader);
                        tt = __shfl_sync(kFull, c2.tri_tests, leader);
                    }
                    const unsigned owner = __fns(batch, 0, hv + 1);
                    if (owner < 32u && lane == static_cast<int>(owner)) {
                        q.s1.have = have != 0;
                        q.s1.t = st;
                        q.s1.key = sk;
                        cray.patch_tests += pt;
                        cray.cell_tests += ct;
                        cray.tri_tests += tt;
                        mode = M_S1_DONE;
                    }
                }
            }
        } else if (G > 1 || W.warp_stage1) {
            unsigned pend = __ballot_sync(kFull, mode == M_S1_WARP);
            while (pend) {
                const int src = __ffs(pend) - 1;
                pend &= pend - 1;
                V3 so, sd;
                so.x = __shfl_sync(kFull, r.o.x, src);
                so.y = __shfl_sync(kFull, r.o.y, src);
                so.z = __shfl_sync(kFull, r.o.z, src);
                sd.x = __shfl_sync(kFull, r.d.x, src);
                sd.y = __shfl_sync(kFull, r.d.y, src);
                sd.z = __shfl_sync(kFull, r.d.z, src);
                const int spidx = __shfl_sync(kFull, q.pidx, src);
                const bool scull = __shfl_sync(kFull, q.use_cull ? 1 : 0, src) != 0;
                CullRay scr;
                scr.ox = __shfl_sync(kFull, q.cr.ox, src);
                scr.oy = __shfl_sync(kFull, q.cr.oy, src);
                scr.oz = __shfl_sync(kFull, q.cr.oz, src);
                scr.ix = __shfl_sync(kFull, q.cr.ix, src);
                scr.iy = __shfl_sync(kFull, q.cr.iy, src);
                scr.iz = __shfl_sync(kFull, q.cr.iz, src);
                scr.delta = __shfl_sync(kFull, q.cr.delta, src);
                CountersT<STATS> c2;
                const Stage1 res = warp_patch_stage1(S, spidx, so, sd, scull, scr, lane, c2);
                long long pt = 0, ct = 0, tt = 0;
                if constexpr (STATS) {
                    pt = __shfl_sync(kFull, c2.patch_tests, 0);
                    ct = __shfl_sync(kFull, c2.cell_tests, 0);
                    tt = __shfl_sync(kFull, c2.tri_tests, 0);
                }
                if (lane == src) {
                    q.s1 = res;
                    cray.patch_tests += pt;
                    cray.cell_tests += ct;
                    cray.tri_tests += tt;
                    mode = M_S1_DONE;
                }
            }
        }
        // Only when some lane's ray left its working modes (one vote in the
        // common case): retire suspended / overflowed / finished rays, then
        // let idle lanes fetch the next runnable ray.
        if (__ballot_sync(0xffffffffu, mode >= M_FINISH) == 0u) continue;
        const long long rs = warp_append(&W.counters[0], mode == M_SUSPEND);
        if (rs >= 0) W.req[rs] = rq;
        const long long os = warp_append(&W.counters[1], mode == M_OVERFLOW);
        if (os >= 0) W.overflow[os] = static_cast<int>(i);
        if (mode == M_SUSPEND || mode == M_OVERFLOW || mode == M_FINISH) {
            add_ray_work(A, i, cray);
            ctr.node_tests += cray.node_tests;
            ctr.patch_tests += cray.patch_tests;
            ctr.cell_tests += cray.cell_tests;
            ctr.tri_tests += cray.tri_tests;
            if (mode == M_SUSPEND) {
                save_ray(W, i, r, nres + 1);
                save_query(W, i, q, stack);
            } else if (mode == M_OVERFLOW) {
                save_ray(W, i, r, nres);
            } else {
                finish_ray(A, i, r);
                tally.bounces += r.bounces;
                tally.hist[r.status]++;
            }
            mode = M_IDLE;
        }
        const bool need = (mode == M_IDLE);
        const long long fs = warp_append(&W.counters[2], need);
        if (need) {
            if (fs < n_run) {
                cray = CountersT<STATS>();
                nres = 0;
                if (W.runnable == nullptr) {
                    i = W.order ? W.order[fs] : fs;
                    init_outputs(A, i);
                    r = start_ray(A, i);
                } else {
                    i = W.runnable[fs].ray;
                    r = load_ray(A, W, i, nres);
                }
                mode = M_FINISH;
                if (r.status < 0) {
                    if (W.runnable != nullptr && resume_query(S, A, W, i, r, q, stack)) {
                        mode = M_LEAF;
                    } else if (r.bounces >= A.max_bounces) {
                        r.status = BBRT_RAY_MAX_BOUNCES;
                    } else {
                        adv_start_query(S, A, W, r, q, stack);
                        mode = M_NODE;
                    }
                }
            } else {
                mode = M_DRAINED;
            }
        }
        if (__all_sync(0xffffffffu, mode == M_DRAINED)) break;
    }
    flush_stats(A, ctr, tally);
}

// Newton on patch pidx in the scene's precision mode.
__device__ __forceinline__ int newton_mode(const DScene& S, int pidx, const V3& o, const V3& d, double u, double v,
                                           double t, QHit& h, long long& iters, long long& iters32) {
    if (S.precision == BBRT_PREC_SPLIT) return newton_split(S, pidx, o, d, u, v, t, h, iters, iters32);
    return newton_exact(S, pidx, o, d, u, v, t, h, iters);
}

// Newton solves of one round, one request per thread.  With a learned guess,
// a confident guess is tried first; its root is kept only when it converges
// inside the patch within guess_t_window patch sizes of the stage-1 t, and
// otherwise the solve restarts from the stage-1 triangle (the reference's start).
__device__ __forceinline__ void newton_thread_body(const DScene& S, const TraceArgs& A, const WaveArgs& W,
                                                   long long n_req) {
    if (blockIdx.x * static_cast<long long>(blockDim.x) >= n_req) return;   // graph launch: spare blocks
    const long long j = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    long long iters = 0, iters32 = 0, used = 0, fallback = 0, off = 0;
    if (j < n_req) {
        const NewtonRequest q = W.req[j];
        if (W.next_req) W.next_req[j] = q;
        const V3 o = load3(W.o + 3LL * q.ray);
        const V3 d = load3(W.d + 3LL * q.ray);
        const int pidx = S.obj_sub[q.obj];
        QHit h;
        h.err = 0;
        h.ev0 = h.ev1 = 0.0;
        h.t = 0.0;
        h.p = h.n = v3(0.0, 0.0, 0.0);
        h.u = h.v = 0.0;
        // One solve for every request, from the guess where it is confident
        // (one call site, so requests of both kinds in a warp run together);
        // a second solve from the triangle only for abandoned guesses.
        double su, sv, st;
        key_to_uv(S, q.key, su, sv);
        st = q.t0;
        double win = 0.0;
        if (W.guess) {
            const double* g = W.guess + 4 * j;
            win = W.guess_t_window * W.frame[16LL * pidx + 12];
            if (g[3] > W.guess_min_logit && isfinite(g[0]) && isfinite(g[1]) && fabs(g[2] - q.t0) <= win) {
                used = 1;
                su = g[0];
                sv = g[1];
                st = g[2];
            }
        }
        const QHit h0 = h;
        const int ok = newton_mode(S, pidx, o, d, su, sv, st, h, iters, iters32);
        if (used && !(ok && fabs(h.t - q.t0) <= win)) {
            fallback = 1;
            h = h0;
            double u0, v0;
            key_to_uv(S, q.key, u0, v0);
            newton_mode(S, pidx, o, d, u0, v0, q.t0, h, iters, iters32);
        }
        if (A.off_patch_miss && h.err == BBRT_RAY_NEWTON_DOMAIN &&
            !guess_inside(W.guess ? W.guess + 4 * j : nullptr, W.guess_min_logit)) {
            off = 1;   // not hit: resolved with t = +inf
            h.err = 0;
            h.t = CUDART_INF;
        }
        if (A.samples && h.err == 0) record_sample(A, 1, o, d, pidx, h.u, h.v, h.t);
        // a root outside the patch teaches the network a miss near the edge
        if (A.samples && h.err == BBRT_RAY_NEWTON_DOMAIN) record_sample(A, 0, o, d, pidx, 0.0, 0.0, 0.0);
        const long long e = static_cast<long long>(q.ray) * kResolved + q.entry;
        double* rd = W.res_data + e * kResData;
        rd[0] = h.t; rd[1] = h.p.x; rd[2] = h.p.y; rd[3] = h.p.z;
        rd[4] = h.n.x; rd[5] = h.n.y; rd[6] = h.n.z; rd[7] = h.u; rd[8] = h.v; rd[9] = h.ev0; rd[10] = h.ev1;
        W.res_err[e] = h.err;
        if (A.ray_work) A.ray_work[4LL * q.ray + 3] += iters + iters32;
    }
    if (A.stats) {
        warp_add(A.stats + ST_NEWTON_ITERS, iters);
        warp_add(A.stats + ST_NEWTON_ITERS_FP32, iters32);
        warp_add(A.stats + ST_GUESS_USED, used);
        warp_add(A.stats + ST_GUESS_FALLBACK, fallback);
        warp_add(A.stats + ST_OFF_PATCH, off);
    }
}

// k_newton with 8 lanes per request (patches of at most 8 nodes per axis):
// the same starts, fallbacks and results, bit for bit.
__device__ __forceinline__ void newton_grp_body(const DScene& S, const TraceArgs& A, const WaveArgs& W,
                                                long long n_req) {
    if (blockIdx.x * static_cast<long long>(blockDim.x) / kGroup >= n_req) return;   // graph launch: spare blocks
    const Grp G = make_grp();
    const long long j = (blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x) / kGroup;
    long long iters = 0, iters32 = 0, used = 0, fallback = 0, off = 0;
    if (j < n_req) {   // uniform over the group
        const NewtonRequest q = W.req[j];
        if (W.next_req && G.g == 0) W.next_req[j] = q;
        const V3 o = load3(W.o + 3LL * q.ray);
        const V3 d = load3(W.d + 3LL * q.ray);
        const int pidx = S.obj_sub[q.obj];
        QHit h;
        h.err = 0;
        h.ev0 = h.ev1 = 0.0;
        h.t = 0.0;
        h.p = h.n = v3(0.0, 0.0, 0.0);
        h.u = h.v = 0.0;
        bool done = false;
        if (W.guess) {
            const double* g = W.guess + 4 * j;
            const double win = W.guess_t_window * W.frame[16LL * pidx + 12];
            if (g[3] > W.guess_min_logit && isfinite(g[0]) && isfinite(g[1]) && fabs(g[2] - q.t0) <= win) {
                used = 1;
                QHit hg = h;
                if (grp_newton_mode(S, pidx, o, d, g[0], g[1], g[2], hg, iters, iters32, G) &&
                    fabs(hg.t - q.t0) <= win) {
                    h = hg;
                    done = true;
                } else {
                    fallback = 1;
                }
            }
        }
        if (!done) {
            double u0, v0;
            key_to_uv(S, q.key, u0, v0);
            grp_newton_mode(S, pidx, o, d, u0, v0, q.t0, h, iters, iters32, G);
        }
        if (A.off_patch_miss && h.err == BBRT_RAY_NEWTON_DOMAIN &&
            !guess_inside(W.guess ? W.guess + 4 * j : nullptr, W.guess_min_logit)) {
            off = 1;
            h.err = 0;
            h.t = CUDART_INF;
        }
        if (G.g == 0) {
            if (A.samples && h.err == 0) record_sample(A, 1, o, d, pidx, h.u, h.v, h.t);
            if (A.samples && h.err == BBRT_RAY_NEWTON_DOMAIN) record_sample(A, 0, o, d, pidx, 0.0, 0.0, 0.0);
            const long long e = static_cast<long long>(q.ray) * kResolved + q.entry;
            double* rd = W.res_data + e * kResData;
            rd[0] = h.t; rd[1] = h.p.x; rd[2] = h.p.y; rd[3] = h.p.z;
            rd[4] = h.n.x; rd[5] = h.n.y; rd[6] = h.n.z; rd[7] = h.u; rd[8] = h.v; rd[9] = h.ev0; rd[10] = h.ev1;
            W.res_err[e] = h.err;
            if (A.ray_work) A.ray_work[4LL * q.ray + 3] += iters + iters32;
        }
    }
    if (G.g != 0) iters = iters32 = used = fallback = off = 0;
    if (A.stats) {
        warp_add(A.stats + ST_NEWTON_ITERS, iters);
        warp_add(A.stats + ST_NEWTON_ITERS_FP32, iters32);
        warp_add(A.stats + ST_GUESS_USED, used);
        warp_add(A.stats + ST_GUESS_FALLBACK, fallback);
        warp_add(A.stats + ST_OFF_PATCH, off);
    }
}

__global__ void __launch_bounds__(128) k_newton(DScene S, TraceArgs A, WaveArgs W, long long n_req) {
    if (W.count_dev) n_req = *W.count_dev;
    newton_thread_body(S, A, W, n_req);
}

__global__ void __launch_bounds__(128) k_newton_grp(DScene S, TraceArgs A, WaveArgs W, long long n_req) {
    if (W.count_dev) n_req = *W.count_dev;
    newton_grp_body(S, A, W, n_req);
}

// A round's Newton solves with the solver picked by the round's size: one
// request per thread for a big round (throughput), 8 lanes per request for a
// small one (at most W.newton_group_max requests, and the grid has their
// lanes), whose time is its slowest solve's latency.  Same results bit for
// bit either way.
__global__ void __launch_bounds__(128) k_newton_auto(DScene S, TraceArgs A, WaveArgs W, long long n_req) {
    if (W.count_dev) n_req = *W.count_dev;
    if (n_req <= W.newton_group_max && n_req * kGroup <= static_cast<long long>(gridDim.x) * blockDim.x)
        newton_grp_body(S, A, W, n_req);
    else
        newton_thread_body(S, A, W, n_req);
}

// Finishes rays from their saved state with inline queries (the tail of a
// wavefront trace, and rays whose query overflowed the resolved list).  The
// current bounce's query restarts from the root, so the result is the same.
__global__ void __launch_bounds__(128) k_resume(DScene S, TraceArgs A, WaveArgs W, const NewtonRequest* reqs,
                                                const int* rays, long long n) {
    if (W.count_dev) {
        n = *W.count_dev;
        if (blockIdx.x * static_cast<long long>(blockDim.x) >= n) return;   // graph launch: spare blocks
    }
    const long long slot = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    Counters ctr;
    RayTally tally;
    if (slot < n) {
        const long long i = reqs ? reqs[slot].ray : rays[slot];
        int nres;
        RayCtx r = load_ray(A, W, i, nres);
        run_ray(S, A, i, r, ctr, tally.queries);
        add_ray_work(A, i, ctr);
        finish_ray(A, i, r);
        tally.bounces += r.bounces;
        tally.hist[r.status]++;
    }
    flush_stats(A, ctr, tally, true);
}

// ---- warp-per-ray form: 32 lanes cooperate on one ray ----------------------
//
// Used for the last rays of a wavefront trace, where too few rays are left
// to fill the GPU and one lane per ray would run each ray's long chain of
// dependent queries alone.  Traversal, bookkeeping and Newton run on every
// lane with identical values (the warp stays converged); the stage-1 box and
// triangle tests of a patch are split over the lanes and the winner is the
// (t, key) minimum over the warp, which is what the reference's ordered loop
// keeps for finite t.  Non-finite rays take the ordered per-lane loop.

// BVH::intersect for one ray with a whole warp (every lane returns the same result).
// Nodes [0, staged) are read from the shared-memory copy (sbox, slink).
template <class Ctr>
__device__ QHit warp_bvh_query(const DScene& S, const V3& o, const V3& d, int cull_flag, int lane, Ctr& ctr,
                               const double* sbox, const float* sbox32, const int* slink, int staged, bool node_f32,
                               bool off_patch_miss, int member) {
    QHit best;
    best.obj = -1;
    best.err = 0;
    best.t = CUDART_INF;
    const double inv[3] = { 1.0 / d.x, 1.0 / d.y, 1.0 / d.z };
    const bool neg[3] = { inv[0] < 0.0, inv[1] < 0.0, inv[2] < 0.0 };
    const bool use_cull = cull_ok(S, member, cull_flag, o, d);
    bool node32 = node_f32 && finite3(o) && finite3(d);
    CullRay cr;
    if (use_cull || node32) cr = make_cull_ray(S, member, o, d);
    float e32 = 0.0f;
    if (node32) node32 = node_margin(S, cr, e32);
    double best_t = CUDART_INF;
    int stack[64];
    int sp = 0;
    stack[sp++] = root_node(S, member);
    while (sp > 0) {
        const int idx = stack[--sp];
        if (lane == 0) ++ctr.node_tests;
        const bool in_smem = idx < staged;
        // FP32 node test where it decides (the staged copy then holds FP32 boxes)
        int dec = -1;
        if (node32) dec = node_box_f32(in_smem ? sbox32 + 6 * idx : S.node_box32 + 6LL * idx, cr, e32, best_t);
        if (dec < 0) {
            if (node32 && lane == 0) ++ctr.node_f64;
            dec = ray_box_exact(o, inv, in_smem && !node_f32 ? sbox + 6 * idx : S.node_box + 6LL * idx, best_t);
        }
        if (!dec) continue;
        const int* link = in_smem ? slink + 4 * idx : S.node_link + 4LL * idx;
        if (link[1] < 0) {
            const int start = link[0], count = link[2];
            for (int k = 0; k < count; ++k) {
                const int obj = S.leaf_objects[start + k];
                QHit h;
                h.err = 0;
                h.ev0 = h.ev1 = 0.0;
                int r = 0;
                if (S.obj_kind[obj] == BBRT_OBJ_PATCH) {
                    const int pidx = S.obj_sub[obj];
                    const Stage1 s1 = warp_patch_stage1(S, pidx, o, d, use_cull, cr, lane, ctr);
                    if (s1.have) {
                        double u0, v0;
                        key_to_uv(S, s1.key, u0, v0);
                        long long it = 0;
                        // One ray per warp: the solve is latency-bound, so
                        // when every patch axis has at most 8 nodes each
                        // 8-lane group evaluates it with one node row per lane
                        // (the same result bit for bit; all four groups agree).
                        if (S.max_nodes <= kGroup) r = grp_newton_exact(S, pidx, o, d, u0, v0, s1.t, h, it, make_grp());
                        else r = newton_exact(S, pidx, o, d, u0, v0, s1.t, h, it);
                        if (lane == 0) ctr.newton_iters += it;
                    }
                } else {
                    CountersT<false> dummy;
                    r = triangle_intersect(S, S.obj_sub[obj], o, d, h, dummy);
                }
                if (off_patch_miss && h.err == BBRT_RAY_NEWTON_DOMAIN) {
                    if (lane == 0) ++ctr.off_patch;
                    continue;
                }
                if (h.err) {
                    h.obj = obj;
                    return h;
                }
                if (r && h.t < best_t) {
                    best_t = h.t;
                    best = h;
                    best.obj = obj;
                }
            }
            continue;
        }
        if (sp + 2 > 64) {
            best.err = BBRT_RAY_STACK_OVERFLOW;
            best.obj = -1;
            return best;
        }
        const int left = link[0], right = link[1];
        if (neg[link[3]]) { stack[sp++] = left; stack[sp++] = right; }
        else              { stack[sp++] = right; stack[sp++] = left; }
    }
    return best;
}

// Finishes rays from their saved state, one warp per ray.
// MINB blocks of 128 threads per SM requested from the register allocator;
// the first S.smem_nodes BVH nodes are staged in shared memory.
template <int MINB, bool STATS>
__global__ void __launch_bounds__(128, MINB) k_resume_warp(DScene S, TraceArgs A, WaveArgs W,
                                                           const NewtonRequest* reqs, const int* rays, long long n) {
    extern __shared__ __align__(16) double smem_tail[];
    // staged nodes: FP64 boxes, or FP32 boxes with the FP32 node test, then links
    const bool f32 = W.node_f32 != 0;
    double* sbox = smem_tail;
    float* sbox32 = reinterpret_cast<float*>(smem_tail);
    int* slink = f32 ? reinterpret_cast<int*>(sbox32 + 6 * S.smem_nodes)
                     : reinterpret_cast<int*>(smem_tail + 6 * S.smem_nodes);
    if (f32) {
        for (int k = threadIdx.x; k < 6 * S.smem_nodes; k += blockDim.x) sbox32[k] = S.node_box32[k];
    } else {
        for (int k = threadIdx.x; k < 6 * S.smem_nodes; k += blockDim.x) sbox[k] = S.node_box[k];
    }
    for (int k = threadIdx.x; k < 4 * S.smem_nodes; k += blockDim.x) slink[k] = S.node_link[k];
    __syncthreads();
    if (W.count_dev) n = *W.count_dev;
    const int lane = threadIdx.x & 31;
    const long long warp = (blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x) >> 5;
    const long long n_warps = (static_cast<long long>(gridDim.x) * blockDim.x) >> 5;
    CountersT<STATS> ctr;
    RayTallyT<STATS> tally;
    // The tail's time is that of its slowest warp: rays are handed out one
    // at a time from a counter, so a warp that drew a long chain takes no
    // further rays while others do (a fixed stride when no counter is given).
    unsigned int* next = W.counters ? W.counters + (reqs ? kWcTailNext : kWcOvfNext) : nullptr;
    auto take = [&](long long fixed) -> long long {
        if (!next) return fixed;
        unsigned int v = 0;
        if (lane == 0) v = atomicAdd(next, 1u);
        return static_cast<long long>(__shfl_sync(0xffffffffu, v, 0));
    };
    for (long long slot = take(warp); slot < n; slot = take(slot + n_warps)) {
        const long long i = reqs ? reqs[slot].ray : rays[slot];
        int nres;
        RayCtx r = load_ray(A, W, i, nres);
        CountersT<STATS> c1;
        while (r.status < 0) {
            if (r.bounces >= A.max_bounces) { r.status = BBRT_RAY_MAX_BOUNCES; break; }
            if (lane == 0) ++tally.queries;
            const QHit h = warp_bvh_query(S, r.o, r.d, A.cull, lane, c1, sbox, sbox32, slink, S.smem_nodes, f32,
                                          A.off_patch_miss != 0, r.member);
            if (!step_ray(S, A, i, r, h, lane == 0)) break;
        }
        if (lane == 0) {
            add_ray_work(A, i, c1);
            finish_ray(A, i, r);
            tally.bounces += r.bounces;
            tally.hist[r.status]++;
        }
        ctr.node_tests += c1.node_tests;
        ctr.patch_tests += c1.patch_tests;
        ctr.cell_tests += c1.cell_tests;
        ctr.tri_tests += c1.tri_tests;
        ctr.newton_iters += c1.newton_iters;
        ctr.off_patch += c1.off_patch;
        ctr.node_f64 += c1.node_f64;
    }
    flush_stats(A, ctr, tally, true);
}

// One query per ray: BVH, brute force over all objects, or one object.
__global__ void __launch_bounds__(128) k_query(DScene S, QueryArgs Q) {
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i >= Q.n) return;
    const V3 o = load3(Q.origins + 3 * i);
    const V3 d = load3(Q.dirs + 3 * i);
    Counters ctr;
    QHit r;
    r.obj = -1;
    r.err = 0;
    r.t = 0.0;
    r.p = r.n = v3(0.0, 0.0, 0.0);
    r.u = r.v = r.ev0 = r.ev1 = 0.0;
    const bool use_cull = cull_ok(S, -1, Q.cull, o, d);
    CullRay cr;
    if (use_cull) cr = make_cull_ray(S, -1, o, d);
    if (Q.mode == BBRT_QUERY_BVH) {
        r = bvh_query(S, o, d, Q.cull, ctr);
    } else if (Q.mode == BBRT_QUERY_BRUTE) {
        bool have = false;
        for (int k = 0; k < S.n_objects; ++k) {
            QHit h;
            const int hit = object_intersect(S, k, o, d, use_cull, cr, h, ctr);
            if (h.err) { r = h; r.obj = k; have = false; break; }
            if (hit && (!have || h.t < r.t)) { r = h; r.obj = k; have = true; }
        }
        if (!have && !r.err) r.obj = -1;
    } else {
        QHit h;
        const int hit = object_intersect(S, Q.object, o, d, use_cull, cr, h, ctr);
        if (h.err) { r = h; r.obj = Q.object; }
        else if (hit) { r = h; r.obj = Q.object; }
    }
    bbrt_hit* out = static_cast<bbrt_hit*>(Q.out) + i;
    bbrt_hit w;
    w.t = 0.0;
    for (int k = 0; k < 3; ++k) { w.point[k] = 0.0; w.normal[k] = 0.0; }
    w.uv[0] = w.uv[1] = 0.0;
    w.object = -1;
    w.status = 0;
    w.err_object = -1;
    w.pad_ = 0;
    w.err_value[0] = w.err_value[1] = 0.0;
    if (r.err) {
        w.status = r.err;
        w.err_object = r.obj;
        w.err_value[0] = r.ev0;
        w.err_value[1] = r.ev1;
    } else if (r.obj >= 0) {
        w.t = r.t;
        w.point[0] = r.p.x; w.point[1] = r.p.y; w.point[2] = r.p.z;
        w.normal[0] = r.n.x; w.normal[1] = r.n.y; w.normal[2] = r.n.z;
        w.uv[0] = r.u; w.uv[1] = r.v;
        w.object = r.obj;
    }
    *out = w;
}

// ---- host launchers -------------------------------------------------------
cudaError_t launch_trace(const DScene& S, const TraceArgs& A, cudaStream_t stream, int sm_count) {
    if (A.n <= 0) return cudaSuccess;
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_trace, 128, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    long long blocks = static_cast<long long>(per_sm) * sm_count;
    const long long need = (A.n + 127) / 128;
    if (blocks > need) blocks = need;
    k_trace<<<static_cast<unsigned>(blocks), 128, 0, stream>>>(S, A);
    return cudaGetLastError();
}

// ---- allocation-free trace (bbrt_trace_noalloc) ----------------------------
//
// The fused trace kernel's scratch — its ray counter, its statistics block
// and per-object hit counters — lives in this file-scope device array
// instead of memory allocated per scene or per call: word 0 is the counter,
// words [1, 1 + ST_COUNT) the statistics, words [kNoAllocHeader,
// kNoAllocHeader + n_objects) the hit counters.  One copy exists per device
// that loads the library, for the life of the process.  Host code must not
// use the array's name as a device address; noalloc_scratch() returns the
// address the device sees.
constexpr int kNoAllocHeader = 32;
static_assert(1 + ST_COUNT <= kNoAllocHeader, "the statistics block would overlap the per-object hit counters");
static __device__ __align__(256) unsigned long long g_noalloc_scratch[kNoAllocHeader + BBRT_NOALLOC_MAX_OBJECTS];

// Device address of g_noalloc_scratch on the current device, looked up with
// cudaGetSymbolAddress the first time each device asks.
cudaError_t noalloc_scratch(unsigned long long** out) {
    constexpr int kMaxDevices = 64;
    static std::mutex mu;
    static void* addr[kMaxDevices] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> g(mu);
    if (addr[dev] == nullptr) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        addr[dev] = p;
    }
    *out = static_cast<unsigned long long*>(addr[dev]);
    return cudaSuccess;
}

// Loads, on the current device, everything bbrt_trace_noalloc needs from this
// module: the scratch array's address and the fused trace kernel.  Under lazy
// module loading the first use of either would otherwise load the module
// (which allocates device memory, the array included) inside the first
// allocation-free call; bbrt_scene_upload calls this instead.
cudaError_t noalloc_prepare() {
    unsigned long long* p = nullptr;
    cudaError_t e = noalloc_scratch(&p);
    if (e != cudaSuccess) return e;
    cudaFuncAttributes fa;
    return cudaFuncGetAttributes(&fa, k_trace);
}

// The fused trace kernel with its scratch in g_noalloc_scratch.  Clears the
// words this call uses first, then traces; hit counters (when asked for) are
// copied to the caller's device array and the statistics to `host_stats`.
cudaError_t launch_trace_noalloc(const DScene& S, TraceArgs A, bool count_hits, long long* hit_counts_out,
                                 long long* host_stats, cudaStream_t stream, int sm_count) {
    unsigned long long* scratch = nullptr;
    cudaError_t e = noalloc_scratch(&scratch);
    if (e != cudaSuccess) return e;
    const size_t words = kNoAllocHeader + (count_hits ? static_cast<size_t>(S.n_objects) : 0);
    e = cudaMemsetAsync(scratch, 0, words * sizeof(unsigned long long), stream);
    if (e != cudaSuccess) return e;
    A.work_counter = scratch;
    A.stats = reinterpret_cast<long long*>(scratch + 1);
    A.hit_counts = count_hits ? scratch + kNoAllocHeader : nullptr;
    e = launch_trace(S, A, stream, sm_count);
    if (e != cudaSuccess) return e;
    if (count_hits) {
        e = cudaMemcpyAsync(hit_counts_out, scratch + kNoAllocHeader, sizeof(long long) * S.n_objects,
                            cudaMemcpyDeviceToDevice, stream);
        if (e != cudaSuccess) return e;
    }
    if (host_stats) {
        e = cudaMemcpyAsync(host_stats, scratch + 1, sizeof(long long) * ST_COUNT, cudaMemcpyDeviceToHost, stream);
        if (e != cudaSuccess) return e;
        e = cudaStreamSynchronize(stream);
    }
    return e;
}

size_t wave_bytes_per_ray() {
    return sizeof(double) * 9 + sizeof(int) * 2 + sizeof(int) * 2 * kResolved + sizeof(double) * kResolved * kResData +
           2 * sizeof(NewtonRequest) + sizeof(int) + sizeof(int) * (kQsInt + kSaveStack) + sizeof(double) * 3;
}

// Carves the wavefront workspace for n rays out of `ws` (wave_bytes_per_ray() * n bytes).
void wave_layout(void* ws, long long n, WaveArgs& W, NewtonRequest*& req_a, NewtonRequest*& req_b) {
    char* p = static_cast<char*>(ws);
    auto take = [&](size_t bytes) { char* q = p; p += (bytes + 255) & ~static_cast<size_t>(255); return q; };
    W.o = reinterpret_cast<double*>(take(sizeof(double) * 3 * n));
    W.d = reinterpret_cast<double*>(take(sizeof(double) * 3 * n));
    W.end = reinterpret_cast<double*>(take(sizeof(double) * 3 * n));
    W.bounces = reinterpret_cast<int*>(take(sizeof(int) * n));
    W.nres = reinterpret_cast<int*>(take(sizeof(int) * n));
    W.res_obj = reinterpret_cast<int*>(take(sizeof(int) * kResolved * n));
    W.res_err = reinterpret_cast<int*>(take(sizeof(int) * kResolved * n));
    W.res_data = reinterpret_cast<double*>(take(sizeof(double) * kResolved * kResData * n));
    req_a = reinterpret_cast<NewtonRequest*>(take(sizeof(NewtonRequest) * n));
    req_b = reinterpret_cast<NewtonRequest*>(take(sizeof(NewtonRequest) * n));
    W.overflow = reinterpret_cast<int*>(take(sizeof(int) * n));
    W.qs_int = reinterpret_cast<int*>(take(sizeof(int) * kQsInt * n));
    W.qs_dbl = reinterpret_cast<double*>(take(sizeof(double) * 3 * n));
    W.qs_stack = reinterpret_cast<int*>(take(sizeof(int) * kSaveStack * n));
}

size_t wave_workspace_bytes(long long n) { return wave_bytes_per_ray() * n + 20 * 256; }

template <int NT, int MINB, bool CHILD, int G, bool STATS>
static cudaError_t launch_advance_stats(const DScene& Sl, const TraceArgs& A, const WaveArgs& W, int sm_count,
                                        cudaStream_t stream) {
    const size_t smem = static_cast<size_t>(Sl.smem_nodes) *
                        ((W.node_f32 ? 6 * sizeof(float) : 6 * sizeof(double)) + 4 * sizeof(int));
    cudaError_t e = cudaFuncSetAttribute(k_advance<NT, MINB, CHILD, G, STATS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_advance<NT, MINB, CHILD, G, STATS>, NT, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    // A small round (the late ones) is spread over every SM: with full blocks
    // whose warps take fewer rays each (W.adapt_lanes, see k_advance), else
    // with smaller blocks rather than packed into the first few SMs.
    int threads = NT;
    long long blocks = static_cast<long long>(per_sm) * sm_count;
    if (W.adapt_lanes) {
        const long long need = (W.n_runnable + NT / 32 - 1) / (NT / 32);   // one ray per warp at least
        if (blocks > need) blocks = need;
    } else {
        const long long per_block = (W.n_runnable + static_cast<long long>(per_sm) * sm_count - 1) /
                                    (static_cast<long long>(per_sm) * sm_count);
        if (per_block < NT) threads = static_cast<int>(std::max<long long>(32, (per_block + 31) / 32 * 32));
        const long long need = (W.n_runnable + threads - 1) / threads;
        if (blocks > need) blocks = need;
    }
    k_advance<NT, MINB, CHILD, G, STATS><<<static_cast<unsigned>(blocks), threads, smem, stream>>>(Sl, A, W);
    return cudaGetLastError();
}

// The statistics-free instance unless the call collects statistics or a per-ray work profile.
template <int NT, int MINB, bool CHILD, int G>
static cudaError_t launch_advance_variant(const DScene& Sl, const TraceArgs& A, const WaveArgs& W, int sm_count,
                                          cudaStream_t stream) {
    if (A.stats || A.ray_work) return launch_advance_stats<NT, MINB, CHILD, G, true>(Sl, A, W, sm_count, stream);
    return launch_advance_stats<NT, MINB, CHILD, G, false>(Sl, A, W, sm_count, stream);
}

template <int NT, int MINB>
static cudaError_t launch_advance_shape(const DScene& S, const TraceArgs& A, const WaveArgs& W, int sm_count,
                                        int max_smem_nodes, cudaStream_t stream) {
    DScene Sl = S;
    if (W.node_f32) {
        // 40 instead of 64 bytes a staged node: the same shared memory holds 1.6 x the nodes
        Sl.smem_nodes = static_cast<int>(std::min<long long>(S.n_nodes, max_smem_nodes * 64LL / 40));
    } else if (Sl.smem_nodes > max_smem_nodes) {
        Sl.smem_nodes = max_smem_nodes;
    }
    // Half-warp stage 1 where a patch's blocks and a block's cells fit 16
    // lanes; else child tests when part of the tree stays in global memory.
    // The two together measured slower than either, and on both measured
    // scenes the half-warp stage 1 beat the child tests.
    if (W.child_test > 0) return launch_advance_variant<NT, MINB, true, 1>(Sl, A, W, sm_count, stream);
    const bool half = W.half_stage1 && W.warp_stage1 && S.n_blocks_side * S.n_blocks_side <= 16 &&
                      S.block_cells * S.block_cells <= 16;
    if (half && W.quarter_stage1) return launch_advance_variant<NT, MINB, false, 4>(Sl, A, W, sm_count, stream);
    if (half) return launch_advance_variant<NT, MINB, false, 2>(Sl, A, W, sm_count, stream);
    const bool child = W.child_test < 0 && S.n_nodes > Sl.smem_nodes;
    return child ? launch_advance_variant<NT, MINB, true, 1>(Sl, A, W, sm_count, stream)
                 : launch_advance_variant<NT, MINB, false, 1>(Sl, A, W, sm_count, stream);
}

// Launch shapes of k_advance: 0 = 128 threads x 3 blocks per SM,
// 1 = 256 threads x 2 blocks per SM, 2 = 128 threads x 4 blocks per SM (fewer
// staged nodes), 3 / 4 / 5 / 6 = 512 / 768 / 1024 / 384 threads x 1 block per SM.
cudaError_t launch_advance(const DScene& S, const TraceArgs& A, const WaveArgs& W, int sm_count, int shape,
                           cudaStream_t stream) {
    if (W.n_runnable <= 0) return cudaSuccess;
    switch (shape) {
        case 1: return launch_advance_shape<256, 2>(S, A, W, sm_count, 1536, stream);
        case 2: return launch_advance_shape<128, 4>(S, A, W, sm_count, 864, stream);
        case 3: return launch_advance_shape<512, 1>(S, A, W, sm_count, 3400, stream);
        case 4: return launch_advance_shape<768, 1>(S, A, W, sm_count, 3400, stream);
        case 5: return launch_advance_shape<1024, 1>(S, A, W, sm_count, 3400, stream);
        case 6: return launch_advance_shape<384, 1>(S, A, W, sm_count, 3400, stream);
        default: return launch_advance_shape<128, 3>(S, A, W, sm_count, 1536, stream);
    }
}

// Round control of the graph-launched trace, after each k_advance: the same
// decision the host-driven loop takes from the round's counters.  No requests,
// or a watchdog stop: the rounds end.  At most wave_tail requests: the rounds
// end and the tail kernel finishes those rays.  Otherwise the requests go to
// Newton and become the next round's runnable set; the loop repeats unless
// this was round max_rounds (flagged for the host as an error).  Every
// repetition raises counters[kWcRounds], so the loop ends after at most
// max_rounds rounds whatever the counts.
__global__ void k_wave_decide(unsigned int* c, long long wave_tail, long long max_rounds,
                              cudaGraphConditionalHandle loop) {
    if (threadIdx.x != 0) return;
    const long long n_req = c[0];
    unsigned int next = 0, tail = 0, go = 0;
    if (c[3] == 0u && n_req > 0) {
        if (n_req <= wave_tail) tail = static_cast<unsigned int>(n_req);
        else next = static_cast<unsigned int>(n_req);
    }
    if (next) {
        const unsigned int r = c[kWcRounds] + 1u;
        c[kWcRounds] = r;
        if (static_cast<long long>(r) >= max_rounds) c[kWcBound] = 1u;
        else go = 1u;
    }
    c[kWcNext] = next;
    c[kWcTail] = tail;
    cudaGraphSetConditional(loop, go);
}

cudaError_t launch_wave_decide(unsigned int* counters, long long wave_tail, long long max_rounds,
                               cudaGraphConditionalHandle loop, cudaStream_t stream) {
    k_wave_decide<<<1, 32, 0, stream>>>(counters, wave_tail, max_rounds, loop);
    return cudaGetLastError();
}

cudaError_t launch_newton(const DScene& S, const TraceArgs& A, const WaveArgs& W, long long n_req, cudaStream_t stream) {
    if (n_req <= 0) return cudaSuccess;
    if (S.max_nodes <= kGroup && W.group_newton) {
        const long long threads = n_req * kGroup;
        k_newton_grp<<<static_cast<unsigned>((threads + 127) / 128), 128, 0, stream>>>(S, A, W, n_req);
    } else if (S.max_nodes <= kGroup && W.newton_group_max > 0) {
        const long long threads = std::max(n_req, std::min(n_req, W.newton_group_max) * kGroup);
        k_newton_auto<<<static_cast<unsigned>((threads + 127) / 128), 128, 0, stream>>>(S, A, W, n_req);
    } else {
        k_newton<<<static_cast<unsigned>((n_req + 127) / 128), 128, 0, stream>>>(S, A, W, n_req);
    }
    return cudaGetLastError();
}

cudaError_t launch_resume(const DScene& S, const TraceArgs& A, const WaveArgs& W, const NewtonRequest* reqs,
                          const int* rays, long long n, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    k_resume<<<static_cast<unsigned>((n + 127) / 128), 128, 0, stream>>>(S, A, W, reqs, rays, n);
    return cudaGetLastError();
}

template <int MINB, bool STATS>
static cudaError_t launch_resume_warp_stats(const DScene& S, const TraceArgs& A, const WaveArgs& W,
                                            const NewtonRequest* reqs, const int* rays, long long n, int sm_count,
                                            int max_smem_nodes, cudaStream_t stream) {
    DScene Sl = S;
    if (Sl.smem_nodes > max_smem_nodes) Sl.smem_nodes = max_smem_nodes;
    const size_t smem = static_cast<size_t>(Sl.smem_nodes) *
                        ((W.node_f32 ? 6 * sizeof(float) : 6 * sizeof(double)) + 4 * sizeof(int));
    cudaError_t e = cudaFuncSetAttribute(k_resume_warp<MINB, STATS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_resume_warp<MINB, STATS>, 128, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    long long blocks = static_cast<long long>(per_sm) * sm_count;
    const long long need = (n + 3) / 4;   // four warps (rays) per block
    if (blocks > need) blocks = need;
    k_resume_warp<MINB, STATS><<<static_cast<unsigned>(blocks), 128, smem, stream>>>(Sl, A, W, reqs, rays, n);
    return cudaGetLastError();
}

// The statistics-free instance unless the call collects statistics or a per-ray work profile.
template <int MINB>
static cudaError_t launch_resume_warp_shape(const DScene& S, const TraceArgs& A, const WaveArgs& W,
                                            const NewtonRequest* reqs, const int* rays, long long n, int sm_count,
                                            int max_smem_nodes, cudaStream_t stream) {
    if (A.stats || A.ray_work)
        return launch_resume_warp_stats<MINB, true>(S, A, W, reqs, rays, n, sm_count, max_smem_nodes, stream);
    return launch_resume_warp_stats<MINB, false>(S, A, W, reqs, rays, n, sm_count, max_smem_nodes, stream);
}

// Tail launch shapes (blocks of 128 threads per SM, BVH nodes staged in
// shared memory): 0 = 3 blocks, none staged; 1 = 4 blocks, 768 nodes;
// 2 = 3 blocks, 1024 nodes; 3 = 2 blocks, 1536 nodes.
cudaError_t launch_resume_warp(const DScene& S, const TraceArgs& A, const WaveArgs& W, const NewtonRequest* reqs,
                               const int* rays, long long n, int sm_count, int shape, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    switch (shape) {
        case 1: return launch_resume_warp_shape<4>(S, A, W, reqs, rays, n, sm_count, 768, stream);
        case 2: return launch_resume_warp_shape<3>(S, A, W, reqs, rays, n, sm_count, 1024, stream);
        case 3: return launch_resume_warp_shape<2>(S, A, W, reqs, rays, n, sm_count, 1536, stream);
        default: return launch_resume_warp_shape<3>(S, A, W, reqs, rays, n, sm_count, 0, stream);
    }
}

// ---- BounceMapDriver::run on the device ------------------------------------

// Launch ray r = (point q, direction ti * phi_n + pj) of the sweep
// (BounceMapDriver.hpp:195-237): the point's frame (origin, t1, t2, n) and
// the direction tables come from the host; the expression and its rounding
// (no fused multiply-add in this file) are the reference's.
__global__ void k_bounce_rays(const double* __restrict__ frames, const double* __restrict__ trig, int theta_n,
                              int phi_n, long long n, double* __restrict__ org, double* __restrict__ dir) {
    const long long r = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (r >= n) return;
    const long long dirs_per = static_cast<long long>(theta_n) * phi_n;
    const long long q = r / dirs_per, dk = r % dirs_per;
    const int ti = static_cast<int>(dk / phi_n), pj = static_cast<int>(dk % phi_n);
    const double* F = frames + 12 * q;
    const double m = trig[ti], st_ = trig[theta_n + ti], cp = trig[2 * theta_n + pj], sp = trig[2 * theta_n + phi_n + pj];
    org[3 * r] = F[0];
    org[3 * r + 1] = F[1];
    org[3 * r + 2] = F[2];
    dir[3 * r] = F[3] * st_ * cp + F[6] * st_ * sp + F[9] * m;
    dir[3 * r + 1] = F[4] * st_ * cp + F[7] * st_ * sp + F[10] * m;
    dir[3 * r + 2] = F[5] * st_ * cp + F[8] * st_ * sp + F[11] * m;
}

// Per grid point: the largest bounce count over non-Error directions, the
// number of Error directions, and the first direction reaching the maximum
// (BounceMapDriver.hpp:199-240).
__global__ void k_bounce_reduce(const int* __restrict__ status, const int* __restrict__ bounces, long long points,
                                int dirs_per, int* __restrict__ max_out, int* __restrict__ err_out,
                                int* __restrict__ best_out) {
    const long long q = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (q >= points) return;
    int best = 0, nerr = 0, bdir = -1;
    for (int k = 0; k < dirs_per; ++k) {
        const long long r = q * dirs_per + k;
        const int s = status[r];
        if (s != BBRT_RAY_ESCAPED && s != BBRT_RAY_MAX_BOUNCES) { ++nerr; continue; }
        const int b = bounces[r];
        if (bdir < 0 || b > best) bdir = k;
        best = b > best ? b : best;
    }
    max_out[q] = best;
    err_out[q] = nerr;
    best_out[q] = bdir;
}

cudaError_t launch_bounce_rays(const double* frames, const double* trig, int theta_n, int phi_n, long long n,
                               double* org, double* dir, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    k_bounce_rays<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(frames, trig, theta_n, phi_n, n, org, dir);
    return cudaGetLastError();
}

cudaError_t launch_bounce_reduce(const int* status, const int* bounces, long long points, int dirs_per, int* max_out,
                                 int* err_out, int* best_out, cudaStream_t st) {
    if (points <= 0) return cudaSuccess;
    k_bounce_reduce<<<static_cast<unsigned>((points + 127) / 128), 128, 0, st>>>(status, bounces, points, dirs_per,
                                                                              max_out, err_out, best_out);
    return cudaGetLastError();
}

// Check of the FP32 node test (bbrt_node_test_check): ray i against box i
// with bound t best[i]: out[2i] = ray_box_exact, out[2i + 1] = node_box_f32
// (-2 when the ray's FP32 values are outside the bound's range).
__global__ void k_node_check(DScene S, const double* __restrict__ o, const double* __restrict__ d,
                             const double* __restrict__ best, long long n, const double* __restrict__ boxes,
                             int* __restrict__ out) {
    const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const V3 oo = load3(o + 3 * i), dd = load3(d + 3 * i);
    const double inv[3] = { 1.0 / dd.x, 1.0 / dd.y, 1.0 / dd.z };
    out[2 * i] = ray_box_exact(oo, inv, boxes + 6 * i, best[i]) ? 1 : 0;
    const CullRay c = make_cull_ray(S, -1, oo, dd);
    float e = 0.0f;
    __align__(8) float b32[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) b32[k] = static_cast<float>(boxes[6 * i + k]);
    const bool ok = finite3(oo) && finite3(dd) && node_margin(S, c, e);
    out[2 * i + 1] = ok ? node_box_f32(b32, c, e, best[i]) : -2;
}

cudaError_t launch_node_check(const DScene& S, const double* o, const double* d, const double* best, long long n,
                              const double* boxes, int* out, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    k_node_check<<<static_cast<unsigned>((n + 255) / 256), 256, 0, stream>>>(S, o, d, best, n, boxes, out);
    return cudaGetLastError();
}

cudaError_t launch_query(const DScene& S, const QueryArgs& Q, cudaStream_t stream) {
    if (Q.n <= 0) return cudaSuccess;
    const long long blocks = (Q.n + 127) / 128;
    k_query<<<static_cast<unsigned>(blocks), 128, 0, stream>>>(S, Q);
    return cudaGetLastError();
}

}  // namespace bbrt
