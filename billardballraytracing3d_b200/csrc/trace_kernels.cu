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

#include "../../include/bbrt.h"
#include "exact.cuh"

namespace bbrt {

struct Counters {
    long long node_tests = 0, patch_tests = 0, cell_tests = 0, tri_tests = 0, newton_iters = 0;
};

// Per-ray data of the FP32 cull test (computed once per query).
struct CullRay {
    float ox, oy, oz, ix, iy, iz, delta;
};

__device__ __forceinline__ bool finite3(const V3& a) {
    return isfinite(a.x) && isfinite(a.y) && isfinite(a.z);
}

// The cull inflation bound is derived for |d| <= 1 (the trace loop always
// normalises d); single queries with longer or non-finite rays skip culling.
__device__ __forceinline__ bool cull_ok(const DScene& S, int cull_flag, const V3& o, const V3& d) {
    return cull_flag && S.cull_enabled && finite3(o) && finite3(d) &&
           d.x * d.x + d.y * d.y + d.z * d.z <= 1.0 + 1e-6;
}

__device__ __forceinline__ CullRay make_cull_ray(const DScene& S, const V3& o, const V3& d) {
    CullRay c;
    const double cx = o.x - S.cull_center[0], cy = o.y - S.cull_center[1], cz = o.z - S.cull_center[2];
    const double L = sqrt(cx * cx + cy * cy + cz * cz) + S.cull_radius;
    const double on = sqrt(o.x * o.x + o.y * o.y + o.z * o.z);
    const double delta = S.cull_a * (L + S.cull_h) + S.cull_b * (L + on + S.cull_coord);
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
__device__ __forceinline__ bool cull_box(const float* __restrict__ b, const CullRay& c) {
    float t1 = (b[0] - c.delta - c.ox) * c.ix, t2 = (b[3] + c.delta - c.ox) * c.ix;
    float tmin = fmaxf(0.0f, fminf(t1, t2)), tmax = fmaxf(t1, t2);
    t1 = (b[1] - c.delta - c.oy) * c.iy; t2 = (b[4] + c.delta - c.oy) * c.iy;
    tmin = fmaxf(tmin, fminf(t1, t2)); tmax = fminf(tmax, fmaxf(t1, t2));
    t1 = (b[2] - c.delta - c.oz) * c.iz; t2 = (b[5] + c.delta - c.oz) * c.iz;
    tmin = fmaxf(tmin, fminf(t1, t2)); tmax = fminf(tmax, fmaxf(t1, t2));
    return tmin <= tmax;
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

// SurfacePatch::intersect: stage 1 over the coarse triangulation (all cells,
// or only cells whose inflated box the ray crosses), then Newton from the
// winning triangle's (u, v) centroid and its t.
__device__ __forceinline__ int patch_intersect(const DScene& S, int pidx, const V3& o, const V3& d, bool use_cull,
                               const CullRay& cr, QHit& h, Counters& ctr) {
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
    if (!best.have) return 0;
    const int cell = best.key / 6;
    const bool second = (best.key & 1) != 0;
    const int bi = cell / nc, bj = cell % nc;
    const double ui = S.coarse_uv[bi], ui1 = S.coarse_uv[bi + 1];
    const double vj = S.coarse_uv[bj], vj1 = S.coarse_uv[bj + 1];
    double u0, v0;
    if (!second) { u0 = (ui + ui1 + ui1) / 3.0; v0 = (vj + vj + vj1) / 3.0; }
    else         { u0 = (ui + ui + ui1) / 3.0; v0 = (vj + vj1 + vj1) / 3.0; }
    return newton_exact(S, pidx, o, d, u0, v0, best.t, h, ctr.newton_iters);
}

// ScatObject::intersect for object `obj`: 1 hit, 0 miss (h.err set on a
// Newton failure).
__device__ __forceinline__ int object_intersect(const DScene& S, int obj, const V3& o, const V3& d, bool use_cull,
                                                const CullRay& cr, QHit& h, Counters& ctr) {
    h.err = 0;
    const int sub = S.obj_sub[obj];
    if (S.obj_kind[obj] == BBRT_OBJ_PATCH) return patch_intersect(S, sub, o, d, use_cull, cr, h, ctr);
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

// BVH::intersect with a 64-entry stack.  Returns the closest hit (obj >= 0),
// a miss (obj < 0, err 0), or the first Newton failure met (err != 0).
__device__ QHit bvh_query(const DScene& S, const V3& o, const V3& d, int cull_flag, Counters& ctr) {
    QHit best;
    best.obj = -1;
    best.err = 0;
    best.t = CUDART_INF;
    const double inv[3] = { 1.0 / d.x, 1.0 / d.y, 1.0 / d.z };
    const bool neg[3] = { inv[0] < 0.0, inv[1] < 0.0, inv[2] < 0.0 };
    const bool use_cull = cull_ok(S, cull_flag, o, d);
    CullRay cr;
    if (use_cull) cr = make_cull_ray(S, o, d);
    double best_t = CUDART_INF;
    int stack[64];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
        const int idx = stack[--sp];
        ++ctr.node_tests;
        if (!ray_box_exact(o, inv, S.node_box + 6LL * idx, best_t)) continue;
        const int* link = S.node_link + 4LL * idx;
        const int right = link[0];
        if (right < 0) {
            const int start = link[1], count = link[2];
            for (int k = 0; k < count; ++k) {
                const int obj = S.leaf_objects[start + k];
                QHit h;
                const int r = object_intersect(S, obj, o, d, use_cull, cr, h, ctr);
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
        const int left = idx + 1;
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

// The bounce loop for one ray (RayTracingDriver::trace_ray).
__device__ void trace_one(const DScene& S, const TraceArgs& A, long long i, Counters& ctr, long long& bounces_out,
                          long long& queries_out, int& status_out) {
    const V3 origin = load3(A.origins + 3 * i);
    const V3 dir_in = load3(A.dirs + 3 * i);
    const int K = A.record;
    for (int k = 0; k < K; ++k) {
        if (A.hit_object) A.hit_object[i * K + k] = -1;
        if (A.hit_point) { double* p = A.hit_point + (i * K + k) * 3; p[0] = 0.0; p[1] = 0.0; p[2] = 0.0; }
        if (A.hit_uv) { double* p = A.hit_uv + (i * K + k) * 2; p[0] = 0.0; p[1] = 0.0; }
    }
    int status = BBRT_RAY_MAX_BOUNCES, bounces = 0, err_obj = -1;
    long long queries = 0;
    double ev0 = 0.0, ev1 = 0.0;
    V3 end = origin;
    V3 d = v3(0.0, 0.0, 0.0);
    const double len2 = dir_in.x * dir_in.x + dir_in.y * dir_in.y + dir_in.z * dir_in.z;
    if (len2 < 1e-300) {
        status = BBRT_RAY_BAD_DIR;
    } else {
        const double len = sqrt(dir_in.x * dir_in.x + dir_in.y * dir_in.y + dir_in.z * dir_in.z);
        d = v3(dir_in.x / len, dir_in.y / len, dir_in.z / len);
        V3 o = origin;
        status = BBRT_RAY_MAX_BOUNCES;
        for (int b = 0; b < A.max_bounces; ++b) {
            ++queries;
            const QHit h = bvh_query(S, o, d, A.cull, ctr);
            if (h.err) {
                status = h.err;
                err_obj = h.obj;
                ev0 = h.ev0;
                ev1 = h.ev1;
                break;
            }
            if (h.obj < 0) {
                status = BBRT_RAY_ESCAPED;
                end = v3(o.x + d.x * S.scene_diagonal, o.y + d.y * S.scene_diagonal, o.z + d.z * S.scene_diagonal);
                break;
            }
            if (vdot(d, h.n) > S.backface_tol) { status = BBRT_RAY_WENT_INSIDE; break; }
            if (bounces < K) {
                if (A.hit_object) A.hit_object[i * K + bounces] = h.obj;
                if (A.hit_point) {
                    double* p = A.hit_point + (i * K + bounces) * 3;
                    p[0] = h.p.x; p[1] = h.p.y; p[2] = h.p.z;
                }
                if (A.hit_uv) { double* p = A.hit_uv + (i * K + bounces) * 2; p[0] = h.u; p[1] = h.v; }
            }
            if (A.hit_counts && bounces >= A.count_from) atomicAdd(A.hit_counts + h.obj, 1ULL);
            ++bounces;
            end = h.p;
            const double dn = d.x * h.n.x + d.y * h.n.y + d.z * h.n.z;
            d = v3(d.x - 2.0 * dn * h.n.x, d.y - 2.0 * dn * h.n.y, d.z - 2.0 * dn * h.n.z);
            const double eps = smax(S.eps_factor * S.scene_diagonal, S.sag_factor * S.obj_pad[h.obj]);
            o = v3(h.p.x + d.x * eps, h.p.y + d.y * eps, h.p.z + d.z * eps);
        }
    }
    if (A.status) A.status[i] = status;
    if (A.bounce_count) A.bounce_count[i] = bounces;
    if (A.exit_dir) { double* p = A.exit_dir + 3 * i; p[0] = d.x; p[1] = d.y; p[2] = d.z; }
    if (A.end_point) { double* p = A.end_point + 3 * i; p[0] = end.x; p[1] = end.y; p[2] = end.z; }
    if (A.err_object) A.err_object[i] = err_obj;
    if (A.err_value) { A.err_value[2 * i] = ev0; A.err_value[2 * i + 1] = ev1; }
    bounces_out = bounces;
    queries_out = queries;
    status_out = status;
}

// Persistent trace kernel: warps pull 32-ray batches until none are left.
__global__ void __launch_bounds__(128) k_trace(DScene S, TraceArgs A) {
    Counters ctr;
    long long bounces = 0, queries = 0;
    long long hist[BBRT_RAY_STATUS_COUNT];
#pragma unroll
    for (int k = 0; k < BBRT_RAY_STATUS_COUNT; ++k) hist[k] = 0;
    const int lane = threadIdx.x & 31;
    while (true) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(A.work_counter, 32ULL);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= static_cast<unsigned long long>(A.n)) break;
        const long long i = static_cast<long long>(base) + lane;
        if (i < A.n) {
            long long b = 0, q = 0;
            int st = 0;
            trace_one(S, A, i, ctr, b, q, st);
            bounces += b;
            queries += q;
            hist[st]++;
        }
    }
    if (A.stats) {
        warp_add(A.stats + ST_BOUNCES, bounces);
        warp_add(A.stats + ST_QUERIES, queries);
        warp_add(A.stats + ST_NODE_TESTS, ctr.node_tests);
        warp_add(A.stats + ST_PATCH_TESTS, ctr.patch_tests);
        warp_add(A.stats + ST_CELL_TESTS, ctr.cell_tests);
        warp_add(A.stats + ST_TRI_TESTS, ctr.tri_tests);
        warp_add(A.stats + ST_NEWTON_ITERS, ctr.newton_iters);
#pragma unroll
        for (int k = 0; k < BBRT_RAY_STATUS_COUNT; ++k) warp_add(A.stats + ST_HIST0 + k, hist[k]);
    }
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
    const bool use_cull = cull_ok(S, Q.cull, o, d);
    CullRay cr;
    if (use_cull) cr = make_cull_ray(S, o, d);
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

cudaError_t launch_query(const DScene& S, const QueryArgs& Q, cudaStream_t stream) {
    if (Q.n <= 0) return cudaSuccess;
    const long long blocks = (Q.n + 127) / 128;
    k_query<<<static_cast<unsigned>(blocks), 128, 0, stream>>>(S, Q);
    return cudaGetLastError();
}

}  // namespace bbrt
