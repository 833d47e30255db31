// Scene compile on the GPU: the per-patch set-up of SurfacePatch's
// constructor — coarse grid, per-cell normal and sagitta, box, centroid,
// padding — and the stage-1 cull boxes, for every patch of a scene at once.
//
// Reference counterparts (manuelarturosantana/BillardBallRayTracing3D):
//   compute_centroid_and_box   include/ScatObjects/SurfacePatch.hpp:380-407
//   compute_coarse_grid        :416-436 (lagrange_interpolation_2D,
//                                        Utils/PatchInterpolation.hpp:54-159)
//   compute_cell_padding       :446-492 (lagrange_basis_1d :518-538,
//                                        eval_scalar_field :542-555)
//
// The host compiler (scene_host.cpp setup_patch, build_cull_tables) computes
// the same values; this file restates each of its expressions in the same
// operand order and is compiled with -fmad=false, so every double (and every
// outward-rounded float of the cull boxes) equals the host's bit for bit:
// IEEE FP64 + - * / and sqrt are correctly rounded on the device as on the
// host, and nothing is contracted into an FMA.  The dgemm order of the
// reference's coarse-grid interpolation is the one the host uses (a left to
// right sum over k, then over m).
//
// One CTA per patch (grid-stride over patches): the patch's node tables and
// position / normal fields are staged in shared memory; threads take coarse
// vertices, then cells, then cull boxes, then cull blocks, with a barrier
// between the phases (each phase reads what the previous one wrote).
#include <cuda_runtime.h>
#include <math_constants.h>

#include <algorithm>

#include "dscene.h"
#include "scene_compile.h"

namespace bbrt {
namespace {

constexpr int kSetupThreads = 128;
constexpr int kMaxN = 16;                  // nodes per axis (scene_host.hpp kMaxNodes)
constexpr int kFieldsPerNode = 12;         // x y z, X_u, X_v, normal (scene_host.hpp kFields)
constexpr double kTol = 1.0e-12;           // EQUAL_TOL, Utils/PatchInterpolation.hpp:21

__device__ __forceinline__ double dmin_(double a, double b) { return (b < a) ? b : a; }   // std::min(a, b)
__device__ __forceinline__ double dmax_(double a, double b) { return (a < b) ? b : a; }   // std::max(a, b)
__device__ __forceinline__ float fmin_(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float fmax_(float a, float b) { return (a < b) ? b : a; }

// First-form Lagrange row at t: w_j / (t - x_j) and the scale prod (t - x_j);
// a node within kTol gives a one-hot row and scale 1.
__device__ __forceinline__ void first_form_row(const double* x, const double* w, int n, double t, double* row,
                                               double& scale) {
    double prod = 1.0;
    int hit = -1;
    for (int j = 0; j < n; ++j) {
        const double diff = t - x[j];
        if (fabs(diff) < kTol) { hit = j; break; }
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

// Second-form basis at t, normalised by the sum of the w_i / (t - x_i).
__device__ __forceinline__ void second_form_basis(const double* x, const double* w, int n, double t, double* b) {
    for (int i = 0; i < n; ++i) b[i] = 0.0;
    for (int i = 0; i < n; ++i)
        if (fabs(t - x[i]) < kTol) { b[i] = 1.0; return; }
    double denom = 0.0;
    for (int i = 0; i < n; ++i) {
        const double li = w[i] / (t - x[i]);
        b[i] = li;
        denom += li;
    }
    for (int i = 0; i < n; ++i) b[i] /= denom;
}

// sum_i bu_i * (sum_j bv_j f_ij), rows with bu_i == 0 skipped.
__device__ __forceinline__ double tensor_eval(const double* f, int I, int J, const double* bu, const double* bv) {
    double sum = 0.0;
    for (int i = 0; i < I; ++i) {
        const double li = bu[i];
        if (li == 0.0) continue;
        const double* r = f + i * J;
        double rs = 0.0;
        for (int j = 0; j < J; ++j) rs += bv[j] * r[j];
        sum += li * rs;
    }
    return sum;
}

__device__ __forceinline__ double block_max(double v, double* red) {
    // non-NaN inputs (each thread's running dmax_ starts from a non-NaN value)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[w] = v;
    __syncthreads();
    double r = red[0];
    for (int k = 1; k < nw; ++k) r = fmax(r, red[k]);
    return r;
}

__global__ void __launch_bounds__(kSetupThreads) k_patch_setup(SetupArgs A) {
    __shared__ double s_nodes[4 * kMaxN];                       // un, vn, uw, vw
    __shared__ double s_f[6][kMaxN * kMaxN];                    // x y z, nu_x nu_y nu_z (row-major i * J + j)
    __shared__ double s_red[kSetupThreads / 32];
    __shared__ double s_lo[3], s_hi[3], s_cen[3];
    const int tid = threadIdx.x;
    const int cn = A.cn, nc = cn - 1;
    const long long cnn = static_cast<long long>(cn) * cn;
    for (int q = blockIdx.x; q < A.n_patches; q += gridDim.x) {
        const int I = A.dims[2 * q], J = A.dims[2 * q + 1];
        const int nn = I * J;
        const double* nd = A.nodes + A.node_off[q];
        const double* fl = A.fields + A.field_off[q];
        __syncthreads();   // the previous patch's readers are done with shared memory
        for (int k = tid; k < 2 * (I + J); k += blockDim.x) {
            // un[I] vn[J] uw[I] vw[J] -> s_nodes at 0, kMaxN, 2 kMaxN, 3 kMaxN
            int dst;
            if (k < I) dst = k;
            else if (k < I + J) dst = kMaxN + (k - I);
            else if (k < 2 * I + J) dst = 2 * kMaxN + (k - I - J);
            else dst = 3 * kMaxN + (k - 2 * I - J);
            s_nodes[dst] = nd[k];
        }
        for (int k = tid; k < 6 * nn; k += blockDim.x) {
            const int c = k / nn, node = k % nn;
            const int fi = c < 3 ? c : 9 + (c - 3);
            s_f[c][node] = fl[static_cast<long long>(node) * kFieldsPerNode + fi];
        }
        __syncthreads();
        const double* un = s_nodes;
        const double* vn = s_nodes + kMaxN;
        const double* uw = s_nodes + 2 * kMaxN;
        const double* vw = s_nodes + 3 * kMaxN;

        // centroid = mean of the nodes (summed in node order); node AABB
        if (tid == 0) {
            double sx = 0.0, sy = 0.0, sz = 0.0;
            double lo[3] = { CUDART_INF, CUDART_INF, CUDART_INF }, hi[3] = { -CUDART_INF, -CUDART_INF, -CUDART_INF };
            for (int i = 0; i < nn; ++i) {
                const double p[3] = { s_f[0][i], s_f[1][i], s_f[2][i] };
                sx += p[0];
                sy += p[1];
                sz += p[2];
                for (int a = 0; a < 3; ++a) {
                    lo[a] = dmin_(lo[a], p[a]);
                    hi[a] = dmax_(hi[a], p[a]);
                }
            }
            const double inv_n = 1.0 / static_cast<double>(nn);
            s_cen[0] = sx * inv_n;
            s_cen[1] = sy * inv_n;
            s_cen[2] = sz * inv_n;
            for (int a = 0; a < 3; ++a) { s_lo[a] = lo[a]; s_hi[a] = hi[a]; }
        }

        // coarse grid: out(i, j) = (sum_m (sum_k ru_ik f_km) rv_jm) * (su_i * sv_j), per coordinate
        double* X = A.c_xyz + static_cast<long long>(q) * cnn * 3;
        for (long long t = tid; t < 3 * cnn; t += blockDim.x) {
            const int c = static_cast<int>(t / cnn);
            const int r = static_cast<int>(t % cnn);
            const int i = r / cn, j = r % cn;
            double ru[kMaxN], rv[kMaxN], su, sv;
            for (int k = 0; k < kMaxN; ++k) { ru[k] = 0.0; rv[k] = 0.0; }
            first_form_row(un, uw, I, A.coarse_uv[i], ru, su);
            first_form_row(vn, vw, J, A.coarse_uv[j], rv, sv);
            const double* f = s_f[c];
            double s2 = 0.0;
            for (int m = 0; m < J; ++m) {
                double s = 0.0;
                for (int k = 0; k < I; ++k) s += ru[k] * f[k * J + m];
                s2 += (1.0 * s) * rv[m];
            }
            X[3LL * r + c] = (1.0 * s2) * (su * sv);
        }
        __syncthreads();   // the coarse vertices are read by the cells below

        // per-cell sagitta at the parameter midpoint and the unit normal there
        double* CC = A.c_cell + static_cast<long long>(q) * nc * nc * 4;
        double ms = 0.0;
        for (int t = tid; t < nc * nc; t += blockDim.x) {
            const int i = t / nc, j = t % nc;
            const double um = 0.5 * (A.coarse_uv[i] + A.coarse_uv[i + 1]);
            const double vm = 0.5 * (A.coarse_uv[j] + A.coarse_uv[j + 1]);
            double bu[kMaxN], bv[kMaxN];
            second_form_basis(un, uw, I, um, bu);
            second_form_basis(vn, vw, J, vm, bv);
            double mid[3], nrm[3];
            for (int c = 0; c < 3; ++c) mid[c] = tensor_eval(s_f[c], I, J, bu, bv);
            for (int c = 0; c < 3; ++c) nrm[c] = tensor_eval(s_f[3 + c], I, J, bu, bv);
            const double nl = sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
            const long long k00 = static_cast<long long>(i) * cn + j, k10 = k00 + cn, k01 = k00 + 1, k11 = k00 + cn + 1;
            double df[3];
            for (int c = 0; c < 3; ++c) {
                const double bil = 0.25 * (X[3 * k00 + c] + X[3 * k10 + c] + X[3 * k01 + c] + X[3 * k11 + c]);
                df[c] = mid[c] - bil;
            }
            const double sag = sqrt(df[0] * df[0] + df[1] * df[1] + df[2] * df[2]);
            double* cell = CC + 4LL * t;
            cell[0] = nrm[0] / nl;
            cell[1] = nrm[1] / nl;
            cell[2] = nrm[2] / nl;
            cell[3] = sag;
            ms = dmax_(ms, sag);
        }
        ms = block_max(ms, s_red);   // also the barrier after the cells' writes
        if (tid == 0) {
            double* po = A.patch_out + 10LL * q;
            for (int a = 0; a < 3; ++a) {
                po[a] = s_lo[a] - ms;
                po[3 + a] = s_hi[a] + ms;
                po[6 + a] = s_cen[a];
            }
            po[9] = ms;
        }
        if (!A.cell_box) continue;

        // cull boxes: AABB of each cell's twelve offset corners, rounded outward
        float* CB = A.cell_box + static_cast<long long>(q) * nc * nc * 6;
        double hmax = 0.0, cmax = 0.0;
        int finite = 1;
        for (int t = tid; t < nc * nc; t += blockDim.x) {
            const int i = t / nc, j = t % nc;
            const double* p[4] = { X + 3LL * (i * cn + j), X + 3LL * ((i + 1) * cn + j), X + 3LL * (i * cn + j + 1),
                                   X + 3LL * ((i + 1) * cn + j + 1) };   // p00 p10 p01 p11
            const double* c = CC + 4LL * t;
            double lo[3] = { CUDART_INF, CUDART_INF, CUDART_INF }, hi[3] = { -CUDART_INF, -CUDART_INF, -CUDART_INF };
            for (int k = 0; k < 3; ++k) {
                const double sg = (k == 0) ? 0.0 : ((k == 1) ? 1.0 : -1.0);
                const double dd = sg * c[3];
                double qv[4][3];
                for (int r = 0; r < 4; ++r)
                    for (int a = 0; a < 3; ++a) {
                        qv[r][a] = p[r][a] + c[a] * dd;
                        lo[a] = dmin_(lo[a], qv[r][a]);
                        hi[a] = dmax_(hi[a], qv[r][a]);
                        finite = finite && isfinite(qv[r][a]);
                        cmax = dmax_(cmax, fabs(qv[r][a]));
                    }
                const int ends[3] = { 1, 3, 2 };
                for (int e : ends) {
                    const double dx = qv[e][0] - qv[0][0], dy = qv[e][1] - qv[0][1], dz = qv[e][2] - qv[0][2];
                    hmax = dmax_(hmax, sqrt(dx * dx + dy * dy + dz * dz));
                }
            }
            float* box = CB + 6LL * t;
            for (int a = 0; a < 3; ++a) {
                box[a] = __double2float_rd(lo[a]);
                box[3 + a] = __double2float_ru(hi[a]);
            }
        }
        const double hm = block_max(hmax, s_red);
        const double cm = block_max(cmax, s_red);
        const int fin = __syncthreads_and(finite);
        if (tid == 0) {
            double* cs = A.cull_stats + 3LL * q;
            cs[0] = hm;
            cs[1] = cm;
            cs[2] = fin ? 1.0 : 0.0;
        }
        // block boxes: the union of their cells' boxes, cells taken in row-major order
        const int B = A.block_cells, NB = A.n_blocks_side;
        float* BBx = A.block_box + static_cast<long long>(q) * NB * NB * 6;
        for (int kb = tid; kb < NB * NB; kb += blockDim.x) {
            const int bi = kb / NB, bj = kb % NB;
            float lo[3] = { CUDART_INF_F, CUDART_INF_F, CUDART_INF_F }, hi[3] = { -CUDART_INF_F, -CUDART_INF_F, -CUDART_INF_F };
            for (int i = bi * B; i < min(nc, (bi + 1) * B); ++i)
                for (int j = bj * B; j < min(nc, (bj + 1) * B); ++j) {
                    const float* box = CB + 6LL * (i * nc + j);
                    for (int a = 0; a < 3; ++a) {
                        lo[a] = fmin_(lo[a], box[a]);
                        hi[a] = fmax_(hi[a], box[3 + a]);
                    }
                }
            for (int a = 0; a < 3; ++a) {
                BBx[6 * kb + a] = lo[a];
                BBx[6 * kb + 3 + a] = hi[a];
            }
        }
    }
}

}  // namespace

cudaError_t launch_patch_setup(const SetupArgs& A, int sm_count, cudaStream_t st) {
    if (A.n_patches <= 0) return cudaSuccess;
    const long long blocks = std::min<long long>(A.n_patches, 16LL * sm_count);
    k_patch_setup<<<static_cast<unsigned>(blocks), kSetupThreads, 0, st>>>(A);
    return cudaGetLastError();
}

}  // namespace bbrt
