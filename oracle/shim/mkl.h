/* Stand-in for the one Intel MKL routine the reference calls.
 *
 * Test infrastructure only: this header lets the reference's own sources
 * (include/Utils/PatchInterpolation.hpp:16,148-149) compile into the
 * reference oracle under oracle/_ref.  MKL itself (pinned to mkl2023.2.0 by
 * SLURM/launch_raytrace.sh:17) is not available here.
 *
 * Semantics: the published BLAS dgemm, C = alpha * op(A) * op(B) + beta * C,
 * row-major only.  Summation order is fixed: for each C[i][j] the K products
 * are accumulated left to right into a zero-initialised double, then scaled by
 * alpha (and beta * C added when beta != 0).  The product's host scene
 * compiler (billardballraytracing3d_b200/csrc/scene_host.cpp) uses exactly
 * this order, so both see bit-identical coarse grids.  MKL's own blocking may
 * differ from this in the last ulp; no reference test pins that boundary.
 */
#pragma once
#include <stdio.h>
#include <stdlib.h>

typedef enum { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_LAYOUT;
typedef enum { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE;

static inline void cblas_dgemm(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb,
                               int M, int N, int K, double alpha,
                               const double* A, int lda, const double* B, int ldb,
                               double beta, double* C, int ldc) {
    if (layout != CblasRowMajor) {
        fprintf(stderr, "oracle mkl shim: only CblasRowMajor is supported\n");
        abort();
    }
    for (int i = 0; i < M; ++i) {
        for (int j = 0; j < N; ++j) {
            double s = 0.0;
            for (int k = 0; k < K; ++k) {
                const double a = (ta == CblasNoTrans) ? A[(long)i * lda + k] : A[(long)k * lda + i];
                const double b = (tb == CblasNoTrans) ? B[(long)k * ldb + j] : B[(long)j * ldb + k];
                s += a * b;
            }
            double* c = &C[(long)i * ldc + j];
            *c = (beta == 0.0) ? alpha * s : alpha * s + beta * (*c);
        }
    }
}
