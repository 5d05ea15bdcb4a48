// exact_lu.cuh -- cone coordinates by an explicitly rounded 3x3 LU (shared
// by the tree assignment and the remesh step).
#pragma once
#include "device_common.cuh"

namespace fss {

// Unnormalised cone coordinates of p in the triangle (v1, v2, v3): the 3x3
// system [v1 v2 v3] c = p solved by LU with partial pivoting in LAPACK
// dgetf2/dgetrs order (helpers.h:137-150 barycoords via dgesv_).  Every
// operation is an explicitly rounded intrinsic, so no multiply-add is fused
// and the result is bit-identical to the host FP64 arithmetic.  Returns true
// when a pivot is exactly zero (then b = p, as dgesv_ leaves it).
__device__ __forceinline__ bool cone_coords_exact(const double* v1, const double* v2, const double* v3,
                                                  const double* p, double* b) {
    double a[9] = {v1[0], v1[1], v1[2], v2[0], v2[1], v2[2], v3[0], v3[1], v3[2]};  // a[i + 3j]
    b[0] = p[0]; b[1] = p[1]; b[2] = p[2];
    int ipiv[3];
    bool singular = false;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        int pr = k;
        double mx = fabs(a[k + 3 * k]);
#pragma unroll
        for (int i = k + 1; i < 3; i++)
            if (fabs(a[i + 3 * k]) > mx) { mx = fabs(a[i + 3 * k]); pr = i; }
        ipiv[k] = pr;
        // mx is |a[pr + 3k]|, so this is the test a[pr + 3k] == 0 (NaN fails both)
        if (mx == 0.0) { singular = true; continue; }
        // row swap written with compile-time indices only, so a[] stays in
        // registers (a run-time row index would put the matrix in local memory)
#pragma unroll
        for (int i = k + 1; i < 3; i++) {
            if (pr == i) {
#pragma unroll
                for (int j = 0; j < 3; j++) { double t = a[k + 3 * j]; a[k + 3 * j] = a[i + 3 * j]; a[i + 3 * j] = t; }
            }
        }
        const double r = __drcp_rn(a[k + 3 * k]);
#pragma unroll
        for (int i = k + 1; i < 3; i++) a[i + 3 * k] = __dmul_rn(a[i + 3 * k], r);
#pragma unroll
        for (int j = k + 1; j < 3; j++)
#pragma unroll
            for (int i = k + 1; i < 3; i++) a[i + 3 * j] = __dsub_rn(a[i + 3 * j], __dmul_rn(a[i + 3 * k], a[k + 3 * j]));
    }
    if (singular) return true;  // dgesv_ leaves b = p
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const int pr = ipiv[k];
#pragma unroll
        for (int i = k + 1; i < 3; i++)
            if (pr == i) { double t = b[k]; b[k] = b[i]; b[i] = t; }
    }
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
        for (int i = k + 1; i < 3; i++) b[i] = __dsub_rn(b[i], __dmul_rn(a[i + 3 * k], b[k]));
#pragma unroll
    for (int k = 2; k >= 0; k--) {
        b[k] = __ddiv_rn(b[k], a[k + 3 * k]);
#pragma unroll
        for (int i = 0; i < 2; i++)
            if (i < k) b[i] = __dsub_rn(b[i], __dmul_rn(a[i + 3 * k], b[k]));
    }
    return false;
}

}  // namespace fss
