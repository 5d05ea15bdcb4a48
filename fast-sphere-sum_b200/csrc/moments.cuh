// moments.cuh -- per-leaf moments of the upward pass (shared by the single
// problem and the ensemble kernels).
#pragma once
#include "device_common.cuh"

namespace fss {

constexpr int kUpThreads = 128;
constexpr int kUpRows = 16;              // basis rows (degree <= 15), zero beyond n
constexpr int kUpLd = kUpThreads + 4;    // padded row: 8 rows of 4 doubles hit distinct banks

// Moments of the particles [a0, a1) of one leaf in the frame of one
// ancestor face (FP64).  Per chunk of 128 particles each thread writes its
// particle's basis W[a][j] = w T_a(u), V[b][j] = T_b(v); then M = W V^T
// (16 x 16, a + b <= n used) on the FP64 tensor cores, warp w taking the 8 x 8
// tile (w / 2, w % 2).  Lane (4 g + t) ends holding M[8 (w/2) + g][8 (w%2) +
// 2t + {0, 1}], written to out[m], m = (a + b)(a + b + 1) / 2 + b.  A tile
// holding no a + b <= n is not formed: (1, 1) never (n <= 12 < 16), (0, 1) and
// (1, 0) not for n < 8.
template <typename T>
__device__ __forceinline__ void leaf_moments(const typename Vec4<T>::type* __restrict__ src, int a0, int a1,
                                             double fx, double fy, double fz, const NodeGeom& ng, int nmax,
                                             double (*W)[kUpLd], double (*V)[kUpLd], double* __restrict__ out) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int ta = warp >> 1, tb = warp & 1, g = lane >> 2, t = lane & 3;
    double d0 = 0.0, d1 = 0.0;
    for (int c0 = a0; c0 < a1; c0 += kUpThreads) {
        const int j = c0 + tid;
        double u = 0.0, v = 0.0, w = 0.0;
        if (j < a1) {
            const typename Vec4<T>::type q = src[j];
            const double x = fx + double(q.x), y = fy + double(q.y), z = fz + double(q.z);
            w = double(q.w);
            const double e0 = ng.minv[0] * x + ng.minv[1] * y + ng.minv[2] * z;
            const double e1 = ng.minv[3] * x + ng.minv[4] * y + ng.minv[5] * z;
            const double e2 = ng.minv[6] * x + ng.minv[7] * y + ng.minv[8] * z;
            const double inv = 1.0 / (e0 + e1 + e2);
            u = 2.0 * (e0 * inv) - 1.0;
            v = 2.0 * (e1 * inv) - 1.0;
        }
        double ta0 = 1.0, ta1 = u, tb0 = 1.0, tb1 = v;
#pragma unroll
        for (int r = 0; r < kUpRows; r++) {
            const double tu = (r == 0) ? 1.0 : (r == 1 ? u : 2.0 * u * ta1 - ta0);
            const double tv = (r == 0) ? 1.0 : (r == 1 ? v : 2.0 * v * tb1 - tb0);
            if (r >= 2) { ta0 = ta1; ta1 = tu; tb0 = tb1; tb1 = tv; }
            W[r][tid] = (r <= nmax) ? w * tu : 0.0;
            V[r][tid] = (r <= nmax) ? tv : 0.0;
        }
        __syncthreads();
        const int nk = (min(kUpThreads, a1 - c0) + 3) >> 2;  // same in every thread
        if (8 * (ta + tb) <= nmax)                            // warp-uniform
            for (int k = 0; k < nk; k++)
                dmma_8x8x4(d0, d1, W[8 * ta + g][4 * k + t], V[8 * tb + g][4 * k + t]);
        __syncthreads();
    }
    const int a = 8 * ta + g;
    for (int i = 0; i < 2; i++) {
        const int b = 8 * tb + 2 * t + i, gg = a + b;
        if (gg <= nmax) out[gg * (gg + 1) / 2 + b] = i ? d1 : d0;
    }
}

}  // namespace fss
