// moments.cuh -- per-leaf moments of the upward pass (shared by the single
// problem and the ensemble kernels).
#pragma once
#include "device_common.cuh"

namespace fss {

constexpr int kUpThreads = 128;          // four warps, one leaf each
constexpr int kUpLeaves = kUpThreads / 32;
constexpr int kUpRows = 16;              // basis rows (degree <= 15), zero beyond n
constexpr int kUpLd = 32 + 4;            // padded row: the 8 rows x 4 doubles a DMMA operand reads hit distinct banks

// Moments of the particles [a0, a1) of one leaf in the frame of one
// ancestor face (FP64), by one warp.  Per chunk of 32 particles each lane
// writes its particle's basis W[a][j] = w T_a(u), V[b][j] = T_b(v) into the
// warp's own shared rows; then the moments M_ab (a + b <= n) as 8 x 8 tiles
// of W V^T on the FP64 tensor cores, over the chunk's groups of four
// particles.  Tile 0 is a, b < 8.  The rest (a >= 8 or b >= 8, so the other
// index <= n - 8) is one tile with rows a = 8..n, 0..n-8 and columns
// b = 0..n-8, 8..n when n <= 11, else the two tiles a >= 8, b < 8 and
// a < 8, b >= 8 (none for n < 8).  Lane (4 g + t) holds D[g][2t + {0, 1}]
// of each tile; every moment is written once, to out[m], m = (a + b)(a + b +
// 1) / 2 + b.  The groups of four particles are taken in particle order, so
// a moment's sum does not depend on which tile forms it or on the chunking.
template <typename T>
__device__ __forceinline__ void leaf_moments(const typename Vec4<T>::type* __restrict__ src, int a0, int a1,
                                             double fx, double fy, double fz, const NodeGeom& ng, int nmax,
                                             double (*W)[kUpLd], double (*V)[kUpLd], double* __restrict__ out) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    // the rows (of W) and columns (of V) of the tiles beyond tile 0
    const int ntiles = nmax < 8 ? 1 : (nmax <= 11 ? 2 : 3);  // warp-uniform
    const int h = nmax - 7;                                    // rows 8..nmax when nmax <= 11
    int ra1, cb1;                                             // tile 1, this lane's row and B column
    if (ntiles == 2) {
        ra1 = g < h ? 8 + g : g - h;
        cb1 = g < h ? g : 8 + (g - h);
    } else {
        ra1 = 8 + g;  // a >= 8, b < 8
        cb1 = g;
    }
    double d00 = 0.0, d01 = 0.0, e00 = 0.0, e01 = 0.0, f00 = 0.0, f01 = 0.0;
    for (int c0 = a0; c0 < a1; c0 += 32) {
        const int j = c0 + lane;
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
            W[r][lane] = (r <= nmax) ? w * tu : 0.0;
            V[r][lane] = (r <= nmax) ? tv : 0.0;
        }
        __syncwarp();
        const int nk = (min(32, a1 - c0) + 3) >> 2;
        for (int k = 0; k < nk; k++) {
            const int p = 4 * k + t;
            dmma_8x8x4(d00, d01, W[g][p], V[g][p]);
            if (ntiles >= 2) dmma_8x8x4(e00, e01, W[ra1][p], V[cb1][p]);
            if (ntiles == 3) dmma_8x8x4(f00, f01, W[g][p], V[8 + g][p]);  // a < 8, b >= 8
        }
        __syncwarp();
    }
    // column index of this lane's two accumulators in tile 1
    auto col1 = [&](int c) { return ntiles == 2 ? (c < h ? c : 8 + (c - h)) : c; };
    for (int i = 0; i < 2; i++) {
        const int c = 2 * t + i;
        int a = g, b = c;  // tile 0
        if (a + b <= nmax) out[(a + b) * (a + b + 1) / 2 + b] = i ? d01 : d00;
        if (ntiles >= 2) {
            a = ra1;
            b = col1(c);
            if (a + b <= nmax && (a >= 8 || b >= 8)) out[(a + b) * (a + b + 1) / 2 + b] = i ? e01 : e00;
        }
        if (ntiles == 3) {
            a = g;
            b = 8 + c;
            if (a + b <= nmax) out[(a + b) * (a + b + 1) / 2 + b] = i ? f01 : f00;
        }
    }
}

}  // namespace fss
