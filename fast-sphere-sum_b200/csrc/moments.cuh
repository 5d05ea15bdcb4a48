// moments.cuh -- per-leaf moments of the upward pass (shared by the single
// problem and the ensemble kernels).
#pragma once
#include "device_common.cuh"

namespace fss {

constexpr int kUpThreads = 128;          // four warps, one leaf each
constexpr int kUpLeaves = kUpThreads / 32;
constexpr int kUpRows = kMaxDegree + 1;  // basis rows (degree <= kMaxDegree)
constexpr int kUpLd = 32 + 4;            // padded row: the 8 rows x 4 doubles a DMMA operand reads hit distinct banks

// Moments of the particles [a0, a1) of one leaf in the frame of one
// ancestor face (FP64), by one warp, up to degree NM.  Per chunk of 32
// particles each lane writes its particle's basis W[a][j] = w T_a(u),
// V[b][j] = T_b(v), a, b <= NM, into the warp's own shared rows; then the
// moments M_ab (a + b <= NM) with a, b < 8 as one 8 x 8 tile of W V^T on the
// FP64 tensor cores, over the chunk's groups of four particles.  The rest
// (a >= 8 or b >= 8, so the other index <= NM - 8): for NM <= 11 at most 20
// moments, each a per-lane FP64 sum of the lane's own particles, added over
// the warp by shuffles at the end (a second tile would be mostly unused,
// and on B200 an FP64 tensor tile costs the FP64 pipe as much as its 256
// FMA); for NM = 12 the two tiles a >= 8, b < 8 and a < 8, b >= 8.  A tile
// row or column index above NM is clamped to NM (a row of this chunk), and
// it only reaches outputs with a + b > NM, which are dropped.  Lane (4 g +
// t) holds D[g][2t + {0, 1}] of each tile; every moment is written once, to
// out[m], m = (a + b)(a + b + 1) / 2 + b.
template <typename T, int NM>
__device__ __forceinline__ void leaf_moments_n(const typename Vec4<T>::type* __restrict__ src, int a0, int a1,
                                               double fx, double fy, double fz, const NodeGeom& ng,
                                               double (*W)[kUpLd], double (*V)[kUpLd], double* __restrict__ out) {
    static_assert(NM >= 0 && NM < kUpRows, "degree beyond the basis rows");
    constexpr int NT = NM < 8 ? 1 : (NM <= 11 ? 2 : 3);  // tiles (NT == 2: one tile and lane sums)
    // NM 8..11: the moments with a or b >= 8 (the other index <= NM - 8 <= 3),
    // XE of them, are per-lane FP64 sums of this lane's particles, added
    // across the warp at the end, instead of a second 8x8x4 tile per four
    // particles that would be mostly unused.  Entry order: for r = 8..NM and
    // s = 0..NM - r, (a, b) = (r, s) then (s, r).
    constexpr int H = NM - 7;
    constexpr int XE = NT == 2 ? H * (H + 1) : 0;
    constexpr int XL = NT == 2 ? H : 1;  // low rows kept in registers (s <= NM - 8)
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int g0 = min(g, NM);      // tile 0's row and column (a, b < 8)
    const int r1 = min(8 + g, NM);  // NT == 3: tile 1's row (a >= 8), tile 2's column (b >= 8)
    double d00 = 0.0, d01 = 0.0, e00 = 0.0, e01 = 0.0, f00 = 0.0, f01 = 0.0;
    double xs[XE > 0 ? XE : 1];
#pragma unroll
    for (int e = 0; e < (XE > 0 ? XE : 1); e++) xs[e] = 0.0;
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
        double wlo[XL], vlo[XL];  // w T_s(u), T_s(v) for s < XL
#pragma unroll
        for (int r = 0; r <= NM; r++) {
            const double tu = (r == 0) ? 1.0 : (r == 1 ? u : 2.0 * u * ta1 - ta0);
            const double tv = (r == 0) ? 1.0 : (r == 1 ? v : 2.0 * v * tb1 - tb0);
            if (r >= 2) { ta0 = ta1; ta1 = tu; tb0 = tb1; tb1 = tv; }
            const double wt = w * tu;
            if (r < 8 || NT == 3) {
                W[r][lane] = wt;
                V[r][lane] = tv;
            }
            if constexpr (NT == 2) {
                if (r < XL) {
                    wlo[r] = wt;
                    vlo[r] = tv;
                }
                if (r >= 8) {
                    const int e0 = (r - 8) * (2 * H - (r - 8) + 1);  // entries before row r
#pragma unroll
                    for (int s2 = 0; s2 <= NM - r; s2++) {
                        xs[e0 + 2 * s2] = fma(wt, vlo[s2], xs[e0 + 2 * s2]);
                        xs[e0 + 2 * s2 + 1] = fma(wlo[s2], tv, xs[e0 + 2 * s2 + 1]);
                    }
                }
            }
        }
        __syncwarp();
        const int nk = (min(32, a1 - c0) + 3) >> 2;
        for (int k = 0; k < nk; k++) {
            const int p = 4 * k + t;
            dmma_8x8x4(d00, d01, W[g0][p], V[g0][p]);
            if constexpr (NT == 3) {
                dmma_8x8x4(e00, e01, W[r1][p], V[g0][p]);  // a >= 8, b < 8
                dmma_8x8x4(f00, f01, W[g0][p], V[r1][p]);  // a < 8, b >= 8
            }
        }
        __syncwarp();
    }
#pragma unroll
    for (int i = 0; i < 2; i++) {
        const int c = 2 * t + i;
        int a = g, b = c;  // tile 0
        if (a + b <= NM) out[(a + b) * (a + b + 1) / 2 + b] = i ? d01 : d00;
        if constexpr (NT == 3) {
            a = 8 + g;
            b = c;
            if (a + b <= NM) out[(a + b) * (a + b + 1) / 2 + b] = i ? e01 : e00;
            a = g;
            b = 8 + c;
            if (a + b <= NM) out[(a + b) * (a + b + 1) / 2 + b] = i ? f01 : f00;
        }
    }
    if constexpr (NT == 2) {
#pragma unroll
        for (int e = 0; e < XE; e++)
            for (int o = 16; o > 0; o >>= 1) xs[e] += __shfl_xor_sync(0xffffffffu, xs[e], o);
        if (lane == 0) {
#pragma unroll
            for (int r = 8; r <= NM; r++) {
                const int e0 = (r - 8) * (2 * H - (r - 8) + 1);
#pragma unroll
                for (int s2 = 0; s2 <= NM - r; s2++) {
                    out[(r + s2) * (r + s2 + 1) / 2 + s2] = xs[e0 + 2 * s2];  // (a, b) = (r, s2)
                    out[(r + s2) * (r + s2 + 1) / 2 + r] = xs[e0 + 2 * s2 + 1];  // (a, b) = (s2, r)
                }
            }
        }
    }
}

// leaf_moments_n for a run-time (warp-uniform) degree nm <= kMaxDegree.
template <typename T>
__device__ __forceinline__ void leaf_moments(const typename Vec4<T>::type* __restrict__ src, int a0, int a1,
                                             double fx, double fy, double fz, const NodeGeom& ng, int nm,
                                             double (*W)[kUpLd], double (*V)[kUpLd], double* __restrict__ out) {
    static_assert(kMaxDegree == 12, "extend the dispatch");
    switch (nm) {
#define FSS_MOMENTS_CASE(N) \
    case N: leaf_moments_n<T, N>(src, a0, a1, fx, fy, fz, ng, W, V, out); break;
        FSS_MOMENTS_CASE(0) FSS_MOMENTS_CASE(1) FSS_MOMENTS_CASE(2) FSS_MOMENTS_CASE(3) FSS_MOMENTS_CASE(4)
        FSS_MOMENTS_CASE(5) FSS_MOMENTS_CASE(6) FSS_MOMENTS_CASE(7) FSS_MOMENTS_CASE(8) FSS_MOMENTS_CASE(9)
        FSS_MOMENTS_CASE(10) FSS_MOMENTS_CASE(11) FSS_MOMENTS_CASE(12)
#undef FSS_MOMENTS_CASE
        default: break;
    }
}

// Sum of R rows, row(i) for i < R, as four chains (rows i = 0, 4, 8, ...;
// 1, 5, ...; ...) added as (s0 + s1) + (s2 + s3): four loads in flight.
// The single problem's and the ensemble's combines both sum this way.
template <typename F>
__device__ __forceinline__ double sum_rows4(F row, int R) {
    double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
    int i = 0;
    for (; i + 4 <= R; i += 4) {
        s0 += row(i + 0);
        s1 += row(i + 1);
        s2 += row(i + 2);
        s3 += row(i + 3);
    }
    for (; i < R; i++) s0 += row(i);
    return (s0 + s1) + (s2 + s3);
}

// Moment rows of the upward pass.  The leaves of a member are numbered so
// that leaves 4g .. 4g + 3 are the four children of one face (and share
// every ancestor above the leaf level).  A block of four warps takes one
// such group on one level l: on the leaf level each warp writes its own
// leaf's row; above it the four rows are added in shared memory as
// (r0 + r1) + (r2 + r3) and written once, into the slot of the group's
// first leaf.  A face on level l < leaf level then sums the rows of every
// fourth leaf of its range (its groups), a leaf-level face its one row.
// The same below for the single problem and the ensemble, so that both
// form every proxy charge from the same additions.
__device__ __forceinline__ int up_row_step(int level, int leaf_level) { return level < leaf_level ? 4 : 1; }

}  // namespace fss
