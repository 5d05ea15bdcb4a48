// k_pairs.cu -- the pair engine shared by the direct sum, the near field and
// the particle-cluster far field.
//
// A block owns up to THREADS*R targets of one leaf (or of one tile of the
// direct sum).  Its sources -- particles of near leaves, proxy charges of far
// clusters, or a chunk of all particles -- arrive as a sequence of
// shared-memory tiles.  Each tile is several source ranges placed back to
// back by bulk TMA copies (cp.async.bulk, issued by one lane of warp 0,
// completion counted on the tile slot's mbarrier; no multicast), in a ring
// of kDepth slots released by the consumer warps through a second mbarrier.
// Each thread keeps R targets in registers.  Per pair (23 algorithmic flops):
//
//   d   = x_j - x_i
//   r2  = |d|^2           (= 2 (1 - x_i.x_j) on the unit sphere, no cancellation)
//   A  += w_j d / r2
//
// and afterwards u_i = -(1/2pi) x_i x A_i, since x_i x x_j = x_i x d and
// G(x_i, x_j) = 2 x_i x d / |d|^2.  Mixed precision sums each tile in FP32
// and folds it into a Kahan-compensated per-target sum; the FP64 path sums
// plainly.  Results go to the work item's partial slot.
#include <cuda_runtime.h>

#include "device_common.cuh"
#include "kernels.h"

namespace fss {

constexpr int kDepth = 4;  // ring depth (tiles in flight)

template <typename T, int R, bool PSI, bool GUARD>
__device__ __forceinline__ void tile_pairs(const typename Vec4<T>::type* __restrict__ s, int cnt, const T* tx,
                                           const T* ty, const T* tz, T* ax, T* ay, T* az, T* ap) {
#pragma unroll 8
    for (int j = 0; j < cnt; j++) {
        const typename Vec4<T>::type q = s[j];
#pragma unroll
        for (int r = 0; r < R; r++) {
            const T dx = q.x - tx[r], dy = q.y - ty[r], dz = q.z - tz[r];
            const T r2 = fma(dz, dz, fma(dy, dy, dx * dx));
            T inv = rcp_fast(r2);
            if (GUARD) inv = (r2 > T(0)) ? inv : T(0);
            const T sc = q.w * inv;
            ax[r] = fma(sc, dx, ax[r]);
            ay[r] = fma(sc, dy, ay[r]);
            az[r] = fma(sc, dz, az[r]);
            if (PSI) {
                T lg = lg2_fast(r2);
                if (GUARD) lg = (r2 > T(0)) ? lg : T(0);
                ap[r] = fma(q.w, lg, ap[r]);
            }
        }
    }
}

template <typename T>
__device__ __forceinline__ void kahan_add(T& sum, T& comp, T x) {
    const T y = x - comp;
    const T t = sum + y;
    comp = (t - sum) - y;
    sum = t;
}

template <typename T, int THREADS, int R, bool PSI, int TILE>
__global__ void __launch_bounds__(THREADS) k_pairs(const typename Vec4<T>::type* __restrict__ src,
                                                   const Copy* __restrict__ copies, const Tile* __restrict__ tiles,
                                                   const WorkItem* __restrict__ items, double4* __restrict__ partials,
                                                   int64_t pstride, int* __restrict__ err) {
    using S4 = typename Vec4<T>::type;
    constexpr bool kKahan = sizeof(T) == 4;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    S4* ring = reinterpret_cast<S4*>(smem_raw);
    __shared__ __align__(8) uint64_t full_bar[kDepth], empty_bar[kDepth];

    const WorkItem it = items[blockIdx.x];
    const int tid = threadIdx.x, lane = tid & 31;

    // Warps whose targets all lie beyond nt have nothing to compute (the
    // tail chunk of a leaf larger than one block): they leave at once, and
    // the slot-release barrier counts only the active warps.
    const int need = (it.nt + 32 * R - 1) / (32 * R);
    const int active_warps = need < THREADS / 32 ? need : THREADS / 32;
    if (tid == 0) {
#pragma unroll
        for (int d = 0; d < kDepth; d++) {
            mbar_init(&full_bar[d], 1);
            mbar_init(&empty_bar[d], active_warps);
        }
        mbar_init_fence();
    }
    __syncthreads();
    if ((tid >> 5) >= active_warps) return;

    T tx[R], ty[R], tz[R];
#pragma unroll
    for (int r = 0; r < R; r++) {
        const int k = tid * R + r;
        const S4 v = src[it.t0 + ((k < it.nt) ? k : 0)];
        tx[r] = v.x; ty[r] = v.y; tz[r] = v.z;
    }
    T ax[R], ay[R], az[R], ap[R];
    T sx[R], sy[R], sz[R], sp[R], cx[R], cy[R], cz[R], cp[R];
#pragma unroll
    for (int r = 0; r < R; r++) {
        ax[r] = ay[r] = az[r] = ap[r] = T(0);
        sx[r] = sy[r] = sz[r] = sp[r] = T(0);
        cx[r] = cy[r] = cz[r] = cp[r] = T(0);
    }

    // Producer: warp 0 as a whole (it never diverges from its own consumer
    // work); lane 0 issues the copies of one tile.
    const bool producer = (tid >> 5) == 0;
    int pk = it.k0;  // next tile to issue
    bool failed = false;
    auto produce = [&]() {
        if (pk >= it.k1) return;
        const int k = pk - it.k0;
        const int slot = k % kDepth;
        bool ok = true;
        if (k >= kDepth) ok = mbar_wait_bounded(&empty_bar[slot], ((k / kDepth) - 1) & 1);
        if (!__all_sync(0xffffffffu, ok)) {
            failed = true;
            return;
        }
        if (lane == 0) {
            const Tile tl = tiles[pk];
            mbar_arrive_expect_tx(&full_bar[slot], uint32_t(tl.count) * uint32_t(sizeof(S4)));
            S4* dst = ring + slot * TILE;
            for (int c = tl.c0; c < tl.c1; c++) {
                const Copy cp = copies[c];
                bulk_g2s(dst, src + cp.start, uint32_t(cp.count) * uint32_t(sizeof(S4)), &full_bar[slot]);
                dst += cp.count;
            }
        }
        __syncwarp();
        pk++;
    };
    if (producer)
        for (int d = 0; d < kDepth - 1 && !failed; d++) produce();

    int kfail = it.k1;
    for (int kt = it.k0; kt < it.k1; kt++) {
        if (producer && !failed) produce();
        const int k = kt - it.k0;
        const int slot = k % kDepth;
        const Tile tl = tiles[kt];
        if (!__all_sync(0xffffffffu, mbar_wait_bounded(&full_bar[slot], (k / kDepth) & 1))) {
            failed = true;
            kfail = kt;
            break;
        }
        const S4* tile = ring + slot * TILE;
        if (tl.guard)
            tile_pairs<T, R, PSI, true>(tile, tl.count, tx, ty, tz, ax, ay, az, ap);
        else
            tile_pairs<T, R, PSI, false>(tile, tl.count, tx, ty, tz, ax, ay, az, ap);
        if (kKahan) {
#pragma unroll
            for (int r = 0; r < R; r++) {
                kahan_add(sx[r], cx[r], ax[r]);
                kahan_add(sy[r], cy[r], ay[r]);
                kahan_add(sz[r], cz[r], az[r]);
                if (PSI) kahan_add(sp[r], cp[r], ap[r]);
                ax[r] = ay[r] = az[r] = ap[r] = T(0);
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty_bar[slot]);
    }
    if (failed) {
        set_error(err, kErrTimeout);
        // wait (bounded) for copies issued but not consumed before leaving
        if (producer && lane == 0)
            for (int kk = kfail; kk < pk; kk++)
                mbar_wait_bounded(&full_bar[(kk - it.k0) % kDepth], ((kk - it.k0) / kDepth) & 1);
        return;
    }
#pragma unroll
    for (int r = 0; r < R; r++) {
        const int kk = tid * R + r;
        if (kk >= it.nt) continue;
        double4 o;
        if (kKahan) {
            o = make_double4(double(sx[r]) - double(cx[r]), double(sy[r]) - double(cy[r]),
                             double(sz[r]) - double(cz[r]), double(sp[r]) - double(cp[r]));
        } else {
            o = make_double4(double(ax[r]), double(ay[r]), double(az[r]), double(ap[r]));
        }
        partials[int64_t(it.part) * pstride + it.t0 + kk] = o;
    }
}

// ---------------------------------------------------------------- dispatch

template <typename T, int THREADS, int R, bool PSI>
static cudaError_t run_pairs(cudaStream_t st, int nitems, const void* src, const Copy* copies, const Tile* tiles,
                             const WorkItem* items, double4* partials, int64_t pstride, int* err) {
    constexpr int TILE = tile_capacity(sizeof(T) == 8);
    constexpr size_t smem = size_t(kDepth) * TILE * sizeof(typename Vec4<T>::type);
    static_assert(smem <= 48 * 1024, "ring must fit the default dynamic shared memory limit");
    if (nitems == 0) return cudaSuccess;
    k_pairs<T, THREADS, R, PSI, TILE><<<nitems, THREADS, smem, st>>>(
        static_cast<const typename Vec4<T>::type*>(src), copies, tiles, items, partials, pstride, err);
    return cudaGetLastError();
}

const std::vector<PairShape>& pair_shapes(bool fp64) {
    static const std::vector<PairShape> f32 = {{128, 1, 256}, {160, 1, 256}, {192, 1, 256}, {256, 1, 256},
                                               {64, 2, 256},  {96, 2, 256},  {128, 2, 256}};
    static const std::vector<PairShape> f64 = {{128, 1, 128}, {160, 1, 128}, {192, 1, 128}, {256, 1, 128}};
    return fp64 ? f64 : f32;
}

PairShape pairs_shape(bool fp64, int threads, int per_thread) {
    for (const PairShape& s : pair_shapes(fp64))
        if (s.threads == threads && s.per_thread == (per_thread > 0 ? per_thread : 1)) return s;
    return pair_shapes(fp64).front();
}

template <typename T, bool PSI>
static cudaError_t dispatch(cudaStream_t st, PairShape sh, int nitems, const void* src, const Copy* copies,
                            const Tile* tiles, const WorkItem* items, double4* partials, int64_t pstride, int* err) {
#define FSS_SHAPE(TH, R)                                                                                   \
    if (sh.threads == TH && sh.per_thread == R)                                                            \
        return run_pairs<T, TH, R, PSI>(st, nitems, src, copies, tiles, items, partials, pstride, err);
    FSS_SHAPE(128, 1)
    FSS_SHAPE(160, 1)
    FSS_SHAPE(192, 1)
    FSS_SHAPE(256, 1)
    if (sizeof(T) == 4) {
        FSS_SHAPE(64, 2)
        FSS_SHAPE(96, 2)
        FSS_SHAPE(128, 2)
    }
#undef FSS_SHAPE
    return cudaErrorInvalidConfiguration;
}

cudaError_t launch_pairs(cudaStream_t st, bool fp64, bool psi, PairShape shape, int nitems, const void* src,
                         const Copy* copies, const Tile* tiles, const WorkItem* items, double4* partials,
                         int64_t pstride, int* err) {
    if (fp64)
        return psi ? dispatch<double, true>(st, shape, nitems, src, copies, tiles, items, partials, pstride, err)
                   : dispatch<double, false>(st, shape, nitems, src, copies, tiles, items, partials, pstride, err);
    return psi ? dispatch<float, true>(st, shape, nitems, src, copies, tiles, items, partials, pstride, err)
               : dispatch<float, false>(st, shape, nitems, src, copies, tiles, items, partials, pstride, err);
}

}  // namespace fss
