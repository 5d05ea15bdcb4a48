// k_pairs.cu -- the pair engine shared by the direct sum, the near field and
// the particle-cluster far field.
//
// A block owns up to THREADS*R targets of one leaf (or of one tile of the
// direct sum) and streams its source ranges -- particles of near leaves,
// proxy charges of far clusters, or a chunk of all particles -- through a
// ring of shared-memory tiles filled by bulk TMA copies (cp.async.bulk, one
// elected thread, completion on an mbarrier; no multicast).  Each thread
// keeps R targets in registers.  Per pair (23 algorithmic flops):
//
//   d   = x_j - x_i                      (local frames: s_j + (D - t_i))
//   r2  = |d|^2           (= 2 (1 - x_i.x_j) on the unit sphere, no cancellation)
//   A  += w_j d / r2
//
// and afterwards u_i = -(1/2pi) x_i x A_i, since x_i x x_j = x_i x d and
// G(x_i, x_j) = 2 x_i x d / |d|^2.  Mixed precision accumulates each tile in
// FP32 and folds it into a Kahan-compensated per-target sum; the FP64 path
// sums plainly.  Results are written per work item to a partial slot.
#include <cuda_runtime.h>

#include "device_common.cuh"
#include "kernels.h"

namespace fss {

constexpr int kDepth = 4;  // ring depth (tiles in flight)

template <typename T, int R, bool PSI, bool GUARD>
__device__ __forceinline__ void tile_pairs(const typename Vec4<T>::type* __restrict__ s, int cnt, const T* ox,
                                           const T* oy, const T* oz, T* ax, T* ay, T* az, T* ap) {
#pragma unroll 4
    for (int j = 0; j < cnt; j++) {
        const typename Vec4<T>::type q = s[j];
#pragma unroll
        for (int r = 0; r < R; r++) {
            const T dx = q.x + ox[r], dy = q.y + oy[r], dz = q.z + oz[r];
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
                                                   const SrcEntry* __restrict__ ents,
                                                   const WorkItem* __restrict__ items, double4* __restrict__ partials,
                                                   int64_t pstride, int* __restrict__ err) {
    using S4 = typename Vec4<T>::type;
    constexpr bool kKahan = sizeof(T) == 4;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    S4* ring = reinterpret_cast<S4*>(smem_raw);
    __shared__ __align__(8) uint64_t full_bar[kDepth], empty_bar[kDepth];

    const WorkItem it = items[blockIdx.x];
    const int tid = threadIdx.x, lane = tid & 31;

    T tx[R], ty[R], tz[R];
#pragma unroll
    for (int r = 0; r < R; r++) {
        const int k = tid + r * THREADS;
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

    if (tid == 0) {
#pragma unroll
        for (int d = 0; d < kDepth; d++) {
            mbar_init(&full_bar[d], 1);
            mbar_init(&empty_bar[d], THREADS / 32);
        }
        mbar_init_fence();
    }
    __syncthreads();

    // Producer: warp 0 as a whole (so that it never diverges from its own
    // consumer work); lane 0 issues.  Cursor = entry, offset within it,
    // tiles issued so far.
    const bool producer = (tid >> 5) == 0;
    int pe = it.e0, po = 0, pk = 0;
    bool failed = false;
    auto produce = [&]() {
        while (pe < it.e1 && po >= ents[pe].count) { pe++; po = 0; }
        if (pe >= it.e1) return;
        const int start = ents[pe].start;
        const int cnt = min(TILE, ents[pe].count - po);
        const int slot = pk % kDepth;
        bool ok = true;
        if (pk >= kDepth) ok = mbar_wait_bounded(&empty_bar[slot], ((pk / kDepth) - 1) & 1);
        if (!__all_sync(0xffffffffu, ok)) {
            failed = true;
            return;
        }
        if (lane == 0) {
            const uint32_t bytes = uint32_t(cnt) * uint32_t(sizeof(S4));
            mbar_arrive_expect_tx(&full_bar[slot], bytes);
            bulk_g2s(ring + slot * TILE, src + start + po, bytes, &full_bar[slot]);
        }
        __syncwarp();
        po += cnt;
        pk++;
    };
    if (producer)
        for (int d = 0; d < kDepth - 1 && !failed; d++) produce();

    const int t_lo = it.t0, t_hi = it.t0 + it.nt;
    int ce = it.e0, co = 0, k = 0;
    for (;;) {
        while (ce < it.e1 && co >= ents[ce].count) { ce++; co = 0; }
        if (ce >= it.e1) break;
        if (producer && !failed) produce();
        const SrcEntry e = ents[ce];
        const int cnt = min(TILE, e.count - co);
        const int gs = e.start + co;
        const int slot = k % kDepth;
        if (!__all_sync(0xffffffffu, mbar_wait_bounded(&full_bar[slot], (k / kDepth) & 1))) {
            set_error(err, kErrTimeout);
            failed = true;
            break;
        }
        T ox[R], oy[R], oz[R];
#pragma unroll
        for (int r = 0; r < R; r++) {
            ox[r] = T(e.dx) - tx[r];
            oy[r] = T(e.dy) - ty[r];
            oz[r] = T(e.dz) - tz[r];
        }
        const S4* tile = ring + slot * TILE;
        const bool overlap = (gs < t_hi) && (gs + cnt > t_lo);
        if (overlap)
            tile_pairs<T, R, PSI, true>(tile, cnt, ox, oy, oz, ax, ay, az, ap);
        else
            tile_pairs<T, R, PSI, false>(tile, cnt, ox, oy, oz, ax, ay, az, ap);
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
        co += cnt;
        k++;
    }
    if (failed) {
        set_error(err, kErrTimeout);
        // drain copies that were issued but not consumed (bounded)
        if (producer && lane == 0)
            for (int kk = k; kk < pk; kk++) mbar_wait_bounded(&full_bar[kk % kDepth], (kk / kDepth) & 1);
        return;
    }
#pragma unroll
    for (int r = 0; r < R; r++) {
        const int kk = tid + r * THREADS;
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
static cudaError_t run_pairs(cudaStream_t st, int nitems, const void* src, const SrcEntry* ents,
                             const WorkItem* items, double4* partials, int64_t pstride, int* err) {
    constexpr int TILE = (sizeof(T) == 4) ? 256 : 128;
    const size_t smem = size_t(kDepth) * TILE * sizeof(typename Vec4<T>::type);
    static_assert(size_t(kDepth) * TILE * sizeof(typename Vec4<T>::type) <= 48 * 1024,
                  "ring must fit the default dynamic shared memory limit");
    auto kern = k_pairs<T, THREADS, R, PSI, TILE>;
    if (nitems == 0) return cudaSuccess;
    kern<<<nitems, THREADS, smem, st>>>(static_cast<const typename Vec4<T>::type*>(src), ents, items, partials,
                                         pstride, err);
    return cudaGetLastError();
}

PairShape pairs_shape(bool fp64, int threads_hint) {
    PairShape s;
    if (fp64) {
        s.threads = 128;
        s.per_thread = 1;
    } else {
        s.threads = (threads_hint == 64) ? 64 : 128;
        s.per_thread = (threads_hint == 64) ? 2 : 1;
    }
    return s;
}

cudaError_t launch_pairs(cudaStream_t st, bool fp64, bool psi, PairShape shape, int nitems, const void* src,
                         const SrcEntry* ents, const WorkItem* items, double4* partials, int64_t pstride, int* err) {
    if (fp64) {
        return psi ? run_pairs<double, 128, 1, true>(st, nitems, src, ents, items, partials, pstride, err)
                   : run_pairs<double, 128, 1, false>(st, nitems, src, ents, items, partials, pstride, err);
    }
    if (shape.threads == 64) {
        return psi ? run_pairs<float, 64, 2, true>(st, nitems, src, ents, items, partials, pstride, err)
                   : run_pairs<float, 64, 2, false>(st, nitems, src, ents, items, partials, pstride, err);
    }
    return psi ? run_pairs<float, 128, 1, true>(st, nitems, src, ents, items, partials, pstride, err)
               : run_pairs<float, 128, 1, false>(st, nitems, src, ents, items, partials, pstride, err);
}

}  // namespace fss
