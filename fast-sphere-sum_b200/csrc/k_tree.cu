// k_tree.cu -- GPU tree build: particle -> face assignment on the
// icosahedral refinement path, stable radix key-sort, leaf ranges, and the
// gather of the particle state into leaf order.
#include <cuda_runtime.h>

#include "device_common.cuh"
#include "exact_lu.cuh"
#include "kernels.h"

namespace fss {

// ---------------------------------------------------------------- assignment

// icos_utils.h:145-170 point_assign for every particle.  Level 0 searches
// the 20 faces, level l the four children of the level l-1 face; the first
// face whose cone coordinates are all >= 0 wins.  In reference mode a
// particle with no match is left out of the level (loc = -1) and the next
// level searches the children of face 0, as the reference does with its
// zero-initialised tree_point_locs.  In complete mode the particle goes to
// the candidate whose smallest cone coordinate is largest, so every particle
// has exactly one leaf.  key[i] = leaf face (complete mode only).
__global__ void k_assign(int64_t n, const double* __restrict__ in5, const double* __restrict__ verts,
                         const int32_t* __restrict__ tri_verts, const int64_t* __restrict__ lev_off,
                         int tree_levels, int reference_mode, int32_t* __restrict__ loc, uint32_t* __restrict__ key,
                         int* __restrict__ err) {
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double p[3] = {in5[5 * i], in5[5 * i + 1], in5[5 * i + 2]};
    if (!isfinite(p[0]) || !isfinite(p[1]) || !isfinite(p[2])) set_error(err, kErrNonFinite);
    int prev = 0;
    for (int l = 0; l < tree_levels; l++) {
        const int lb = (l > 0) ? 4 * prev : 0, ub = (l > 0) ? lb + 4 : 20;
        int found = -1, best = lb;
        double best_min = -1e300;
        for (int j = lb; j < ub; j++) {
            const int32_t* tv = tri_verts + 3 * (lev_off[l] + j);
            double c[3];
            cone_coords_exact(verts + 3 * int64_t(tv[0]), verts + 3 * int64_t(tv[1]), verts + 3 * int64_t(tv[2]), p, c);
            if (c[0] >= 0 && c[1] >= 0 && c[2] >= 0) { found = j; break; }
            const double m = fmin(c[0], fmin(c[1], c[2]));
            if (m > best_min) { best_min = m; best = j; }
        }
        if (reference_mode) {
            if (loc) loc[int64_t(l) * n + i] = found;
            prev = (found >= 0) ? found : 0;
        } else {
            const int f = (found >= 0) ? found : best;
            if (loc) loc[int64_t(l) * n + i] = f;
            prev = f;
        }
    }
    if (key) key[i] = uint32_t(prev);
}

// Per-face member counts of every level from loc (reference-mode parity).
__global__ void k_level_hist(int64_t n, int tree_levels, const int32_t* __restrict__ loc,
                             const int64_t* __restrict__ lev_off, int32_t* __restrict__ counts) {
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int l = 0; l < tree_levels; l++) {
        const int32_t f = loc[int64_t(l) * n + i];
        if (f >= 0) atomicAdd(&counts[lev_off[l] + f], 1);
    }
}

// ---------------------------------------------------------------- radix sort
// Stable LSD radix sort of (key, value) with 8-bit digits.  Each block owns
// a tile of kSortTile consecutive elements; warps own consecutive 512-element
// slices of it, so ranks computed warp by warp, round by round, lane by lane
// preserve the input order within every digit.

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortPerWarp = 512;
constexpr int kSortTile = kSortWarps * kSortPerWarp;  // 4096

__global__ void __launch_bounds__(kSortThreads) k_radix_hist(int64_t n, const uint32_t* __restrict__ keys, int shift,
                                                             uint32_t* __restrict__ hist, int nblk) {
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const int64_t base = int64_t(blockIdx.x) * kSortTile;
    for (int k = threadIdx.x; k < kSortTile; k += kSortThreads) {
        const int64_t i = base + k;
        if (i < n) atomicAdd(&h[(keys[i] >> shift) & 255u], 1u);
    }
    __syncthreads();
    hist[int64_t(threadIdx.x) * nblk + blockIdx.x] = h[threadIdx.x];
}

// Exclusive scan of 32-bit counts by blocks of 1024 threads, in chunks of
// 1024 x kScanPer entries staged through shared memory (coalesced loads and
// stores; each thread scans kScanPer consecutive entries; warp-shuffle scan
// of the thread sums).  scan_chunk scans one chunk from a carry and returns
// the carry after it (all threads).
constexpr int kScanPer = 8;
constexpr int64_t kScanChunk = 1024 * kScanPer;

struct ScanSmem {
    uint32_t buf[kScanChunk];
    uint32_t wsum[32];
    uint32_t carry;
};

__device__ __forceinline__ uint32_t scan_chunk(uint32_t* __restrict__ a, int64_t m, int64_t base, uint32_t carry,
                                               ScanSmem& sm) {
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    for (int k = 0; k < kScanPer; k++) {
        const int64_t i = base + int64_t(k) * 1024 + t;
        sm.buf[k * 1024 + t] = (i < m) ? a[i] : 0u;
    }
    __syncthreads();
    uint32_t v[kScanPer], s = 0;
    for (int k = 0; k < kScanPer; k++) {
        v[k] = sm.buf[t * kScanPer + k];
        s += v[k];
    }
    // inclusive scan of the thread sums
    uint32_t x = s;
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= d) x += y;
    }
    if (lane == 31) sm.wsum[w] = x;
    __syncthreads();
    if (w == 0) {
        uint32_t z = sm.wsum[lane];
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, z, d);
            if (lane >= d) z += y;
        }
        sm.wsum[lane] = z;
    }
    __syncthreads();
    uint32_t run = carry + (x - s) + (w > 0 ? sm.wsum[w - 1] : 0u);
    for (int k = 0; k < kScanPer; k++) {
        sm.buf[t * kScanPer + k] = run;
        run += v[k];
    }
    __syncthreads();
    if (t == 1023) sm.carry = run;
    for (int k = 0; k < kScanPer; k++) {
        const int64_t i = base + int64_t(k) * 1024 + t;
        if (i < m) a[i] = sm.buf[k * 1024 + t];
    }
    __syncthreads();
    return sm.carry;
}

// One block, all chunks in turn.
__global__ void __launch_bounds__(1024) k_scan_exclusive(uint32_t* __restrict__ a, int64_t m) {
    __shared__ ScanSmem sm;
    uint32_t carry = 0;
    for (int64_t base = 0; base < m; base += kScanChunk) carry = scan_chunk(a, m, base, carry, sm);
}

// Large scans: chunk totals, one-block scan of the totals, then every chunk
// scanned from its offset by its own block.
__global__ void __launch_bounds__(1024) k_chunk_totals(const uint32_t* __restrict__ a, int64_t m,
                                                       uint32_t* __restrict__ tot) {
    __shared__ uint32_t wsum[32];
    const int64_t base = int64_t(blockIdx.x) * kScanChunk;
    uint32_t s = 0;
    for (int k = 0; k < kScanPer; k++) {
        const int64_t i = base + int64_t(k) * 1024 + threadIdx.x;
        if (i < m) s += a[i];
    }
    for (int d = 16; d > 0; d >>= 1) s += __shfl_xor_sync(0xffffffffu, s, d);
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = wsum[threadIdx.x];
        for (int d = 16; d > 0; d >>= 1) s += __shfl_xor_sync(0xffffffffu, s, d);
        if (threadIdx.x == 0) tot[blockIdx.x] = s;
    }
}

__global__ void __launch_bounds__(1024) k_chunk_scan(uint32_t* __restrict__ a, int64_t m,
                                                     const uint32_t* __restrict__ off) {
    __shared__ ScanSmem sm;
    scan_chunk(a, m, int64_t(blockIdx.x) * kScanChunk, off[blockIdx.x], sm);
}

__global__ void __launch_bounds__(kSortThreads) k_radix_scatter(int64_t n, const uint32_t* __restrict__ kin,
                                                                const int32_t* __restrict__ vin,
                                                                uint32_t* __restrict__ kout, int32_t* __restrict__ vout,
                                                                int shift, const uint32_t* __restrict__ gofs,
                                                                int nblk) {
    __shared__ uint32_t cnt[kSortWarps][256];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int d = lane; d < 256; d += 32) cnt[w][d] = 0;
    __syncwarp();
    const int64_t base = int64_t(blockIdx.x) * kSortTile + int64_t(w) * kSortPerWarp;
    for (int r = 0; r < kSortPerWarp / 32; r++) {
        const int64_t i = base + r * 32 + lane;
        if (i < n) atomicAdd(&cnt[w][(kin[i] >> shift) & 255u], 1u);
    }
    __syncthreads();
    // per digit: exclusive prefix over warps
    {
        const int d = threadIdx.x;  // 256 threads <-> 256 digits
        uint32_t run = 0;
        for (int ww = 0; ww < kSortWarps; ww++) {
            const uint32_t c = cnt[ww][d];
            cnt[ww][d] = run;
            run += c;
        }
    }
    __syncthreads();
    const uint32_t lt_mask = (1u << lane) - 1u;
    for (int r = 0; r < kSortPerWarp / 32; r++) {
        const int64_t i = base + r * 32 + lane;
        const bool valid = i < n;
        const uint32_t k = valid ? kin[i] : 0u;
        const uint32_t d = (k >> shift) & 255u;
        const uint32_t tag = valid ? d : (256u + lane);
        const uint32_t peers = __match_any_sync(0xffffffffu, tag);
        const uint32_t rank = __popc(peers & lt_mask);
        uint32_t basepos = 0;
        if (valid) basepos = cnt[w][d];
        __syncwarp();
        if (valid) {
            const uint64_t pos = uint64_t(gofs[int64_t(d) * nblk + blockIdx.x]) + basepos + rank;
            kout[pos] = k;
            vout[pos] = vin ? vin[i] : int32_t(i);
            if ((__ffs(peers) - 1) == lane) cnt[w][d] += __popc(peers);
        }
        __syncwarp();
    }
}

// leaf_start[k] = first sorted position whose key is >= k (k = 0..nleaf).
__global__ void k_leaf_bounds(int64_t n, const uint32_t* __restrict__ skey, int32_t nleaf,
                              int32_t* __restrict__ leaf_start) {
    const int64_t s = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (s > n) return;
    const int64_t prev = (s == 0) ? -1 : int64_t(skey[s - 1]);
    const int64_t cur = (s == n) ? int64_t(nleaf) : int64_t(skey[s]);
    for (int64_t k = prev + 1; k <= cur && k <= nleaf; k++) leaf_start[k] = int32_t(s);
}

// ---------------------------------------------------------------- gather

// Sorted (leaf-order) FP64 state from the caller's AoS state, and the
// interaction sources: local coordinates against the leaf's frame centre
// (mixed precision) or absolute coordinates (FP64 / direct sum), w = zeta*A.
template <typename T>
__global__ void k_gather(int64_t n, const double* __restrict__ in5, const double* __restrict__ area_in,
                         const int32_t* __restrict__ perm, const uint32_t* __restrict__ leaf_of,
                         const double4* __restrict__ frame, double4* __restrict__ s0, double4* __restrict__ xs,
                         double* __restrict__ area_s, double* __restrict__ tracer_s,
                         typename Vec4<T>::type* __restrict__ src) {
    const int64_t s = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int64_t i = perm ? perm[s] : s;
    const double4 v = make_double4(in5[5 * i], in5[5 * i + 1], in5[5 * i + 2], in5[5 * i + 3]);
    const double a = area_in[i];
    if (s0) s0[s] = v;
    xs[s] = v;
    area_s[s] = a;
    if (tracer_s) tracer_s[s] = in5[5 * i + 4];
    double cx = 0, cy = 0, cz = 0;
    if (frame && leaf_of) {
        const double4 f = frame[leaf_of[s]];
        cx = f.x; cy = f.y; cz = f.z;
    }
    typename Vec4<T>::type o;
    o.x = T(v.x - cx);
    o.y = T(v.y - cy);
    o.z = T(v.z - cz);
    o.w = T(v.w * a);
    src[s] = o;
}

// ---------------------------------------------------------------- re-sort

// Particles move between RK4 steps; at the start of a step each is put in
// the leaf it is in now.  Its previous leaf key[s] is kept when the
// particle is still inside it (all cone coordinates >= 0), otherwise it
// descends from the 20 root faces (the first child that contains it, else
// the most-inside one).  Cone coordinates c = Minv p come from each face's
// inverse vertex matrix (FP64); the initial build's exact-rounding LU is
// only needed for parity with the reference's assignment.  With `leaves`
// the keys are global leaf indices of an ensemble (each member's leaf level
// and the leaf's index on it from the table; a member's leaves are
// consecutive); without, leaf indices of one tree with leaves on
// `leaf_level`.
__device__ __forceinline__ double min_cone(const NodeGeom& g, double x, double y, double z) {
    const double c0 = g.minv[0] * x + g.minv[1] * y + g.minv[2] * z;
    const double c1 = g.minv[3] * x + g.minv[4] * y + g.minv[5] * z;
    const double c2 = g.minv[6] * x + g.minv[7] * y + g.minv[8] * z;
    return fmin(c0, fmin(c1, c2));
}

// Leaf index on level LL reached from the 20 root faces: on each level the
// first child that contains the point, else the most-inside one.  With l0 >
// 0 the walk starts below face `prev` of level l0 - 1.
__device__ __forceinline__ int descend(const NodeGeom* __restrict__ node, const int64_t* __restrict__ lev_off, int LL,
                                       double4 q, int l0 = 0, int prev = 0) {
    for (int l = l0; l <= LL; l++) {
        const int lb = (l > 0) ? 4 * prev : 0, ub = (l > 0) ? lb + 4 : 20;
        int best = lb;
        double best_min = -1e300;
        for (int j = lb; j < ub; j++) {
            const double m = min_cone(node[lev_off[l] + j], q.x, q.y, q.z);
            if (m >= 0.0) { best = j; break; }
            if (m > best_min) { best_min = m; best = j; }
        }
        prev = best;
    }
    return prev;
}

__global__ void k_reassign(int64_t n, const double4* __restrict__ pos, const EnsLeaf* __restrict__ leaves,
                           int leaf_level, const NodeGeom* __restrict__ node, const int64_t* __restrict__ lev_off,
                           uint32_t* __restrict__ key, int* __restrict__ err) {
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double4 q = pos[i];
    // a non-finite position (a diverged state) fails every cone test and
    // would send the particle down the first-child chain: all such particles
    // would pile into one leaf and one block.  It keeps its leaf instead,
    // and the call reports the error.
    if (!isfinite(q.x) || !isfinite(q.y) || !isfinite(q.z)) {
        set_error(err, kErrNonFinite);
        return;
    }
    const uint32_t g = key[i];
    int LL = leaf_level, local = int(g);
    if (leaves) {
        const EnsLeaf lf = leaves[g];
        LL = lf.leaf_level;
        local = lf.local;
    }
    if (min_cone(node[lev_off[LL] + local], q.x, q.y, q.z) >= 0.0) return;
    key[i] = uint32_t(int64_t(g) - local + descend(node, lev_off, LL, q));
}

// New order q (sorted position -> old position): the step state, areas,
// tracers and caller indices gathered into the free stage buffers (xs, and
// acc as {area, tracer, caller index, 0}).
__global__ void k_resort_gather(int64_t n, const int32_t* __restrict__ q, const double4* __restrict__ s0,
                                const double* __restrict__ area, const double* __restrict__ tracer,
                                const int32_t* __restrict__ perm, double4* __restrict__ xs, double4* __restrict__ acc) {
    const int64_t s = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int64_t j = q[s];
    xs[s] = s0[j];
    acc[s] = make_double4(area[j], tracer[j], double(perm[j]), 0.0);
}

// Back into place, with the stage-1 state (xs = s0) and interaction
// sources (x, y, z, zeta A) of the new order; with ls_new, the new leaf
// ranges (nls entries) copied into leaf_start as well.
template <typename T>
__global__ void k_resort_commit(int64_t n, const double4* __restrict__ xs, const double4* __restrict__ acc,
                                double4* __restrict__ s0, double* __restrict__ area, double* __restrict__ tracer,
                                int32_t* __restrict__ perm, typename Vec4<T>::type* __restrict__ src,
                                const uint32_t* __restrict__ ls_new, int32_t* __restrict__ leaf_start, int64_t nls) {
    const int64_t s = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (ls_new && s < nls) leaf_start[s] = int32_t(ls_new[s]);
    if (s >= n) return;
    const double4 v = xs[s];
    const double4 t = acc[s];
    s0[s] = v;
    area[s] = t.x;
    tracer[s] = t.y;
    perm[s] = int32_t(t.z);
    typename Vec4<T>::type o;
    o.x = T(v.x);
    o.y = T(v.y);
    o.z = T(v.z);
    o.w = T(v.w * t.x);
    src[s] = o;
}

// ---------------------------------------------------------------- re-sort by partition
// Between two steps few particles change leaves, so the stable key sort of
// the new leaf keys is built from the old order instead of sorted again:
// within new leaf k, a stable sort puts first the particles that come from
// old positions before leaf k's old range, then the ones that stayed (in
// their old order), then the ones from after it (each group in old order).
// The stayers' places follow from the old ranges and one scan of the new
// leaf counts; only the movers are bucketed by new leaf and ranked there by
// old position.  The result is the unique stable order, the same as the
// radix sort's.
//
// Scratch words: in[m], out[m], fill[m] (zeroed before every re-sort),
// ns[m + 1] (new leaf starts), mo[m + 1] (bucket starts), m = leaf count.
constexpr int kPartThreads = 256;
// Cone-coordinate margin of the descent's shortcut.  Cone coordinates of a
// point inside a face are O(1) at every level; their FP64 rounding error is
// a few ulp times the row sums of M^-1, which grow like 1 / face size (at
// most 243 on level 7), so about 1e-13: far below the margin.  A face of a
// coarser level is at most 2^7 times larger, so a point that far inside
// one face is still clearly outside every other face of the levels above.
constexpr double kInsideMargin = 1e-6;
constexpr uint32_t kNoLeaf = 0xffffffffu;

// Lanes of a warp that add 1 to the same counter add their count once
// (movers of a warp mostly share their old and their new leaf).  idx =
// kNoLeaf adds nothing.  All 32 lanes call it.
__device__ __forceinline__ void warp_count_add(uint32_t* __restrict__ cnt, uint32_t idx) {
    const unsigned peers = __match_any_sync(0xffffffffu, idx);
    if (idx != kNoLeaf && int(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&cnt[idx], uint32_t(__popc(peers)));
}

// Every particle's new leaf: the old one while the particle is still
// inside it, else the descent's; the counts into and out of every leaf.
__global__ void __launch_bounds__(kPartThreads) k_part_keys(int64_t n, const double4* __restrict__ pos,
                                                            const NodeGeom* __restrict__ node,
                                                            const int64_t* __restrict__ lev_off, int leaf_level,
                                                            const uint32_t* __restrict__ key,
                                                            uint32_t* __restrict__ key_new,
                                                            uint32_t* __restrict__ scratch, int64_t m,
                                                            int* __restrict__ err) {
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    uint32_t from = kNoLeaf, to = kNoLeaf;
    if (i < n) {
        const double4 q = pos[i];
        const uint32_t g = key[i];
        uint32_t g2 = g;
        // a non-finite position keeps its leaf (see k_reassign)
        if (!isfinite(q.x) || !isfinite(q.y) || !isfinite(q.z)) {
            set_error(err, kErrNonFinite);
        } else if (min_cone(node[lev_off[leaf_level] + g], q.x, q.y, q.z) < 0.0) {
            // The lowest ancestor of the old leaf that holds the particle
            // with a margin: every other face of its level and of the levels
            // above lies at least that far away, so each of them fails its
            // test and the descent from the root passes through this
            // ancestor.  Start below it (the root's walk when none qualifies).
            int l = leaf_level - 1;
            uint32_t f = g >> 2;
            for (; l >= 0; l--, f >>= 2)
                if (min_cone(node[lev_off[l] + f], q.x, q.y, q.z) > kInsideMargin) break;
            g2 = uint32_t(l >= 0 ? descend(node, lev_off, leaf_level, q, l + 1, int(f))
                                 : descend(node, lev_off, leaf_level, q));
        }
        key_new[i] = g2;
        if (g2 != g) {
            from = g;
            to = g2;
        }
    }
    warp_count_add(scratch, to);        // in
    warp_count_add(scratch + m, from);  // out
}

// One block of 1024 threads: ns = exclusive scan of the new leaf counts
// (old count - out + in), mo = exclusive scan of in; entry m holds the
// totals.  Chunks of 4096 entries pass through shared memory, so that the
// global loads and stores are coalesced.
__device__ void part_scan(int64_t m, const int32_t* __restrict__ ls, const uint32_t* __restrict__ in,
                          const uint32_t* __restrict__ out, uint32_t* __restrict__ ns, uint32_t* __restrict__ mo) {
    constexpr int R = 4, T = 1024, C = R * T;
    __shared__ uint32_t ba[C], bb[C];
    __shared__ uint32_t wa[T / 32], wb[T / 32];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    uint32_t ca = 0, cb = 0;  // carries (block-uniform)
    for (int64_t base = 0; base < m; base += C) {
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int64_t k = base + int64_t(r) * T + t;
            uint32_t va = 0, vb = 0;
            if (k < m) {
                vb = in[k];
                va = uint32_t(ls[k + 1] - ls[k]) - out[k] + vb;
            }
            ba[r * T + t] = va;
            bb[r * T + t] = vb;
        }
        __syncthreads();
        uint32_t va[R], vb[R], sa = 0, sb = 0;  // thread t: entries [R t, R t + R) of the chunk
#pragma unroll
        for (int r = 0; r < R; r++) {
            va[r] = ba[t * R + r];
            vb[r] = bb[t * R + r];
            sa += va[r];
            sb += vb[r];
        }
        uint32_t xa = sa, xb = sb;  // inclusive warp scan
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t ya = __shfl_up_sync(0xffffffffu, xa, d), yb = __shfl_up_sync(0xffffffffu, xb, d);
            if (lane >= d) { xa += ya; xb += yb; }
        }
        if (lane == 31) { wa[w] = xa; wb[w] = xb; }
        __syncthreads();
        uint32_t oa = ca, ob = cb, ta = 0, tb = 0;
        for (int v = 0; v < T / 32; v++) {
            if (v < w) { oa += wa[v]; ob += wb[v]; }
            ta += wa[v];
            tb += wb[v];
        }
        oa += xa - sa;
        ob += xb - sb;
#pragma unroll
        for (int r = 0; r < R; r++) {
            ba[t * R + r] = oa;
            bb[t * R + r] = ob;
            oa += va[r];
            ob += vb[r];
        }
        ca += ta;
        cb += tb;
        __syncthreads();
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int64_t k = base + int64_t(r) * T + t;
            if (k < m) {
                ns[k] = ba[r * T + t];
                mo[k] = bb[r * T + t];
            }
        }
        __syncthreads();
    }
    if (t == 0) { ns[m] = ca; mo[m] = cb; }
}

// The scan of the counts, by one block of kScanThreads.
constexpr int kScanThreads = 1024;
__global__ void __launch_bounds__(kScanThreads) k_part_scan(uint32_t* __restrict__ scratch, int64_t m,
                                                           const int32_t* __restrict__ ls) {
    uint32_t* ns = scratch + 3 * m;
    part_scan(m, ls, scratch, scratch + m, ns, ns + m + 1);
}

// Movers into their new leaf's bucket (unordered within it).
__global__ void __launch_bounds__(kPartThreads) k_part_bucket(int64_t n, const uint32_t* __restrict__ key,
                                                              const uint32_t* __restrict__ key_new,
                                                              uint32_t* __restrict__ scratch, int64_t m,
                                                              int32_t* __restrict__ bucket) {
    uint32_t* fill = scratch + 2 * m;
    const uint32_t* mo = scratch + 3 * m + (m + 1);
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    uint32_t to = kNoLeaf;
    if (i < n) {
        const uint32_t g2 = key_new[i];
        if (g2 != key[i]) to = g2;
    }
    // lanes bound for the same leaf reserve their slots with one atomic
    const unsigned peers = __match_any_sync(0xffffffffu, to);
    const int leader = __ffs(peers) - 1;
    uint32_t slot = 0;
    if (to != kNoLeaf && lane == leader) slot = atomicAdd(&fill[to], uint32_t(__popc(peers)));
    slot = __shfl_sync(0xffffffffu, slot, leader);
    if (to != kNoLeaf) bucket[mo[to] + slot + uint32_t(__popc(peers & ((1u << lane) - 1u)))] = int32_t(i);
}

// One block per new leaf k: its movers ranked by old position, its stayers
// in old order, each particle's state gathered into its new place (xs, and
// acc as {area, tracer, caller index, 0}), the new sorted keys written.
constexpr int kPlaceThreads = 128;
constexpr int kPlaceStage = 512;  // movers into one leaf ranked from shared memory
__global__ void __launch_bounds__(kPlaceThreads) k_part_place(
    int64_t m, const int32_t* __restrict__ ls, const uint32_t* __restrict__ key_new,
    const uint32_t* __restrict__ scratch, const int32_t* __restrict__ bucket, const double4* __restrict__ s0,
    const double* __restrict__ area, const double* __restrict__ tracer, const int32_t* __restrict__ perm,
    double4* __restrict__ xs, double4* __restrict__ acc, uint32_t* __restrict__ key) {
    constexpr int W = kPlaceThreads / 32;
    __shared__ uint32_t wcnt[W];
    const int64_t k = blockIdx.x;
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const uint32_t* in = scratch;
    const uint32_t* out = scratch + m;
    const uint32_t* ns = scratch + 3 * m;
    const uint32_t* mo = ns + m + 1;
    const int32_t a = ls[k], b = ls[k + 1];
    const uint32_t base = ns[k], c = in[k], m0 = mo[k];
    const uint32_t stays = uint32_t(b - a) - out[k];
    auto place = [&](int64_t p, int64_t dst) {
        xs[dst] = s0[p];
        acc[dst] = make_double4(area[p], tracer[p], double(perm[p]), 0.0);
    };
    // movers: rank = number of movers into k with a smaller old position
    // (the bucket staged in shared memory when it fits)
    __shared__ int32_t bk[kPlaceStage];
    const bool staged = c <= uint32_t(kPlaceStage);
    if (staged)
        for (uint32_t u = t; u < c; u += kPlaceThreads) bk[u] = bucket[m0 + u];
    uint32_t below = 0;
    for (uint32_t u0 = 0; u0 < c; u0 += kPlaceThreads) {
        const uint32_t u = u0 + t;
        below += uint32_t(__syncthreads_count(u < c && (staged ? bk[u] : bucket[m0 + u]) < a));
    }
    for (uint32_t j = t; j < c; j += kPlaceThreads) {
        const int32_t p = staged ? bk[j] : bucket[m0 + j];
        uint32_t r = 0;
        if (staged)
            for (uint32_t u = 0; u < c; u++) r += bk[u] < p ? 1u : 0u;
        else
            for (uint32_t u = 0; u < c; u++) r += bucket[m0 + u] < p ? 1u : 0u;
        place(p, int64_t(base) + r + (p >= a ? stays : 0u));
    }
    // stayers, in old order after the movers from below
    uint32_t run = base + below;
    for (int32_t p0 = a; p0 < b; p0 += kPlaceThreads) {
        const int32_t p = p0 + t;
        const bool st = p < b && key_new[p] == uint32_t(k);
        const unsigned bal = __ballot_sync(0xffffffffu, st);
        if (lane == 0) wcnt[w] = uint32_t(__popc(bal));
        __syncthreads();
        uint32_t off = 0, tot = 0;
#pragma unroll
        for (int v = 0; v < W; v++) {
            const uint32_t x = wcnt[v];
            if (v < w) off += x;
            tot += x;
        }
        if (st) place(p, int64_t(run) + off + uint32_t(__popc(bal & ((1u << lane) - 1u))));
        run += tot;
        __syncthreads();
    }
    const uint32_t cnt = stays + c;
    for (uint32_t j = t; j < cnt; j += kPlaceThreads) key[base + j] = uint32_t(k);
}

// ---------------------------------------------------------------- launchers

void launch_assign(cudaStream_t st, int64_t n, const double* in5, const double* verts, const int32_t* tri_verts,
                   const int64_t* lev_off, int tree_levels, int reference_mode, int32_t* loc, uint32_t* key, int* err) {
    if (n == 0) return;
    k_assign<<<unsigned((n + 127) / 128), 128, 0, st>>>(n, in5, verts, tri_verts, lev_off, tree_levels, reference_mode,
                                                        loc, key, err);
}

void launch_level_hist(cudaStream_t st, int64_t n, int tree_levels, const int32_t* loc, const int64_t* lev_off,
                       int32_t* counts) {
    if (n == 0) return;
    k_level_hist<<<unsigned((n + 255) / 256), 256, 0, st>>>(n, tree_levels, loc, lev_off, counts);
}

int64_t scan_part_words(int64_t m) { return (m + kScanChunk - 1) / kScanChunk; }

void launch_scan_u32(cudaStream_t st, uint32_t* a, int64_t m, uint32_t* part) {
    if (m <= 0) return;
    const int64_t nchunk = scan_part_words(m);
    if (nchunk <= 4 || !part) {
        k_scan_exclusive<<<1, 1024, 0, st>>>(a, m);
        return;
    }
    k_chunk_totals<<<unsigned(nchunk), 1024, 0, st>>>(a, m, part);
    k_scan_exclusive<<<1, 1024, 0, st>>>(part, nchunk);
    k_chunk_scan<<<unsigned(nchunk), 1024, 0, st>>>(a, m, part);
}

// Digit histograms (256 per block), then the scan's chunk totals.
int64_t sort_scratch_words(int64_t n) {
    const int64_t nblk = (n + kSortTile - 1) / kSortTile;
    return 256 * nblk + scan_part_words(256 * nblk);
}

int sort_launch_count(int64_t n, int bits) {
    if (n == 0) return 0;
    const int64_t nblk = (n + kSortTile - 1) / kSortTile;
    const int scan = scan_part_words(256 * nblk) <= 4 ? 1 : 3;
    return ((bits + 7) / 8) * (2 + scan);
}

void launch_sort(cudaStream_t st, int64_t n, int bits, uint32_t* keys, uint32_t* keys_tmp, int32_t* vals,
                 int32_t* vals_tmp, uint32_t* hist) {
    if (n == 0) return;
    const int nblk = int((n + kSortTile - 1) / kSortTile);
    uint32_t *ki = keys, *ko = keys_tmp;
    int32_t *vi = nullptr, *vo = vals;
    int pass = 0;
    for (int shift = 0; shift < bits; shift += 8, pass++) {
        k_radix_hist<<<nblk, kSortThreads, 0, st>>>(n, ki, shift, hist, nblk);
        launch_scan_u32(st, hist, int64_t(256) * nblk, hist + int64_t(256) * nblk);
        k_radix_scatter<<<nblk, kSortThreads, 0, st>>>(n, ki, vi, ko, vo, shift, hist, nblk);
        std::swap(ki, ko);
        vi = vo;
        vo = (vo == vals) ? vals_tmp : vals;
    }
    // results end in (ki, vi); make sure they are in (keys, vals)
    if (ki != keys) cudaMemcpyAsync(keys, ki, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st);
    if (vi != vals) cudaMemcpyAsync(vals, vi, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, st);
}

void launch_leaf_bounds(cudaStream_t st, int64_t n, const uint32_t* skey, int32_t nleaf, int32_t* leaf_start) {
    k_leaf_bounds<<<unsigned((n + 1 + 255) / 256), 256, 0, st>>>(n, skey, nleaf, leaf_start);
}

void launch_gather(cudaStream_t st, bool fp64, int64_t n, const double* in5, const double* area_in, const int32_t* perm,
                   const uint32_t* leaf_of, const double4* frame, double4* s0, double4* xs, double* area_s,
                   double* tracer_s, void* src) {
    if (n == 0) return;
    const unsigned g = unsigned((n + 255) / 256);
    if (fp64)
        k_gather<double><<<g, 256, 0, st>>>(n, in5, area_in, perm, leaf_of, frame, s0, xs, area_s, tracer_s,
                                            static_cast<double4*>(src));
    else
        k_gather<float><<<g, 256, 0, st>>>(n, in5, area_in, perm, leaf_of, frame, s0, xs, area_s, tracer_s,
                                           static_cast<float4*>(src));
}

void launch_reassign(cudaStream_t st, int64_t n, const double4* pos, const EnsLeaf* leaves, int leaf_level,
                     const NodeGeom* node, const int64_t* lev_off, uint32_t* key, int* err) {
    if (n == 0) return;
    k_reassign<<<unsigned((n + 255) / 256), 256, 0, st>>>(n, pos, leaves, leaf_level, node, lev_off, key, err);
}

void launch_resort(cudaStream_t st, bool fp64, int64_t n, const int32_t* q, double4* s0, double* area,
                   double* tracer, int32_t* perm, double4* xs, double4* acc, void* src) {
    if (n == 0) return;
    const unsigned g = unsigned((n + 255) / 256);
    k_resort_gather<<<g, 256, 0, st>>>(n, q, s0, area, tracer, perm, xs, acc);
    if (fp64)
        k_resort_commit<double><<<g, 256, 0, st>>>(n, xs, acc, s0, area, tracer, perm, static_cast<double4*>(src),
                                                   nullptr, nullptr, 0);
    else
        k_resort_commit<float><<<g, 256, 0, st>>>(n, xs, acc, s0, area, tracer, perm, static_cast<float4*>(src),
                                                  nullptr, nullptr, 0);
}

int64_t partition_scratch_words(int64_t nleaf) { return 3 * nleaf + 2 * (nleaf + 1); }

void launch_resort_partition(cudaStream_t st, bool fp64, int64_t n, int64_t nleaf, int leaf_level,
                             const NodeGeom* node, const int64_t* lev_off, uint32_t* key, uint32_t* key_new,
                             int32_t* leaf_start, int32_t* bucket, uint32_t* scratch, double4* s0, double* area,
                             double* tracer, int32_t* perm, double4* xs, double4* acc, void* src, int* err) {
    if (n == 0) return;
    cudaMemsetAsync(scratch, 0, sizeof(uint32_t) * size_t(3 * nleaf), st);
    const unsigned grid = unsigned((n + kPartThreads - 1) / kPartThreads);
    k_part_keys<<<grid, kPartThreads, 0, st>>>(n, s0, node, lev_off, leaf_level, key, key_new, scratch, nleaf, err);
    k_part_scan<<<1, kScanThreads, 0, st>>>(scratch, nleaf, leaf_start);
    k_part_bucket<<<grid, kPartThreads, 0, st>>>(n, key, key_new, scratch, nleaf, bucket);
    k_part_place<<<unsigned(nleaf), kPlaceThreads, 0, st>>>(
        nleaf, leaf_start, key_new, scratch, bucket, s0, area, tracer, perm, xs, acc, key);
    const uint32_t* ns = scratch + 3 * nleaf;
    const unsigned g = unsigned((std::max(n, nleaf + 1) + 255) / 256);
    if (fp64)
        k_resort_commit<double><<<g, 256, 0, st>>>(n, xs, acc, s0, area, tracer, perm, static_cast<double4*>(src),
                                                   ns, leaf_start, nleaf + 1);
    else
        k_resort_commit<float><<<g, 256, 0, st>>>(n, xs, acc, s0, area, tracer, perm, static_cast<float4*>(src), ns,
                                                  leaf_start, nleaf + 1);
}

}  // namespace fss
