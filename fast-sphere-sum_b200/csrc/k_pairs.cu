// k_pairs.cu -- the pair engine shared by the direct sum, the near field and
// the particle-cluster far field.
//
// A block works on one work item: the targets of one leaf (taken in chunks
// of the consumer count; the leaf's current particle range is read from
// leaf_start on the device, since particles are re-sorted into the leaves
// they have moved into) or an explicit target range (direct sum).  Its
// sources are a list of segments -- the particles of a run of leaves (range
// read at run time) or a fixed range of far-cluster proxies -- which warp 0
// packs back to back into shared-memory tiles as it goes, issuing one bulk
// TMA copy (cp.async.bulk, no multicast) per piece with completion counted
// on the tile slot's mbarrier.  Tiles circulate in a ring of DEPTH slots
// (kDepth = 4; kClusterDepth = 3 for the target-cluster launch's small
// blocks) released by the consumer warps through a second mbarrier; an
// empty tile ends a chunk.  Warp 0 only produces (and, in FP32, converts each landed
// tile to pair-interleaved order for the packed f32x2 pipe); the other warps
// consume, one target per thread.  Per pair (23 algorithmic flops):
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
constexpr int kClusterDepth = 3;  // ring depth of the target-cluster launch
constexpr int TILE_F32 = tile_capacity(false);
constexpr float kSelfR2 = 1e-30f;  // r^2 bias of the FP32 loop (a normal float; 1 / kSelfR2 finite)

// Sources j = j0, j0 + step, ... < cnt of an FP64 tile (step 1: all of them).
template <typename T, bool PSI, bool GUARD, bool STRIDED>
__device__ __forceinline__ void tile_pairs(const typename Vec4<T>::type* __restrict__ s, int cnt, int j0, int step,
                                           T tx, T ty, T tz, T& ax, T& ay, T& az, T& ap) {
    if (!STRIDED) {
        j0 = 0;
        step = 1;
    }
#pragma unroll(STRIDED ? 2 : 8)
    for (int j = j0; j < cnt; j += step) {
        const typename Vec4<T>::type q = s[j];
        const T dx = q.x - tx, dy = q.y - ty, dz = q.z - tz;
        const T r2 = fma(dz, dz, fma(dy, dy, dx * dx));
        T inv = rcp_fast(r2);
        if (GUARD) inv = (r2 > T(0)) ? inv : T(0);
        const T sc = q.w * inv;
        ax = fma(sc, dx, ax);
        ay = fma(sc, dy, ay);
        az = fma(sc, dz, az);
        if (PSI) {
            T lg = lg2_fast(r2);
            if (GUARD) lg = (r2 > T(0)) ? lg : T(0);
            ap = fma(q.w, lg, ap);
        }
    }
}

// FP32 tiles in SoA order: x[TILE], y[TILE], z[TILE], w[TILE], padded to a
// multiple of 4 sources with w = 0 at the origin (|x_i - 0|^2 = 1, no
// contribution).  One 128-bit shared load brings a component of four
// sources; each pair of sources goes through the packed f32x2 pipe: per
// four sources 4 shared loads, 20 packed operations and 4 reciprocals.
// The self pair (and any source at the target's position) needs no select:
// r^2 starts from kSelfR2 = 1e-30 inside the first FMA, so it gets
// 1 / r^2 = 1e30 and w 1e30 * (x_j - x_i) = 0; every other pair's r^2 (at
// least ~1e-12 between distinct particles on the unit sphere) is unchanged
// by the bias except when the exact d_x^2 falls on a rounding tie.  Only
// the stream function's log needs the guard (GUARD: tiles holding targets).
// Quads q = q0, q0 + step, ... < nquad of the tile (step 1: all of them).
template <bool PSI, bool GUARD, bool STRIDED>
__device__ __forceinline__ void tile_pairs_soa(const float* __restrict__ s, int nquad, int q0, int step, f2 ntx,
                                               f2 nty, f2 ntz, f2& ax, f2& ay, f2& az, float& ap) {
    constexpr int T = TILE_F32;
    if (!STRIDED) {
        q0 = 0;
        step = 1;
    }
    const f2 eps = f2_pack(kSelfR2, kSelfR2);
#pragma unroll 4
    for (int q = q0; q < nquad; q += step) {
        const float4 X = reinterpret_cast<const float4*>(s)[q];
        const float4 Y = reinterpret_cast<const float4*>(s + T)[q];
        const float4 Z = reinterpret_cast<const float4*>(s + 2 * T)[q];
        const float4 W = reinterpret_cast<const float4*>(s + 3 * T)[q];
        const f2 qx[2] = {f2_pack(X.x, X.y), f2_pack(X.z, X.w)};
        const f2 qy[2] = {f2_pack(Y.x, Y.y), f2_pack(Y.z, Y.w)};
        const f2 qz[2] = {f2_pack(Z.x, Z.y), f2_pack(Z.z, Z.w)};
        const f2 qw[2] = {f2_pack(W.x, W.y), f2_pack(W.z, W.w)};
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const f2 dx = f2_add(qx[h], ntx);
            const f2 dy = f2_add(qy[h], nty);
            const f2 dz = f2_add(qz[h], ntz);
            const f2 r2 = f2_fma(dz, dz, f2_fma(dy, dy, f2_fma(dx, dx, eps)));
            float r0, r1;
            f2_unpack(r2, r0, r1);
            const float i0 = rcp_fast(r0), i1 = rcp_fast(r1);
            const f2 sc = f2_mul(qw[h], f2_pack(i0, i1));
            ax = f2_fma(sc, dx, ax);
            ay = f2_fma(sc, dy, ay);
            az = f2_fma(sc, dz, az);
            if (PSI) {
                float l0 = lg2_fast(r0), l1 = lg2_fast(r1);
                if (GUARD) {
                    l0 = (r0 > kSelfR2) ? l0 : 0.f;
                    l1 = (r1 > kSelfR2) ? l1 : 0.f;
                }
                float w0, w1;
                f2_unpack(qw[h], w0, w1);
                ap = fmaf(w0, l0, fmaf(w1, l1, ap));
            }
        }
    }
}

// Transposition of a landed FP32 tile of `cnt` float4 sources into SoA
// order, by one warp: lane L reads sources [8L, 8L + 8) and writes their 8
// entries of each component array (padding [cnt, 4 ceil(cnt / 4)) with
// zeros).
__device__ __forceinline__ void tile_to_soa(const float4* __restrict__ in, float* __restrict__ out, int cnt) {
    constexpr int T = TILE_F32;
    const int lane = threadIdx.x & 31;
    const int j0 = 8 * lane;
    const int padded = (cnt + 3) & ~3;
    if (j0 >= padded) return;
#pragma unroll
    for (int half = 0; half < 2; half++) {
        const int j = j0 + 4 * half;
        if (j >= padded) break;
        float4 v[4];
#pragma unroll
        for (int k = 0; k < 4; k++) v[k] = (j + k < cnt) ? in[j + k] : make_float4(0.f, 0.f, 0.f, 0.f);
        reinterpret_cast<float4*>(out + j)[0] = make_float4(v[0].x, v[1].x, v[2].x, v[3].x);
        reinterpret_cast<float4*>(out + T + j)[0] = make_float4(v[0].y, v[1].y, v[2].y, v[3].y);
        reinterpret_cast<float4*>(out + 2 * T + j)[0] = make_float4(v[0].z, v[1].z, v[2].z, v[3].z);
        reinterpret_cast<float4*>(out + 3 * T + j)[0] = make_float4(v[0].w, v[1].w, v[2].w, v[3].w);
    }
}

template <typename T>
__device__ __forceinline__ void kahan_add(T& sum, T& comp, T x) {
    const T y = x - comp;
    const T t = sum + y;
    comp = (t - sum) - y;
    sum = t;
}

// Sum over the L lanes of each group [L t, L t + L) of the warp (segmented
// tree of shuffles, L warp-uniform); the group's first lane (sub = 0) holds
// the sum.
template <typename T>
__device__ __forceinline__ T group_sum(T x, int sub, int L) {
    for (int off = 1; off < L; off <<= 1) {
        const T y = __shfl_down_sync(0xffffffffu, x, off);
        if (sub + off < L) x += y;
    }
    return x;
}

// Producer side of the ring: warp 0 packs the next tile of a work item's
// sources.  Lane i resolves segment g + i to its range [lo, hi) (kind 0
// through leaf_start), a warp scan places the ranges back to back, and each
// lane issues the bulk copy of its piece; the segment cut by the end of the
// tile is resumed at `off` by the next tile.  Returns the tile's source
// count (0: the item's sources are exhausted); `guard` is set when a piece
// overlaps the targets [t0, t1) (a source that is one of the block's own
// targets must skip the self pair).  The transaction bytes of each round
// are expected on `bar` by lane 0 before any lane issues its copy.
template <typename S4, int TILE>
__device__ __forceinline__ int pack_tile(const Segment* __restrict__ segs, const int32_t* __restrict__ leaf_start,
                                         int g1, int& g, int& off, int t0, int t1, const S4* __restrict__ src,
                                         S4* dst, uint64_t* bar, bool& guard) {
    const int lane = threadIdx.x & 31;
    int count = 0;
    bool gd = false;
    while (g < g1 && count < TILE) {
        const int gi = g + lane;
        int lo = 0, hi = 0;
        if (gi < g1) {
            const Segment sg = segs[gi];
            if (sg.kind == 0) {
                lo = leaf_start[sg.a];
                hi = leaf_start[sg.b];
            } else {
                lo = sg.a;
                hi = sg.b;
            }
            if (lane == 0) lo += off;
        }
        const int len = max(hi - lo, 0);
        int incl = len;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += y;
        }
        const int excl = incl - len;
        const int room = TILE - count;
        const int take = max(0, min(len, room - excl));
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        const int placed = min(total, room);
        if (lane == 0 && placed > 0) mbar_expect_tx(bar, uint32_t(placed) * uint32_t(sizeof(S4)));
        __syncwarp();
        if (take > 0) {
            bulk_g2s(dst + count + excl, src + lo, uint32_t(take) * uint32_t(sizeof(S4)), bar);
            if (lo < t1 && lo + take > t0) gd = true;
        }
        if (total <= room) {
            g = min(g + 32, g1);
            off = 0;
            count += total;
        } else {
            const int k = __ffs(__ballot_sync(0xffffffffu, incl > room)) - 1;
            const int ek = __shfl_sync(0xffffffffu, excl, k);
            off = (k == 0 ? off : 0) + (room - ek);
            g += k;
            count = TILE;
        }
    }
    guard = __any_sync(0xffffffffu, gd) != 0;
    return count;
}

// Tile header written by the producer before the slot's arrive (the
// consumers read it after the slot's phase completes).
struct SlotHdr {
    int count, guard;
};

struct RingState {
    int64_t issued, consumed, converted;
    bool failed;
};

// One work item: every chunk of targets against every tile of its segments.
// Warp 0 is the producer: it packs and issues the tiles and (FP32) converts
// each landed tile to the pair-interleaved order, releasing it through
// ready_bar; it computes nothing.  Warps 1.. are the consumers, one target
// per thread (THREADS - 32 targets per chunk); they wait on ready_bar (FP32)
// or full_bar (FP64) and release a slot through empty_bar.
template <typename T, int THREADS, int TILE, bool PSI, int DEPTH>
__device__ __forceinline__ void run_item(const WorkItem& it, const typename Vec4<T>::type* __restrict__ src,
                                         const Segment* __restrict__ segs, const int32_t* __restrict__ leaf_start,
                                         double4* __restrict__ partials, int64_t pstride,
                                         typename Vec4<T>::type* ring, float* soa, SlotHdr* hdr, uint64_t* full_bar,
                                         uint64_t* empty_bar, uint64_t* ready_bar, RingState& rs,
                                         const PairCtl& ctl, bool hold) {
    using S4 = typename Vec4<T>::type;
    constexpr bool kPacked = sizeof(T) == 4;
    constexpr int kTargets = THREADS - 32;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    int t0 = it.t0, nt = it.nt;
    if (it.leaf >= 0) {
        t0 = leaf_start[it.leaf];
        nt = leaf_start[it.leaf + 1] - t0;
    }
    for (int c0 = 0; c0 < nt && !rs.failed; c0 += kTargets) {
        const int cn = min(kTargets, nt - c0);
        if (warp == 0) {
            // ------------------------------------------------ producer
            int pg = it.g0, poff = 0;
            bool pdone = false;
            for (;;) {
                // convert every produced tile (each waits for its copies)
                while (kPacked && rs.converted < rs.issued && !rs.failed) {
                    const int slot = int(rs.converted % DEPTH);
                    if (!__all_sync(0xffffffffu, mbar_wait_bounded(&full_bar[slot], uint32_t(rs.converted / DEPTH) & 1,
                                                                   ctl.wait_ns))) {
                        rs.failed = true;
                        break;
                    }
                    tile_to_soa(reinterpret_cast<const float4*>(ring + slot * TILE), soa + slot * 4 * TILE,
                                hdr[slot].count);
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&ready_bar[slot]);
                    rs.converted++;
                }
                if (pdone || rs.failed) break;
                // the next tile, once its slot is free (then the empty tile
                // that ends the chunk)
                const int slot = int(rs.issued % DEPTH);
                bool ok = true;
                if (rs.issued >= DEPTH)
                    ok = mbar_wait_bounded(&empty_bar[slot], uint32_t((rs.issued / DEPTH) - 1) & 1, ctl.wait_ns);
                if (!__all_sync(0xffffffffu, ok)) {
                    rs.failed = true;
                    break;
                }
                bool gd = false;
                int cnt = 1;
                if (hold && rs.issued == 0) {
                    // test hook: the first tile is neither copied nor signalled
                    if (lane == 0) hdr[slot].count = cnt;
                } else {
                    cnt = pack_tile<S4, TILE>(segs, leaf_start, it.g1, pg, poff, t0 + c0, t0 + c0 + cn, src,
                                              ring + slot * TILE, &full_bar[slot], gd);
                    if (lane == 0) {
                        hdr[slot].count = cnt;
                        hdr[slot].guard = gd ? 1 : 0;
                        mbar_arrive(&full_bar[slot]);
                    }
                }
                __syncwarp();
                if (cnt == 0) pdone = true;
                rs.issued++;
            }
            rs.consumed = rs.issued;
        } else {
            // ------------------------------------------------ consumers
            // consumer warp cw takes targets [32 cw, 32 cw + 32) of the chunk;
            // the last, partial warp (r < 32 targets) gives every target
            // L = 32 / r lanes, which split each tile's sources between them
            // and add their sums by shuffles, so that few of its lanes compute
            // for no target (a block's time per tile is set by its full warps)
            const int cw = warp - 1;
            const int r = min(32, cn - 32 * cw);
            const bool active = r > 0;
            const int L = (r > 0 && r < 32) ? 32 / r : 1;
            const int tl = lane / L, sub = lane - tl * L;
            const bool has_t = active && tl < r;
            const int tgt = 32 * cw + tl;
            const S4 v = src[t0 + c0 + (has_t ? tgt : 0)];
            T ax = 0, ay = 0, az = 0, ap = 0, sx = 0, sy = 0, sz = 0, sp = 0, cx = 0, cy = 0, cz = 0, cp = 0;
            f2 ntx = 0, nty = 0, ntz = 0;
            if (kPacked) {
                ntx = f2_pack(-float(v.x), -float(v.x));
                nty = f2_pack(-float(v.y), -float(v.y));
                ntz = f2_pack(-float(v.z), -float(v.z));
            }
            for (;;) {
                const int slot = int(rs.consumed % DEPTH);
                uint64_t* wait_bar = kPacked ? &ready_bar[slot] : &full_bar[slot];
                if (!__all_sync(0xffffffffu,
                                mbar_wait_bounded(wait_bar, uint32_t(rs.consumed / DEPTH) & 1, ctl.wait_ns))) {
                    rs.failed = true;
                    break;
                }
                const SlotHdr h = hdr[slot];
                if (active && h.count > 0) {
                    if constexpr (kPacked) {
                        const float* tile = soa + slot * 4 * TILE;
                        const int nq = (h.count + 3) >> 2;
                        f2 px = 0, py = 0, pz = 0;
                        float pw = 0.f;
                        // (the velocity needs no guard; only the stream function's log does)
                        if (L == 1) {
                            if (PSI && h.guard)
                                tile_pairs_soa<PSI, true, false>(tile, nq, 0, 1, ntx, nty, ntz, px, py, pz, pw);
                            else
                                tile_pairs_soa<PSI, false, false>(tile, nq, 0, 1, ntx, nty, ntz, px, py, pz, pw);
                        } else {
                            if (PSI && h.guard)
                                tile_pairs_soa<PSI, true, true>(tile, nq, sub, L, ntx, nty, ntz, px, py, pz, pw);
                            else
                                tile_pairs_soa<PSI, false, true>(tile, nq, sub, L, ntx, nty, ntz, px, py, pz, pw);
                        }
                        float a0, a1;
                        f2_unpack(px, a0, a1);
                        float tx = a0 + a1;
                        f2_unpack(py, a0, a1);
                        float ty = a0 + a1;
                        f2_unpack(pz, a0, a1);
                        float tz = a0 + a1;
                        if (L > 1) {
                            tx = group_sum(tx, sub, L);
                            ty = group_sum(ty, sub, L);
                            tz = group_sum(tz, sub, L);
                            if (PSI) pw = group_sum(pw, sub, L);
                        }
                        kahan_add(sx, cx, T(tx));
                        kahan_add(sy, cy, T(ty));
                        kahan_add(sz, cz, T(tz));
                        if (PSI) kahan_add(sp, cp, T(pw));
                    } else {
                        const S4* tile = ring + slot * TILE;
                        if (L == 1) {
                            if (h.guard)
                                tile_pairs<T, PSI, true, false>(tile, h.count, 0, 1, v.x, v.y, v.z, ax, ay, az, ap);
                            else
                                tile_pairs<T, PSI, false, false>(tile, h.count, 0, 1, v.x, v.y, v.z, ax, ay, az, ap);
                        } else {
                            if (h.guard)
                                tile_pairs<T, PSI, true, true>(tile, h.count, sub, L, v.x, v.y, v.z, ax, ay, az, ap);
                            else
                                tile_pairs<T, PSI, false, true>(tile, h.count, sub, L, v.x, v.y, v.z, ax, ay, az, ap);
                        }
                    }
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(&empty_bar[slot]);
                rs.consumed++;
                if (h.count == 0) break;
            }
            if (!kPacked && L > 1) {  // the FP64 path sums plainly: add the lanes' shares once
                ax = group_sum(ax, sub, L);
                ay = group_sum(ay, sub, L);
                az = group_sum(az, sub, L);
                if (PSI) ap = group_sum(ap, sub, L);
            }
            if (!rs.failed && has_t && sub == 0) {
                double4 o;
                if (kPacked)
                    o = make_double4(double(sx) - double(cx), double(sy) - double(cy), double(sz) - double(cz),
                                     double(sp) - double(cp));
                else
                    o = make_double4(double(ax), double(ay), double(az), double(ap));
                partials[int64_t(it.part) * pstride + t0 + c0 + tgt] = o;
            }
            rs.issued = rs.consumed;
        }
        // every tile produced for this chunk has been consumed, so the
        // counters agree in every warp unless a wait gave up
        rs.failed = __syncthreads_or(rs.failed) != 0;
        if (rs.failed) {
            // no bulk copy may still be landing in this block's shared memory
            // when it exits: the producer waits (bounded) for the tiles not
            // known to have landed -- at most the last DEPTH it issued
            if (warp == 0) {
                int64_t t = rs.issued - DEPTH;
                if (kPacked && rs.converted > t) t = rs.converted;
                for (t = (t < 0) ? 0 : t; t < rs.issued; t++)
                    mbar_wait_bounded(&full_bar[t % DEPTH], uint32_t(t / DEPTH) & 1, ctl.wait_ns);
            }
            return;
        }
    }
}

// Shared memory of a pair block: the landing ring (DEPTH tiles as copied)
// and, in FP32, the SoA ring the consumers read.
template <typename T, int TILE, int DEPTH = kDepth>
FSS_HD constexpr size_t ring_bytes() { return size_t(DEPTH) * TILE * sizeof(typename Vec4<T>::type); }
template <typename T, int TILE, int DEPTH = kDepth>
FSS_HD constexpr size_t pair_smem_bytes() {
    return ring_bytes<T, TILE, DEPTH>() + (sizeof(T) == 4 ? size_t(DEPTH) * 4 * TILE * sizeof(float) : 0);
}

__device__ __forceinline__ void init_ring(uint64_t* full_bar, uint64_t* empty_bar, uint64_t* ready_bar, int warps,
                                          int depth) {
    if (threadIdx.x == 0) {
        for (int d = 0; d < depth; d++) {
            mbar_init(&full_bar[d], 1);
            mbar_init(&empty_bar[d], warps - 1);  // consumer warps
            mbar_init(&ready_bar[d], 1);
        }
        mbar_init_fence();
    }
    __syncthreads();
}

// One block per work item; a ring of DEPTH tile slots.
template <typename T, int THREADS, bool PSI, int TILE, int DEPTH>
__global__ void __launch_bounds__(THREADS) k_pairs(const typename Vec4<T>::type* __restrict__ src,
                                                   const Segment* __restrict__ segs,
                                                   const int32_t* __restrict__ leaf_start,
                                                   const WorkItem* __restrict__ items, double4* __restrict__ partials,
                                                   int64_t pstride, int* __restrict__ err, const PairCtl ctl) {
    using S4 = typename Vec4<T>::type;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full_bar[DEPTH], empty_bar[DEPTH], ready_bar[DEPTH];
    __shared__ SlotHdr hdr[DEPTH];
    init_ring(full_bar, empty_bar, ready_bar, THREADS / 32, DEPTH);
    RingState rs{0, 0, 0, false};
    const WorkItem it = items[blockIdx.x];
    run_item<T, THREADS, TILE, PSI, DEPTH>(it, src, segs, leaf_start, partials, pstride,
                                           reinterpret_cast<S4*>(smem_raw),
                                           reinterpret_cast<float*>(smem_raw + ring_bytes<T, TILE, DEPTH>()), hdr,
                                           full_bar, empty_bar, ready_bar, rs, ctl,
                                           int(blockIdx.x) == ctl.hold_block);
    if (rs.failed && threadIdx.x == 0) set_error(err, kErrTimeout);
}

// Persistent blocks pulling work items from one global queue (reset to 0
// before every launch); the ring counters run on from item to item.  Six
// blocks per SM: the compiler's own choice (71 registers) leaves room for
// five 160-thread blocks; capped at 64 it spills 20 bytes, and a 16-member
// ensemble runs 1% faster (14.96-15.02 against 14.80 RK4 steps/s).
template <typename T, int THREADS, int TILE>
__global__ void __launch_bounds__(THREADS, 6) k_pairs_persistent(const typename Vec4<T>::type* __restrict__ src,
                                                              const Segment* __restrict__ segs,
                                                              const int32_t* __restrict__ leaf_start,
                                                              const WorkItem* __restrict__ items, int nitems,
                                                              int* __restrict__ queue, double4* __restrict__ partials,
                                                              int64_t pstride, int* __restrict__ err,
                                                              const PairCtl ctl) {
    using S4 = typename Vec4<T>::type;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full_bar[kDepth], empty_bar[kDepth], ready_bar[kDepth];
    __shared__ SlotHdr hdr[kDepth];
    __shared__ int next_item;
    init_ring(full_bar, empty_bar, ready_bar, THREADS / 32, kDepth);
    RingState rs{0, 0, 0, false};
    for (;;) {
        if (threadIdx.x == 0) next_item = atomicAdd(queue, 1);
        __syncthreads();
        const int item = next_item;
        __syncthreads();
        if (item >= nitems) break;
        const WorkItem it = items[item];
        run_item<T, THREADS, TILE, false, kDepth>(it, src, segs, leaf_start, partials, pstride,
                                          reinterpret_cast<S4*>(smem_raw),
                                          reinterpret_cast<float*>(smem_raw + ring_bytes<T, TILE>()), hdr, full_bar,
                                          empty_bar, ready_bar, rs, ctl, false);
        if (rs.failed) break;
    }
    if (rs.failed && threadIdx.x == 0) set_error(err, kErrTimeout);
}

// ---------------------------------------------------------------- dispatch

template <typename T, int THREADS, bool PSI, int DEPTH>
static cudaError_t run_pairs(cudaStream_t st, int nitems, const void* src, const Segment* segs,
                             const int32_t* leaf_start, const WorkItem* items, double4* partials, int64_t pstride,
                             int* err, PairCtl ctl) {
    constexpr int TILE = tile_capacity(sizeof(T) == 8);
    constexpr size_t smem = pair_smem_bytes<T, TILE, DEPTH>();
    static_assert(smem <= 48 * 1024, "ring must fit the default dynamic shared memory limit");
    if (nitems == 0) return cudaSuccess;
    k_pairs<T, THREADS, PSI, TILE, DEPTH><<<nitems, THREADS, smem, st>>>(static_cast<const typename Vec4<T>::type*>(src),
                                                                   segs, leaf_start, items, partials,
                                                                   pstride, err, ctl);
    return cudaGetLastError();
}

const std::vector<PairShape>& pair_shapes(bool fp64) {
    static const std::vector<PairShape> f32 = {{160, 1, 256}, {192, 1, 256}, {224, 1, 256}, {288, 1, 256}};
    static const std::vector<PairShape> f64 = {{160, 1, 128}, {192, 1, 128}, {224, 1, 128}, {288, 1, 128}};
    return fp64 ? f64 : f32;
}

PairShape pairs_shape(bool fp64, int threads, int per_thread) {
    (void)per_thread;
    for (const PairShape& s : pair_shapes(fp64))
        if (s.threads == threads) return s;
    return pair_shapes(fp64).front();
}

PairShape cluster_shape(bool fp64, int k) {
    const int tile = tile_capacity(fp64);
    const int depth = kClusterDepth;
    if (k <= 32) return PairShape{64, 1, tile, depth};
    if (k <= 64) return PairShape{96, 1, tile, depth};
    if (k <= 96) return PairShape{128, 1, tile, depth};
    return PairShape{160, 1, tile, depth};
}

template <typename T, bool PSI>
static cudaError_t dispatch(cudaStream_t st, PairShape sh, int nitems, const void* src, const Segment* segs,
                            const int32_t* leaf_start, const WorkItem* items, double4* partials,
                            int64_t pstride, int* err, PairCtl ctl) {
#define FSS_SHAPE(TH)                                                                                            \
    if (sh.threads == TH)                                                                                        \
        return run_pairs<T, TH, PSI, kDepth>(st, nitems, src, segs, leaf_start, items, partials, pstride, err, ctl);
#define FSS_SHAPE3(TH)                                                                                           \
    if (sh.threads == TH && sh.depth == 3)                                                                       \
        return run_pairs<T, TH, PSI, 3>(st, nitems, src, segs, leaf_start, items, partials, pstride, err, ctl);
    FSS_SHAPE3(64)
    FSS_SHAPE3(96)
    FSS_SHAPE3(128)
    FSS_SHAPE3(160)
#undef FSS_SHAPE3
    FSS_SHAPE(64)
    FSS_SHAPE(96)
    FSS_SHAPE(128)
    FSS_SHAPE(160)
    FSS_SHAPE(192)
    FSS_SHAPE(224)
    FSS_SHAPE(288)
#undef FSS_SHAPE
    return cudaErrorInvalidConfiguration;
}

cudaError_t launch_pairs(cudaStream_t st, bool fp64, bool psi, PairShape shape, int nitems, const void* src,
                         const Segment* segs, const int32_t* leaf_start, const WorkItem* items,
                         double4* partials, int64_t pstride, int* err, PairCtl ctl) {
    if (fp64)
        return psi ? dispatch<double, true>(st, shape, nitems, src, segs, leaf_start, items, partials, pstride, err, ctl)
                   : dispatch<double, false>(st, shape, nitems, src, segs, leaf_start, items, partials, pstride, err,
                                             ctl);
    return psi ? dispatch<float, true>(st, shape, nitems, src, segs, leaf_start, items, partials, pstride, err, ctl)
               : dispatch<float, false>(st, shape, nitems, src, segs, leaf_start, items, partials, pstride, err, ctl);
}

cudaError_t launch_pairs_persistent(cudaStream_t st, int nitems, const void* src, const Segment* segs,
                                    const int32_t* leaf_start, const WorkItem* items, int* queue,
                                    double4* partials, int64_t pstride, int* err, int blocks, PairCtl ctl) {
    constexpr int TILE = tile_capacity(false);
    constexpr size_t smem = pair_smem_bytes<float, TILE>();
    if (nitems == 0) return cudaSuccess;
    k_pairs_persistent<float, kPersistentThreads, TILE><<<blocks, kPersistentThreads, smem, st>>>(
        static_cast<const float4*>(src), segs, leaf_start, items, nitems, queue, partials, pstride, err, ctl);
    return cudaGetLastError();
}

int persistent_blocks_per_sm() {
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_pairs_persistent<float, kPersistentThreads, tile_capacity(false)>,
                                                  kPersistentThreads, pair_smem_bytes<float, tile_capacity(false)>());
    return nb > 0 ? nb : 1;
}

}  // namespace fss
