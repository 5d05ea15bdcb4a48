// fss_internal.h -- structures shared by the host orchestration (C++) and the
// sm_100a kernels (CUDA).  Plain data only; no CUDA types in the host-only
// parts.
#pragma once
#include <cstdint>

#if defined(__CUDACC__)
#define FSS_HD __host__ __device__
#else
#define FSS_HD
#endif

namespace fss {

// Error codes a kernel records in the context's device error word.
enum : int { kErrNone = 0, kErrTimeout = 1, kErrTree = 2, kErrNonFinite = 3 };

// One run of sources of a work item.  The pair kernel resolves it to a
// range [lo, hi) of the unified source array (particles [0, n), proxies
// after them) when it runs:
//   kind 0: the particles of leaves [a, b), i.e. [leaf_start[a],
//           leaf_start[b]) -- read on the device, since particles are
//           re-sorted into the leaves they have moved into;
//   kind 1: the fixed range [a, b) (far-cluster proxies, or a chunk of the
//           direct sum).
// The kernel packs consecutive runs into shared-memory tiles as it goes.
struct Segment {
    int32_t kind;
    int32_t a, b;
    int32_t pad;
};

// One block's work.  leaf >= 0: the targets are that leaf's current
// particles, taken in chunks of the block size; leaf < 0: the targets are
// [t0, t0 + nt).  Sources: segments [g0, g1).  Results go to partial slot
// `part`.
struct WorkItem {
    int32_t t0, nt;
    int32_t g0, g1;
    int32_t part;
    int32_t leaf;
};

// Default limit of a bounded wait, in nanoseconds of %globaltimer (a context
// can set its own).
constexpr uint64_t kWaitLimitNs = 2000000000ull;  // 2 s

// Run-time controls of a pair launch: the limit of every bounded wait
// (nanoseconds of %globaltimer) and a test hook, hold_block >= 0: that block
// never issues its first source tile nor signals its arrival, so that its
// waits run out (the launch then reports kErrTimeout).
struct PairCtl {
    uint64_t wait_ns;
    int32_t hold_block;
    int32_t pad;
};

// Sources per shared-memory tile: 256 float4 (4 KB) or 128 double4 (4 KB).
FSS_HD constexpr int tile_capacity(bool fp64) { return fp64 ? 128 : 256; }

// Upward-pass combine work: node `node` (global index, levels concatenated)
// on `level`; proxies of degree set `degmask` (bit d = degree d) written at
// proxy offsets off[d] (index into the unified source array).
struct ProxyJob {
    int32_t level, node, local;   // local = index within its level
    int32_t leaf_lo, leaf_hi;     // leaves under the node
    int32_t degmask;
    int32_t off[16];              // by degree (0..kMaxDegree), -1 when not wanted
};

// One leaf of an ensemble member for the batched upward pass: its index in
// the concatenated leaf_start (particles [leaf_start[g], leaf_start[g+1])
// of the concatenated arrays), its member's leaf level, its index on that
// level, the first of its (leaf_level + 1) x K moment slots, and the levels
// whose faces carry proxies in its member.
struct EnsLeaf {
    int32_t gleaf;
    int32_t leaf_level, local;
    int32_t level_mask;
    int64_t part_base;
};

// Downward pass: a target cluster, a face that receives far sources at its
// K = nproxy(deg) interpolation points (fast_rhs.h cp and cc): unified
// indices [slot, slot + K).  Its field there becomes K coefficients of the
// Chebyshev product basis (double4 from `coef`), which every particle below
// the face evaluates directly (as cp evaluates the interpolant at the
// targets, fast_rhs.h:228-235).
struct DownJob {
    int32_t level, node, deg;  // node = global face index
    int32_t slot;              // first interpolation point (unified index)
    int32_t coef;              // first coefficient (double4 units)
    int32_t pad[3];
};

// A block of the batched V^-1 products (proxy charges of the upward pass,
// coefficients of the downward pass): `count` tasks of degree `deg`, task
// indices tasks[first .. first + count) (a proxy job or a target cluster).
struct TaskBlock {
    int32_t deg, first, count, pad;
};

// One target cluster above a leaf, as the leaf's evaluation reads it:
// coefficients from `coef`, degree, face (global index); coef < 0 ends a
// leaf's list.
struct LeafAnc {
    int32_t coef, deg, node, pad;
};

// Per-node geometry for the upward pass: inverse of [v1 v2 v3] (columns),
// row-major, and the frame centre.
struct NodeGeom {
    double minv[9];
    double cx, cy, cz;
};

constexpr int kMaxDegree = 12;
constexpr int kMaxK = (kMaxDegree + 1) * (kMaxDegree + 2) / 2;  // 91
constexpr int kMaxLevels = 8;  // tree_levels supported

FSS_HD inline int nproxy(int n) { return (n + 1) * (n + 2) / 2; }

}  // namespace fss
