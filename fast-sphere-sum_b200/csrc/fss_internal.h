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
enum : int { kErrNone = 0, kErrTimeout = 1, kErrTree = 2 };

// One contiguous run of sources seen by one target leaf: `count` entries of
// the unified source array starting at `start` (particles [0, n), proxies
// after them).  Host-side list element before packing into tiles.
struct SrcEntry {
    int32_t start;
    int32_t count;
    int32_t kind;   // 0 particles (near or small far cluster), 1 proxies
    int32_t pad;
};

// One bulk copy global -> shared: `count` sources from `start`.
struct Copy {
    int32_t start;
    int32_t count;
};

// One shared-memory tile: copies [c0, c1) placed back to back, `count`
// sources in all; guard = 1 when a copy overlaps the block's own targets
// (the self pair must be skipped).
struct Tile {
    int32_t c0, c1;
    int32_t count;
    int32_t guard;
};

// One block's work: targets [t0, t0 + nt) (one leaf, sorted order) against
// tiles [k0, k1); results go to partial slot `part`.
struct WorkItem {
    int32_t t0, nt;
    int32_t k0, k1;
    int32_t part;
    int32_t leaf;
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
    int32_t off[12];              // by degree, -1 when not wanted
    int32_t pad;
};

// Per-node geometry for the upward pass: inverse of [v1 v2 v3] (columns),
// row-major, and the frame centre.
struct NodeGeom {
    double minv[9];
    double cx, cy, cz;
};

constexpr int kMaxDegree = 10;
constexpr int kMaxK = (kMaxDegree + 1) * (kMaxDegree + 2) / 2;  // 66
constexpr int kMaxLevels = 8;  // tree_levels supported

FSS_HD inline int nproxy(int n) { return (n + 1) * (n + 2) / 2; }

}  // namespace fss
