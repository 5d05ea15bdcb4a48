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
// after them).  (dx, dy, dz) = source frame centre - target frame centre; the
// kernels add it to the source's local coordinates so that displacements are
// formed from small numbers (frames are leaf/node circumcentres in mixed
// precision and the origin in FP64).
struct SrcEntry {
    int32_t start;
    int32_t count;
    int32_t kind;   // 0 particles (near or small far cluster), 1 proxies
    int32_t pad;
    double dx, dy, dz;
};

// One block's work: targets [t0, t0 + nt) (one leaf, sorted order) against
// entries [e0, e1); results go to partial slot `part`.
struct WorkItem {
    int32_t t0, nt;
    int32_t e0, e1;
    int32_t part;
    int32_t leaf;
};

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
