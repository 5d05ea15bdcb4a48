// traverse.h -- interaction lists of the icosahedral treecode (host).
#pragma once
#include <cstdint>
#include <vector>

#include "fss_internal.h"
#include "geometry.h"

namespace fss {

// One record of fast_rhs.h:16-91 tree_traverse (struct_list.h:6-14
// interaction_pair) plus whether it came from the well-separated branch.
struct Pair {
    int32_t lt, ls, t, s, nt, ns, type;  // type: 0 pp, 1 pc, 2 cp, 3 cc
    int32_t far;
    int32_t deg;  // interpolation degree of the pair (-1: the context's)
};

// The reference's dual traversal, bit-exact: FIFO over (target, source)
// faces seeded with all 20x20 level-0 pairs; counts are per-face particle
// counts (levels concatenated).
std::vector<Pair> dual_traverse(const TreeGeometry& g, const std::vector<int32_t>& counts, double theta,
                                int many_count);

// Dual traversal with parameters per target face (per-leaf choices carried
// up the tree): the pair (T, S) is well separated when (r_T + r_S)/d <
// theta_T, and T's degree n_T sets the cluster threshold K(n_T) of both
// faces; otherwise the same FIFO and refinement rules as dual_traverse.
// face_theta / face_deg are per global face.
std::vector<Pair> dual_traverse_faces(const TreeGeometry& g, const std::vector<int32_t>& counts,
                                      const std::vector<double>& face_theta, const std::vector<int32_t>& face_deg);

// Per-face parameters from per-leaf ones: theta_T = min and n_T = max over
// the leaves under T (so every leaf is served at least as accurately as its
// own choice asks).
void face_params(const TreeGeometry& g, int leaf_level, const std::vector<int32_t>& leaf_deg,
                 const std::vector<double>& leaf_theta, std::vector<int32_t>& face_deg,
                 std::vector<double>& face_theta);

// Source of one target leaf before materialisation: the particles of face
// (level, node), or the degree-`deg` proxies of that face.
struct ASrc {
    int32_t proxy;  // 0 particles, 1 proxies
    int32_t level, node, deg;
};

// Sources of one target cluster, a face whose interpolation points are the
// targets (fast_rhs.h cp: source particles; cc: source proxies).
struct TList {
    int32_t level, node, deg;  // node: index on its level
    std::vector<ASrc> src;
};

struct ListInput {
    const TreeGeometry* g = nullptr;
    int leaf_level = 0;                 // tree_levels - 1
    int64_t n = 0;                      // particles
    const int32_t* leaf_start = nullptr;  // nleaf + 1 (sorted order) at the build; estimates only
    int threads = 128, per_thread = 1;  // targets per block chunk = threads * per_thread
    int tile = 256;                     // sources per shared-memory tile
    int parts = 1;                      // source-list split
    bool all_leaves = false;            // items also for leaves empty at the build
};

struct ListOutput {
    std::vector<Segment> segs;      // per work item, in list order
    std::vector<WorkItem> items;    // target-leaf items, then target-cluster items
    int64_t n_leaf_items = 0;
    int max_cluster_k = 0;          // largest interpolation point count of a target cluster
    std::vector<ProxyJob> jobs;
    std::vector<DownJob> down;      // target clusters
    std::vector<LeafAnc> leaf_anc;  // per leaf, kMaxLevels records: the target clusters above it, coarse to fine
    int64_t n_coef = 0;             // down-pass coefficients (double4)
    std::vector<double> proxy_pos;  // 4 doubles per proxy slot: y (on sphere) and pad
    std::vector<int32_t> proxy_node;  // proxy slot -> face (global index)
    int64_t n_proxy = 0;            // proxy slots after the n particles
    int64_t n_tiles = 0;            // shared-memory tiles per RHS at the build's leaf counts
    double pp_pairs = 0, pc_pairs = 0;
    double cp_pairs = 0, cc_pairs = 0;  // at target-cluster interpolation points
    int max_degree = 0;
};

// Per-target-leaf source lists from the reference's pair list: every pair
// (T, S) gives each leaf under T either S's proxies (well separated and S
// holds more than many_count particles) or S's particles, leaf by leaf.
// With `clusters`, a well-separated pair whose target T holds more than
// many_count particles (the reference's cp and cc types) goes to T's
// interpolation points instead (fast_rhs.h cp/cc), one TList per such T.
std::vector<std::vector<ASrc>> lists_from_pairs(const TreeGeometry& g, int leaf_level,
                                                const std::vector<Pair>& pairs, int many_count, int degree,
                                                std::vector<TList>* clusters = nullptr);

// Per-target-leaf traversal with its own (degree, theta): a source face is
// taken as proxies when (r_t + r_s)/d < theta and it holds more particles
// than its proxy count, as particles when well separated but small or when
// it is a leaf, otherwise its four children are visited.  Faces empty at
// the build are skipped, unless keep_empty (particles re-sorted every step
// may move into them): then every leaf gets a list and an empty face is
// taken as particles, whatever it holds when the kernel runs.
std::vector<std::vector<ASrc>> lists_per_leaf(const TreeGeometry& g, int leaf_level,
                                              const std::vector<int32_t>& counts,
                                              const std::vector<int32_t>& leaf_degree,
                                              const std::vector<double>& leaf_theta, bool keep_empty);

// Materialise segments, work items (one per target leaf or target cluster
// and source part), proxy slots, upward-pass and downward-pass jobs.  A
// face's particles become a kind-0 segment over its leaves (adjacent ones
// merged), a face's proxies a kind-1 segment over its proxy slots.  A target
// cluster's items have targets [slot, slot + K) of the unified array (its
// interpolation points, which share the slot of the face's source proxies).
void build_lists(const ListInput& in, const std::vector<std::vector<ASrc>>& lists,
                 const std::vector<TList>& clusters, ListOutput& out);

// Contiguous ranges of units for nranks ranks with near-equal summed cost:
// bounds[r] .. bounds[r + 1] for rank r (nranks + 1 entries, bounds[0] = 0,
// bounds[nranks] = cost.size()); every rank gets at least one unit when
// there are enough; uniform costs when they sum to zero.
std::vector<int64_t> shard_partition(const std::vector<double>& cost, int nranks);

// Proxy node set: barycentric interpolation points of degree n on a
// triangle (Blyth-Pozrikidis construction on Chebyshev-Lobatto points) and
// the inverse of the Vandermonde matrix of the Chebyshev product basis
// T_a(2 l1 - 1) T_b(2 l2 - 1), a + b <= n.  nodes: 3 doubles each; vinv: K x K
// row-major with vinv[m*K + k] = coefficient of basis m in Lagrange poly k.
void interp_nodes(int n, std::vector<double>& nodes, std::vector<double>& vinv);

}  // namespace fss
