// ctx.h -- the context behind fss_ctx (private to the library).
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <string>
#include <vector>

#include "fss.h"
#include "geometry.h"
#include "kernels.h"
#include "traverse.h"

namespace fss {

struct ProfEntry {
    double ms = 0;
    int64_t launches = 0;
};

// One profiled range: its events and the number of kernels launched in it.
struct ProfPending {
    std::string name;
    cudaEvent_t a, b;
    int kernels;
};

}  // namespace fss

struct fss_ctx {
    using DBuf = fss::DBuf;
    using ProfEntry = fss::ProfEntry;
    using ProfPending = fss::ProfPending;
    using TreeGeometry = fss::TreeGeometry;
    using Pair = fss::Pair;
    using ListOutput = fss::ListOutput;
    using ASrc = fss::ASrc;
    using PairShape = fss::PairShape;
    fss_config cfg{};
    std::string err;
    int dev = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    // second stream of a treecode RHS with target clusters: the target-leaf
    // pair launch runs on it beside the upward/downward passes (fork and
    // join through events, so graph capture records them as edges)
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_up = nullptr, ev_join = nullptr;
    bool fp64 = false;
    bool tree = true;
    bool resort = false;  // re-sort particles into their current leaves every RK4 step
    // one problem sharded over ranks (shard_nranks == 0: not sharded): this
    // rank's targets are units [shard_bounds[rank], shard_bounds[rank + 1]) --
    // faces of level shard_unit_level (treecode) or blocks of target rows
    // (direct sum) -- i.e. leaves or rows [shard_lo, shard_hi)
    int shard_rank = 0, shard_nranks = 0, shard_unit_level = 0;
    int64_t shard_lo = 0, shard_hi = 0;
    std::vector<int64_t> shard_bounds;
    std::vector<double> shard_cost;
    uint64_t wait_ns = 0;  // limit of the pair kernel's bounded waits
    int hold_block = -1;   // test hook: block of the next target-leaf launch that withholds a tile
    int hold_stage = -1;   // test hook: 0 / 1, block 0 of the next proxy / coefficient launch withholds its matrix
    int resort_mode = 0;   // test hook: per-step re-sort by partition of the old order (0) or radix key sort (1)

    int64_t n = 0;
    bool have = false;
    bool stage_dirty = false;  // xs/src hold a stand-alone rhs input, not s0

    // tree
    int tree_levels = 0, leaf_level = 0;
    int64_t nleaf = 1;
    TreeGeometry geom;
    std::vector<int32_t> leaf_start_h;
    std::vector<int32_t> counts_h;
    std::vector<Pair> pairs;
    std::vector<int32_t> ref_loc_h, cmp_loc_h;
    int64_t unassigned = 0;
    ListOutput lists;
    std::vector<std::vector<ASrc>> alists;  // per-leaf sources before packing
    std::vector<fss::TList> tlists;         // target clusters (cp/cc) and their sources
    std::vector<std::pair<fss::PairShape, double>> tuned;  // autotuner: shape, ms per pair pass
    std::vector<std::pair<int, double>> tuned_depth;       // autotuner: tree levels, ms per RHS
    std::vector<std::pair<int, double>> tuned_parts;       // autotuner: src_parts, ms per right-hand side
    int64_t depth_n = -1;  // particle count the tuned depth belongs to
    int depth_tl = 0;      // tuned tree levels (0: none)
    int src_parts_given = 0;  // src_parts of the configuration (0: the autotuner may choose)
    std::vector<int32_t> leaf_deg;
    std::vector<double> leaf_theta;
    int nmax = 0, level_mask = 0;
    int parts = 1;
    int64_t pstride = 0;  // partial slot stride: n, or n + proxy slots with target clusters
    int n_up_blocks = 0, n_dn_blocks = 0;  // blocks of the batched V^-1 products
    int down_max_deg = 0;                  // highest target-cluster degree
    PairShape shape;
    double direct_pairs = 0;

    // device
    DBuf in5, area_in, perm, key, key_tmp, vals_tmp, hist, leaf_start, s0, xs, acc, area_s, tracer_s, src, partials,
        segs, items, jobs, frame, node, lev_off, verts, tri_verts, part_up, proxy_pos, out5, psi,
        wtotal, err_flag, loc, sortq, grid3, rm_target, rm_tris, rm_off, rm_adj, down_jobs, down_anc, down_coef, vpad, vtpad, vpad_off, up_deg, up_tblocks, up_tasks,
        dn_tblocks, dn_tasks, msum, part_scratch;
    int64_t src_count = 0;

    // graph
    cudaGraphExec_t graph = nullptr;
    double graph_dt = 0, graph_omega = 0;

    // profiling
    bool prof = false;
    std::vector<ProfPending> pending;
    std::vector<cudaEvent_t> ev_pool;
    std::map<std::string, ProfEntry> prof_acc;
    std::vector<std::string> prof_order;

    std::unique_ptr<fss_ctx> alt;  // the other method, created on demand
    // remesh: device triangles and adjacency of the last call, kept while
    // the caller's triangles (host copy) and the particle count are unchanged
    fss::RemeshScratch rm;
    std::vector<int32_t> rm_tris_host;
    int64_t rm_n = -1;

    ~fss_ctx() {
        if (graph) cudaGraphExecDestroy(graph);
        for (auto& p : pending) {
            cudaEventDestroy(p.a);
            cudaEventDestroy(p.b);
        }
        for (auto e : ev_pool) cudaEventDestroy(e);
        for (cudaEvent_t e : {ev_fork, ev_up, ev_join})
            if (e) cudaEventDestroy(e);
        if (side) cudaStreamDestroy(side);
        if (own_stream) cudaStreamDestroy(own_stream);
    }
};

