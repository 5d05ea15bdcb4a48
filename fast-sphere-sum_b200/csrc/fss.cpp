// fss.cpp -- context, orchestration and the C ABI (include/fss.h).
#include "fss.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "amr_internal.h"
#include "ctx.h"
#include "geometry.h"
#include "kernels.h"
#include "traverse.h"

using namespace fss;

namespace {

thread_local std::string g_last_error;

}  // namespace

namespace {

int fail(fss_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    g_last_error = msg;
    return code;
}

#define CU(call)                                                                                       \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess)                                                                         \
            return fail(c, e_ == cudaErrorMemoryAllocation ? FSS_ERR_NOMEM : FSS_ERR_CUDA,             \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                           \
    } while (0)

#define TRY(call)                        \
    do {                                 \
        int r_ = (call);                 \
        if (r_ != FSS_OK) return r_;     \
    } while (0)

cudaEvent_t ev_get(fss_ctx* c) {
    if (!c->ev_pool.empty()) {
        cudaEvent_t e = c->ev_pool.back();
        c->ev_pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}

// Device time of a range of launches (`kernels` of them) under profiling.
struct ProfScope {
    fss_ctx* c;
    const char* name;
    int kernels;
    cudaEvent_t a = nullptr, b = nullptr;
    ProfScope(fss_ctx* ctx, const char* nm, int nk = 1) : c(ctx), name(nm), kernels(nk) {
        if (c->prof) {
            a = ev_get(c);
            b = ev_get(c);
            cudaEventRecord(a, c->stream);
        }
    }
    ~ProfScope() {
        if (c->prof) {
            cudaEventRecord(b, c->stream);
            c->pending.push_back({name, a, b, kernels});
        }
    }
};

void prof_resolve(fss_ctx* c) {
    if (c->pending.empty()) return;
    cudaStreamSynchronize(c->stream);
    for (auto& p : c->pending) {
        float ms = 0;
        cudaEventElapsedTime(&ms, p.a, p.b);
        if (!c->prof_acc.count(p.name)) c->prof_order.push_back(p.name);
        c->prof_acc[p.name].ms += ms;
        c->prof_acc[p.name].launches += p.kernels;
        c->ev_pool.push_back(p.a);
        c->ev_pool.push_back(p.b);
    }
    c->pending.clear();
}

int check_device_error(fss_ctx* c) {
    int h = 0;
    CU(cudaMemcpyAsync(&h, c->err_flag.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CU(cudaStreamSynchronize(c->stream));
    prof_resolve(c);
    if (h != 0) {
        cudaMemsetAsync(c->err_flag.p, 0, sizeof(int), c->stream);
        if (h == kErrNonFinite) return fail(c, FSS_ERR_INVALID, "non-finite particle position (diverged state?)");
        return fail(c, h == kErrTimeout ? FSS_ERR_TIMEOUT : FSS_ERR_TREE,
                    h == kErrTimeout ? "a kernel's bounded wait timed out" : "tree build error");
    }
    return FSS_OK;
}

template <typename T>
int upload(fss_ctx* c, DBuf& b, const std::vector<T>& v) {
    CU(b.ensure(sizeof(T) * std::max<size_t>(v.size(), 1)));
    if (!v.empty()) CU(cudaMemcpyAsync(b.p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, c->stream));
    return FSS_OK;
}

// Blocks of the batched V^-1 products: tasks (index, degree) grouped by
// degree (stable, so a block's tasks keep list order), at most per_block a
// block.
void make_task_blocks(const std::vector<std::pair<int32_t, int32_t>>& tasks, int per_block,
                      std::vector<TaskBlock>& blocks, std::vector<int32_t>& index) {
    blocks.clear();
    index.clear();
    for (int d = 0; d <= kMaxDegree; d++) {
        const int32_t first = int32_t(index.size());
        for (const auto& t : tasks)
            if (t.second == d) index.push_back(t.first);
        for (int32_t b = first; b < int32_t(index.size()); b += per_block)
            blocks.push_back(TaskBlock{d, b, std::min<int32_t>(per_block, int32_t(index.size()) - b), 0});
    }
}

int auto_tree_levels(const fss_config& cfg, int64_t n) {
    if (cfg.tree_levels > 0) return cfg.tree_levels;
    const int target = cfg.leaf_target > 0 ? cfg.leaf_target : 64;
    int ll = 0;
    while (ll + 1 < kMaxLevels && double(n) / (20.0 * std::pow(4.0, ll + 1)) >= target) ll++;
    return ll + 1;
}

int src_size_ensure(fss_ctx* c, int64_t count) {
    const size_t es = c->fp64 ? sizeof(double4) : sizeof(float4);
    void* before = c->src.p;
    CU(c->src.ensure(es * size_t(std::max<int64_t>(count, 1))));
    if (c->src.p != before) c->stage_dirty = true;  // particle sources must be rewritten
    c->src_count = count;
    return FSS_OK;
}

// Lists of the direct sum: blocks of targets x P chunks of the sources.
int build_direct_lists(fss_ctx* c) {
    const int64_t n = c->n;
    c->shape = pairs_shape(c->fp64, c->cfg.block_threads, c->cfg.targets_per_thread);
    const int TB = c->shape.targets();
    const int64_t tiles = (n + TB - 1) / TB;
    int P = c->cfg.src_parts;
    if (P <= 0) {
        const int64_t want = 148 * 8 * 3;
        P = int(std::max<int64_t>(1, (want + tiles - 1) / std::max<int64_t>(tiles, 1)));
        P = int(std::min<int64_t>(P, std::max<int64_t>(1, n / 512)));
        P = std::min(P, 64);
    }
    c->parts = P;
    ListOutput& L = c->lists;
    L = ListOutput();
    for (int p = 0; p < P; p++) L.segs.push_back(Segment{1, int32_t(n * p / P), int32_t(n * (p + 1) / P), 0});
    // sharded: this rank's blocks of target rows (direct_sum_mpi.cpp:74-82
    // splits the rows over ranks in equal blocks)
    int64_t t_lo = 0, t_hi = tiles;
    if (c->shard_nranks > 0) {
        c->shard_unit_level = 0;
        c->shard_cost.assign(size_t(tiles), 0.0);
        for (int64_t t = 0; t < tiles; t++) c->shard_cost[t] = double(std::min<int64_t>(TB, n - t * TB)) * double(n - 1);
        c->shard_bounds = shard_partition(c->shard_cost, c->shard_nranks);
        t_lo = c->shard_bounds[c->shard_rank];
        t_hi = c->shard_bounds[c->shard_rank + 1];
        c->shard_lo = t_lo * TB;
        c->shard_hi = std::min<int64_t>(n, t_hi * TB);
    }
    for (int64_t t = t_lo; t < t_hi; t++) {
        const int64_t t0 = t * TB, nt = std::min<int64_t>(TB, n - t0);
        for (int p = 0; p < P; p++) {
            L.items.push_back(WorkItem{int32_t(t0), int32_t(nt), p, p + 1, p, -1});
            L.n_tiles += (L.segs[p].b - L.segs[p].a + c->shape.tile - 1) / c->shape.tile;
        }
    }
    L.n_leaf_items = int64_t(L.items.size());
    L.pp_pairs = double(c->shard_nranks > 0 ? c->shard_hi - c->shard_lo : n) * double(n - 1);
    c->direct_pairs = L.pp_pairs;
    TRY(upload(c, c->segs, L.segs));
    TRY(upload(c, c->items, L.items));
    TRY(src_size_ensure(c, n));
    c->pstride = n;
    CU(c->partials.ensure(sizeof(double4) * size_t(P) * size_t(std::max<int64_t>(n, 1))));
    return FSS_OK;
}

// Per-leaf source lists of the configured mode.  With re-sorting, faces
// empty at the build may fill later, so no face is pruned for being empty.
void make_alists(fss_ctx* c, const std::vector<int32_t>& dual_counts) {
    const int LL = c->leaf_level;
    c->tlists.clear();
    std::vector<int32_t> cc = dual_counts;
    if (c->resort)
        for (int32_t& x : cc) x = std::max(x, 1);
    if (c->cfg.list_mode == FSS_LIST_LEAF && c->cfg.cluster_targets) {
        // per-leaf (n, theta) carried up to the target faces of a dual traversal
        std::vector<int32_t> fdeg;
        std::vector<double> fth;
        face_params(c->geom, LL, c->leaf_deg, c->leaf_theta, fdeg, fth);
        c->alists = lists_from_pairs(c->geom, LL, dual_traverse_faces(c->geom, cc, fth, fdeg), 0, c->cfg.degree,
                                     &c->tlists);
        return;
    }
    if (c->cfg.list_mode == FSS_LIST_LEAF) {
        c->alists = lists_per_leaf(c->geom, LL, c->counts_h, c->leaf_deg, c->leaf_theta, c->resort);
        return;
    }
    const int many = (c->cfg.many_count < 0) ? nproxy(c->cfg.degree) : c->cfg.many_count;
    c->alists = lists_from_pairs(c->geom, LL, dual_traverse(c->geom, cc, c->cfg.theta, many), many, c->cfg.degree,
                                 c->cfg.cluster_targets ? &c->tlists : nullptr);
}

// The lists of the current tree: the reference's pair list as built (static
// tree, complete assignment, dual lists) or those of the configured mode.
void make_lists(fss_ctx* c) {
    const int LL = c->leaf_level;
    const int many = (c->cfg.many_count < 0) ? nproxy(c->cfg.degree) : c->cfg.many_count;
    if (c->cfg.list_mode == FSS_LIST_DUAL && !c->resort && c->cfg.assign_mode != FSS_ASSIGN_REFERENCE) {
        c->tlists.clear();
        c->alists = lists_from_pairs(c->geom, LL, c->pairs, many, c->cfg.degree,
                                     c->cfg.cluster_targets ? &c->tlists : nullptr);
    } else {
        make_alists(c, c->counts_h);
    }
}

// Sharded treecode: the units are the faces of the shallowest level holding
// a target cluster (every target cluster and the downward pass below it then
// lie within one unit), or the leaves; each unit costs the interactions of
// its target leaves and clusters at the build's counts.  The ranks take
// contiguous unit ranges of near-equal cost (every rank computes the same
// plan from the same tree), and this rank keeps the source lists of its own
// leaves and clusters only.
int shard_filter(fss_ctx* c) {
    if (c->shard_nranks <= 0) return FSS_OK;
    const int LL = c->leaf_level;
    int u = LL;
    for (const TList& t : c->tlists) u = std::min(u, int(t.level));
    const int64_t nunits = int64_t(20) << (2 * u);
    if (nunits < c->shard_nranks)
        return fail(c, FSS_ERR_INVALID, "more ranks than units (faces of level " + std::to_string(u) + ")");
    auto count = [&](const ASrc& a) -> double {
        return a.proxy ? double(nproxy(a.deg)) : double(c->counts_h[c->geom.lev_off[a.level] + a.node]);
    };
    std::vector<double> cost(size_t(nunits), 0.0);
    for (int64_t lf = 0; lf < c->nleaf; lf++) {
        double sc = 0;
        for (const ASrc& a : c->alists[lf]) sc += count(a);
        cost[size_t(lf >> (2 * (LL - u)))] += double(c->leaf_start_h[lf + 1] - c->leaf_start_h[lf]) * sc;
    }
    for (const TList& t : c->tlists) {
        double sc = 0;
        for (const ASrc& a : t.src) sc += count(a);
        cost[size_t(t.node >> (2 * (t.level - u)))] += double(nproxy(t.deg)) * sc;
    }
    c->shard_unit_level = u;
    c->shard_cost = cost;
    c->shard_bounds = shard_partition(cost, c->shard_nranks);
    const int64_t u0 = c->shard_bounds[c->shard_rank], u1 = c->shard_bounds[c->shard_rank + 1];
    c->shard_lo = u0 << (2 * (LL - u));
    c->shard_hi = u1 << (2 * (LL - u));
    for (int64_t lf = 0; lf < c->nleaf; lf++)
        if (lf < c->shard_lo || lf >= c->shard_hi) c->alists[lf].clear();
    std::vector<TList> own;
    for (TList& t : c->tlists) {
        const int64_t unit = t.node >> (2 * (t.level - u));
        if (unit >= u0 && unit < u1) own.push_back(std::move(t));
    }
    c->tlists = std::move(own);
    return FSS_OK;
}

int ensure_particle_buffers(fss_ctx* c, int64_t n) {
    const size_t N = size_t(std::max<int64_t>(n, 1));
    CU(c->in5.ensure(sizeof(double) * 5 * N));
    CU(c->area_in.ensure(sizeof(double) * N));
    CU(c->s0.ensure(sizeof(double4) * N));
    CU(c->xs.ensure(sizeof(double4) * N));
    CU(c->acc.ensure(sizeof(double4) * N));
    CU(c->area_s.ensure(sizeof(double) * N));
    CU(c->tracer_s.ensure(sizeof(double) * N));
    CU(c->out5.ensure(sizeof(double) * 5 * N));
    CU(c->psi.ensure(sizeof(double) * N));
    CU(c->wtotal.ensure(sizeof(double)));
    return FSS_OK;
}

int build_tree(fss_ctx* c);
PairShape choose_shape(fss_ctx* c);
int materialize(fss_ctx* c, PairShape shape);
int autotune(fss_ctx* c, bool depth);
int refresh_stage(fss_ctx* c);
int eval(fss_ctx* c, EpiArgs& ea, bool want_psi);

int gather(fss_ctx* c, bool write_s0) {
    const bool treec = c->tree;
    ProfScope ps(c, "gather");
    launch_gather(c->stream, c->fp64, c->n, c->in5.as<double>(), c->area_in.as<double>(),
                  treec ? c->perm.as<int32_t>() : nullptr, treec ? c->key.as<uint32_t>() : nullptr,
                  nullptr, write_s0 ? c->s0.as<double4>() : nullptr,
                  c->xs.as<double4>(), c->area_s.as<double>(), c->tracer_s.as<double>(), c->src.p);
    CU(cudaGetLastError());
    return FSS_OK;
}

void invalidate_graph(fss_ctx* c) {
    if (c->graph) cudaGraphExecDestroy(c->graph);
    c->graph = nullptr;
}

int set_particles(fss_ctx* c, int64_t n, const double* state5, const double* area) {
    if (n < 2) return fail(c, FSS_ERR_INVALID, "need at least 2 particles");
    if (n > (int64_t(1) << 30)) return fail(c, FSS_ERR_INVALID, "too many particles");
    if (!state5 || !area) return fail(c, FSS_ERR_INVALID, "null state or area");
    invalidate_graph(c);
    c->n = n;
    TRY(ensure_particle_buffers(c, n));
    // host or device arrays (unified addressing)
    CU(cudaMemcpyAsync(c->in5.p, state5, sizeof(double) * 5 * n, cudaMemcpyDefault, c->stream));
    CU(cudaMemcpyAsync(c->area_in.p, area, sizeof(double) * n, cudaMemcpyDefault, c->stream));
    // the positions given here are the grid the remesh step returns to
    CU(c->grid3.ensure(sizeof(double) * 3 * size_t(n)));
    CU(cudaMemcpy2DAsync(c->grid3.p, 3 * sizeof(double), c->in5.p, 5 * sizeof(double), 3 * sizeof(double), size_t(n),
                         cudaMemcpyDeviceToDevice, c->stream));
    if (c->tree) {
        TRY(build_tree(c));
    } else {
        TRY(build_direct_lists(c));
    }
    TRY(gather(c, true));
    c->have = true;
    c->stage_dirty = false;
    if (c->tree && c->cfg.autotune) TRY(autotune(c, true));
    TRY(refresh_stage(c));
    return check_device_error(c);
}

int build_tree(fss_ctx* c) {
    const int64_t n = c->n;
    // automatic depth: the autotuner's choice for this particle count, if any
    const int TL = (c->cfg.tree_levels == 0 && c->depth_n == n && c->depth_tl > 0) ? c->depth_tl
                                                                                   : auto_tree_levels(c->cfg, n);
    c->resort = c->cfg.rebuild == FSS_REBUILD_RESORT ||
                (c->cfg.rebuild == FSS_REBUILD_AUTO && c->cfg.assign_mode != FSS_ASSIGN_REFERENCE);
    if (TL < 1 || TL > kMaxLevels) return fail(c, FSS_ERR_INVALID, "tree_levels out of range");
    if (TL != c->tree_levels || c->geom.tree_levels != TL) {
        c->geom = build_tree_geometry(TL);
        c->tree_levels = TL;
        c->leaf_level = TL - 1;
        c->nleaf = int64_t(20) << (2 * c->leaf_level);
        TRY(upload(c, c->verts, c->geom.verts));
        TRY(upload(c, c->tri_verts, c->geom.tri_verts));
        TRY(upload(c, c->lev_off, c->geom.lev_off));
        TRY(upload(c, c->node, c->geom.node));
        std::vector<double4> fr(c->nleaf);
        for (int64_t l = 0; l < c->nleaf; l++) {
            const double* ti = &c->geom.tri_info[4 * (c->geom.lev_off[c->leaf_level] + l)];
            fr[l] = make_double4(ti[0], ti[1], ti[2], 0.0);
        }
        TRY(upload(c, c->frame, fr));
        if ((int)c->leaf_deg.size() != c->nleaf) {
            c->leaf_deg.assign(c->nleaf, c->cfg.degree);
            c->leaf_theta.assign(c->nleaf, c->cfg.theta);
        }
    }
    const int LL = c->leaf_level;
    const int64_t nfaces = c->geom.lev_off[TL];
    // assignment
    CU(c->key.ensure(sizeof(uint32_t) * n));
    CU(c->key_tmp.ensure(sizeof(uint32_t) * n));
    CU(c->perm.ensure(sizeof(int32_t) * n));
    CU(c->vals_tmp.ensure(sizeof(int32_t) * n));
    CU(c->sortq.ensure(sizeof(int32_t) * n));
    CU(c->hist.ensure(sizeof(uint32_t) * sort_scratch_words(n)));
    CU(c->part_scratch.ensure(sizeof(uint32_t) * partition_scratch_words(c->nleaf)));
    CU(c->leaf_start.ensure(sizeof(int32_t) * (c->nleaf + 1)));
    c->ref_loc_h.clear();
    c->unassigned = 0;
    std::vector<int32_t> ref_counts;
    if (c->cfg.assign_mode == FSS_ASSIGN_REFERENCE) {
        CU(c->loc.ensure(sizeof(int32_t) * size_t(TL) * n));
        DBuf cnt;
        CU(cnt.ensure(sizeof(int32_t) * nfaces));
        CU(cudaMemsetAsync(cnt.p, 0, sizeof(int32_t) * nfaces, c->stream));
        {
            ProfScope ps(c, "tree_assign");
            launch_assign(c->stream, n, c->in5.as<double>(), c->verts.as<double>(), c->tri_verts.as<int32_t>(),
                          c->lev_off.as<int64_t>(), TL, 1, c->loc.as<int32_t>(), nullptr, c->err_flag.as<int>());
        }
        launch_level_hist(c->stream, n, TL, c->loc.as<int32_t>(), c->lev_off.as<int64_t>(), cnt.as<int32_t>());
        c->ref_loc_h.resize(size_t(TL) * n);
        ref_counts.resize(nfaces);
        CU(cudaMemcpyAsync(c->ref_loc_h.data(), c->loc.p, sizeof(int32_t) * TL * n, cudaMemcpyDeviceToHost, c->stream));
        CU(cudaMemcpyAsync(ref_counts.data(), cnt.p, sizeof(int32_t) * nfaces, cudaMemcpyDeviceToHost, c->stream));
        CU(cudaStreamSynchronize(c->stream));
        for (int64_t i = 0; i < n; i++)
            if (c->ref_loc_h[size_t(LL) * n + i] < 0) c->unassigned++;
    }
    {
        ProfScope ps(c, "tree_assign");
        launch_assign(c->stream, n, c->in5.as<double>(), c->verts.as<double>(), c->tri_verts.as<int32_t>(),
                      c->lev_off.as<int64_t>(), TL, 0, nullptr, c->key.as<uint32_t>(), c->err_flag.as<int>());
    }
    int bits = 0;
    while ((int64_t(1) << bits) < c->nleaf) bits++;
    {
        ProfScope ps(c, "tree_sort");
        launch_sort(c->stream, n, std::max(bits, 1), c->key.as<uint32_t>(), c->key_tmp.as<uint32_t>(),
                    c->perm.as<int32_t>(), c->vals_tmp.as<int32_t>(), c->hist.as<uint32_t>());
        launch_leaf_bounds(c->stream, n, c->key.as<uint32_t>(), int32_t(c->nleaf), c->leaf_start.as<int32_t>());
    }
    CU(cudaGetLastError());
    c->leaf_start_h.resize(c->nleaf + 1);
    CU(cudaMemcpyAsync(c->leaf_start_h.data(), c->leaf_start.p, sizeof(int32_t) * (c->nleaf + 1),
                       cudaMemcpyDeviceToHost, c->stream));
    CU(cudaStreamSynchronize(c->stream));
    // stop here on non-finite input positions (before lists and autotuning)
    TRY(check_device_error(c));
    // per-face counts on every level from the leaf ranges
    c->counts_h.assign(nfaces, 0);
    for (int l = 0; l <= LL; l++) {
        const int64_t span = int64_t(1) << (2 * (LL - l));
        const int64_t nf = c->geom.level_count(l);
        for (int64_t f = 0; f < nf; f++)
            c->counts_h[c->geom.lev_off[l] + f] = c->leaf_start_h[(f + 1) * span] - c->leaf_start_h[f * span];
    }
    const int K = nproxy(c->cfg.degree);
    const int many = (c->cfg.many_count < 0) ? K : c->cfg.many_count;
    // the reference-format pair list (fss_get_tree) of this build
    c->pairs = dual_traverse(c->geom, (c->cfg.assign_mode == FSS_ASSIGN_REFERENCE) ? ref_counts : c->counts_h,
                             c->cfg.theta, many);
    make_lists(c);
    TRY(shard_filter(c));
    TRY(materialize(c, choose_shape(c)));
    return FSS_OK;
}

// Block shape for the treecode's pair kernel: the configured one, or the
// smallest supported block whose consumer threads cover the largest leaf (so
// that no leaf needs a second chunk).
PairShape choose_shape(fss_ctx* c) {
    if (c->cfg.block_threads > 0) return pairs_shape(c->fp64, c->cfg.block_threads, c->cfg.targets_per_thread);
    int maxleaf = 1;
    for (int64_t l = 0; l < c->nleaf; l++) maxleaf = std::max(maxleaf, c->leaf_start_h[l + 1] - c->leaf_start_h[l]);
    for (const PairShape& sh : pair_shapes(c->fp64))
        if (sh.per_thread == 1 && sh.targets() >= maxleaf) return sh;
    return pair_shapes(c->fp64).back();
}

// Work items, tiles and copies of the current lists for one block shape;
// proxy slots, upward-pass jobs and interpolation tables.
int materialize(fss_ctx* c, PairShape shape) {
    const int64_t n = c->n;
    const int LL = c->leaf_level;
    c->shape = shape;
    ListInput in;
    in.g = &c->geom;
    in.leaf_level = LL;
    in.n = n;
    in.leaf_start = c->leaf_start_h.data();
    in.tile = shape.tile;
    in.threads = shape.targets();
    in.per_thread = 1;
    int P = c->cfg.src_parts;
    if (P <= 0) {
        int64_t chunks = 0;
        const int TB = in.threads * in.per_thread;
        for (int64_t l = 0; l < c->nleaf; l++) chunks += (c->leaf_start_h[l + 1] - c->leaf_start_h[l] + TB - 1) / TB;
        const double waves = double(chunks) / (148.0 * 8.0);
        P = waves >= 3.0 ? 1 : (waves >= 1.0 ? 2 : 4);
    }
    in.parts = P;
    in.all_leaves = c->resort;
    c->parts = P;
    build_lists(in, c->alists, c->tlists, c->lists);
    const ListOutput& L = c->lists;
    // interpolation tables for the degrees in use
    c->nmax = std::max(L.max_degree, 0);
    c->level_mask = 0;
    // per face, the highest proxy degree it serves (-1: no proxies), so the
    // upward pass forms only the moments some list uses
    std::vector<int8_t> up_deg(c->geom.node.size(), int8_t(-1));
    for (const ProxyJob& j : L.jobs) {
        c->level_mask |= 1 << j.level;
        for (int d = 0; d <= kMaxDegree; d++)
            if ((j.degmask >> d) & 1) {
                c->nmax = std::max(c->nmax, d);
                up_deg[size_t(j.node)] = int8_t(std::max<int>(up_deg[size_t(j.node)], d));
            }
    }
    TRY(upload(c, c->up_deg, up_deg));
    // Vinv of every degree in use for the batched products, rows padded to a
    // multiple of 4 doubles (Vinv[m][k] by rows m, and the transpose by rows
    // k), each a bulk copy of K * Kp doubles
    std::vector<double> vpad_all, vtpad_all;
    std::vector<int32_t> vpad_off(kMaxDegree + 1, 0);
    for (int d = 0; d <= c->nmax; d++) {
        std::vector<double> nodes, vi;
        interp_nodes(d, nodes, vi);
        const int K = nproxy(d), Kp = (K + 3) & ~3;
        vpad_off[d] = int32_t(vpad_all.size());
        for (int r = 0; r < K; r++)
            for (int q = 0; q < Kp; q++) {
                vpad_all.push_back(q < K ? vi[size_t(r) * K + q] : 0.0);
                vtpad_all.push_back(q < K ? vi[size_t(q) * K + r] : 0.0);
            }
    }
    TRY(upload(c, c->vpad, vpad_all));
    TRY(upload(c, c->vtpad, vtpad_all));
    TRY(upload(c, c->vpad_off, vpad_off));
    TRY(upload(c, c->segs, L.segs));
    TRY(upload(c, c->items, L.items));
    TRY(upload(c, c->jobs, L.jobs));
    TRY(upload(c, c->down_jobs, L.down));
    {
        std::vector<std::pair<int32_t, int32_t>> up, dn;
        for (size_t j = 0; j < L.jobs.size(); j++)
            for (int d = 0; d <= kMaxDegree; d++)
                if ((L.jobs[j].degmask >> d) & 1) up.emplace_back(int32_t(j), d);
        c->down_max_deg = 0;
        for (size_t j = 0; j < L.down.size(); j++) {
            dn.emplace_back(int32_t(j), L.down[j].deg);
            c->down_max_deg = std::max(c->down_max_deg, int(L.down[j].deg));
        }
        CU(batch_prepare());
        CU(c->msum.ensure(sizeof(double) * std::max<size_t>(L.jobs.size(), 1) * size_t(nproxy(c->nmax))));
        std::vector<TaskBlock> blocks;
        std::vector<int32_t> index;
        make_task_blocks(up, batch_tasks(), blocks, index);
        c->n_up_blocks = int(blocks.size());
        TRY(upload(c, c->up_tblocks, blocks));
        TRY(upload(c, c->up_tasks, index));
        make_task_blocks(dn, batch_tasks(), blocks, index);
        c->n_dn_blocks = int(blocks.size());
        TRY(upload(c, c->dn_tblocks, blocks));
        TRY(upload(c, c->dn_tasks, index));
    }
    TRY(upload(c, c->down_anc, L.leaf_anc));
    CU(c->down_coef.ensure(sizeof(double4) * size_t(std::max<int64_t>(L.n_coef, 1))));
    std::vector<double4> pp(L.proxy_pos.size() / 4);
    for (size_t i = 0; i < pp.size(); i++)
        pp[i] = make_double4(L.proxy_pos[4 * i], L.proxy_pos[4 * i + 1], L.proxy_pos[4 * i + 2], 0.0);
    TRY(upload(c, c->proxy_pos, pp));
    TRY(src_size_ensure(c, n + L.n_proxy));
    // target clusters write partials at their interpolation points (slots
    // after the particles) and the down pass one more slot per particle
    const bool down = !L.down.empty();
    c->pstride = down ? n + L.n_proxy : n;
    CU(c->partials.ensure(sizeof(double4) * size_t(P + (down ? 1 : 0)) * size_t(c->pstride)));
    CU(c->part_up.ensure(sizeof(double) * size_t(c->nleaf) * (LL + 1) * nproxy(c->nmax)));
    return FSS_OK;
}

// The pair kernel over all work items: target leaves with the block shape
// of the context, target clusters with a block fitted to their
// interpolation point count.
int launch_leaf_pairs(fss_ctx* c, cudaStream_t st, bool want_psi) {
    const PairCtl ctl{c->wait_ns, c->hold_block, 0};
    c->hold_block = -1;  // the test hook holds one launch only
    CU(launch_pairs(st, c->fp64, want_psi, c->shape, int(c->lists.n_leaf_items), c->src.p, c->segs.as<Segment>(),
                    c->leaf_start.as<int32_t>(), c->items.as<WorkItem>(), c->partials.as<double4>(), c->pstride,
                    c->err_flag.as<int>(), ctl));
    return FSS_OK;
}

int launch_cluster_pairs(fss_ctx* c, cudaStream_t st, bool want_psi) {
    const ListOutput& L = c->lists;
    const int nl = int(L.n_leaf_items), nall = int(L.items.size());
    if (nall > nl)
        CU(launch_pairs(st, c->fp64, want_psi, cluster_shape(c->fp64, L.max_cluster_k), nall - nl, c->src.p,
                        c->segs.as<Segment>(), c->leaf_start.as<int32_t>(), c->items.as<WorkItem>() + nl,
                        c->partials.as<double4>(), c->pstride, c->err_flag.as<int>(), PairCtl{c->wait_ns, -1, 0}));
    return FSS_OK;
}

int launch_all_pairs(fss_ctx* c, bool want_psi) {
    TRY(launch_leaf_pairs(c, c->stream, want_psi));
    return launch_cluster_pairs(c, c->stream, want_psi);
}

// The partial sums of one right-hand side on the current stage state
// (xs/src): every pair launch and the downward pass, joined on the
// context's stream; *down is set when the downward pass wrote its slot.
int eval_partials(fss_ctx* c, bool want_psi, bool* down_out) {
    // With target clusters, the target-leaf pair launch (compute-bound) runs
    // on the side stream beside the chain upward pass -> target-cluster
    // pairs -> downward pass (mostly latency-bound); it waits for the upward
    // pass only when a leaf takes proxies.  Partial slots of the two are
    // disjoint (particles vs interpolation points).  Sequential while
    // profiling, so that every range times its own kernels.
    const bool overlap = c->tree && !c->lists.down.empty() && !c->prof;
    const bool leaf_needs_up = c->lists.pc_pairs > 0;
    if (overlap) {
        CU(cudaEventRecord(c->ev_fork, c->stream));
        CU(cudaStreamWaitEvent(c->side, c->ev_fork, 0));
        if (!leaf_needs_up) TRY(launch_leaf_pairs(c, c->side, want_psi));
    }
    if (c->tree && !c->lists.jobs.empty()) {
        {
            ProfScope ps(c, "upward_leaf");
            launch_up_leaf(c->stream, c->fp64, int(c->nleaf), c->src.p, c->leaf_start.as<int32_t>(), nullptr,
                           c->node.as<NodeGeom>(), c->lev_off.as<int64_t>(),
                           c->leaf_level, c->nmax, c->level_mask, c->up_deg.as<int8_t>(), c->part_up.as<double>());
        }
        {
            ProfScope ps(c, "upward_combine", 2);  // k_up_sums, k_up_proxies
            launch_up_proxies(c->stream, c->fp64, int(c->lists.jobs.size()), c->jobs.as<ProxyJob>(),
                              c->part_up.as<double>(), c->leaf_level, c->nmax, c->msum.as<double>(),
                              c->n_up_blocks, c->up_tblocks.as<TaskBlock>(), c->up_tasks.as<int32_t>(),
                              c->vpad.as<double>(), c->vpad_off.as<int32_t>(), c->proxy_pos.as<double4>(), c->n,
                              c->src.p, c->err_flag.as<int>(), c->wait_ns, c->hold_stage == 0 ? 0 : -1);
            if (c->hold_stage == 0) c->hold_stage = -1;  // the test hook holds one launch only
        }
    }
    if (overlap) {
        if (leaf_needs_up) {
            CU(cudaEventRecord(c->ev_up, c->stream));
            CU(cudaStreamWaitEvent(c->side, c->ev_up, 0));
            TRY(launch_leaf_pairs(c, c->side, want_psi));
        }
        TRY(launch_cluster_pairs(c, c->stream, want_psi));
    } else {
        ProfScope ps(c, c->fp64 ? "pairs_fp64" : "pairs_mixed", c->lists.n_leaf_items < int64_t(c->lists.items.size()) ? 2 : 1);
        TRY(launch_all_pairs(c, want_psi));
    }
    const bool down = c->tree && !c->lists.down.empty();
    if (down) {
        DownArgs d;
        d.njobs = int(c->lists.down.size());
        d.jobs = c->down_jobs.as<DownJob>();
        d.ncoef_blocks = c->n_dn_blocks;
        d.max_deg = c->down_max_deg;
        d.fp32_eval = !c->fp64;
        d.coef_blocks = c->dn_tblocks.as<TaskBlock>();
        d.coef_tasks = c->dn_tasks.as<int32_t>();
        d.partials = c->partials.as<double4>();
        d.parts = c->parts;
        d.pstride = c->pstride;
        d.vtpad = c->vtpad.as<double>();
        d.vpad_off = c->vpad_off.as<int32_t>();
        d.err = c->err_flag.as<int>();
        d.wait_ns = c->wait_ns;
        d.hold_block = c->hold_stage == 1 ? 0 : -1;
        if (c->hold_stage == 1) c->hold_stage = -1;  // the test hook holds one launch only
        d.node = c->node.as<NodeGeom>();
        d.coef = c->down_coef.as<double4>();
        d.nleaf = int(c->nleaf);
        d.xs = c->xs.as<double4>();
        d.leaf_start = c->leaf_start.as<int32_t>();
        d.leaf_anc = c->down_anc.as<LeafAnc>();
        d.out = c->partials.as<double4>() + int64_t(c->parts) * c->pstride;
        ProfScope ps(c, "downward", down_launch_count(d));
        launch_down(c->stream, want_psi, d);
    }
    if (overlap) {  // join: the epilogue needs the target-leaf partials
        CU(cudaEventRecord(c->ev_join, c->side));
        CU(cudaStreamWaitEvent(c->stream, c->ev_join, 0));
    }
    *down_out = down;
    return FSS_OK;
}

// One right-hand side on the current stage state (xs/src).
int eval(fss_ctx* c, EpiArgs& ea, bool want_psi) {
    bool down = false;
    TRY(eval_partials(c, want_psi, &down));
    if (want_psi) launch_wsum(c->stream, c->n, c->xs.as<double4>(), c->area_s.as<double>(), c->wtotal.as<double>());
    ea.n = c->n;
    ea.parts = c->parts + (down ? 1 : 0);
    ea.pstride = c->pstride;
    ea.partials = c->partials.as<double4>();
    ea.xs = c->xs.as<double4>();
    ea.area = c->area_s.as<double>();
    ea.wtotal = c->wtotal.as<double>();
    ea.perm = c->tree ? c->perm.as<int32_t>() : nullptr;
    ea.src = c->src.p;
    ea.leaf_of = nullptr;
    ea.frame = nullptr;  // interaction sources in absolute coordinates
    {
        ProfScope ps(c, "epilogue");
        launch_epilogue(c->stream, c->fp64, ea);
    }
    CU(cudaGetLastError());
    return FSS_OK;
}

// Device time (ms, mean of `reps`) of `step` on the context's stream, after
// one untimed run.
struct TuneEvents {
    cudaEvent_t a = nullptr, b = nullptr;
    ~TuneEvents() {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
    }
};

template <class Step>
int time_ms(fss_ctx* c, TuneEvents& ev, int reps, Step&& step, double* ms) {
    TRY(step());
    CU(cudaEventRecord(ev.a, c->stream));
    for (int r = 0; r < reps; r++) TRY(step());
    CU(cudaEventRecord(ev.b, c->stream));
    CU(cudaEventSynchronize(ev.b));
    float t = 0;
    CU(cudaEventElapsedTime(&t, ev.a, ev.b));
    *ms = double(t) / reps;
    return FSS_OK;
}

// One whole right-hand side on the current stage state (for tuning).
int tune_rhs(fss_ctx* c) {
    EpiArgs ea;
    ea.mode = EPI_RHS;
    ea.out5 = c->out5.as<double>();
    return eval(c, ea, false);
}

// Autotuner, run by fss_set_particles.  autotune >= 1: the pair kernel's
// block shape -- every supported shape timed on the current lists (after
// the upward pass), the fastest kept.  autotune >= 2 also: the tree depth
// (leaf size), when the configuration leaves it automatic -- the automatic
// depth and one level either side, each built and timed on a whole
// right-hand side (the fastest is kept for this particle count); and the
// source split (src_parts 1, 2, 4), when automatic, timed on a whole
// right-hand side (more parts balance the pair launches but add partial
// slots for the epilogue to sum).
// depth = false (lists rebuilt for per-leaf parameters, which belong to the
// current leaves) keeps the tree.
int autotune(fss_ctx* c, bool depth) {
    c->tuned.clear();
    const bool prof_was = c->prof;
    c->prof = false;
    TuneEvents ev;
    CU(cudaEventCreate(&ev.a));
    CU(cudaEventCreate(&ev.b));
    if (depth && c->cfg.autotune >= 2 && c->tree && c->cfg.tree_levels == 0 && c->depth_n != c->n) {
        const int base = c->tree_levels;
        int best_tl = base;
        double best_ms = 1e30;
        c->depth_n = c->n;
        for (int tl = base - 1; tl <= base + 1; tl++) {
            if (tl < 2 || tl > kMaxLevels) continue;
            if (double(c->n) / (20.0 * std::pow(4.0, tl - 1)) < 8.0) continue;  // leaves under 8 particles
            c->depth_tl = tl;
            TRY(build_tree(c));
            TRY(gather(c, true));
            c->stage_dirty = false;
            double ms = 0;
            TRY(time_ms(c, ev, 2, [&] { return tune_rhs(c); }, &ms));
            c->tuned_depth.push_back({tl, ms});
            if (ms < best_ms) {
                best_ms = ms;
                best_tl = tl;
            }
        }
        c->depth_tl = best_tl;
        if (c->tree_levels != best_tl) {
            TRY(build_tree(c));
            TRY(gather(c, true));
            c->stage_dirty = false;
        }
    }
    PairShape best = c->shape;
    double best_ms = 1e30;
    for (const PairShape& sh : pair_shapes(c->fp64)) {
        TRY(materialize(c, sh));
        TRY(refresh_stage(c));
        TRY(tune_rhs(c));  // proxies of the upward pass for the pair launches
        double ms = 0;
        TRY(time_ms(c, ev, 2, [&] { return launch_all_pairs(c, false); }, &ms));
        c->tuned.push_back({sh, ms});
        if (ms < best_ms) {
            best_ms = ms;
            best = sh;
        }
    }
    if (c->cfg.autotune >= 2 && c->cfg.src_parts == 0) {
        c->tuned_parts.clear();
        int best_p = 1;
        double best_p_ms = 1e30;
        for (int p : {1, 2, 4}) {
            c->cfg.src_parts = p;
            TRY(materialize(c, best));
            TRY(refresh_stage(c));
            double ms = 0;
            TRY(time_ms(c, ev, 3, [&] { return tune_rhs(c); }, &ms));
            c->tuned_parts.push_back({p, ms});
            if (ms < best_p_ms) {
                best_p_ms = ms;
                best_p = p;
            }
        }
        c->cfg.src_parts = best_p;
    }
    TRY(materialize(c, best));
    c->prof = prof_was;
    c->stage_dirty = true;  // the timing passes overwrote the stage sources
    return FSS_OK;
}

// Particles into the leaves they are in now (start of an RK4 step): keys,
// the stable order of the new keys, state permuted in place, leaf ranges,
// stage-1 sources.  The order comes from partitioning the old one (few
// particles change leaves in a step); the radix key sort of the initial
// build gives the same order and stays selectable by a test hook.
int resort(fss_ctx* c) {
    const int64_t n = c->n;
    if (c->resort_mode == 0) {
        // keys, scan, bucket, place, commit
        ProfScope ps(c, "resort", 5);
        launch_resort_partition(c->stream, c->fp64, n, c->nleaf, c->leaf_level, c->node.as<NodeGeom>(),
                                c->lev_off.as<int64_t>(), c->key.as<uint32_t>(), c->key_tmp.as<uint32_t>(),
                                c->leaf_start.as<int32_t>(), c->vals_tmp.as<int32_t>(),
                                c->part_scratch.as<uint32_t>(), c->s0.as<double4>(), c->area_s.as<double>(),
                                c->tracer_s.as<double>(), c->perm.as<int32_t>(), c->xs.as<double4>(),
                                c->acc.as<double4>(), c->src.p, c->err_flag.as<int>());
        CU(cudaGetLastError());
        return FSS_OK;
    }
    int bits = 0;
    while ((int64_t(1) << bits) < c->nleaf) bits++;
    bits = std::max(bits, 1);
    // reassign, 3 per 8-bit sort pass, gather + commit, leaf bounds
    ProfScope ps(c, "resort", 1 + sort_launch_count(c->n, bits) + 2 + 1);
    launch_reassign(c->stream, n, c->s0.as<double4>(), nullptr, c->leaf_level, c->node.as<NodeGeom>(),
                    c->lev_off.as<int64_t>(), c->key.as<uint32_t>(), c->err_flag.as<int>());
    launch_sort(c->stream, n, bits, c->key.as<uint32_t>(), c->key_tmp.as<uint32_t>(),
                c->sortq.as<int32_t>(), c->vals_tmp.as<int32_t>(), c->hist.as<uint32_t>());
    launch_resort(c->stream, c->fp64, n, c->sortq.as<int32_t>(), c->s0.as<double4>(), c->area_s.as<double>(),
                  c->tracer_s.as<double>(), c->perm.as<int32_t>(), c->xs.as<double4>(), c->acc.as<double4>(),
                  c->src.p);
    launch_leaf_bounds(c->stream, n, c->key.as<uint32_t>(), int32_t(c->nleaf), c->leaf_start.as<int32_t>());
    CU(cudaGetLastError());
    return FSS_OK;
}

int rk4_once(fss_ctx* c, double dt, double omega) {
    if (c->tree && c->resort) TRY(resort(c));
    for (int stage = 1; stage <= 4; stage++) {
        EpiArgs ea;
        ea.mode = EPI_RK4;
        ea.stage = stage;
        ea.dt = dt;
        ea.omega = omega;
        ea.s0 = c->s0.as<double4>();
        ea.acc = c->acc.as<double4>();
        TRY(eval(c, ea, false));
    }
    return FSS_OK;
}

int refresh_stage(fss_ctx* c) {
    if (!c->stage_dirty) return FSS_OK;
    launch_refresh(c->stream, c->fp64, c->n, c->s0.as<double4>(), c->area_s.as<double>(), nullptr, nullptr,
                   c->xs.as<double4>(), c->src.p);
    CU(cudaGetLastError());
    c->stage_dirty = false;
    return FSS_OK;
}

int rk4_steps(fss_ctx* c, double dt, double omega, int nsteps) {
    if (!c->have) return fail(c, FSS_ERR_STATE, "no particles set");
    if (nsteps < 0) return fail(c, FSS_ERR_INVALID, "nsteps < 0");
    TRY(refresh_stage(c));
    // a held tile (test hook) is taken by one eager step, never baked into a graph
    const bool use_graph = c->cfg.use_graph && !c->prof && c->hold_block < 0 && c->hold_stage < 0;
    if (!use_graph) {
        for (int s = 0; s < nsteps; s++) TRY(rk4_once(c, dt, omega));
        return FSS_OK;
    }
    if (!c->graph || c->graph_dt != dt || c->graph_omega != omega) {
        invalidate_graph(c);
        cudaGraph_t g;
        CU(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        int r = rk4_once(c, dt, omega);
        cudaError_t e = cudaStreamEndCapture(c->stream, &g);
        if (r != FSS_OK) return r;
        if (e != cudaSuccess) return fail(c, FSS_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
        e = cudaGraphInstantiate(&c->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return fail(c, FSS_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
        c->graph_dt = dt;
        c->graph_omega = omega;
    }
    for (int s = 0; s < nsteps; s++) CU(cudaGraphLaunch(c->graph, c->stream));
    return FSS_OK;
}

int rhs_host(fss_ctx* c, const double* state5, const double* area, double omega, double* modify5, double* psi) {
    if (!state5 || !area || !modify5) return fail(c, FSS_ERR_INVALID, "null pointer");
    if (!c->have) return fail(c, FSS_ERR_STATE, "no particles set");
    CU(cudaMemcpyAsync(c->in5.p, state5, sizeof(double) * 5 * c->n, cudaMemcpyHostToDevice, c->stream));
    CU(cudaMemcpyAsync(c->area_in.p, area, sizeof(double) * c->n, cudaMemcpyHostToDevice, c->stream));
    TRY(gather(c, false));
    c->stage_dirty = true;
    EpiArgs ea;
    ea.mode = EPI_RHS;
    ea.omega = omega;
    ea.out5 = c->out5.as<double>();
    ea.psi = psi ? c->psi.as<double>() : nullptr;
    TRY(eval(c, ea, psi != nullptr));
    CU(cudaMemcpyAsync(modify5, c->out5.p, sizeof(double) * 5 * c->n, cudaMemcpyDeviceToHost, c->stream));
    if (psi) CU(cudaMemcpyAsync(psi, c->psi.p, sizeof(double) * c->n, cudaMemcpyDeviceToHost, c->stream));
    return check_device_error(c);
}

fss_ctx* other_method(fss_ctx* c, int method, int* rc) {
    *rc = FSS_OK;
    if ((method == FSS_METHOD_TREECODE) == c->tree) return c;
    if (!c->alt) {
        fss_config cfg = c->cfg;
        cfg.method = method;
        fss_ctx* a = nullptr;
        *rc = fss_create(&cfg, &a);
        if (*rc != FSS_OK) return nullptr;
        c->alt.reset(a);
        c->alt->stream = c->stream;
    }
    c->alt->stream = c->stream;
    return c->alt.get();
}

}  // namespace

namespace fss {
// Message for fss_last_error(NULL), for entry points outside this file.
void set_last_error(const std::string& msg) { g_last_error = msg; }

// Interaction lists again from the current mode and per-leaf parameters.
int internal_relist(fss_ctx* c) {
    invalidate_graph(c);
    make_alists(c, c->counts_h);
    TRY(shard_filter(c));
    TRY(materialize(c, choose_shape(c)));
    c->stage_dirty = true;
    if (c->cfg.autotune) {  // block shape (and source split) for the new lists
        if (c->cfg.autotune >= 2 && c->src_parts_given == 0) c->cfg.src_parts = 0;  // tune it again
        TRY(autotune(c, false));
    }
    TRY(refresh_stage(c));
    return check_device_error(c);
}

// Velocity of the current stage state into a host array (caller's order).
int internal_rhs_current(fss_ctx* c, std::vector<double>& out5) {
    TRY(refresh_stage(c));
    EpiArgs ea;
    ea.mode = EPI_RHS;
    ea.omega = 2 * M_PI;
    ea.out5 = c->out5.as<double>();
    TRY(eval(c, ea, false));
    out5.resize(5 * c->n);
    CU(cudaMemcpyAsync(out5.data(), c->out5.p, sizeof(double) * 5 * c->n, cudaMemcpyDeviceToHost, c->stream));
    return check_device_error(c);
}
}  // namespace fss

// =================================================================== C ABI

extern "C" {

void fss_config_init(fss_config* cfg) {
    if (!cfg) return;
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->device = 0;
    cfg->precision = FSS_PREC_MIXED;
    cfg->method = FSS_METHOD_TREECODE;
    cfg->tree_levels = 0;
    cfg->leaf_target = 64;
    cfg->degree = 8;
    cfg->theta = 0.7;
    cfg->many_count = -1;
    cfg->assign_mode = FSS_ASSIGN_COMPLETE;
    cfg->list_mode = FSS_LIST_DUAL;
    cfg->use_graph = 1;
    cfg->src_parts = 0;
    cfg->block_threads = 0;
    cfg->targets_per_thread = 1;
    cfg->autotune = 0;
}

int fss_create(const fss_config* cfg, fss_ctx** out) {
    fss_ctx* c = nullptr;
    if (!cfg || !out) return fail(c, FSS_ERR_INVALID, "null argument");
    *out = nullptr;
    if (cfg->degree < 0 || cfg->degree > kMaxDegree) return fail(c, FSS_ERR_INVALID, "degree must be in 0..12");
    if (!(cfg->theta > 0)) return fail(c, FSS_ERR_INVALID, "theta must be positive");
    if (cfg->tree_levels < 0 || cfg->tree_levels > kMaxLevels) return fail(c, FSS_ERR_INVALID, "tree_levels out of range");
    if (cfg->wait_limit_us < 0) return fail(c, FSS_ERR_INVALID, "wait_limit_us < 0");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(c, FSS_ERR_UNSUPPORTED, "no CUDA device");
    }
    if (cfg->device < 0 || cfg->device >= ndev) return fail(c, FSS_ERR_INVALID, "bad device ordinal");
    std::unique_ptr<fss_ctx> ctx(new fss_ctx());
    c = ctx.get();
    c->cfg = *cfg;
    c->dev = cfg->device;
    c->fp64 = cfg->precision == FSS_PREC_FP64;
    c->tree = cfg->method == FSS_METHOD_TREECODE;
    c->wait_ns = cfg->wait_limit_us > 0 ? uint64_t(cfg->wait_limit_us) * 1000ull : kWaitLimitNs;
    c->src_parts_given = cfg->src_parts;
    CU(cudaSetDevice(c->dev));
    cudaDeviceProp prop;
    CU(cudaGetDeviceProperties(&prop, c->dev));
    if (prop.major < 10) return fail(c, FSS_ERR_UNSUPPORTED, "this build targets sm_100a (Blackwell B200)");
    // the latency-bound chain of an RHS (upward pass, target-cluster pairs,
    // downward pass) runs on the context's stream at the highest priority;
    // the compute-bound target-leaf pairs beside it at the lowest
    int prio_least = 0, prio_greatest = 0;
    CU(cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest));
    CU(cudaStreamCreateWithPriority(&c->own_stream, cudaStreamNonBlocking, prio_greatest));
    c->stream = c->own_stream;
    CU(cudaStreamCreateWithPriority(&c->side, cudaStreamNonBlocking, prio_least));
    CU(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
    CU(cudaEventCreateWithFlags(&c->ev_up, cudaEventDisableTiming));
    CU(cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming));
    CU(c->err_flag.ensure(sizeof(int)));
    CU(cudaMemsetAsync(c->err_flag.p, 0, sizeof(int), c->stream));
    CU(cudaStreamSynchronize(c->stream));
    *out = ctx.release();
    return FSS_OK;
}

void fss_destroy(fss_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->dev);
    cudaStreamSynchronize(ctx->stream);
    delete ctx;
}

const char* fss_last_error(const fss_ctx* ctx) { return ctx ? ctx->err.c_str() : g_last_error.c_str(); }

int fss_set_stream(fss_ctx* c, void* s) {
    if (!c) return fail(c, FSS_ERR_INVALID, "null context");
    invalidate_graph(c);
    c->stream = s ? static_cast<cudaStream_t>(s) : c->own_stream;
    if (c->alt) c->alt->stream = c->stream;
    return FSS_OK;
}

int fss_get_stream(fss_ctx* c, void** s) {
    if (!c || !s) return fail(c, FSS_ERR_INVALID, "null argument");
    *s = static_cast<void*>(c->stream);
    return FSS_OK;
}

int fss_set_particles(fss_ctx* c, int64_t n, const double* state5, const double* area) {
    if (!c) return fail(c, FSS_ERR_INVALID, "null context");
    CU(cudaSetDevice(c->dev));
    return set_particles(c, n, state5, area);
}

int fss_rebuild_tree(fss_ctx* c) {
    if (!c) return fail(c, FSS_ERR_INVALID, "null context");
    if (!c->have) return fail(c, FSS_ERR_STATE, "no particles set");
    CU(cudaSetDevice(c->dev));
    // current state back to the caller's order, then rebuild from it
    launch_scatter_state(c->stream, c->n, c->tree ? c->perm.as<int32_t>() : nullptr, c->s0.as<double4>(),
                         c->tracer_s.as<double>(), c->in5.as<double>());
    std::vector<double> s5(5 * c->n), a(c->n);
    CU(cudaMemcpyAsync(s5.data(), c->in5.p, sizeof(double) * 5 * c->n, cudaMemcpyDeviceToHost, c->stream));
    CU(cudaMemcpyAsync(a.data(), c->area_in.p, sizeof(double) * c->n, cudaMemcpyDeviceToHost, c->stream));
    CU(cudaStreamSynchronize(c->stream));
    return set_particles(c, c->n, s5.data(), a.data());
}

int fss_rhs(fss_ctx* c, const double* state5, const double* area, double omega, double* modify5, double* psi) {
    if (!c) return fail(c, FSS_ERR_INVALID, "null context");
    CU(cudaSetDevice(c->dev));
    return rhs_host(c, state5, area, omega, modify5, psi);
}

static int rhs_method(fss_ctx* c, int method, const double* state5, const double* area, double omega, double* modify5,
                      double* psi, int64_t n_hint) {
    if (!c) return fail(c, FSS_ERR_INVALID, "null context");
    CU(cudaSetDevice(c->dev));
    int rc;
    fss_ctx* t = other_method(c, method, &rc);
    if (!t) return fail(c, rc, fss_last_error(nullptr));
    if (!t->have || t->n != n_hint) {
        if (n_hint <= 0) return fail(c, FSS_ERR_STATE, "no particles set");
        rc = set_particles(t, n_hint, state5, area);
        if (rc != FSS_OK) return fail(c, rc, t->err);
    }
    rc = rhs_host(t, state5, area, omega, modify5, psi);
    if (rc != FSS_OK) return fail(c, rc, t->err);
    return FSS_OK;
}

int fss_rhs_direct(fss_ctx* c, const double* state5, const double* area, double omega, double* modify5, double* psi) {
    if (!c) return fail(c, FSS_ERR_INVALID, "null context");
    return rhs_method(c, FSS_METHOD_DIRECT, state5, area, omega, modify5, psi, c->n);
}

int fss_rhs_treecode(fss_ctx* c, const double* state5, const double* area, double omega, double* modify5, double* psi) {
    if (!c) return fail(c, FSS_ERR_INVALID, "null context");
    return rhs_method(c, FSS_METHOD_TREECODE, state5, area, omega, modify5, psi, c->n);
}

int fss_rk4_step(fss_ctx* c, double dt, double omega, int32_t nsteps) {
    if (!c) return fail(c, FSS_ERR_INVALID, "null context");
    CU(cudaSetDevice(c->dev));
    TRY(rk4_steps(c, dt, omega, nsteps));
    if (c->prof) prof_resolve(c);
    return FSS_OK;
}

int fss_rk4_step_host(fss_ctx* c, double* state5, double dt, double omega, int32_t nsteps) {
    if (!c || !state5) return fail(c, FSS_ERR_INVALID, "null argument");
    if (!c->have) return fail(c, FSS_ERR_STATE, "no particles set");
    CU(cudaSetDevice(c->dev));
    CU(cudaMemcpyAsync(c->in5.p, state5, sizeof(double) * 5 * c->n, cudaMemcpyHostToDevice, c->stream));
    TRY(gather(c, true));
    c->stage_dirty = false;
    TRY(rk4_steps(c, dt, omega, nsteps));
    launch_scatter_state(c->stream, c->n, c->tree ? c->perm.as<int32_t>() : nullptr, c->s0.as<double4>(),
                         c->tracer_s.as<double>(), c->out5.as<double>());
    CU(cudaMemcpyAsync(state5, c->out5.p, sizeof(double) * 5 * c->n, cudaMemcpyDeviceToHost, c->stream));
    return check_device_error(c);
}

int fss_get_state(fss_ctx* c, double* state5) {
    if (!c || !state5) return fail(c, FSS_ERR_INVALID, "null argument");
    if (!c->have) return fail(c, FSS_ERR_STATE, "no particles set");
    CU(cudaSetDevice(c->dev));
    launch_scatter_state(c->stream, c->n, c->tree ? c->perm.as<int32_t>() : nullptr, c->s0.as<double4>(),
                         c->tracer_s.as<double>(), c->out5.as<double>());
    CU(cudaMemcpyAsync(state5, c->out5.p, sizeof(double) * 5 * c->n, cudaMemcpyDeviceToHost, c->stream));
    return check_device_error(c);
}

int fss_rhs_current(fss_ctx* c, double omega, double* modify5, double* psi) {
    if (!c || !modify5) return fail(c, FSS_ERR_INVALID, "null argument");
    if (!c->have) return fail(c, FSS_ERR_STATE, "no particles set");
    CU(cudaSetDevice(c->dev));
    TRY(refresh_stage(c));
    EpiArgs ea;
    ea.mode = EPI_RHS;
    ea.omega = omega;
    ea.out5 = c->out5.as<double>();
    ea.psi = psi ? c->psi.as<double>() : nullptr;
    TRY(eval(c, ea, psi != nullptr));
    CU(cudaMemcpyAsync(modify5, c->out5.p, sizeof(double) * 5 * c->n, cudaMemcpyDeviceToHost, c->stream));
    if (psi) CU(cudaMemcpyAsync(psi, c->psi.p, sizeof(double) * c->n, cudaMemcpyDeviceToHost, c->stream));
    return check_device_error(c);
}

namespace {
// Pair evaluations the consumer lanes of a pair launch perform on items
// [i0, i1) with `targets` consumer threads per block: per chunk of targets,
// every full warp evaluates every source of the item (padded to whole
// quads) on each lane; the last, partial warp (r targets) splits them over
// 32 / r lanes per target, each lane taking every (32 / r)-th quad.
double lane_pairs(const fss_ctx* c, int64_t i0, int64_t i1, int targets) {
    const ListOutput& L = c->lists;
    double sum = 0;
    for (int64_t i = i0; i < i1; i++) {
        const WorkItem& it = L.items[i];
        double src = 0;
        for (int g = it.g0; g < it.g1; g++) {
            const Segment& sg = L.segs[g];
            src += sg.kind == 0 ? double(c->leaf_start_h[sg.b] - c->leaf_start_h[sg.a]) : double(sg.b - sg.a);
        }
        const double quads = std::ceil(src / 4.0);
        const int nt = it.leaf >= 0 ? c->leaf_start_h[it.leaf + 1] - c->leaf_start_h[it.leaf] : it.nt;
        for (int c0 = 0; c0 < nt; c0 += targets) {
            const int cn = std::min(targets, nt - c0);
            sum += 32.0 * double(cn / 32) * 4.0 * quads;
            if (cn % 32) sum += 32.0 * 4.0 * std::ceil(quads / double(32 / (cn % 32)));
        }
    }
    return sum;
}
}  // namespace

int fss_get_tree_info(fss_ctx* c, fss_tree_info* info) {
    if (!c || !info) return fail(c, FSS_ERR_INVALID, "null argument");
    std::memset(info, 0, sizeof(*info));
    info->tree_levels = c->tree ? c->tree_levels : 0;
    info->leaf_count = c->tree ? int32_t(c->nleaf) : 0;
    info->degree = c->cfg.degree;
    info->n_proxy = nproxy(c->cfg.degree);
    info->n_pairs = int64_t(c->pairs.size());
    info->n_list_entries = int64_t(c->lists.segs.size());
    info->n_tiles = c->lists.n_tiles;
    info->n_items = int64_t(c->lists.items.size());
    info->unassigned = c->unassigned;
    info->pp_interactions = c->lists.pp_pairs;
    info->pc_interactions = c->lists.pc_pairs;
    info->block_threads = c->shape.threads;
    info->targets_per_thread = c->shape.per_thread;
    info->src_parts = c->parts;
    info->target_clusters = int32_t(c->lists.down.size());
    info->cp_interactions = c->lists.cp_pairs;
    info->cc_interactions = c->lists.cc_pairs;
    info->max_degree = c->tree ? c->nmax : 0;
    info->max_cluster_points = c->lists.down.empty() ? 0 : int32_t(c->lists.max_cluster_k);
    if (c->tree && c->have) {
        const int64_t nl = c->lists.n_leaf_items, na = int64_t(c->lists.items.size());
        info->lane_pairs_leaf = lane_pairs(c, 0, nl, c->shape.targets());
        if (na > nl)
            info->lane_pairs_cluster = lane_pairs(c, nl, na, cluster_shape(c->fp64, c->lists.max_cluster_k).targets());
    }
    return FSS_OK;
}

int fss_get_tree(fss_ctx* c, int32_t* loc, int32_t* counts, int32_t* pairs, int64_t cap) {
    if (!c) return fail(c, FSS_ERR_INVALID, "null context");
    if (!c->have || !c->tree) return fail(c, FSS_ERR_STATE, "no tree built");
    const int TL = c->tree_levels, LL = c->leaf_level;
    const int64_t n = c->n, nfaces = c->geom.lev_off[TL];
    if (loc) {
        if (c->cfg.assign_mode == FSS_ASSIGN_REFERENCE) {
            std::memcpy(loc, c->ref_loc_h.data(), sizeof(int32_t) * TL * n);
        } else {
            std::vector<int32_t> perm(n);
            std::vector<uint32_t> skey(n);
            CU(cudaMemcpyAsync(perm.data(), c->perm.p, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, c->stream));
            CU(cudaMemcpyAsync(skey.data(), c->key.p, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, c->stream));
            CU(cudaStreamSynchronize(c->stream));
            for (int64_t s = 0; s < n; s++)
                for (int l = 0; l < TL; l++) loc[int64_t(l) * n + perm[s]] = int32_t(skey[s] >> (2 * (LL - l)));
        }
    }
    if (counts) {
        if (c->cfg.assign_mode == FSS_ASSIGN_REFERENCE) {
            std::vector<int32_t> cc(nfaces, 0);
            for (int l = 0; l < TL; l++)
                for (int64_t i = 0; i < n; i++) {
                    const int32_t f = c->ref_loc_h[size_t(l) * n + i];
                    if (f >= 0) cc[c->geom.lev_off[l] + f]++;
                }
            std::memcpy(counts, cc.data(), sizeof(int32_t) * nfaces);
        } else {
            std::memcpy(counts, c->counts_h.data(), sizeof(int32_t) * nfaces);
        }
    }
    if (pairs) {
        if (int64_t(c->pairs.size()) > cap) return fail(c, FSS_ERR_CAPACITY, "pairs buffer too small");
        for (size_t i = 0; i < c->pairs.size(); i++) {
            const Pair& p = c->pairs[i];
            int32_t* r = pairs + 7 * i;
            r[0] = p.lt; r[1] = p.ls; r[2] = p.t; r[3] = p.s; r[4] = p.nt; r[5] = p.ns; r[6] = p.type;
        }
    }
    return FSS_OK;
}

int fss_set_leaf_params(fss_ctx* c, int32_t nleaf, const int32_t* degree, const double* theta) {
    if (!c || !degree || !theta) return fail(c, FSS_ERR_INVALID, "null argument");
    for (int32_t i = 0; i < nleaf; i++) {
        if (degree[i] < 0 || degree[i] > kMaxDegree) return fail(c, FSS_ERR_INVALID, "degree out of range");
        if (!(theta[i] > 0)) return fail(c, FSS_ERR_INVALID, "theta must be positive");
    }
    c->leaf_deg.assign(degree, degree + nleaf);
    c->leaf_theta.assign(theta, theta + nleaf);
    return FSS_OK;
}

int fss_profile_enable(fss_ctx* c, int32_t on) {
    if (!c) return fail(c, FSS_ERR_INVALID, "null context");
    prof_resolve(c);
    c->prof = on != 0;
    c->prof_acc.clear();
    c->prof_order.clear();
    return FSS_OK;
}

int fss_profile_read(fss_ctx* c, char* names, int32_t names_cap, double* ms, int64_t* launches, int32_t cap,
                     int32_t* count) {
    if (!c) return fail(c, FSS_ERR_INVALID, "null context");
    prof_resolve(c);
    std::string all;
    int32_t k = 0;
    for (const std::string& nm : c->prof_order) {
        if (k < cap) {
            if (ms) ms[k] = c->prof_acc[nm].ms;
            if (launches) launches[k] = c->prof_acc[nm].launches;
        }
        all += nm;
        all += '\n';
        k++;
    }
    if (count) *count = k;
    if (names && names_cap > 0) {
        std::strncpy(names, all.c_str(), size_t(names_cap) - 1);
        names[names_cap - 1] = 0;
    }
    return FSS_OK;
}

int fss_work_per_rhs(fss_ctx* c, double* interactions, double* upward_bytes) {
    if (!c) return fail(c, FSS_ERR_INVALID, "null context");
    if (interactions) *interactions = c->lists.pp_pairs + c->lists.pc_pairs + c->lists.cp_pairs + c->lists.cc_pairs;
    if (upward_bytes) {
        double b = 0;
        if (c->tree && !c->lists.jobs.empty()) {
            int levels = 0;
            for (int l = 0; l <= c->leaf_level; l++) levels += (c->level_mask >> l) & 1;
            const double es = c->fp64 ? 32.0 : 16.0;
            b = double(c->n) * es * levels + double(c->lists.n_proxy) * es;
        }
        *upward_bytes = b;
    }
    return FSS_OK;
}

int fss_icos_counts(int32_t level, int64_t* nv, int64_t* nf) {
    if (level < 0 || level > 11) return fail(nullptr, FSS_ERR_INVALID, "level out of range");
    if (nv) *nv = 10 * (int64_t(1) << (2 * level)) + 2;
    if (nf) *nf = 20 * (int64_t(1) << (2 * level));
    return FSS_OK;
}

int fss_icos_grid(int32_t level, double* xyz, int32_t* faces) {
    if (level < 0 || level > 11) return fail(nullptr, FSS_ERR_INVALID, "level out of range");
    std::vector<double> v;
    std::vector<int32_t> f;
    icos_grid(level, v, f);
    if (xyz) std::memcpy(xyz, v.data(), sizeof(double) * v.size());
    if (faces) std::memcpy(faces, f.data(), sizeof(int32_t) * f.size());
    return FSS_OK;
}

int fss_area_init(int64_t n, const double* state5, int64_t nf, const int32_t* faces, double* area) {
    if (!state5 || !faces || !area) return fail(nullptr, FSS_ERR_INVALID, "null argument");
    area_init(n, state5, nf, faces, area);
    return FSS_OK;
}

int fss_vorticity_rh4_ref(int64_t n, double* state5) {
    if (!state5) return fail(nullptr, FSS_ERR_INVALID, "null argument");
    vorticity_rh4_ref(n, state5);
    return FSS_OK;
}

int fss_vorticity_rh_vortices(int64_t n, double* state5, const double* area, double amp, int32_t nv, double width,
                              uint64_t seed) {
    if (!state5) return fail(nullptr, FSS_ERR_INVALID, "null argument");
    vorticity_rh_vortices(n, state5, area, amp, nv, width, seed);
    return FSS_OK;
}

int fss_tree_traverse(int32_t tree_levels, double theta, int32_t many_count, const int32_t* counts, int32_t* pairs,
                      int64_t cap, int64_t* n_pairs) {
    if (tree_levels < 1 || tree_levels > kMaxLevels || !counts)
        return fail(nullptr, FSS_ERR_INVALID, "bad tree_levels or counts");
    TreeGeometry g = build_tree_geometry(tree_levels);
    std::vector<int32_t> cnt(counts, counts + g.lev_off[tree_levels]);
    std::vector<Pair> pp = dual_traverse(g, cnt, theta, many_count);
    if (n_pairs) *n_pairs = int64_t(pp.size());
    if (int64_t(pp.size()) > cap) return fail(nullptr, FSS_ERR_CAPACITY, "pairs buffer too small");
    if (pairs)
        for (size_t i = 0; i < pp.size(); i++) {
            int32_t* r = pairs + 7 * i;
            r[0] = pp[i].lt; r[1] = pp[i].ls; r[2] = pp[i].t; r[3] = pp[i].s;
            r[4] = pp[i].nt; r[5] = pp[i].ns; r[6] = pp[i].type;
        }
    return FSS_OK;
}

int fss_interp_nodes(int32_t degree, double* nodes, double* vinv) {
    if (degree < 0 || degree > kMaxDegree) return fail(nullptr, FSS_ERR_INVALID, "degree must be in 0..12");
    std::vector<double> nd, vi;
    interp_nodes(degree, nd, vi);
    if (nodes) std::memcpy(nodes, nd.data(), sizeof(double) * nd.size());
    if (vinv) std::memcpy(vinv, vi.data(), sizeof(double) * vi.size());
    return FSS_OK;
}

int fss_tree_geometry(int32_t tree_levels, double* tri_info) {
    if (tree_levels < 1 || tree_levels > kMaxLevels || !tri_info)
        return fail(nullptr, FSS_ERR_INVALID, "bad tree_levels");
    TreeGeometry g = build_tree_geometry(tree_levels);
    std::memcpy(tri_info, g.tri_info.data(), sizeof(double) * 4 * g.lev_off[tree_levels]);
    return FSS_OK;
}

// ------------------------------------------------------------------ sharding

int fss_shard_partition(int64_t nunits, const double* cost, int32_t nranks, int64_t* bounds) {
    if (nunits < 1 || nranks < 1 || !cost || !bounds) return fail(nullptr, FSS_ERR_INVALID, "bad partition arguments");
    if (nranks > nunits) return fail(nullptr, FSS_ERR_INVALID, "more ranks than units");
    const std::vector<int64_t> b = shard_partition(std::vector<double>(cost, cost + nunits), nranks);
    std::memcpy(bounds, b.data(), sizeof(int64_t) * b.size());
    return FSS_OK;
}

int fss_shard_set(fss_ctx* c, int32_t rank, int32_t nranks) {
    if (!c) return fail(c, FSS_ERR_INVALID, "null context");
    if (nranks < 0 || (nranks > 0 && (rank < 0 || rank >= nranks))) return fail(c, FSS_ERR_INVALID, "bad rank");
    CU(cudaSetDevice(c->dev));
    invalidate_graph(c);
    c->shard_rank = nranks > 0 ? rank : 0;
    c->shard_nranks = nranks;
    c->shard_bounds.clear();
    c->shard_cost.clear();
    c->shard_lo = 0;
    c->shard_hi = c->tree ? c->nleaf : c->n;
    if (!c->have) return FSS_OK;  // applied when the particles are set
    if (c->tree) {
        make_lists(c);
        TRY(shard_filter(c));
        TRY(materialize(c, c->shape));
    } else {
        TRY(build_direct_lists(c));
    }
    c->stage_dirty = true;
    TRY(refresh_stage(c));
    return check_device_error(c);
}

int fss_shard_get_info(fss_ctx* c, fss_shard_info* info) {
    if (!c || !info) return fail(c, FSS_ERR_INVALID, "null argument");
    std::memset(info, 0, sizeof(*info));
    info->rank = c->shard_rank;
    info->nranks = c->shard_nranks;
    if (c->shard_nranks <= 0 || c->shard_bounds.empty()) return FSS_OK;
    info->unit_level = c->tree ? c->shard_unit_level : -1;
    info->units = int64_t(c->shard_cost.size());
    info->unit_lo = c->shard_bounds[c->shard_rank];
    info->unit_hi = c->shard_bounds[c->shard_rank + 1];
    info->target_lo = c->shard_lo;
    info->target_hi = c->shard_hi;
    for (size_t u = 0; u < c->shard_cost.size(); u++) {
        info->cost_total += c->shard_cost[u];
        if (int64_t(u) >= info->unit_lo && int64_t(u) < info->unit_hi) info->cost_own += c->shard_cost[u];
    }
    return FSS_OK;
}

int fss_shard_stage(fss_ctx* c, int32_t stage, void* exchange) {
    if (!c || !exchange) return fail(c, FSS_ERR_INVALID, "null argument");
    if (!c->have) return fail(c, FSS_ERR_STATE, "no particles set");
    if (c->shard_nranks <= 0) return fail(c, FSS_ERR_STATE, "context not sharded (fss_shard_set)");
    if (stage < 1 || stage > 4) return fail(c, FSS_ERR_INVALID, "stage must be 1..4");
    CU(cudaSetDevice(c->dev));
    if (stage == 1) {
        TRY(refresh_stage(c));
        if (c->tree && c->resort) TRY(resort(c));
    }
    bool down = false;
    TRY(eval_partials(c, false, &down));
    {
        ProfScope ps(c, "shard_reduce");
        launch_shard_reduce(c->stream, c->n, c->parts + (down ? 1 : 0), c->pstride, c->partials.as<double4>(),
                            c->tree ? c->leaf_start.as<int32_t>() : nullptr, c->shard_lo, c->shard_hi, c->shard_lo,
                            c->shard_hi, static_cast<double4*>(exchange));
    }
    CU(cudaGetLastError());
    return FSS_OK;
}

int fss_shard_combine(fss_ctx* c, int32_t stage, double dt, double omega, const void* exchange) {
    if (!c || !exchange) return fail(c, FSS_ERR_INVALID, "null argument");
    if (!c->have) return fail(c, FSS_ERR_STATE, "no particles set");
    if (c->shard_nranks <= 0) return fail(c, FSS_ERR_STATE, "context not sharded (fss_shard_set)");
    if (stage < 1 || stage > 4) return fail(c, FSS_ERR_INVALID, "stage must be 1..4");
    CU(cudaSetDevice(c->dev));
    EpiArgs ea;
    ea.mode = EPI_RK4;
    ea.stage = stage;
    ea.dt = dt;
    ea.omega = omega;
    ea.s0 = c->s0.as<double4>();
    ea.acc = c->acc.as<double4>();
    ea.n = c->n;
    ea.parts = 1;
    ea.pstride = c->n;
    ea.partials = static_cast<const double4*>(exchange);
    ea.xs = c->xs.as<double4>();
    ea.area = c->area_s.as<double>();
    ea.wtotal = c->wtotal.as<double>();
    ea.perm = c->tree ? c->perm.as<int32_t>() : nullptr;
    ea.src = c->src.p;
    ea.leaf_of = nullptr;
    ea.frame = nullptr;
    {
        ProfScope ps(c, "epilogue");
        launch_epilogue(c->stream, c->fp64, ea);
    }
    CU(cudaGetLastError());
    if (c->prof && stage == 4) prof_resolve(c);
    return FSS_OK;
}

int fss_test_hold_tile(fss_ctx* c, int32_t block) {
    if (!c) return fail(c, FSS_ERR_INVALID, "null context");
    invalidate_graph(c);
    c->hold_block = block < 0 ? -1 : block;
    return FSS_OK;
}

int fss_test_hold_stage(fss_ctx* c, int32_t which) {
    if (!c) return fail(c, FSS_ERR_INVALID, "null context");
    if (which > 1) return fail(c, FSS_ERR_INVALID, "which must be 0 (proxy charges) or 1 (cluster coefficients)");
    invalidate_graph(c);
    c->hold_stage = which < 0 ? -1 : which;
    return FSS_OK;
}

int fss_test_resort_mode(fss_ctx* c, int32_t mode) {
    if (!c) return fail(c, FSS_ERR_INVALID, "null context");
    if (mode != 0 && mode != 1) return fail(c, FSS_ERR_INVALID, "mode must be 0 (partition) or 1 (radix key sort)");
    invalidate_graph(c);
    c->resort_mode = mode;
    return FSS_OK;
}

const char* fss_version(void) { return "fss-b200 0.1 (sm_100a; direct sum + icosahedral BLTC; FP64 and FP32/Kahan)"; }

// ------------------------------------------------------------------ remesh


namespace {
// fss_remesh's device buffers, kept per device between calls (never freed:
// they live until the process ends) and used under a lock.
struct RemeshHost {
    std::mutex mu;
    cudaStream_t st = nullptr;
    DBuf dm, dt, dtri, doff, dadj;
    fss::RemeshScratch rs;
    std::vector<int32_t> tris_host;
    int64_t n = -1;
};
constexpr int kMaxDevices = 64;
RemeshHost* remesh_host(int dev) {
    static std::mutex mu;
    static RemeshHost* h[kMaxDevices] = {};
    std::lock_guard<std::mutex> g(mu);
    if (!h[dev]) h[dev] = new RemeshHost;
    return h[dev];
}
}  // namespace

int fss_remesh(int64_t n, const double* moved5, double* target5, int64_t ntri, const int32_t* tris, double omega,
               int64_t* n_fallback, int64_t* n_not_found) {
    fss_ctx* c = nullptr;  // for the error macros: messages go to fss_last_error(NULL)
    if (n < 3 || ntri < 1 || !moved5 || !target5 || !tris) return fail(c, FSS_ERR_INVALID, "bad remesh arguments");
    if (n > (int64_t(1) << 30) || 3 * ntri > (int64_t(1) << 31) - 1)
        return fail(c, FSS_ERR_INVALID, "too many particles or triangles");
    int dev = 0;
    CU(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fail(c, FSS_ERR_UNSUPPORTED, "device index out of range");
    RemeshHost& h = *remesh_host(dev);
    std::lock_guard<std::mutex> lock(h.mu);
    if (!h.st) CU(cudaStreamCreateWithFlags(&h.st, cudaStreamNonBlocking));
    cudaStream_t st = h.st;
    CU(h.dm.ensure(sizeof(double) * 5 * size_t(n)));
    CU(h.dt.ensure(sizeof(double) * 5 * size_t(n)));
    CU(cudaMemcpyAsync(h.dm.p, moved5, sizeof(double) * 5 * n, cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(h.dt.p, target5, sizeof(double) * 5 * n, cudaMemcpyHostToDevice, st));
    const bool same = h.n == n && h.tris_host.size() == size_t(3 * ntri) &&
                      std::memcmp(h.tris_host.data(), tris, sizeof(int32_t) * 3 * ntri) == 0;
    if (!same) {
        h.n = -1;
        h.tris_host.assign(tris, tris + 3 * ntri);
        CU(h.dtri.ensure(sizeof(int32_t) * 3 * size_t(ntri)));
        CU(h.doff.ensure(sizeof(uint32_t) * size_t(n + 1)));
        CU(h.dadj.ensure(sizeof(int32_t) * 3 * size_t(ntri)));
        CU(cudaMemcpyAsync(h.dtri.p, h.tris_host.data(), sizeof(int32_t) * 3 * ntri, cudaMemcpyHostToDevice, st));
        bool valid = false;
        CU(launch_remesh_adjacency(st, n, ntri, h.dtri.as<int32_t>(), nullptr, h.doff.as<uint32_t>(),
                                   h.dadj.as<int32_t>(), h.rs, &valid));
        if (!valid) {
            h.tris_host.clear();
            return fail(c, FSS_ERR_INVALID, "triangle vertex out of range");
        }
        h.n = n;
    }
    CU(launch_remesh(st, n, h.dm.as<double>(), h.dt.as<double>(), ntri, h.dtri.as<int32_t>(), h.doff.as<uint32_t>(),
                     h.dadj.as<int32_t>(), omega, h.rs, n_fallback, n_not_found));
    CU(cudaMemcpyAsync(target5, h.dt.p, sizeof(double) * 5 * n, cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    return FSS_OK;
}

int fss_remesh_lists(int64_t n, const double* moved5, double* target5, int64_t ntri, const int32_t* tris,
                     const int32_t* vt_off, const int32_t* vt_adj, double omega, int64_t* n_fallback,
                     int64_t* n_not_found) {
    fss_ctx* c = nullptr;  // for the error macros: messages go to fss_last_error(NULL)
    if (n < 3 || ntri < 1 || !moved5 || !target5 || !tris || !vt_off || !vt_adj)
        return fail(c, FSS_ERR_INVALID, "bad remesh arguments");
    if (n > (int64_t(1) << 30) || 3 * ntri > (int64_t(1) << 31) - 1)
        return fail(c, FSS_ERR_INVALID, "too many particles or triangles");
    for (int64_t j = 0; j < 3 * ntri; j++)
        if (tris[j] < 0 || tris[j] >= n) return fail(c, FSS_ERR_INVALID, "triangle vertex out of range");
    if (vt_off[0] != 0) return fail(c, FSS_ERR_INVALID, "vert_tris offsets must start at 0");
    for (int64_t i = 0; i < n; i++)
        if (vt_off[i + 1] < vt_off[i]) return fail(c, FSS_ERR_INVALID, "vert_tris offsets must not decrease");
    const int64_t na = vt_off[n];
    // the remesh kernels read corner ids (3 t + c) and use the triangle t
    std::vector<uint32_t> off(size_t(n) + 1);
    std::vector<int32_t> adj(size_t(std::max<int64_t>(na, 1)));
    for (int64_t i = 0; i <= n; i++) off[i] = uint32_t(vt_off[i]);
    for (int64_t a = 0; a < na; a++) {
        if (vt_adj[a] < 0 || vt_adj[a] >= ntri) return fail(c, FSS_ERR_INVALID, "vert_tris triangle out of range");
        adj[a] = 3 * vt_adj[a];
    }
    cudaStream_t st;
    CU(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } guard{st};
    DBuf dm, dt, dtri, doff, dadj;
    RemeshScratch rs;
    CU(dm.ensure(sizeof(double) * 5 * size_t(n)));
    CU(dt.ensure(sizeof(double) * 5 * size_t(n)));
    CU(dtri.ensure(sizeof(int32_t) * 3 * size_t(ntri)));
    CU(doff.ensure(sizeof(uint32_t) * off.size()));
    CU(dadj.ensure(sizeof(int32_t) * adj.size()));
    CU(cudaMemcpyAsync(dm.p, moved5, sizeof(double) * 5 * n, cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(dt.p, target5, sizeof(double) * 5 * n, cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(dtri.p, tris, sizeof(int32_t) * 3 * ntri, cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(doff.p, off.data(), sizeof(uint32_t) * off.size(), cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(dadj.p, adj.data(), sizeof(int32_t) * adj.size(), cudaMemcpyHostToDevice, st));
    CU(launch_remesh(st, n, dm.as<double>(), dt.as<double>(), ntri, dtri.as<int32_t>(), doff.as<uint32_t>(),
                     dadj.as<int32_t>(), omega, rs, n_fallback, n_not_found));
    CU(cudaMemcpyAsync(target5, dt.p, sizeof(double) * 5 * n, cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    return FSS_OK;
}

int fss_remesh_current(fss_ctx* c, int64_t ntri, const int32_t* tris, double omega, int64_t* n_fallback,
                       int64_t* n_not_found) {
    if (!c) return fail(c, FSS_ERR_INVALID, "null context");
    if (!c->have) return fail(c, FSS_ERR_STATE, "no particles set");
    const int64_t n = c->n;
    if (!tris) {  // the triangles of the previous call
        if (ntri != 0 || c->rm_n != n || c->rm_tris_host.empty())
            return fail(c, FSS_ERR_STATE, "no triangles from a previous remesh to reuse");
        ntri = int64_t(c->rm_tris_host.size() / 3);
        tris = c->rm_tris_host.data();
    }
    if (ntri < 1) return fail(c, FSS_ERR_INVALID, "bad remesh arguments");
    if (3 * ntri > (int64_t(1) << 31) - 1) return fail(c, FSS_ERR_INVALID, "too many triangles");
    CU(cudaSetDevice(c->dev));
    // triangles and adjacency: rebuilt on the device only when they changed
    const bool same = c->rm_n == n && c->rm_tris_host.size() == size_t(3 * ntri) &&
                      (tris == c->rm_tris_host.data() ||
                       std::memcmp(c->rm_tris_host.data(), tris, sizeof(int32_t) * 3 * ntri) == 0);
    if (!same) {
        c->rm_n = -1;
        c->rm_tris_host.assign(tris, tris + 3 * ntri);
        CU(c->rm_tris.ensure(sizeof(int32_t) * 3 * size_t(ntri)));
        CU(c->rm_off.ensure(sizeof(uint32_t) * size_t(n + 1)));
        CU(c->rm_adj.ensure(sizeof(int32_t) * 3 * size_t(ntri)));
        CU(cudaMemcpyAsync(c->rm_tris.p, c->rm_tris_host.data(), sizeof(int32_t) * 3 * ntri, cudaMemcpyHostToDevice,
                           c->stream));
        bool valid = false;
        CU(launch_remesh_adjacency(c->stream, n, ntri, c->rm_tris.as<int32_t>(), nullptr, c->rm_off.as<uint32_t>(),
                                   c->rm_adj.as<int32_t>(), c->rm, &valid));
        if (!valid) {
            c->rm_tris_host.clear();
            return fail(c, FSS_ERR_INVALID, "triangle vertex out of range");
        }
        c->rm_n = n;
    }
    CU(c->rm_target.ensure(sizeof(double) * 5 * size_t(n)));
    TRY(refresh_stage(c));
    // moved state in the caller's order, targets = grid positions
    launch_scatter_state(c->stream, n, c->tree ? c->perm.as<int32_t>() : nullptr, c->s0.as<double4>(),
                         c->tracer_s.as<double>(), c->out5.as<double>());
    launch_remesh_targets(c->stream, n, c->grid3.as<double>(), c->out5.as<double>(), c->rm_target.as<double>());
    CU(launch_remesh(c->stream, n, c->out5.as<double>(), c->rm_target.as<double>(), ntri, c->rm_tris.as<int32_t>(),
                     c->rm_off.as<uint32_t>(), c->rm_adj.as<int32_t>(), omega, c->rm, n_fallback, n_not_found));
    // the regridded state becomes the step state (sorted order of the
    // context), then particles go back into the leaves of their grid points
    CU(cudaMemcpyAsync(c->in5.p, c->rm_target.p, sizeof(double) * 5 * n, cudaMemcpyDeviceToDevice, c->stream));
    TRY(gather(c, true));
    c->stage_dirty = false;
    if (c->tree && c->resort) TRY(resort(c));
    return check_device_error(c);
}

int fss_amr_refine_current(fss_ctx* c, fss_amr* a, double vorticity_tol, double circulation_tol, double omega,
                           int64_t* point_count) {
    if (!c || !a) return fail(c, FSS_ERR_INVALID, "null argument");
    if (!c->have) return fail(c, FSS_ERR_STATE, "no particles set");
    if (a->broken) return fail(c, FSS_ERR_STATE, "amr handle unusable after a capacity error");
    if (a->n != c->n) return fail(c, FSS_ERR_INVALID, "the context's particles are not the mesh's points");
    if (a->dev != c->dev) return fail(c, FSS_ERR_INVALID, "the context and the mesh are on different devices");
    CU(cudaSetDevice(c->dev));
    const int64_t n0 = c->n;
    if (n0 < a->max_points) {  // config1.point_count >= config1.max_count: amr() does nothing
        // the current state in the caller's order, and its areas, into the mesh
        TRY(refresh_stage(c));
        launch_scatter_state(c->stream, n0, c->tree ? c->perm.as<int32_t>() : nullptr, c->s0.as<double4>(),
                             c->tracer_s.as<double>(), c->out5.as<double>());
        CU(cudaMemcpyAsync(a->state5.p, c->out5.p, sizeof(double) * 5 * n0, cudaMemcpyDeviceToDevice, c->stream));
        CU(cudaMemcpyAsync(a->area.p, c->area_in.p, sizeof(double) * n0, cudaMemcpyDeviceToDevice, c->stream));
        CU(cudaStreamSynchronize(c->stream));
        if (int rc = amr_refine_device(a, vorticity_tol, circulation_tol)) {
            a->broken = true;
            return fail(c, rc, fss_last_error(nullptr));
        }
        // the new midpoints onto the sphere (the step's own projection placed
        // the others there), then the new particle set
        amr_project(a->st, n0, a->n, a->state5.as<double>(), omega);
        CU(cudaStreamSynchronize(a->st));
        if (a->n > n0) TRY(set_particles(c, a->n, a->state5.as<double>(), a->area.as<double>()));
    }
    if (point_count) *point_count = c->n;
    return FSS_OK;
}

}  // extern "C"
