// ensemble.cpp -- many independent problems of uneven size advanced
// together (mixed-precision treecode, RK4).
//
// Every member is set up by the single-problem path (tree build on the GPU,
// interaction lists on the host); the ensemble then concatenates the
// members' leaf-ordered particles, their leaves (global leaf index = member
// leaf offset + local index), their far-cluster proxy slots and their work
// lists (indices shifted), so that per RK stage one batched upward pass,
// ONE persistent pair-kernel launch over a global (member, target leaf,
// source run) work queue and one epilogue advance all members.  With
// re-sorting, the particles of all members are put into their current
// leaves at the start of each step by one key sort over global leaf
// indices (a member's leaves are consecutive, so its particles stay in its
// own range).  The re-sort and the four stages of a step are captured in
// one CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "ctx.h"
#include "fss.h"
#include "kernels.h"

namespace fss {
void set_last_error(const std::string& msg);
}

using namespace fss;

struct fss_ensemble {
    fss_config cfg{};
    int dev = 0;
    cudaStream_t stream = nullptr, own = nullptr;
    std::vector<fss_ctx*> members;
    std::vector<int64_t> poff, pxoff, loff;  // particle, proxy-slot and leaf offsets per member
    int64_t ntot = 0, nprox = 0, nleaf = 0;
    int nmax = 0, blocks = 0;
    int max_leaf_level = 0;  // deepest member's leaf level
    double interactions = 0;
    bool built = false, resort = false;
    DBuf s0, xs, acc, area, tracer, perm, src, partials, segs, items, jobs, leaves, leaf_start, part, proxy_pos, vinv,
        vinv_off, node, lev_off, verts, tri_verts, queue, err, key, key_tmp, sortq, vals_tmp, hist;
    int64_t nitems = 0, njobs = 0;
    cudaGraphExec_t graph = nullptr;
    double gdt = 0, gomega = 0;
    fss::PairCtl ctl() const {
        return fss::PairCtl{cfg.wait_limit_us > 0 ? uint64_t(cfg.wait_limit_us) * 1000ull : fss::kWaitLimitNs, -1, 0};
    }
    ~fss_ensemble() {
        if (graph) cudaGraphExecDestroy(graph);
        for (fss_ctx* m : members) fss_destroy(m);
        if (own) cudaStreamDestroy(own);
    }
};

namespace {

int efail(int code, const std::string& m) {
    set_last_error(m);
    return code;
}

#define ECU(call)                                                                                        \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess)                                                                           \
            return efail(e_ == cudaErrorMemoryAllocation ? FSS_ERR_NOMEM : FSS_ERR_CUDA,                 \
                         std::string(#call) + ": " + cudaGetErrorString(e_));                            \
    } while (0)

template <typename T>
int eupload(fss_ensemble* e, DBuf& b, const std::vector<T>& v) {
    ECU(b.ensure(sizeof(T) * std::max<size_t>(v.size(), 1)));
    if (!v.empty()) ECU(cudaMemcpyAsync(b.p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, e->stream));
    return FSS_OK;
}

// Every member's particles into the leaves they are in now.
int resort(fss_ensemble* e) {
    const int64_t n = e->ntot;
    launch_reassign(e->stream, n, e->s0.as<double4>(), e->leaves.as<EnsLeaf>(), 0, e->node.as<NodeGeom>(),
                    e->lev_off.as<int64_t>(), e->key.as<uint32_t>(), e->err.as<int>());
    int bits = 0;
    while ((int64_t(1) << bits) < e->nleaf) bits++;
    launch_sort(e->stream, n, std::max(bits, 1), e->key.as<uint32_t>(), e->key_tmp.as<uint32_t>(),
                e->sortq.as<int32_t>(), e->vals_tmp.as<int32_t>(), e->hist.as<uint32_t>());
    launch_resort(e->stream, false, n, e->sortq.as<int32_t>(), e->s0.as<double4>(), e->area.as<double>(),
                  e->tracer.as<double>(), e->perm.as<int32_t>(), e->xs.as<double4>(), e->acc.as<double4>(), e->src.p);
    launch_leaf_bounds(e->stream, n, e->key.as<uint32_t>(), int32_t(e->nleaf), e->leaf_start.as<int32_t>());
    ECU(cudaGetLastError());
    return FSS_OK;
}

int stage(fss_ensemble* e, int st, double dt, double omega) {
    if (st == 1 && e->resort) {
        const int r = resort(e);
        if (r) return r;
    }
    launch_up_leaf_batch(e->stream, int(e->nleaf), e->src.p, e->leaves.as<EnsLeaf>(), e->leaf_start.as<int32_t>(),
                         e->node.as<NodeGeom>(), e->lev_off.as<int64_t>(), e->nmax, e->max_leaf_level,
                         e->part.as<double>());
    launch_up_combine_batch(e->stream, int(e->njobs), e->jobs.as<ProxyJob>(), e->leaves.as<EnsLeaf>(),
                            e->part.as<double>(), e->nmax, e->vinv.as<double>(), e->vinv_off.as<int32_t>(),
                            e->proxy_pos.as<double4>(), e->ntot, e->src.p);
    ECU(cudaMemsetAsync(e->queue.p, 0, sizeof(int), e->stream));
    ECU(launch_pairs_persistent(e->stream, int(e->nitems), e->src.p, e->segs.as<Segment>(),
                                e->leaf_start.as<int32_t>(), e->items.as<WorkItem>(), e->queue.as<int>(),
                                e->partials.as<double4>(), e->ntot, e->err.as<int>(), e->blocks, e->ctl()));
    EpiArgs a;
    a.n = e->ntot;
    a.parts = 1;
    a.pstride = e->ntot;
    a.partials = e->partials.as<double4>();
    a.xs = e->xs.as<double4>();
    a.area = e->area.as<double>();
    a.omega = omega;
    a.mode = EPI_RK4;
    a.stage = st;
    a.dt = dt;
    a.s0 = e->s0.as<double4>();
    a.acc = e->acc.as<double4>();
    a.src = e->src.p;
    launch_epilogue(e->stream, false, a);
    ECU(cudaGetLastError());
    return FSS_OK;
}

}  // namespace

extern "C" {

int fss_ensemble_create(const fss_config* cfg, fss_ensemble** out) {
    if (!cfg || !out) return efail(FSS_ERR_INVALID, "null argument");
    *out = nullptr;
    if (cfg->precision != FSS_PREC_MIXED || cfg->method != FSS_METHOD_TREECODE)
        return efail(FSS_ERR_UNSUPPORTED, "ensembles run the mixed-precision treecode");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return efail(FSS_ERR_UNSUPPORTED, "no CUDA device");
    }
    std::unique_ptr<fss_ensemble> e(new fss_ensemble());
    e->cfg = *cfg;
    e->cfg.block_threads = kPersistentThreads;  // items hold at most one block of targets
    e->cfg.targets_per_thread = 1;
    e->cfg.src_parts = 1;
    e->cfg.autotune = 0;
    e->cfg.use_graph = 0;
    e->cfg.cluster_targets = 0;  // members' far fields are summed at their particles
    e->dev = cfg->device;
    ECU(cudaSetDevice(e->dev));
    ECU(cudaStreamCreateWithFlags(&e->own, cudaStreamNonBlocking));
    e->stream = e->own;
    *out = e.release();
    return FSS_OK;
}

void fss_ensemble_destroy(fss_ensemble* e) {
    if (!e) return;
    cudaSetDevice(e->dev);
    cudaStreamSynchronize(e->stream);
    delete e;
}

int fss_ensemble_set_stream(fss_ensemble* e, void* stream) {
    if (!e) return efail(FSS_ERR_INVALID, "null ensemble");
    if (e->graph) cudaGraphExecDestroy(e->graph);
    e->graph = nullptr;
    e->stream = stream ? static_cast<cudaStream_t>(stream) : e->own;
    return FSS_OK;
}

int fss_ensemble_add(fss_ensemble* e, int64_t n, const double* state5, const double* area, int32_t* member) {
    if (!e) return efail(FSS_ERR_INVALID, "null ensemble");
    if (e->built) return efail(FSS_ERR_STATE, "ensemble already built");
    fss_ctx* c = nullptr;
    int rc = fss_create(&e->cfg, &c);
    if (rc) return rc;
    rc = fss_set_particles(c, n, state5, area);
    if (rc) {
        set_last_error(fss_last_error(c));
        fss_destroy(c);
        return rc;
    }
    if (member) *member = int32_t(e->members.size());
    e->members.push_back(c);
    return FSS_OK;
}

int fss_ensemble_build(fss_ensemble* e) {
    if (!e || e->members.empty()) return efail(FSS_ERR_STATE, "no members");
    ECU(cudaSetDevice(e->dev));
    // offsets
    e->ntot = e->nprox = e->nleaf = 0;
    e->poff.clear(); e->pxoff.clear(); e->loff.clear();
    int maxTL = 1;
    e->nmax = 0;
    for (fss_ctx* c : e->members) {
        e->poff.push_back(e->ntot);
        e->pxoff.push_back(e->nprox);
        e->loff.push_back(e->nleaf);
        e->ntot += c->n;
        e->nprox += c->lists.n_proxy;
        e->nleaf += c->nleaf;
        maxTL = std::max(maxTL, c->tree_levels);
        e->nmax = std::max(e->nmax, c->nmax);
    }
    // concatenated work lists
    std::vector<Segment> segs;
    std::vector<WorkItem> items;
    std::vector<double> cost;
    std::vector<ProxyJob> jobs;
    std::vector<EnsLeaf> leaves;
    std::vector<int32_t> lstart;
    std::vector<uint32_t> keys;
    std::vector<double4> ppos;
    int64_t part_base = 0;
    const int KM = nproxy(e->nmax);
    e->interactions = 0;
    e->resort = false;
    for (size_t m = 0; m < e->members.size(); m++) {
        fss_ctx* c = e->members[m];
        const ListOutput& L = c->lists;
        const int64_t po = e->poff[m], pxo = e->ntot + e->pxoff[m], lo = e->loff[m];
        const std::vector<int32_t>& ls = c->leaf_start_h;
        e->resort = e->resort || c->resort;
        const int32_t sbase = int32_t(segs.size());
        for (Segment sg : L.segs) {
            if (sg.kind == 0) {
                sg.a += int32_t(lo);
                sg.b += int32_t(lo);
            } else {
                const int64_t sh = (sg.a >= c->n) ? pxo - c->n : po;
                sg.a = int32_t(sg.a + sh);
                sg.b = int32_t(sg.b + sh);
            }
            segs.push_back(sg);
        }
        for (WorkItem it : L.items) {
            double w = 0;
            for (int32_t k = it.g0; k < it.g1; k++) {
                const Segment& sg = L.segs[k];
                w += (sg.kind == 0) ? double(ls[sg.b] - ls[sg.a]) : double(sg.b - sg.a);
            }
            it.t0 = int32_t(it.t0 + po);
            it.g0 += sbase;
            it.g1 += sbase;
            it.part = 0;
            if (it.leaf >= 0) it.leaf += int32_t(lo);
            items.push_back(it);
            cost.push_back(w);
        }
        for (ProxyJob j : L.jobs) {
            j.leaf_lo += int32_t(lo);
            j.leaf_hi += int32_t(lo);
            for (int d = 0; d <= kMaxDegree; d++)
                if (j.off[d] >= 0) j.off[d] = int32_t(j.off[d] - c->n + pxo);
            jobs.push_back(j);
        }
        for (int64_t l = 0; l < c->nleaf; l++) {
            EnsLeaf lf{};
            lf.gleaf = int32_t(lo + l);
            lf.leaf_level = c->leaf_level;
            lf.local = int32_t(l);
            lf.part_base = part_base;
            lf.level_mask = c->level_mask;
            part_base += int64_t(c->leaf_level + 1) * KM;
            leaves.push_back(lf);
            lstart.push_back(int32_t(ls[l] + po));
            for (int32_t s = ls[l]; s < ls[l + 1]; s++) keys.push_back(uint32_t(lo + l));
        }
        for (size_t i = 0; i < L.proxy_pos.size() / 4; i++)
            ppos.push_back(make_double4(L.proxy_pos[4 * i], L.proxy_pos[4 * i + 1], L.proxy_pos[4 * i + 2], 0.0));
        e->interactions += L.pp_pairs + L.pc_pairs;
    }
    lstart.push_back(int32_t(e->ntot));
    e->max_leaf_level = maxTL - 1;
    // longest source lists first across all members
    {
        std::vector<size_t> order(items.size());
        for (size_t k = 0; k < order.size(); k++) order[k] = k;
        std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return cost[a] > cost[b]; });
        std::vector<WorkItem> sorted;
        sorted.reserve(items.size());
        for (size_t k : order) sorted.push_back(items[k]);
        items.swap(sorted);
    }
    e->nitems = int64_t(items.size());
    e->njobs = int64_t(jobs.size());
    int r;
    if ((r = eupload(e, e->segs, segs)) || (r = eupload(e, e->items, items)) || (r = eupload(e, e->jobs, jobs)) ||
        (r = eupload(e, e->leaves, leaves)) || (r = eupload(e, e->leaf_start, lstart)) ||
        (r = eupload(e, e->key, keys)) || (r = eupload(e, e->proxy_pos, ppos)))
        return r;
    // tree geometry of the deepest member serves every member (the
    // refinement numbers faces the same way at every depth)
    TreeGeometry g = build_tree_geometry(maxTL);
    if ((r = eupload(e, e->node, g.node)) || (r = eupload(e, e->lev_off, g.lev_off)) ||
        (r = eupload(e, e->verts, g.verts)) || (r = eupload(e, e->tri_verts, g.tri_verts)))
        return r;
    std::vector<double> vall;
    std::vector<int32_t> voff(kMaxDegree + 1, 0);
    for (int d = 0; d <= e->nmax; d++) {
        std::vector<double> nodes, vi;
        interp_nodes(d, nodes, vi);
        voff[d] = int32_t(vall.size());
        vall.insert(vall.end(), vi.begin(), vi.end());
    }
    if ((r = eupload(e, e->vinv, vall)) || (r = eupload(e, e->vinv_off, voff))) return r;
    // particle state and sources from the members (device to device)
    const size_t N = size_t(e->ntot);
    ECU(e->s0.ensure(sizeof(double4) * N));
    ECU(e->xs.ensure(sizeof(double4) * N));
    ECU(e->acc.ensure(sizeof(double4) * N));
    ECU(e->area.ensure(sizeof(double) * N));
    ECU(e->tracer.ensure(sizeof(double) * N));
    ECU(e->perm.ensure(sizeof(int32_t) * N));
    ECU(e->key_tmp.ensure(sizeof(uint32_t) * N));
    ECU(e->sortq.ensure(sizeof(int32_t) * N));
    ECU(e->vals_tmp.ensure(sizeof(int32_t) * N));
    ECU(e->hist.ensure(sizeof(uint32_t) * size_t(sort_scratch_words(e->ntot))));
    ECU(e->src.ensure(sizeof(float4) * size_t(e->ntot + e->nprox)));
    ECU(e->partials.ensure(sizeof(double4) * N));
    ECU(e->part.ensure(sizeof(double) * size_t(std::max<int64_t>(part_base, 1))));
    ECU(e->queue.ensure(sizeof(int)));
    ECU(e->err.ensure(sizeof(int)));
    ECU(cudaMemsetAsync(e->err.p, 0, sizeof(int), e->stream));
    for (size_t m = 0; m < e->members.size(); m++) {
        fss_ctx* c = e->members[m];
        ECU(cudaStreamSynchronize(c->stream));
        const int64_t po = e->poff[m];
        ECU(cudaMemcpyAsync(e->s0.as<double4>() + po, c->s0.p, sizeof(double4) * c->n, cudaMemcpyDeviceToDevice, e->stream));
        ECU(cudaMemcpyAsync(e->xs.as<double4>() + po, c->s0.p, sizeof(double4) * c->n, cudaMemcpyDeviceToDevice, e->stream));
        ECU(cudaMemcpyAsync(e->area.as<double>() + po, c->area_s.p, sizeof(double) * c->n, cudaMemcpyDeviceToDevice,
                            e->stream));
        ECU(cudaMemcpyAsync(e->tracer.as<double>() + po, c->tracer_s.p, sizeof(double) * c->n,
                            cudaMemcpyDeviceToDevice, e->stream));
        ECU(cudaMemcpyAsync(e->perm.as<int32_t>() + po, c->perm.p, sizeof(int32_t) * c->n, cudaMemcpyDeviceToDevice,
                            e->stream));
    }
    // sources of the step state
    launch_refresh(e->stream, false, e->ntot, e->s0.as<double4>(), e->area.as<double>(), nullptr, nullptr,
                   e->xs.as<double4>(), e->src.p);
    const int per_sm = persistent_blocks_per_sm();
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e->dev);
    e->blocks = per_sm * sms;
    ECU(cudaStreamSynchronize(e->stream));
    e->built = true;
    return FSS_OK;
}

int fss_ensemble_rk4_step(fss_ensemble* e, double dt, double omega, int32_t nsteps) {
    if (!e || !e->built) return efail(FSS_ERR_STATE, "ensemble not built");
    ECU(cudaSetDevice(e->dev));
    if (!e->graph || e->gdt != dt || e->gomega != omega) {
        if (e->graph) cudaGraphExecDestroy(e->graph);
        e->graph = nullptr;
        cudaGraph_t g;
        ECU(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
        int r = FSS_OK;
        for (int st = 1; st <= 4 && r == FSS_OK; st++) r = stage(e, st, dt, omega);
        const cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
        if (r) return r;
        if (ce != cudaSuccess) return efail(FSS_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
        const cudaError_t ie = cudaGraphInstantiate(&e->graph, g, 0);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) return efail(FSS_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie));
        e->gdt = dt;
        e->gomega = omega;
    }
    for (int s = 0; s < nsteps; s++) ECU(cudaGraphLaunch(e->graph, e->stream));
    return FSS_OK;
}

int fss_ensemble_time_pairs(fss_ensemble* e, int32_t reps, double* ms) {
    if (!e || !e->built || !ms) return efail(FSS_ERR_STATE, "ensemble not built");
    if (reps < 1) return efail(FSS_ERR_INVALID, "reps < 1");
    ECU(cudaSetDevice(e->dev));
    cudaEvent_t a, b;
    ECU(cudaEventCreate(&a));
    ECU(cudaEventCreate(&b));
    struct Ev {
        cudaEvent_t a, b;
        ~Ev() { cudaEventDestroy(a); cudaEventDestroy(b); }
    } guard{a, b};
    float total = 0;
    for (int r = 0; r <= reps; r++) {  // launch 0 untimed
        ECU(cudaMemsetAsync(e->queue.p, 0, sizeof(int), e->stream));
        ECU(cudaEventRecord(a, e->stream));
        ECU(launch_pairs_persistent(e->stream, int(e->nitems), e->src.p, e->segs.as<Segment>(),
                                    e->leaf_start.as<int32_t>(), e->items.as<WorkItem>(), e->queue.as<int>(),
                                    e->partials.as<double4>(), e->ntot, e->err.as<int>(), e->blocks, e->ctl()));
        ECU(cudaEventRecord(b, e->stream));
        ECU(cudaEventSynchronize(b));
        float t = 0;
        ECU(cudaEventElapsedTime(&t, a, b));
        if (r) total += t;
    }
    int err = 0;
    ECU(cudaMemcpy(&err, e->err.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) return efail(FSS_ERR_TIMEOUT, "a kernel's bounded wait timed out");
    *ms = double(total) / reps;
    return FSS_OK;
}

int fss_ensemble_get_state(fss_ensemble* e, int32_t member, double* state5) {
    if (!e || !e->built || !state5) return efail(FSS_ERR_STATE, "ensemble not built");
    if (member < 0 || member >= int32_t(e->members.size())) return efail(FSS_ERR_INVALID, "bad member");
    ECU(cudaSetDevice(e->dev));
    fss_ctx* c = e->members[member];
    const int64_t n = c->n, po = e->poff[member];
    std::vector<double4> s(n);
    std::vector<double> tr(n);
    std::vector<int32_t> perm(n);
    int err = 0;
    ECU(cudaMemcpyAsync(s.data(), e->s0.as<double4>() + po, sizeof(double4) * n, cudaMemcpyDeviceToHost, e->stream));
    ECU(cudaMemcpyAsync(tr.data(), e->tracer.as<double>() + po, sizeof(double) * n, cudaMemcpyDeviceToHost, e->stream));
    ECU(cudaMemcpyAsync(perm.data(), e->perm.as<int32_t>() + po, sizeof(int32_t) * n, cudaMemcpyDeviceToHost,
                        e->stream));
    ECU(cudaMemcpyAsync(&err, e->err.p, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
    ECU(cudaStreamSynchronize(e->stream));
    if (err == kErrNonFinite) return efail(FSS_ERR_INVALID, "non-finite particle position (diverged state?)");
    if (err) return efail(FSS_ERR_TIMEOUT, "a kernel's bounded wait timed out");
    for (int64_t k = 0; k < n; k++) {
        double* o = state5 + 5 * int64_t(perm[k]);
        o[0] = s[k].x; o[1] = s[k].y; o[2] = s[k].z; o[3] = s[k].w; o[4] = tr[k];
    }
    return FSS_OK;
}

int fss_ensemble_info(fss_ensemble* e, int32_t* members, int64_t* particles, double* interactions_per_rhs,
                      int64_t* work_items) {
    if (!e) return efail(FSS_ERR_INVALID, "null ensemble");
    if (members) *members = int32_t(e->members.size());
    if (particles) *particles = e->ntot;
    if (interactions_per_rhs) *interactions_per_rhs = e->interactions;
    if (work_items) *work_items = e->nitems;
    return FSS_OK;
}

}  // extern "C"
