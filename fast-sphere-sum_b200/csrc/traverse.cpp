// traverse.cpp -- treecode interaction lists (host).
//
// dual_traverse() is compiled with -ffp-contract=off and follows
// fast_rhs.h:16-91 tree_traverse operation for operation, so its pair list
// is bit-identical to the reference's for the same per-face counts.
#include "traverse.h"

#include <algorithm>
#include <cmath>
#include <map>
#include <stdexcept>

namespace fss {

std::vector<Pair> dual_traverse(const TreeGeometry& g, const std::vector<int32_t>& counts, double theta,
                                int many_count) {
    const int L = g.tree_levels;
    std::vector<Pair> out;
    struct Q { int32_t t, s, lt, ls; };
    std::vector<Q> q;
    q.reserve(1 << 16);
    size_t head = 0;
    for (int i = 0; i < 20; i++)
        for (int j = 0; j < 20; j++) q.push_back({i, j, 0, 0});
    while (head < q.size()) {
        const Q e = q[head++];
        const int nt = counts[g.lev_off[e.lt] + e.t], ns = counts[g.lev_off[e.ls] + e.s];
        if (nt == 0 || ns == 0) continue;  // fast_rhs.h:40
        const double* ti = &g.tri_info[4 * (g.lev_off[e.lt] + e.t)];
        const double* si = &g.tri_info[4 * (g.lev_off[e.ls] + e.s)];
        const double dist = great_circ_dist(ti, si, 1.0);
        const double sep = (ti[3] + si[3]) / dist;
        if (dist > 0 && sep < theta) {  // fast_rhs.h:46-58
            const int ty = ((nt > many_count) ? 2 : 0) + ((ns > many_count) ? 1 : 0);
            out.push_back({e.lt, e.ls, e.t, e.s, nt, ns, ty, 1, -1});
        } else if (nt < many_count && ns < many_count) {  // :60
            out.push_back({e.lt, e.ls, e.t, e.s, nt, ns, 0, 0, -1});
        } else if (e.lt == L - 1 && e.ls == L - 1) {  // :63
            out.push_back({e.lt, e.ls, e.t, e.s, nt, ns, 0, 0, -1});
        } else if (e.lt == L - 1) {  // :66 refine the source
            for (int c = 0; c < 4; c++) q.push_back({e.t, 4 * e.s + c, e.lt, e.ls + 1});
        } else if (e.ls == L - 1) {  // :71 refine the target
            for (int c = 0; c < 4; c++) q.push_back({4 * e.t + c, e.s, e.lt + 1, e.ls});
        } else if (nt >= ns) {  // :77
            for (int c = 0; c < 4; c++) q.push_back({4 * e.t + c, e.s, e.lt + 1, e.ls});
        } else {
            for (int c = 0; c < 4; c++) q.push_back({e.t, 4 * e.s + c, e.lt, e.ls + 1});
        }
        if (head > (1u << 20) && head * 2 > q.size()) {  // keep the FIFO compact
            q.erase(q.begin(), q.begin() + head);
            head = 0;
        }
    }
    return out;
}

std::vector<Pair> dual_traverse_faces(const TreeGeometry& g, const std::vector<int32_t>& counts,
                                      const std::vector<double>& face_theta, const std::vector<int32_t>& face_deg) {
    const int L = g.tree_levels;
    std::vector<Pair> out;
    struct Q { int32_t t, s, lt, ls; };
    std::vector<Q> q;
    q.reserve(1 << 16);
    size_t head = 0;
    for (int i = 0; i < 20; i++)
        for (int j = 0; j < 20; j++) q.push_back({i, j, 0, 0});
    while (head < q.size()) {
        const Q e = q[head++];
        const int64_t gt = g.lev_off[e.lt] + e.t, gs = g.lev_off[e.ls] + e.s;
        const int nt = counts[gt], ns = counts[gs];
        if (nt == 0 || ns == 0) continue;
        const int deg = face_deg[gt];
        const int many = nproxy(deg);
        const double* ti = &g.tri_info[4 * gt];
        const double* si = &g.tri_info[4 * gs];
        const double dist = great_circ_dist(ti, si, 1.0);
        if (dist > 0 && (ti[3] + si[3]) / dist < face_theta[gt]) {
            const int ty = ((nt > many) ? 2 : 0) + ((ns > many) ? 1 : 0);
            out.push_back({e.lt, e.ls, e.t, e.s, nt, ns, ty, 1, deg});
        } else if ((nt < many && ns < many) || (e.lt == L - 1 && e.ls == L - 1)) {
            out.push_back({e.lt, e.ls, e.t, e.s, nt, ns, 0, 0, deg});
        } else if (e.lt == L - 1) {
            for (int c = 0; c < 4; c++) q.push_back({e.t, 4 * e.s + c, e.lt, e.ls + 1});
        } else if (e.ls == L - 1 || nt >= ns) {
            for (int c = 0; c < 4; c++) q.push_back({4 * e.t + c, e.s, e.lt + 1, e.ls});
        } else {
            for (int c = 0; c < 4; c++) q.push_back({e.t, 4 * e.s + c, e.lt, e.ls + 1});
        }
        if (head > (1u << 20) && head * 2 > q.size()) {
            q.erase(q.begin(), q.begin() + head);
            head = 0;
        }
    }
    return out;
}

void face_params(const TreeGeometry& g, int leaf_level, const std::vector<int32_t>& leaf_deg,
                 const std::vector<double>& leaf_theta, std::vector<int32_t>& face_deg,
                 std::vector<double>& face_theta) {
    const int64_t nf = g.lev_off[leaf_level + 1];
    face_deg.assign(nf, 0);
    face_theta.assign(nf, 1e300);
    const int64_t nleaf = g.level_count(leaf_level);
    for (int64_t l = 0; l < nleaf; l++) {
        face_deg[g.lev_off[leaf_level] + l] = leaf_deg[l];
        face_theta[g.lev_off[leaf_level] + l] = leaf_theta[l];
    }
    for (int lv = leaf_level - 1; lv >= 0; lv--)
        for (int64_t f = 0; f < g.level_count(lv); f++) {
            const int64_t p = g.lev_off[lv] + f;
            for (int c = 0; c < 4; c++) {
                const int64_t ch = g.lev_off[lv + 1] + 4 * f + c;
                face_deg[p] = std::max(face_deg[p], face_deg[ch]);
                face_theta[p] = std::min(face_theta[p], face_theta[ch]);
            }
        }
}

std::vector<std::vector<ASrc>> lists_from_pairs(const TreeGeometry& g, int leaf_level, const std::vector<Pair>& pairs,
                                                int many_count, int degree, std::vector<TList>* clusters) {
    const int64_t nleaf = int64_t(20) << (2 * leaf_level);
    std::vector<std::vector<ASrc>> lists(nleaf);
    std::map<int64_t, size_t> cl_of;  // global face -> cluster list
    if (clusters) clusters->clear();
    for (const Pair& p : pairs) {
        const int deg = p.deg >= 0 ? p.deg : degree;
        const int many = p.deg >= 0 ? nproxy(p.deg) : many_count;
        const ASrc src = (p.far && p.ns > many) ? ASrc{1, p.ls, p.s, deg} : ASrc{0, p.ls, p.s, 0};
        if (clusters && p.far && p.nt > many) {  // fast_rhs.h cp / cc
            const int64_t gf = g.lev_off[p.lt] + p.t;
            auto it = cl_of.find(gf);
            if (it == cl_of.end()) {
                it = cl_of.emplace(gf, clusters->size()).first;
                clusters->push_back(TList{p.lt, p.t, deg, {}});
            }
            (*clusters)[it->second].src.push_back(src);
            continue;
        }
        const int64_t span = int64_t(1) << (2 * (leaf_level - p.lt));
        for (int64_t lf = p.t * span; lf < (p.t + 1) * span; lf++) lists[lf].push_back(src);
    }
    return lists;
}

std::vector<std::vector<ASrc>> lists_per_leaf(const TreeGeometry& g, int leaf_level, const std::vector<int32_t>& counts,
                                              const std::vector<int32_t>& leaf_degree,
                                              const std::vector<double>& leaf_theta, bool keep_empty) {
    const int64_t nleaf = int64_t(20) << (2 * leaf_level);
    std::vector<std::vector<ASrc>> lists(nleaf);
    struct S { int32_t l, s; };
    std::vector<S> st;
    for (int64_t lf = 0; lf < nleaf; lf++) {
        if (!keep_empty && counts[g.lev_off[leaf_level] + lf] == 0) continue;
        const int deg = leaf_degree[lf];
        const int K = nproxy(deg);
        const double th = leaf_theta[lf];
        const double* ti = &g.tri_info[4 * (g.lev_off[leaf_level] + lf)];
        st.clear();
        for (int r = 19; r >= 0; r--) st.push_back({0, r});
        while (!st.empty()) {
            const S e = st.back();
            st.pop_back();
            const int ns = counts[g.lev_off[e.l] + e.s];
            if (ns == 0) {
                if (keep_empty) lists[lf].push_back({0, e.l, e.s, 0});
                continue;
            }
            const double* si = &g.tri_info[4 * (g.lev_off[e.l] + e.s)];
            const double dist = great_circ_dist(ti, si, 1.0);
            if (dist > 0 && (ti[3] + si[3]) / dist < th) {
                lists[lf].push_back(ns > K ? ASrc{1, e.l, e.s, deg} : ASrc{0, e.l, e.s, 0});
            } else if (e.l == leaf_level) {
                lists[lf].push_back({0, e.l, e.s, 0});
            } else {
                for (int c = 3; c >= 0; c--) st.push_back({e.l + 1, 4 * e.s + c});
            }
        }
    }
    return lists;
}

void build_lists(const ListInput& in, const std::vector<std::vector<ASrc>>& lists,
                 const std::vector<TList>& clusters, ListOutput& out) {
    const TreeGeometry& g = *in.g;
    const int LL = in.leaf_level;
    const int64_t nleaf = int64_t(20) << (2 * LL);
    out = ListOutput();
    // proxy slots in first-use order
    std::map<std::pair<int64_t, int>, int64_t> slot;  // (global face, degree) -> offset
    std::map<int64_t, size_t> job_of;                 // global face -> job index
    std::map<int, std::vector<double>> node_cache;    // degree -> barycentric nodes
    // proxy slot of (face, degree), created in first-use order with its
    // upward-pass job (which writes the slot's positions and charges)
    auto need_slot = [&](int level, int node, int deg) -> int64_t {
        const int64_t gf = g.lev_off[level] + node;
        auto key = std::make_pair(gf, deg);
        auto found = slot.find(key);
        if (found != slot.end()) return found->second;
        slot[key] = out.n_proxy;
        auto it = job_of.find(gf);
        if (it == job_of.end()) {
            ProxyJob j{};
            j.level = level;
            j.node = int32_t(gf);
            j.local = node;
            const int64_t span = int64_t(1) << (2 * (LL - level));
            j.leaf_lo = int32_t(node * span);
            j.leaf_hi = int32_t((node + 1) * span);
            for (int d = 0; d < 16; d++) j.off[d] = -1;
            job_of[gf] = out.jobs.size();
            out.jobs.push_back(j);
            it = job_of.find(gf);
        }
        ProxyJob& j = out.jobs[it->second];
        j.degmask |= 1 << deg;
        j.off[deg] = int32_t(in.n + out.n_proxy);
        out.max_degree = std::max(out.max_degree, deg);
        // proxy positions: y_k = normalise(sum_m l_km v_m)
        if (!node_cache.count(deg)) {
            std::vector<double> vinv;
            interp_nodes(deg, node_cache[deg], vinv);
        }
        const std::vector<double>& nodes = node_cache[deg];
        const int K = nproxy(deg);
        const int32_t* tv = &g.tri_verts[3 * gf];
        const double* v[3] = {&g.verts[3 * int64_t(tv[0])], &g.verts[3 * int64_t(tv[1])], &g.verts[3 * int64_t(tv[2])]};
        for (int k = 0; k < K; k++) {
            double y[3];
            for (int c = 0; c < 3; c++) y[c] = nodes[3 * k] * v[0][c] + nodes[3 * k + 1] * v[1][c] + nodes[3 * k + 2] * v[2][c];
            const double nn = std::sqrt(y[0] * y[0] + y[1] * y[1] + y[2] * y[2]);
            out.proxy_pos.push_back(y[0] / nn);
            out.proxy_pos.push_back(y[1] / nn);
            out.proxy_pos.push_back(y[2] / nn);
            out.proxy_pos.push_back(0.0);
            out.proxy_node.push_back(int32_t(gf));
        }
        const int64_t off = out.n_proxy;
        out.n_proxy += K;
        return off;
    };
    for (int64_t lf = 0; lf < nleaf; lf++)
        for (const ASrc& a : lists[lf])
            if (a.proxy) need_slot(a.level, a.node, a.deg);
    for (const TList& t : clusters) {
        need_slot(t.level, t.node, t.deg);
        for (const ASrc& a : t.src)
            if (a.proxy) need_slot(a.level, a.node, a.deg);
    }
    // segments and items
    const int TB = in.threads * in.per_thread;
    const int P = std::max(1, in.parts);
    struct Cost { double cost; WorkItem it; };
    std::vector<Cost> items;
    // sources of every entry of one list for nt targets; `self_leaf` is the
    // target leaf (-1 for a target cluster); returns pp and proxy pair counts
    std::vector<double> est;
    auto count_sources = [&](const std::vector<ASrc>& list, double nt, int64_t self_leaf, double& npp, double& npc) {
        est.clear();
        npp = npc = 0;
        for (const ASrc& a : list) {
            double cnt;
            if (a.proxy) {
                cnt = nproxy(a.deg);
                npc += nt * cnt;
            } else {
                const int64_t span = int64_t(1) << (2 * (LL - a.level));
                const int32_t lo = int32_t(a.node * span), hi = int32_t((a.node + 1) * span);
                cnt = in.leaf_start[hi] - in.leaf_start[lo];
                const bool self = (self_leaf >= lo && self_leaf < hi);
                npp += nt * cnt - (self ? nt : 0);
            }
            est.push_back(cnt);
        }
    };
    // the list split into P parts of similar source counts -- cut between
    // entries of the list itself, so that the cut does not depend on which
    // proxy slots happen to be adjacent -- each part merged into segments (a
    // face's particles as a kind-0 run over its leaves, adjacent ones merged;
    // a face's proxies as a kind-1 run over its slots) and queued as one item
    auto add_items = [&](const std::vector<ASrc>& list, int32_t t0, int32_t nt_item, int32_t leaf, int nt_est) {
        double total = 0;
        for (double c : est) total += c;
        std::vector<size_t> cut(P + 1, list.size());
        cut[0] = 0;
        {
            double acc = 0;
            int p = 1;
            for (size_t k = 0; k < list.size() && p < P; k++) {
                acc += est[k];
                if (acc >= total * p / P) cut[p++] = k + 1;
            }
        }
        const int chunks = std::max(1, (nt_est + TB - 1) / TB);
        for (int p = 0; p < P; p++) {
            const int32_t base = int32_t(out.segs.size());
            double w = 0;
            for (size_t k = cut[p]; k < cut[p + 1]; k++) {
                const ASrc& a = list[k];
                const int64_t gf = g.lev_off[a.level] + a.node;
                Segment e{};
                if (a.proxy) {
                    e.kind = 1;
                    e.a = int32_t(in.n + slot[std::make_pair(gf, a.deg)]);
                    e.b = e.a + nproxy(a.deg);
                } else {
                    const int64_t span = int64_t(1) << (2 * (LL - a.level));
                    e.kind = 0;
                    e.a = int32_t(a.node * span);
                    e.b = int32_t((a.node + 1) * span);
                }
                if (int32_t(out.segs.size()) > base && out.segs.back().kind == e.kind && out.segs.back().b == e.a)
                    out.segs.back().b = e.b;
                else
                    out.segs.push_back(e);
                w += est[k];
            }
            out.n_tiles += int64_t(chunks) * (int64_t(w + in.tile - 1) / in.tile);
            // a block's run time follows its source count (its warps run
            // side by side), so the longest source lists go first
            items.push_back({w * chunks, WorkItem{t0, nt_item, base, int32_t(out.segs.size()), p, leaf}});
        }
    };
    auto flush_items = [&]() {
        std::stable_sort(items.begin(), items.end(), [](const Cost& a, const Cost& b) { return a.cost > b.cost; });
        for (auto& c : items) out.items.push_back(c.it);
        items.clear();
    };
    for (int64_t lf = 0; lf < nleaf; lf++) {
        const int32_t nt = in.leaf_start[lf + 1] - in.leaf_start[lf];
        if (lists[lf].empty() || (nt == 0 && !in.all_leaves)) continue;
        double npp, npc;
        count_sources(lists[lf], nt, lf, npp, npc);
        out.pp_pairs += npp;
        out.pc_pairs += npc;
        add_items(lists[lf], 0, 0, int32_t(lf), nt);
    }
    flush_items();
    out.n_leaf_items = int64_t(out.items.size());
    // target clusters: their interpolation points are the targets
    const int64_t nfaces = g.lev_off[LL + 1];
    std::vector<int32_t> job_of_face;
    if (!clusters.empty()) job_of_face.assign(nfaces, -1);
    for (const TList& t : clusters) {
        const int K = nproxy(t.deg);
        const int64_t gf = g.lev_off[t.level] + t.node;
        const int32_t s0 = int32_t(in.n + slot[std::make_pair(gf, t.deg)]);
        double npp, npc;
        count_sources(t.src, K, -1, npp, npc);
        out.cp_pairs += npp;
        out.cc_pairs += npc;
        add_items(t.src, s0, K, -1, K);
        job_of_face[gf] = int32_t(out.down.size());
        out.down.push_back(DownJob{t.level, int32_t(gf), t.deg, s0, int32_t(out.n_coef), {0, 0, 0}});
        out.n_coef += K;
        out.max_cluster_k = std::max(out.max_cluster_k, K);
    }
    flush_items();
    // downward pass: every leaf below a target cluster evaluates that
    // cluster's interpolant at its particles; per leaf the clusters on its
    // path to the root, coarse to fine
    if (!clusters.empty()) {
        out.leaf_anc.assign(size_t(nleaf) * kMaxLevels, LeafAnc{-1, 0, 0, 0});
        for (int64_t lf = 0; lf < nleaf; lf++) {
            int k = 0;
            for (int l = 0; l <= LL; l++) {
                const int64_t gf = g.lev_off[l] + (lf >> (2 * (LL - l)));
                const int32_t j = job_of_face[gf];
                if (j < 0) continue;
                out.leaf_anc[size_t(lf) * kMaxLevels + k++] = LeafAnc{out.down[j].coef, out.down[j].deg, int32_t(gf), 0};
            }
        }
    }
}

// ---------------------------------------------------------------- sharding

std::vector<int64_t> shard_partition(const std::vector<double>& cost_in, int nranks) {
    const int64_t U = int64_t(cost_in.size());
    std::vector<double> cost(cost_in.size());
    double total = 0, biggest = 0;
    for (int64_t i = 0; i < U; i++) {
        cost[i] = std::max(cost_in[i], 0.0);
        total += cost[i];
        biggest = std::max(biggest, cost[i]);
    }
    if (!(total > 0)) {
        std::fill(cost.begin(), cost.end(), 1.0);
        total = double(U);
        biggest = 1.0;
    }
    // ranges a greedy left-to-right fill needs when no range may exceed t
    auto greedy = [&](double t, std::vector<int64_t>* cuts) {
        int64_t ranges = 1;
        double acc = 0;
        if (cuts) cuts->assign(1, 0);
        for (int64_t i = 0; i < U; i++) {
            if (acc + cost[i] > t && acc > 0) {
                ranges++;
                acc = 0;
                if (cuts) cuts->push_back(i);
            }
            acc += cost[i];
        }
        if (cuts) cuts->push_back(U);
        return ranges;
    };
    // the least bound on a range's cost that nranks ranges can meet
    double lo = std::max(biggest, total / nranks), hi = total;
    for (int it = 0; it < 100 && hi - lo > 1e-12 * total; it++) {
        const double mid = 0.5 * (lo + hi);
        if (greedy(mid, nullptr) <= nranks) hi = mid; else lo = mid;
    }
    std::vector<int64_t> b;
    greedy(hi, &b);
    // fewer ranges than ranks: split the costliest range of two or more units
    // at its cost midpoint until every rank has one (when units allow)
    while (int64_t(b.size()) - 1 < nranks) {
        int best = -1;
        double best_cost = -1;
        for (size_t r = 0; r + 1 < b.size(); r++) {
            if (b[r + 1] - b[r] < 2) continue;
            double c = 0;
            for (int64_t i = b[r]; i < b[r + 1]; i++) c += cost[i];
            if (c > best_cost) {
                best_cost = c;
                best = int(r);
            }
        }
        if (best < 0) {  // fewer units than ranks: empty ranges at the end
            while (int64_t(b.size()) - 1 < nranks) b.push_back(U);
            break;
        }
        double acc = 0;
        int64_t k = b[best] + 1;
        for (int64_t i = b[best]; i < b[best + 1] - 1; i++) {
            acc += cost[i];
            k = i + 1;
            if (acc >= 0.5 * best_cost) break;
        }
        b.insert(b.begin() + best + 1, k);
    }
    return b;
}

// ---------------------------------------------------------------- interpolation

void interp_nodes(int n, std::vector<double>& nodes, std::vector<double>& vinv) {
    const int K = nproxy(n);
    nodes.assign(3 * K, 0.0);
    if (n == 0) {
        nodes[0] = nodes[1] = nodes[2] = 1.0 / 3.0;
        vinv.assign(1, 1.0);
        return;
    }
    std::vector<double> v(n + 1);
    for (int m = 0; m <= n; m++) v[m] = 0.5 * (1.0 - std::cos(M_PI * m / n));
    int k = 0;
    for (int i = 0; i <= n; i++)
        for (int j = 0; j <= n - i; j++, k++) {
            const int l = n - i - j;
            nodes[3 * k] = (1 + 2 * v[i] - v[j] - v[l]) / 3.0;
            nodes[3 * k + 1] = (1 + 2 * v[j] - v[i] - v[l]) / 3.0;
            nodes[3 * k + 2] = 1.0 - nodes[3 * k] - nodes[3 * k + 1];
        }
    // Vandermonde V[k][m], basis m <-> (a, b): degree g = a + b, m = g(g+1)/2 + b
    std::vector<double> V(size_t(K) * K);
    std::vector<double> Ta(n + 1), Tb(n + 1);
    for (int q = 0; q < K; q++) {
        const double x = 2 * nodes[3 * q] - 1, y = 2 * nodes[3 * q + 1] - 1;
        Ta[0] = 1; Tb[0] = 1;
        if (n >= 1) { Ta[1] = x; Tb[1] = y; }
        for (int a = 2; a <= n; a++) { Ta[a] = 2 * x * Ta[a - 1] - Ta[a - 2]; Tb[a] = 2 * y * Tb[a - 1] - Tb[a - 2]; }
        for (int gdeg = 0, m = 0; gdeg <= n; gdeg++)
            for (int b = 0; b <= gdeg; b++, m++) V[size_t(q) * K + m] = Ta[gdeg - b] * Tb[b];
    }
    // Gauss-Jordan inverse with partial pivoting
    std::vector<double> A(V), I(size_t(K) * K, 0.0);
    for (int i = 0; i < K; i++) I[size_t(i) * K + i] = 1;
    for (int c = 0; c < K; c++) {
        int p = c;
        for (int r = c + 1; r < K; r++)
            if (std::fabs(A[size_t(r) * K + c]) > std::fabs(A[size_t(p) * K + c])) p = r;
        if (A[size_t(p) * K + c] == 0.0) throw std::runtime_error("singular interpolation matrix");
        if (p != c)
            for (int j = 0; j < K; j++) {
                std::swap(A[size_t(p) * K + j], A[size_t(c) * K + j]);
                std::swap(I[size_t(p) * K + j], I[size_t(c) * K + j]);
            }
        const double inv = 1.0 / A[size_t(c) * K + c];
        for (int j = 0; j < K; j++) { A[size_t(c) * K + j] *= inv; I[size_t(c) * K + j] *= inv; }
        for (int r = 0; r < K; r++) {
            if (r == c) continue;
            const double f = A[size_t(r) * K + c];
            if (f == 0.0) continue;
            for (int j = 0; j < K; j++) {
                A[size_t(r) * K + j] -= f * A[size_t(c) * K + j];
                I[size_t(r) * K + j] -= f * I[size_t(c) * K + j];
            }
        }
    }
    // I = V^{-1}: I[m][k]; l_k(x) = sum_m I[m][k] phi_m(x)
    vinv = I;
}

}  // namespace fss
