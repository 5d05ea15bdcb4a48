// selector.cpp -- learned per-leaf interpolation degree and MAC.
//
// For every target leaf the selector chooses one of 12 classes c = 3 i + j,
//   target-leaf evaluation: (n, theta) in {4, 6, 8, 10} x {0.5, 0.6, 0.7}  (n = 4 + 2i, theta = 0.5 + 0.1 j),
//   target clusters:        (n, theta) in {6, 8, 10, 12} x {0.7, 0.8, 0.9}  (n = 6 + 2i, theta = 0.7 + 0.1 j)
// (with target clusters a face takes the most accurate choice of its
// leaves and interpolates at both ends, so its useful range sits higher),
// so that the relative L2 velocity error stays below a tolerance at least
// interaction count.  A target leaf's velocity error depends only on its own
// class (its far clusters and their degree-n proxies), and squared errors
// add over leaves, so with e_l(c) the error of leaf l the constraint is
//   sum_l e_l(c_l)^2 <= tol^2 ||u||^2.
// The network predicts y_l(c) = log10(e_l(c) / U) with U the RMS speed
// (from 16 leaf features: geometry, charge statistics and far-field
// statistics of the leaf's theta = 0.7 interaction list); the costs cost_l(c)
// are exact interaction counts from one traversal per theta (per class, with
// target clusters, whose work is shared among their leaves).  The choice
// minimises sum cost + mu sum 10^(2y) leaf by leaf, with mu set by bisection
// so that the predicted budget sum_l 10^(2 y_l) <= (tol / safety)^2 N holds.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "ctx.h"
#include "fss.h"
#include "geometry.h"
#include "traverse.h"

namespace fss {

int internal_relist(fss_ctx* c);                                 // fss.cpp
int internal_rhs_current(fss_ctx* c, std::vector<double>& out5);  // fss.cpp
void set_last_error(const std::string& msg);

constexpr int kClasses = 12;
constexpr int kFeatures = 16;
inline int class_degree(int c, bool clusters) { return (clusters ? 6 : 4) + 2 * (c / 3); }
inline double class_theta(int c, bool clusters) { return (clusters ? 0.7 : 0.5) + 0.1 * (c % 3); }
constexpr double kFeatureTheta = 0.7;  // far-field features come from this traversal

struct ThetaLists {
    std::vector<int64_t> near;               // near-field particles per leaf
    std::vector<std::vector<int32_t>> far;   // far source faces (global index) per leaf
};

// Per-leaf traversal with one theta: well-separated faces are far, leaves
// that are not are near (the same acceptance as lists_per_leaf).
static ThetaLists traverse_theta(const TreeGeometry& g, int LL, const std::vector<int32_t>& counts, double theta) {
    const int64_t nleaf = int64_t(20) << (2 * LL);
    ThetaLists out;
    out.near.assign(nleaf, 0);
    out.far.assign(nleaf, {});
    struct S { int32_t l, s; };
    std::vector<S> st;
    for (int64_t lf = 0; lf < nleaf; lf++) {
        if (counts[g.lev_off[LL] + lf] == 0) continue;
        const double* ti = &g.tri_info[4 * (g.lev_off[LL] + lf)];
        st.clear();
        for (int r = 19; r >= 0; r--) st.push_back({0, r});
        while (!st.empty()) {
            const S e = st.back();
            st.pop_back();
            const int64_t gf = g.lev_off[e.l] + e.s;
            const int ns = counts[gf];
            if (ns == 0) continue;
            const double* si = &g.tri_info[4 * gf];
            const double dist = great_circ_dist(ti, si, 1.0);
            if (dist > 0 && (ti[3] + si[3]) / dist < theta) {
                out.far[lf].push_back(int32_t(gf));
            } else if (e.l == LL) {
                out.near[lf] += ns;
            } else {
                for (int c = 3; c >= 0; c--) st.push_back({e.l + 1, 4 * e.s + c});
            }
        }
    }
    return out;
}

// Lagrangian choice: per leaf argmin cost + mu * 10^(2y); mu by bisection so
// that sum 10^(2y) <= budget (or the least-error choice where unattainable).
static void select(int64_t nleaf, int ncls, const double* y, const double* cost, double budget, int32_t* choice) {
    std::vector<double> E(size_t(nleaf) * ncls);
    for (size_t i = 0; i < E.size(); i++) E[i] = std::pow(10.0, 2 * y[i]);
    auto pick = [&](double mu, double* total) {
        double tot = 0;
        for (int64_t l = 0; l < nleaf; l++) {
            int best = 0;
            double bv = 1e300;
            for (int k = 0; k < ncls; k++) {
                const double v = cost[l * ncls + k] + mu * E[l * ncls + k];
                if (v < bv) { bv = v; best = k; }
            }
            choice[l] = best;
            tot += E[l * ncls + best];
        }
        *total = tot;
    };
    double lo = -40, hi = 60, tot = 0;
    pick(std::pow(10.0, hi), &tot);
    if (tot > budget) return;  // cannot be met: least-error choices stay
    for (int it = 0; it < 80; it++) {
        const double mid = 0.5 * (lo + hi);
        pick(std::pow(10.0, mid), &tot);
        if (tot <= budget) hi = mid; else lo = mid;
    }
    pick(std::pow(10.0, hi), &tot);
    // Spend the slack the relaxation leaves: repeatedly take the move to a
    // cheaper class with the largest saving that still fits the budget.
    for (;;) {
        double best_save = 0, best_de = 0;
        int64_t bl = -1;
        int bk = -1;
        for (int64_t l = 0; l < nleaf; l++) {
            const int cur = choice[l];
            const double ecur = E[l * ncls + cur];
            for (int k = 0; k < ncls; k++) {
                const double save = cost[l * ncls + cur] - cost[l * ncls + k];
                if (save <= best_save) continue;
                const double de = E[l * ncls + k] - ecur;
                if (tot + de <= budget) { best_save = save; best_de = de; bl = l; bk = k; }
            }
        }
        if (bl < 0) break;
        choice[bl] = bk;
        tot += best_de;
    }
}

// Features (16 per leaf) and exact per-class costs (12 per leaf).
static int features_and_costs(fss_ctx* c, std::vector<float>& feat, std::vector<double>& cost, double* u_rms) {
    const int LL = c->leaf_level;
    const int64_t nleaf = c->nleaf, n = c->n;
    const TreeGeometry& g = c->geom;
    // RMS speed from one right-hand side with the current lists (this also
    // brings the stage state up to date)
    std::vector<double> u5;
    int rc = internal_rhs_current(c, u5);
    if (rc) return rc;
    double u2 = 0;
    for (int64_t i = 0; i < n; i++) u2 += u5[5 * i] * u5[5 * i] + u5[5 * i + 1] * u5[5 * i + 1] + u5[5 * i + 2] * u5[5 * i + 2];
    const double U = std::sqrt(u2 / double(std::max<int64_t>(n, 1)));
    if (u_rms) *u_rms = U;
    // charges in leaf order
    std::vector<double4> xs(n);
    std::vector<double> area(n);
    if (cudaMemcpyAsync(xs.data(), c->xs.p, sizeof(double4) * n, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
        cudaMemcpyAsync(area.data(), c->area_s.p, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
        cudaStreamSynchronize(c->stream) != cudaSuccess) {
        cudaGetLastError();
        return FSS_ERR_CUDA;
    }
    std::vector<double> labs(nleaf, 0), lsum(nleaf, 0), lmax(nleaf, 0);
    double Wabs = 0;
    for (int64_t l = 0; l < nleaf; l++)
        for (int32_t s = c->leaf_start_h[l]; s < c->leaf_start_h[l + 1]; s++) {
            const double w = xs[s].w * area[s];
            labs[l] += std::fabs(w);
            lsum[l] += w;
            lmax[l] = std::max(lmax[l], std::fabs(w));
            Wabs += std::fabs(w);
        }
    if (!(Wabs > 0)) Wabs = 1e-300;
    // |Q| per face on every level (faces cover leaf ranges)
    const int64_t nfaces = g.lev_off[LL + 1];
    std::vector<double> qabs(nfaces, 0);
    for (int l = 0; l <= LL; l++) {
        const int64_t span = int64_t(1) << (2 * (LL - l));
        for (int64_t f = 0; f < g.level_count(l); f++) {
            double q = 0;
            for (int64_t k = f * span; k < (f + 1) * span; k++) q += labs[k];
            qabs[g.lev_off[l] + f] = q;
        }
    }
    // costs per class: exact interaction counts of each class used everywhere
    cost.assign(size_t(nleaf) * kClasses, 0);
    ThetaLists t07 = traverse_theta(g, LL, c->counts_h, kFeatureTheta);
    const bool clusters = c->cfg.cluster_targets != 0;
    if (clusters) {
        // dual traversal per class; a target cluster's work (its
        // interpolation points against its sources) is shared among its
        // leaves by particle count
        for (int k = 0; k < kClasses; k++) {
            const int K = nproxy(class_degree(k, true));
            const std::vector<Pair> pairs = dual_traverse(g, c->counts_h, class_theta(k, true), K);
            for (const Pair& p : pairs) {
                const int64_t span = int64_t(1) << (2 * (LL - p.lt));
                const bool cl = p.far && p.nt > K;
                const double per_src = (p.far && p.ns > K) ? K : p.ns;
                for (int64_t lf = p.t * span; lf < (p.t + 1) * span; lf++) {
                    const double nl = c->leaf_start_h[lf + 1] - c->leaf_start_h[lf];
                    cost[size_t(lf) * kClasses + k] += cl ? double(K) * per_src * nl / double(p.nt) : nl * per_src;
                }
            }
        }
    } else {
        for (int j = 0; j < 3; j++) {
            const double th = class_theta(j, false);
            const ThetaLists tl = (th == kFeatureTheta) ? ThetaLists() : traverse_theta(g, LL, c->counts_h, th);
            const ThetaLists& t = (th == kFeatureTheta) ? t07 : tl;
            for (int64_t l = 0; l < nleaf; l++) {
                const double nt = c->leaf_start_h[l + 1] - c->leaf_start_h[l];
                for (int i = 0; i < 4; i++) {
                    const int K = nproxy(class_degree(3 * i, false));
                    double s = double(t.near[l]);
                    for (int32_t gf : t.far[l]) s += std::min<double>(K, c->counts_h[gf]);
                    cost[size_t(l) * kClasses + 3 * i + j] = nt * s;
                }
            }
        }
    }
    // features
    feat.assign(size_t(nleaf) * kFeatures, 0.f);
    double rmean = 0;
    for (int64_t l = 0; l < nleaf; l++) rmean += g.tri_info[4 * (g.lev_off[LL] + l) + 3];
    rmean /= double(nleaf);
    const double navg = double(n) / double(nleaf);
    auto lg = [](double x) { return float(std::log10(x + 1e-30)); };
    for (int64_t l = 0; l < nleaf; l++) {
        float* f = &feat[size_t(l) * kFeatures];
        const double* ti = &g.tri_info[4 * (g.lev_off[LL] + l)];
        const double nt = c->leaf_start_h[l + 1] - c->leaf_start_h[l];
        f[0] = float(ti[0]); f[1] = float(ti[1]); f[2] = float(ti[2]);
        f[3] = float(std::log10(ti[3] / rmean));
        f[4] = float(nt / navg);
        f[5] = lg(labs[l] / (Wabs / double(nleaf)));
        f[6] = lg(lmax[l] / (Wabs / double(n)));
        f[7] = float(lsum[l] / (labs[l] + 1e-300));
        double s1 = 0, s5 = 0, s7 = 0, s9 = 0, s11 = 0;
        for (int32_t gf : t07.far[l]) {
            const double* si = &g.tri_info[4 * gf];
            const double d = great_circ_dist(ti, si, 1.0), r = si[3] / d;
            const double q = qabs[gf] / Wabs / d;
            const double r2 = r * r, r4 = r2 * r2, r5 = r4 * r;
            s1 += q; s5 += q * r5; s7 += q * r5 * r2; s9 += q * r5 * r4; s11 += q * r5 * r4 * r2;
        }
        f[8] = lg(s1); f[9] = lg(s5); f[10] = lg(s7); f[11] = lg(s9); f[12] = lg(s11);
        f[13] = float(double(t07.far[l].size()) / 100.0);
        f[14] = float(double(t07.near[l]) / 2000.0);
        f[15] = lg(U / Wabs);
    }
    return FSS_OK;
}

}  // namespace fss

using namespace fss;

extern "C" {

int fss_selector_features(fss_ctx* c, float* features, double* costs, double* u_rms) {
    if (!c || !c->have || !c->tree) {
        set_last_error("fss_selector_features: needs a treecode context with particles");
        return FSS_ERR_STATE;
    }
    if (cudaSetDevice(c->dev) != cudaSuccess) return FSS_ERR_CUDA;
    std::vector<float> f;
    std::vector<double> k;
    int rc = features_and_costs(c, f, k, u_rms);
    if (rc) return rc;
    if (features) std::memcpy(features, f.data(), sizeof(float) * f.size());
    if (costs) std::memcpy(costs, k.data(), sizeof(double) * k.size());
    return FSS_OK;
}

int fss_selector_class_table(int32_t clusters, int32_t* degree, double* theta) {
    if (!degree || !theta) {
        set_last_error("fss_selector_class_table: null argument");
        return FSS_ERR_INVALID;
    }
    for (int k = 0; k < kClasses; k++) {
        degree[k] = class_degree(k, clusters != 0);
        theta[k] = class_theta(k, clusters != 0);
    }
    return FSS_OK;
}

int fss_select_classes(int64_t nleaf, int32_t nclass, const double* pred_log_err, const double* cost, double budget,
                       int32_t* choice) {
    if (nleaf < 0 || nclass <= 0 || !pred_log_err || !cost || !choice) {
        set_last_error("fss_select_classes: bad argument");
        return FSS_ERR_INVALID;
    }
    select(nleaf, nclass, pred_log_err, cost, budget, choice);
    return FSS_OK;
}

int fss_selector_apply(fss_ctx* c, fss_mlp* m, const float* feat_mean, const float* feat_std, double tol,
                       double safety, int32_t* choice_out) {
    if (!c || !m || !feat_mean || !feat_std || !(tol > 0) || !(safety > 0)) {
        set_last_error("fss_selector_apply: bad argument");
        return FSS_ERR_INVALID;
    }
    if (!c->have || !c->tree) {
        set_last_error("fss_selector_apply: needs a treecode context with particles");
        return FSS_ERR_STATE;
    }
    std::vector<float> f;
    std::vector<double> k;
    double U = 0;
    int rc = features_and_costs(c, f, k, &U);
    if (rc) return rc;
    const int64_t nleaf = c->nleaf;
    for (int64_t l = 0; l < nleaf; l++)
        for (int j = 0; j < kFeatures; j++) {
            float& v = f[size_t(l) * kFeatures + j];
            v = (v - feat_mean[j]) / (feat_std[j] > 0 ? feat_std[j] : 1.f);
        }
    std::vector<float> y(size_t(nleaf) * kClasses);
    rc = fss_mlp_predict(m, nleaf, f.data(), y.data());
    if (rc) return rc;
    std::vector<double> yd(y.begin(), y.end());
    std::vector<int32_t> choice(nleaf, 0);
    const double budget = (tol / safety) * (tol / safety) * double(c->n);
    select(nleaf, kClasses, yd.data(), k.data(), budget, choice.data());
    const bool clusters = c->cfg.cluster_targets != 0;
    for (int64_t l = 0; l < nleaf; l++) {
        c->leaf_deg[l] = class_degree(choice[l], clusters);
        c->leaf_theta[l] = class_theta(choice[l], clusters);
    }
    if (choice_out) std::memcpy(choice_out, choice.data(), sizeof(int32_t) * nleaf);
    c->cfg.list_mode = FSS_LIST_LEAF;  // with cluster_targets: per-face dual traversal
    return internal_relist(c);
}

}  // extern "C"
