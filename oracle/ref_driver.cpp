// ref_driver.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Thin extern "C" driver around the reference's own hot-path headers
// (cygnari/fast-sphere-sum Old-BVE-code/*.h), compiled from the reference's
// sources in place by oracle/Makefile into oracle/_ref/libref.so.  Nothing
// of the reference is copied here: this file includes its headers and calls
// its functions.  Used by tests (bit-exact pins of the oracle) and by the
// CPU baseline of the benchmark.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <thread>
#include <vector>
#include <unistd.h>

#include "helpers.h"
#include "struct_list.h"
#include "vorticity_functions.h"
#include "rhs_eval.h"
#include "icos_utils.h"
#include "fast_rhs.h"
#include "interp_utils.h"
#include "remesh.h"
#include "amr.h"

using std::vector;

static vector<double> to_state(int64_t n, const double* s5) { return vector<double>(s5, s5 + 5 * n); }

extern "C" {

// icos_utils.h:15 icos_init.  Outputs as in oracle/fss_oracle.c orc_icos_init.
int64_t ref_icos_init(int levels, double radius, double* verts, int* tri_verts, double* tri_info) {
    run_information c;
    icos_init(c, levels, radius);
    for (size_t i = 0; i < c.tree_verts.size(); i++)
        for (int k = 0; k < 3; k++) verts[3 * i + k] = c.tree_verts[i][k];
    int64_t f = 0;
    for (size_t l = 0; l < c.tree_tri_verts.size(); l++)
        for (size_t j = 0; j < c.tree_tri_verts[l].size(); j++, f++)
            for (int k = 0; k < 3; k++) {
                tri_verts[3 * f + k] = c.tree_tri_verts[l][j][k];
                if (tri_info) tri_info[4 * f + k] = c.tree_tri_info[l][j][k];
                if (tri_info && k == 2) tri_info[4 * f + 3] = c.tree_tri_info[l][j][3];
            }
    return (int64_t)c.tree_verts.size();
}

// helpers.h:344 area_init
void ref_area_init(int64_t n, const double* state5, int64_t ntri, const int* tris, double* area) {
    vector<double> s = to_state(n, state5), a(n, 0.0);
    vector<vector<int>> t(ntri, vector<int>(3));
    for (int64_t i = 0; i < ntri; i++)
        for (int k = 0; k < 3; k++) t[i][k] = tris[3 * i + k];
    area_init(s, a, t, (int)ntri);
    std::memcpy(area, a.data(), sizeof(double) * n);
}

// vorticity_functions.h:13 rossby_haurwitz_4
void ref_rossby_haurwitz_4(int64_t n, double* state5) {
    vector<double> s = to_state(n, state5);
    rossby_haurwitz_4(s, (int)n);
    std::memcpy(state5, s.data(), sizeof(double) * 5 * n);
}

// vorticity_functions.h:26 gauss_vortex
void ref_gauss_vortex(int64_t n, double* state5, const double* area) {
    vector<double> s = to_state(n, state5), a(area, area + n);
    gauss_vortex(s, a, (int)n);
    std::memcpy(state5, s.data(), sizeof(double) * 5 * n);
}

// rhs_eval.h:47 rhs_func with use_fast == false (direct sum).
void ref_rhs_func_direct(int64_t n, const double* state5, const double* area, double omega,
                         double* modify5) {
    run_information c;
    c.point_count = (int)n;
    c.use_fast = false;
    vector<double> s = to_state(n, state5), a(area, area + n), m(5 * n, 0.0);
    rhs_func(m, s, a, omega, c);
    std::memcpy(modify5, m.data(), sizeof(double) * 5 * n);
}

// The loop of rhs_eval.h:15-32 rhs_direct_sum restricted to a set of target
// rows (the row-range form the reference's MPI program uses,
// direct_sum_mpi.cpp:18-55), built on the reference's own BVE_gfunc, slice,
// scalar_mult and vec_add, and scaled by -1/(4 pi) as rhs_func does.
// Rows are split over `threads` OS threads.
void ref_rhs_direct_rows(int64_t n, const double* state5, const double* area, int64_t nrows,
                         const int64_t* rows, double* out3, int threads) {
    vector<double> s = to_state(n, state5);
    vector<double> a(area, area + n);
    if (threads < 1) threads = 1;
    auto work = [&](int64_t lo, int64_t hi) {
        vector<double> pos_change, particle_i, particle_j, contribution;
        for (int64_t r = lo; r < hi; r++) {
            int64_t i = rows ? rows[r] : r;
            pos_change = {0, 0, 0};
            particle_i = slice(s, 5 * (int)i, 1, 3);
            for (int64_t j = 0; j < n; j++) {
                if (i != j) {
                    particle_j = slice(s, 5 * (int)j, 1, 3);
                    contribution = BVE_gfunc(particle_i, particle_j);
                    scalar_mult(contribution, s[5 * j + 3] * a[j]);
                    vec_add(pos_change, contribution);
                }
            }
            scalar_mult(pos_change, -1.0 / (4.0 * M_PI));
            for (int k = 0; k < 3; k++) out3[3 * r + k] = pos_change[k];
        }
    };
    if (threads == 1) { work(0, nrows); return; }
    vector<std::thread> th;
    for (int t = 0; t < threads; t++)
        th.emplace_back(work, nrows * t / threads, nrows * (t + 1) / threads);
    for (auto& x : th) x.join();
}

// helpers.h:362 project_points
void ref_project_points(int64_t n, double* state5, double omega) {
    vector<double> s = to_state(n, state5);
    project_points(s, (int)n, omega);
    std::memcpy(state5, s.data(), sizeof(double) * 5 * n);
}

// One RK4 step in the order of new_dynamics.cpp:281-340 (the loop as it is
// meant to run: its stage buffers intermediate_1..3 and c_1..c_4 are only
// commented-out declarations there), built from the reference's rhs_func,
// scalar_mult, vec_add and project_points with the direct sum.
void ref_rk4_step(int64_t n, double* state5, const double* area, double omega, double dt) {
    run_information c;
    c.point_count = (int)n;
    c.use_fast = false;
    vector<double> s = to_state(n, state5), a(area, area + n);
    vector<double> c_1(5 * n), c_2(5 * n), c_3(5 * n), c_4(5 * n), c1234;
    vector<double> intermediate_1, intermediate_2, intermediate_3;
    rhs_func(c_1, s, a, omega, c);
    intermediate_1 = c_1;
    scalar_mult(intermediate_1, dt / 2);
    vec_add(intermediate_1, s);
    project_points(intermediate_1, (int)n, omega);
    rhs_func(c_2, intermediate_1, a, omega, c);
    intermediate_2 = c_2;
    scalar_mult(intermediate_2, dt / 2);
    vec_add(intermediate_2, s);
    project_points(intermediate_2, (int)n, omega);
    rhs_func(c_3, intermediate_2, a, omega, c);
    intermediate_3 = c_3;
    scalar_mult(intermediate_3, dt);
    vec_add(intermediate_3, s);
    project_points(intermediate_3, (int)n, omega);
    rhs_func(c_4, intermediate_3, a, omega, c);
    c1234 = c_1;
    scalar_mult(c_2, 2);
    vec_add(c1234, c_2);
    scalar_mult(c_3, 2);
    vec_add(c1234, c_3);
    vec_add(c1234, c_4);
    scalar_mult(c1234, dt / 6);
    vec_add(s, c1234);
    project_points(s, (int)n, omega);
    std::memcpy(state5, s.data(), sizeof(double) * 5 * n);
}

// icos_utils.h:135 icosahedron_init + :172 points_assign + fast_rhs.h:16
// tree_traverse.  loc[l*n+i] = face holding particle i on level l or -1;
// counts = faces' member counts (levels concatenated); pairs = 7 ints per
// interaction (lev_t, lev_s, t, s, n_t, n_s, type 0 pp / 1 pc / 2 cp / 3 cc).
// Returns the number of interactions (or -needed if pairs_cap is short).
int64_t ref_tree(int tree_levels, double theta, int many_count, int64_t n, const double* state5,
                 int* loc, int* counts, int* pairs, int64_t pairs_cap) {
    run_information c;
    c.point_count = (int)n;
    c.tree_levels = tree_levels;
    c.theta = theta;
    c.many_count = many_count;
    icosahedron_init(c, 1.0);
    vector<double> s = to_state(n, state5);
    points_assign(c, s);
    tree_traverse(c);
    int64_t f = 0;
    for (int l = 0; l < tree_levels; l++) {
        for (int64_t i = 0; i < n; i++) loc[l * n + i] = -1;
        for (size_t j = 0; j < c.tree_tri_points[l].size(); j++, f++) {
            counts[f] = (int)c.tree_tri_points[l][j].size();
            for (int id : c.tree_tri_points[l][j]) loc[l * n + id] = (int)j;
        }
    }
    int64_t np = (int64_t)c.tree_interactions.size();
    if (np > pairs_cap) return -np;
    for (int64_t i = 0; i < np; i++) {
        const interaction_pair& p = c.tree_interactions[i];
        int ty = (p.type[0] == 'c' ? 2 : 0) + (p.type[1] == 'c' ? 1 : 0);
        int* r = pairs + 7 * i;
        r[0] = p.lev_target; r[1] = p.lev_source; r[2] = p.curr_target; r[3] = p.curr_source;
        r[4] = p.count_target; r[5] = p.count_source; r[6] = ty;
    }
    return np;
}

// Ordered member list of one face (for membership comparisons).
int64_t ref_tree_members(int tree_levels, int64_t n, const double* state5, int level, int face,
                         int* out, int64_t cap) {
    run_information c;
    c.point_count = (int)n;
    c.tree_levels = tree_levels;
    icosahedron_init(c, 1.0);
    vector<double> s = to_state(n, state5);
    points_assign(c, s);
    const vector<int>& m = c.tree_tri_points[level][face];
    for (size_t i = 0; i < m.size() && (int64_t)i < cap; i++) out[i] = m[i];
    return (int64_t)m.size();
}

// The reference's fast sum end to end (interp_utils.h:61 interp_init,
// points_assign, tree_traverse, rhs_func with use_fast): its only working
// setting is degree 2.  Returns dgetrf's info for the interpolation matrix.
int ref_rhs_fast(int64_t n, const double* state5, const double* area, double omega, int tree_levels,
                 double theta, int many_count, int degree, double* modify5) {
    run_information c;
    c.point_count = (int)n;
    c.tree_levels = tree_levels;
    c.theta = theta;
    c.many_count = many_count;
    c.degree = degree;
    icosahedron_init(c, 1.0);
    interp_init(c);
    vector<double> s = to_state(n, state5), a(area, area + n), m(5 * n, 0.0);
    points_assign(c, s);
    tree_traverse(c);
    c.use_fast = true;
    rhs_func(m, s, a, omega, c);
    std::memcpy(modify5, m.data(), sizeof(double) * 5 * n);
    return c.info;
}

// The reference's fast sum with its set-up and its evaluation timed apart
// (set-up: icosahedron_init, interp_init, points_assign, tree_traverse, as
// new_dynamics.cpp:87-88 runs once before the time loop; evaluation: what
// rhs_func does per call), after one set-up: the evaluation on one thread
// (rhs_func itself, into modify1), and, when modifyp is given, split over
// `threads` threads the way fast_sum_mpi.cpp:324-338 splits it over MPI
// ranks: rank r owns the top-level target faces [r * (20 / P), (r + 1) *
// (20 / P)), the last rank the rest, and evaluates the interactions whose
// target face descends from its own.  Here the ranks are threads with
// private modify buffers, summed afterwards (every target gets its
// contributions from one thread only, in the single-thread order), then
// scaled as rhs_func scales.  times[0] = set-up s, times[1] = one-thread
// evaluation s, times[2] = split evaluation s.  Returns dgetrf's info.
int ref_rhs_fast_timed(int64_t n, const double* state5, const double* area, double omega, int tree_levels,
                       double theta, int many_count, int degree, int threads, double* modify1, double* modifyp,
                       double* times) {
    using clk = std::chrono::steady_clock;
    auto secs = [](clk::time_point a, clk::time_point b) { return std::chrono::duration<double>(b - a).count(); };
    if (threads < 1) threads = 1;
    if (threads > 20) threads = 20;
    vector<double> s = to_state(n, state5), a(area, area + n), m(5 * n, 0.0);
    run_information c;
    c.point_count = (int)n;
    c.tree_levels = tree_levels;
    c.theta = theta;
    c.many_count = many_count;
    c.degree = degree;
    c.use_fast = true;
    const auto t0 = clk::now();
    icosahedron_init(c, 1.0);
    interp_init(c);
    points_assign(c, s);
    tree_traverse(c);
    const auto t1 = clk::now();
    rhs_func(m, s, a, omega, c);
    const auto t2 = clk::now();
    std::memcpy(modify1, m.data(), sizeof(double) * 5 * n);
    double t_split = 0.0;
    if (modifyp) {
        // per-thread copies of the configuration, each with its share of the
        // interactions (made before the timed evaluation)
        const int per = 20 / threads;
        vector<run_information> part(threads, c);
        for (auto& p : part) p.tree_interactions.clear();
        for (const interaction_pair& ip : c.tree_interactions) {
            const int top = ip.curr_target >> (2 * ip.lev_target);
            part[std::min(top / per, threads - 1)].tree_interactions.push_back(ip);
        }
        vector<vector<double>> mt(threads, vector<double>(5 * n, 0.0));
        const auto t3 = clk::now();
        vector<std::thread> th;
        for (int r = 0; r < threads; r++)
            th.emplace_back([&, r] { rhs_fast_sum(mt[r], s, a, part[r], omega); });
        for (auto& x : th) x.join();
        std::fill(m.begin(), m.end(), 0.0);
        for (int r = 0; r < threads; r++)
            for (int64_t k = 0; k < 5 * n; k++) m[k] += mt[r][k];
        scalar_mult(m, -1.0 / (4.0 * M_PI));
        for (int64_t i = 0; i < n; i++) m[5 * i + 3] = -2 * omega * m[5 * i + 2];
        t_split = secs(t3, clk::now());
        std::memcpy(modifyp, m.data(), sizeof(double) * 5 * n);
    }
    if (times) {
        times[0] = secs(t0, t1);
        times[1] = secs(t1, t2);
        times[2] = t_split;
    }
    return c.info;
}

// remesh.h:109-178 regrid_points2 on the reference's own code, with the
// vertex -> triangles adjacency built from `tris` in increasing index order
// (the reference reads it from a CSV file it does not contain).  Returns 0,
// or -1 when a target lies in no triangle (the reference throws).  Only
// targets lb <= i < ub are regridded (the reference's own lb/ub arguments).
int ref_regrid_range(int64_t n, const double* moved5, double* target5, int64_t ntri, const int* tris, double omega,
                     int64_t lb, int64_t ub) {
    vector<double> moved(moved5, moved5 + 5 * n), target(target5, target5 + 5 * n);
    vector<vector<int>> triangles(ntri, vector<int>(3)), vert_tris(n);
    for (int64_t j = 0; j < ntri; j++)
        for (int k = 0; k < 3; k++) {
            triangles[j][k] = tris[3 * j + k];
            vert_tris[tris[3 * j + k]].push_back(int(j));
        }
    std::streambuf* old = std::cout.rdbuf(nullptr);  // the reference prints its counts
    int rc = 0;
    try {
        regrid_points2(moved, target, triangles, vert_tris, int(n), int(ntri), omega, int(lb), int(ub), 0);
    } catch (...) {
        rc = -1;
    }
    std::cout.rdbuf(old);
    std::memcpy(target5, target.data(), sizeof(double) * 5 * n);
    return rc;
}

// regrid_points2 with explicit vert_tris lists (CSR), e.g. those amr() kept.
int ref_regrid_csr(int64_t n, const double* moved5, double* target5, int64_t ntri, const int* tris, const int* vt_off,
                   const int* vt_adj, double omega) {
    vector<double> moved(moved5, moved5 + 5 * n), target(target5, target5 + 5 * n);
    vector<vector<int>> triangles(ntri, vector<int>(3)), vert_tris(n);
    for (int64_t j = 0; j < ntri; j++)
        for (int k = 0; k < 3; k++) triangles[j][k] = tris[3 * j + k];
    for (int64_t i = 0; i < n; i++) vert_tris[i].assign(vt_adj + vt_off[i], vt_adj + vt_off[i + 1]);
    std::streambuf* old = std::cout.rdbuf(nullptr);
    int rc = 0;
    try {
        regrid_points2(moved, target, triangles, vert_tris, int(n), int(ntri), omega, 0, int(n), 0);
    } catch (...) {
        rc = -1;
    }
    std::cout.rdbuf(old);
    std::memcpy(target5, target.data(), sizeof(double) * 5 * n);
    return rc;
}

int ref_regrid(int64_t n, const double* moved5, double* target5, int64_t ntri, const int* tris, double omega) {
    return ref_regrid_range(n, moved5, target5, ntri, tris, omega, 0, n);
}

// helpers.h:299 read_points itself: it opens ../<N>points_rh4.csv,
// ../<N>tris.csv, ../<N>vert_tris.csv and ../<N>vert_tri_count.csv relative
// to the working directory, so it runs from `run_dir` (a directory below
// the files) and the working directory is restored after.  Outputs: state
// (x, y, z, zeta; tracer 0), triangles, vert_tris as CSR.
int ref_read_points(const char* run_dir, int64_t n, int64_t ntri, double* state5, int* tris, int* vt_off, int* vt_adj,
                    int64_t cap) {
    char cwd[4096];
    if (!getcwd(cwd, sizeof(cwd)) || chdir(run_dir) != 0) return -1;
    run_information config1;
    config1.point_count = int(n);
    config1.tri_count = int(ntri);
    config1.amr_vert_tris.assign(n, vector<int>());
    config1.dynamics_tris.assign(ntri, vector<int>(3));
    vector<double> curr_state(5 * n, 0.0);
    read_points(config1, curr_state);
    if (chdir(cwd) != 0) return -1;
    std::memcpy(state5, curr_state.data(), sizeof(double) * 5 * n);
    for (int64_t j = 0; j < ntri; j++)
        for (int k = 0; k < 3; k++) tris[3 * j + k] = config1.dynamics_tris[j][k];
    int64_t a = 0;
    for (int64_t i = 0; i < n; i++) {
        vt_off[i] = int(a);
        for (int t : config1.amr_vert_tris[i]) {
            if (a >= cap) return -2;
            vt_adj[a++] = t;
        }
    }
    vt_off[n] = int(a);
    return 0;
}

// amr.h:13 amr on the reference's own structures built from flat arrays:
// dynamics_tris from `tris`, amr_vert_tris in increasing triangle order,
// amr_parent_verts of max_count pairs ((0, 0), or parent_in for the first n
// points).  Writes the new counts, state, areas, triangles, parents (for the
// n_out points) and the vert_tris lists as CSR (vt_off[n_out + 1], vt_adj).
// Returns 0, or -2 when an output capacity is too small.
int ref_amr(int64_t n, int64_t max_count, int64_t ntri, const double* state5, const double* area, const int* tris,
            const int* parent_in, int64_t cap_points, int64_t cap_tris, int64_t* n_out, int64_t* ntri_out,
            double* state5_out, double* area_out, int* tris_out, int* parent_out, int* vt_off, int* vt_adj) {
    run_information config1;
    config1.point_count = int(n);
    config1.tri_count = int(ntri);
    config1.max_count = int(max_count);
    config1.dynamics_tris.assign(ntri, vector<int>(3));
    config1.amr_vert_tris.assign(n, vector<int>());
    for (int64_t j = 0; j < ntri; j++)
        for (int k = 0; k < 3; k++) {
            config1.dynamics_tris[j][k] = tris[3 * j + k];
            config1.amr_vert_tris[tris[3 * j + k]].push_back(int(j));
        }
    config1.amr_parent_verts.assign(max_count, vector<int>(2, 0));
    if (parent_in)
        for (int64_t i = 0; i < n; i++) {
            config1.amr_parent_verts[i][0] = parent_in[2 * i];
            config1.amr_parent_verts[i][1] = parent_in[2 * i + 1];
        }
    vector<double> st(state5, state5 + 5 * n), ar(area, area + n);
    amr(st, ar, config1);
    const int64_t np = config1.point_count, nt = config1.tri_count;
    *n_out = np;
    *ntri_out = nt;
    if (np > cap_points || nt > cap_tris) return -2;
    std::memcpy(state5_out, st.data(), sizeof(double) * 5 * np);
    std::memcpy(area_out, ar.data(), sizeof(double) * np);
    for (int64_t j = 0; j < nt; j++)
        for (int k = 0; k < 3; k++) tris_out[3 * j + k] = config1.dynamics_tris[j][k];
    int64_t a = 0;
    for (int64_t i = 0; i < np; i++) {
        parent_out[2 * i] = config1.amr_parent_verts[i][0];
        parent_out[2 * i + 1] = config1.amr_parent_verts[i][1];
        vt_off[i] = int(a);
        for (int t : config1.amr_vert_tris[i]) vt_adj[a++] = t;
    }
    vt_off[np] = int(a);
    return 0;
}

}  // extern "C"
