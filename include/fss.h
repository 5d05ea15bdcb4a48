/*
 * fss.h -- C ABI of the B200 barotropic-vorticity right-hand side.
 *
 * Drop-in replacement for the right-hand-side evaluators of
 * cygnari/fast-sphere-sum (Old-BVE-code/rhs_eval.h):
 *
 *   rhs_func(modify, curr_state, area, omega, run_information&)  rhs_eval.h:47-56
 *   rhs_direct_sum(modify, curr_state, area, omega, points)     rhs_eval.h:15-32
 *   rhs_fast_sum(modify, curr_state, area, config1, omega)      rhs_eval.h:34-45
 *
 * plus the tree set-up those evaluators read from run_information
 * (icos_utils.h:135 icosahedron_init, :172 points_assign, fast_rhs.h:16
 * tree_traverse, interp_utils.h:61 interp_init) and the RK4 particle loop
 * that calls them (new_dynamics.cpp:281-340, helpers.h:362 project_points).
 *
 * Conventions (the reference's): particle state is an array of 5 doubles per
 * particle {x, y, z, zeta (relative vorticity), tracer}; area is one double
 * per particle; modify has the same layout as the state and is fully
 * overwritten with {u_x, u_y, u_z, dzeta/dt = -2 omega u_z, 0}.  Time is in
 * days, the sphere has radius 1, omega = 2 pi.
 *
 * Every entry point returns an fss_status (0 = success); no exception
 * crosses this boundary.  A context is not thread-safe: one host thread at a
 * time.  Host pointers are plain (pageable or pinned) host memory unless a
 * function says "device".
 */
#ifndef FSS_H
#define FSS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum fss_status {
    FSS_OK = 0,
    FSS_ERR_INVALID = 1,      /* bad argument or configuration */
    FSS_ERR_CUDA = 2,         /* CUDA runtime error (see fss_last_error) */
    FSS_ERR_NOMEM = 3,        /* device or host allocation failed */
    FSS_ERR_TIMEOUT = 4,      /* a kernel's bounded wait ran out */
    FSS_ERR_TREE = 5,         /* tree build failed (e.g. unassigned particles) */
    FSS_ERR_STATE = 6,        /* call order (e.g. no particles set) */
    FSS_ERR_UNSUPPORTED = 7,  /* compiled without this feature / no GPU */
    FSS_ERR_CAPACITY = 8      /* an output buffer is too small */
} fss_status;

typedef enum fss_precision {
    FSS_PREC_FP64 = 0,   /* FP64 everywhere (the plain FP64 path) */
    FSS_PREC_MIXED = 1   /* FP32 interactions + Kahan, FP64 RK4/renorm/interp */
} fss_precision;

typedef enum fss_method {
    FSS_METHOD_DIRECT = 0,    /* rhs_direct_sum: all pairs */
    FSS_METHOD_TREECODE = 1   /* icosahedral-tree barycentric Lagrange treecode */
} fss_method;

typedef enum fss_assign_mode {
    FSS_ASSIGN_COMPLETE = 0,  /* reference first-match rule; particles it drops
                                 go to their most-inside child instead */
    FSS_ASSIGN_REFERENCE = 1  /* exactly the reference's points_assign
                                 (membership/pair parity only) */
} fss_assign_mode;

typedef enum fss_list_mode {
    FSS_LIST_DUAL = 0,   /* the reference's dual traversal (fast_rhs.h:16) */
    FSS_LIST_LEAF = 1    /* per-target-leaf traversal with per-leaf (n, theta) */
} fss_list_mode;

/* What happens to the tree as particles move (treecode). */
typedef enum fss_rebuild_policy {
    FSS_REBUILD_AUTO = 0,    /* RESORT, or STATIC with FSS_ASSIGN_REFERENCE */
    FSS_REBUILD_STATIC = 1,  /* the reference's: membership and lists of the last
                                build are kept (new_dynamics.cpp:87-88 assigns
                                once before the time loop) */
    FSS_REBUILD_RESORT = 2   /* at the start of every RK4 step each particle is
                                put in the leaf it is in now and the particles
                                are re-sorted on the GPU; leaf geometry and
                                interaction lists (which refer to leaves, not
                                particles) stay those of the last build */
} fss_rebuild_policy;

typedef struct fss_config {
    int32_t device;        /* CUDA device ordinal */
    int32_t precision;     /* fss_precision */
    int32_t method;        /* fss_method (reference: run_information::use_fast) */
    int32_t tree_levels;   /* reference -l: levels 0..tree_levels-1, leaves on the
                              last; 0 = smallest depth whose mean leaf holds at
                              least leaf_target particles */
    int32_t leaf_target;   /* for tree_levels == 0 (default 64) */
    int32_t degree;        /* interpolation degree n (K = (n+1)(n+2)/2 proxies) */
    double theta;          /* MAC (reference -h, default 0.7) */
    int32_t many_count;    /* reference cluster threshold; < 0 means K */
    int32_t assign_mode;   /* fss_assign_mode */
    int32_t list_mode;     /* fss_list_mode */
    int32_t use_graph;     /* capture the RK4 step in a CUDA graph */
    int32_t src_parts;     /* split each target's source list in this many parts
                              (0 = automatic) */
    int32_t block_threads; /* threads per interaction block: one producer warp
                              plus one consumer thread per target, 160, 192,
                              224 or 288 (0 = automatic: the smallest block
                              whose consumers hold the largest leaf) */
    int32_t targets_per_thread; /* 1 */
    int32_t autotune;      /* at fss_set_particles: 1 = time every supported
                              block shape of the pair kernel on the actual
                              lists and keep the fastest; 2 = also, when
                              tree_levels is 0, the tree depth (leaf size: the
                              automatic depth and one level either side, each
                              timed on a whole right-hand side, the fastest kept
                              for this particle count) and, when src_parts is
                              0, the source split (1, 2, 4: the fastest kept) */
    int32_t rebuild;       /* fss_rebuild_policy */
    int32_t cluster_targets; /* 1 = the reference's cp/cc interaction types
                              (fast_rhs.h cp, cc): a well-separated target face
                              holding more than many_count particles takes its
                              far sources at its interpolation points,
                              interpolated down to its particles; 0 = every far
                              source is summed at the target particles.  With
                              FSS_LIST_LEAF the per-leaf (n, theta) are carried
                              up to the faces of a dual traversal (theta = min,
                              n = max over a face's leaves) */
    int32_t wait_limit_us; /* every wait of the pair kernel on its tile ring,
                              and of the batched V^-1 kernels on their bulk
                              copy, gives up after this many microseconds and
                              the call returns FSS_ERR_TIMEOUT, the context
                              staying usable (0 = 2 s) */
    int32_t reserved[3];
} fss_config;

typedef struct fss_ctx fss_ctx;

/* Defaults: mixed precision treecode, degree 8, theta 0.7, automatic depth
 * (leaves of >= 64 particles), complete assignment, dual (reference)
 * traversal, CUDA graph on, device 0. */
void fss_config_init(fss_config* cfg);

int fss_create(const fss_config* cfg, fss_ctx** out);
void fss_destroy(fss_ctx* ctx);
/* Message for the last failing call on this context (or on a NULL context). */
const char* fss_last_error(const fss_ctx* ctx);
/* Launch stream for all later work (a cudaStream_t; NULL = the context's own). */
int fss_set_stream(fss_ctx* ctx, void* cuda_stream);
/* The stream the context launches on now (its own unless fss_set_stream gave
 * one), for ordering the caller's work -- e.g. the collective of a sharded
 * step -- after the context's. */
int fss_get_stream(fss_ctx* ctx, void** cuda_stream);

/* Upload a particle set (host, 5 doubles per particle, in the caller's order)
 * and, for the treecode, build the tree, as the reference does before its
 * time loop (new_dynamics.cpp:87-88).  The lists stay fixed until the next
 * fss_set_particles or fss_rebuild_tree; with FSS_REBUILD_RESORT the
 * particles are re-sorted into their current leaves at every RK4 step. */
int fss_set_particles(fss_ctx* ctx, int64_t n, const double* state5, const double* area);
/* Re-assign particles and rebuild the interaction lists from the current
 * device state (new_dynamics.cpp:335, after AMR, calls points_assign again). */
int fss_rebuild_tree(fss_ctx* ctx);

/* rhs_eval.h:47 rhs_func.  state5/area/modify5 are host arrays in the
 * caller's order; psi (nullable) receives the stream function.  The tree of
 * fss_set_particles is reused; if the particle count differs, the particles
 * are set first.  Uses the context's method. */
int fss_rhs(fss_ctx* ctx, const double* state5, const double* area, double omega,
            double* modify5, double* psi);
/* rhs_eval.h:15 rhs_direct_sum (then scaled and dzeta/dt set as rhs_func). */
int fss_rhs_direct(fss_ctx* ctx, const double* state5, const double* area, double omega,
                   double* modify5, double* psi);
/* rhs_eval.h:34 rhs_fast_sum, through the treecode (then scaled as rhs_func). */
int fss_rhs_treecode(fss_ctx* ctx, const double* state5, const double* area, double omega,
                     double* modify5, double* psi);

/* RK4 steps on the device-resident state (new_dynamics.cpp:281-340 order:
 * stage states projected onto the sphere, zeta adjusted by -2 omega dz). */
int fss_rk4_step(fss_ctx* ctx, double dt, double omega, int32_t nsteps);
/* Same, with the state uploaded from and downloaded to host memory. */
int fss_rk4_step_host(fss_ctx* ctx, double* state5, double dt, double omega, int32_t nsteps);
/* Download the device-resident state (caller's order, 5 doubles each). */
int fss_get_state(fss_ctx* ctx, double* state5);
/* Velocity of the device-resident state into host modify5 (and psi). */
int fss_rhs_current(fss_ctx* ctx, double omega, double* modify5, double* psi);

/* remesh.h:109-178 regrid_points2 (helpers.h:251-265 tri_interp): particles
 * that moved with the flow are put back on the grid.  Every target point
 * keeps its position and takes the absolute vorticity (zeta + 2 omega z) and
 * tracer interpolated, with normalised barycentric coordinates, from the
 * first triangle of the moved mesh (vertices moved5, triangles tris: 3
 * vertex indices each) that contains it: first among the triangles adjacent
 * to its own vertex, in increasing index order (the reference reads that
 * adjacency from a file), then among all triangles.  A point found in no
 * triangle keeps its values.  Host arrays, 5 doubles per particle; target5
 * is read (positions, kept values) and written.  *n_fallback: points that
 * needed the search over all triangles; *n_not_found: points found nowhere
 * (the reference throws).  Either may be NULL.  The search over all
 * triangles runs on a cell grid of triangle caps (same first triangle as the
 * reference's linear scan), so its cost stays near linear in the points.
 * Device buffers and the triangles' adjacency are kept per device between
 * calls (until the process ends); calls on one device are serialised. */
int fss_remesh(int64_t n, const double* moved5, double* target5, int64_t ntri, const int32_t* tris,
               double omega, int64_t* n_fallback, int64_t* n_not_found);
/* The same on the context's device-resident state (new_dynamics.cpp:213-216,
 * use_remesh): the targets are the positions given to fss_set_particles; the
 * remeshed state becomes the context's state (and, with re-sorting, the
 * particles go back into the leaves of their grid points).  A point found in
 * no triangle keeps its current zeta and tracer.  tris = NULL with ntri = 0
 * reuses the triangles of the previous call (skipping the comparison with
 * them that a repeated array costs). */
int fss_remesh_current(fss_ctx* ctx, int64_t ntri, const int32_t* tris, double omega, int64_t* n_fallback,
                       int64_t* n_not_found);

/* regrid_points2 with the vertex -> triangles lists given explicitly (CSR:
 * vert_tris of vertex i = vt_adj[vt_off[i] .. vt_off[i + 1]), e.g. as read
 * from the reference's <N>vert_tris.csv by fss_read_vert_tris_csv); the
 * adjacent triangles are tried in list order.  Otherwise as fss_remesh. */
int fss_remesh_lists(int64_t n, const double* moved5, double* target5, int64_t ntri, const int32_t* tris,
                     const int32_t* vt_off, const int32_t* vt_adj, double omega, int64_t* n_fallback,
                     int64_t* n_not_found);

/* ------------------------------------------------------------- state files
 * The reference's output (new_dynamics.cpp:123-139, 228-236): per step, one
 * line "x,y,z,zeta,tracer,area" per particle, each number as a default C++
 * stream writes a double (%g, 6 significant digits), appended to
 * output_<name>.csv; the particle count appended to point_counts_<name>.csv;
 * <name> as fss_output_name builds it from the run's flags.  The binary
 * equivalent appends per step the 8 bytes "FSSSTAT1", the count (int64)
 * and count x 6 float64 (x, y, z, zeta, tracer, area), little-endian. */
int fss_state_csv_append(const char* path, int64_t n, const double* state5, const double* area);
int fss_point_count_append(const char* path, int64_t n);
int fss_output_name(char* buf, int64_t cap, int64_t point_count, const char* init_cond, int use_fast,
                    int tree_levels, int use_amr, int use_mpi, int use_remesh, int64_t time_steps);
int fss_state_bin_append(const char* path, int64_t n, const double* state5, const double* area);
/* Step `step` (from 0) of a binary state file: *n_out = its count;
 * FSS_ERR_CAPACITY when that exceeds cap (state5/area may be NULL). */
int fss_state_bin_read(const char* path, int64_t step, int64_t cap, double* state5, double* area, int64_t* n_out);
/* The reference's inputs (helpers.h:299-340 read_points): <N>points_rh4.csv
 * (x, y, z, zeta: the first 4 fields of each of n lines; the tracer is not
 * read), <N>tris.csv (3 vertex indices per line), <N>vert_tris.csv with
 * <N>vert_tri_count.csv (each vertex's triangles; CSR into off[n + 1] and
 * adj[cap]).  Fields are parsed as stod does, then truncated for indices. */
int fss_read_points_csv(const char* path, int64_t n, double* state5);
int fss_read_tris_csv(const char* path, int64_t ntri, int32_t* tris);
int fss_read_vert_tris_csv(const char* lists_path, const char* counts_path, int64_t n, int32_t* off, int32_t* adj,
                           int64_t cap);

/* ------------------------------------------------------------- AMR
 * amr.h:13-178 amr.  The handle holds the triangle mesh, the reference's
 * vert_tris lists (one ordering key per triangle corner: a vertex's list is
 * its triangles in increasing key order; initial lists in increasing
 * triangle order) and the parent pairs (amr_parent_verts: (0, 0) for a
 * primitive point), on the device.  max_count is the reference's point
 * limit; max_tris bounds the triangle count. */
typedef struct fss_amr fss_amr;
int fss_amr_create(int64_t n, int64_t ntri, const int32_t* tris, const int32_t* parent_verts, int64_t max_count,
                   int64_t max_tris, int device, fss_amr** out);
void fss_amr_destroy(fss_amr* a);
int fss_amr_counts(const fss_amr* a, int64_t* point_count, int64_t* tri_count);
/* One amr() call.  state5 and area are host arrays with room for max_count
 * points; *point_count must be the mesh's count and becomes the new one.
 * Triangles are visited in index order while their count grows; a triangle
 * whose vorticity range exceeds vorticity_tol or whose circulation
 * A |z1 + z2 + z3| / 3 exceeds circulation_tol (the reference: 0.2 and
 * 0.0025) is split in four; new edge midpoints (unprojected averages of all
 * five components) are appended; areas move A/6 from corners to midpoints.
 * Nothing happens when *point_count >= max_count (as the reference).  More
 * points than max_count or triangles than max_tris within the call (the
 * reference: undefined) returns FSS_ERR_CAPACITY, leaves the host arrays
 * unchanged and the handle unusable. */
int fss_amr_refine(fss_amr* a, int64_t* point_count, double* state5, double* area, double vorticity_tol,
                   double circulation_tol);
/* amr() on the context's current particles, device-resident
 * (new_dynamics.cpp:219-228): the context's particles must be the mesh's
 * points (same count, same order); the new midpoints are projected onto the
 * sphere (zeta += -2 omega dz, as project_points) and the context takes the
 * new particle set (tree and lists rebuilt; the remesh grid becomes the new
 * positions).  *point_count receives the new count. */
int fss_amr_refine_current(fss_ctx* ctx, fss_amr* a, double vorticity_tol, double circulation_tol, double omega,
                           int64_t* point_count);
/* The mesh: tris (3 per triangle), corner_keys (3 per triangle), parent
 * pairs (2 per point); any may be NULL. */
int fss_amr_get_mesh(const fss_amr* a, int32_t* tris, uint64_t* corner_keys, int32_t* parent_verts);
/* regrid_points2 on the handle's mesh with its vert_tris lists (the order
 * amr() leaves them in); as fss_remesh otherwise. */
int fss_amr_remesh(fss_amr* a, const double* moved5, double* target5, double omega, int64_t* n_fallback,
                   int64_t* n_not_found);

/* Tree summary of the last build. */
typedef struct fss_tree_info {
    int32_t tree_levels;     /* levels 0..tree_levels-1 */
    int32_t leaf_count;      /* 20 * 4^(tree_levels-1) */
    int32_t degree, n_proxy; /* n and K */
    int64_t n_pairs;         /* reference-format interactions (dual traversal) */
    int64_t n_list_entries;  /* source segments (leaf runs, proxy runs) over all items */
    int64_t n_items;         /* interaction work items (blocks) per RHS */
    int64_t n_tiles;         /* shared-memory source tiles over all items at the
                                build's leaf counts */
    int64_t unassigned;      /* particles without a leaf (reference mode) */
    double pp_interactions;  /* particle-particle pair count per RHS */
    double pc_interactions;  /* particle-proxy pair count per RHS */
    int32_t block_threads;   /* pair-kernel block shape in use */
    int32_t targets_per_thread;
    int32_t src_parts;
    int32_t target_clusters; /* faces evaluated at interpolation points (cp/cc) */
    double cp_interactions;  /* interpolation point-particle pairs per RHS */
    double cc_interactions;  /* interpolation point-proxy pairs per RHS */
    double lane_pairs_leaf;    /* pair evaluations the target-leaf launch's
                                  consumer lanes perform per RHS at the build's
                                  leaf counts, discarded lanes included */
    double lane_pairs_cluster; /* the same for the target-cluster launch */
    int32_t max_degree;        /* highest degree among the lists' proxies and
                                  target clusters (the upward pass forms
                                  moments up to it) */
    int32_t max_cluster_points; /* largest target cluster (interpolation points) */
} fss_tree_info;
int fss_get_tree_info(fss_ctx* ctx, fss_tree_info* info);

/* Membership and interaction list of the last build, in the reference's
 * formats: loc[l*n + i] = face of particle i on level l or -1 (icos_utils.h
 * tree_point_locs / tree_tri_points); counts = member counts per face, levels
 * concatenated; pairs = 7 ints per interaction {lev_t, lev_s, t, s, n_t, n_s,
 * type} with type 0 "pp", 1 "pc", 2 "cp", 3 "cc" (struct_list.h:6-14), in the
 * order tree_traverse emits them.  Any pointer may be NULL. */
int fss_get_tree(fss_ctx* ctx, int32_t* loc, int32_t* counts, int32_t* pairs, int64_t pairs_cap);

/* Per-leaf (degree, theta) choice for FSS_LIST_LEAF, applied at the next
 * build: degree[leaf], theta[leaf] for every leaf. */
int fss_set_leaf_params(fss_ctx* ctx, int32_t nleaf, const int32_t* degree, const double* theta);

/* Per-kernel device time.  When enabled, every launch is bracketed by CUDA
 * events on the launch stream (graphs are not used while enabled). */
int fss_profile_enable(fss_ctx* ctx, int32_t on);
/* names: '\n'-separated kernel names; ms[i], launches[i] per kernel; returns
 * the number of kernels through *count. */
int fss_profile_read(fss_ctx* ctx, char* names, int32_t names_cap, double* ms, int64_t* launches,
                     int32_t cap, int32_t* count);
/* Algorithmic work of one RHS evaluation: pair interactions (23 flops each;
 * pp + pc + cp + cc), and bytes of the upward pass. */
int fss_work_per_rhs(fss_ctx* ctx, double* interactions, double* upward_bytes);

/* ----------------------------------------------------------------- inputs
 * Synthetic inputs: the reference's missing CSV initial conditions
 * (helpers.h:299 read_points) are regenerated from icos_init. */

/* Vertices and faces after `level` refinements (icos_utils.h:15 icos_init,
 * same vertex order): n = 10*4^level + 2, faces = 20*4^level. */
int fss_icos_counts(int32_t level, int64_t* n_verts, int64_t* n_faces);
int fss_icos_grid(int32_t level, double* xyz, int32_t* faces);
/* helpers.h:344 area_init */
int fss_area_init(int64_t n, const double* state5, int64_t n_faces, const int32_t* faces, double* area);
/* vorticity_functions.h:13 rossby_haurwitz_4 (zeta and tracer). */
int fss_vorticity_rh4_ref(int64_t n, double* state5);
/* Rossby-Haurwitz R=4 with w = K = amp (per day), zeta = 2 w sin(lat) -
 * K (R+1)(R+2) cos^R(lat) sin(lat) cos(R lon), plus n_vortex Gaussian vortices
 * a exp(-(d/width)^2) (centres uniform on the sphere, a ~ N(0, 2 pi^2)) from
 * a 64-bit Mersenne twister seeded with `seed`, area-weighted mean removed;
 * tracer = 2 + lat. */
int fss_vorticity_rh_vortices(int64_t n, double* state5, const double* area, double amp,
                              int32_t n_vortex, double width, uint64_t seed);

/* Host-only, no GPU needed. ---------------------------------------------- */

/* fast_rhs.h:16 tree_traverse on given per-face particle counts (levels
 * 0..tree_levels-1 concatenated, 20*4^l faces on level l): the reference's
 * pair list, 7 ints per pair as in fss_get_tree, into pairs[cap*7]; the
 * number of pairs goes to *n_pairs (FSS_ERR_CAPACITY if it exceeds cap). */
int fss_tree_traverse(int32_t tree_levels, double theta, int32_t many_count, const int32_t* counts,
                      int32_t* pairs, int64_t cap, int64_t* n_pairs);
/* Interpolation points of degree n (K = (n+1)(n+2)/2 barycentric triples)
 * and the K x K inverse Vandermonde matrix of the Chebyshev product basis
 * (vinv[m*K + k]: coefficient of basis function m in Lagrange polynomial k);
 * replaces interp_utils.h:12-75 (fekete_init / interp_mat_init). */
int fss_interp_nodes(int32_t degree, double* nodes, double* vinv);
/* icos_utils.h:15 icos_init tree geometry for levels 0..tree_levels-1:
 * circumcentre and circumradius per face (4 doubles), levels concatenated. */
int fss_tree_geometry(int32_t tree_levels, double* tri_info);

/* ------------------------------------------------------------ ensemble
 * Many independent problems of uneven size (mixed-precision treecode) that
 * advance together: per RK stage one batched upward pass, one persistent
 * pair-kernel launch over a global (member, target leaf, source run) work
 * queue and one epilogue; each RK4 step is one CUDA graph.  No counterpart in
 * the reference (which runs one problem per process). */
typedef struct fss_ensemble fss_ensemble;
/* cfg: precision FSS_PREC_MIXED, method FSS_METHOD_TREECODE; degree, theta,
 * tree_levels (0 = automatic per member) apply to every member. */
int fss_ensemble_create(const fss_config* cfg, fss_ensemble** out);
void fss_ensemble_destroy(fss_ensemble* e);
int fss_ensemble_set_stream(fss_ensemble* e, void* cuda_stream);
/* Add one member (host state, 5 doubles per particle, and areas); its tree
 * and lists are built now.  *member receives its index. */
int fss_ensemble_add(fss_ensemble* e, int64_t n, const double* state5, const double* area, int32_t* member);
/* Concatenate all members' state and work lists on the device. */
int fss_ensemble_build(fss_ensemble* e);
int fss_ensemble_rk4_step(fss_ensemble* e, double dt, double omega, int32_t nsteps);
int fss_ensemble_get_state(fss_ensemble* e, int32_t member, double* state5);
int fss_ensemble_info(fss_ensemble* e, int32_t* members, int64_t* particles, double* interactions_per_rhs,
                      int64_t* work_items);
/* Device time (ms) of one persistent pair launch on the current stage
 * sources, the mean of `reps` launches after an untimed one (CUDA events on
 * the ensemble's stream); the launches only rewrite the partial sums that
 * the next stage rewrites anyway, so the state is unchanged. */
int fss_ensemble_time_pairs(fss_ensemble* e, int32_t reps, double* ms);

/* ------------------------------------------------------------ selector
 * Learned per-leaf interpolation degree and MAC (no counterpart in the
 * reference, which fixes degree 2 and one theta: new_dynamics.cpp:78-79,
 * run_config.h:100).  Classes c = 0..11: degree 4 + 2 (c / 3), theta
 * 0.5 + 0.1 (c % 3).  The network is a 16-64-64-12 MLP (ReLU) with BF16
 * weights and FP32 accumulation; it predicts log10(e_l(c) / U) for every
 * leaf l, e_l the L2 velocity error over the leaf's particles and U the RMS
 * speed. */
#define FSS_SELECTOR_CLASSES 12
#define FSS_SELECTOR_FEATURES 16
typedef struct fss_mlp fss_mlp;
int fss_mlp_create(int32_t device, fss_mlp** out);
void fss_mlp_destroy(fss_mlp* m);
/* Number of parameters: W1[64][16], b1[64], W2[64][64], b2[64], W3[12][64], b3[12]. */
int32_t fss_mlp_param_count(void);
int fss_mlp_init(fss_mlp* m, uint64_t seed);
int fss_mlp_set_params(fss_mlp* m, const float* params);
int fss_mlp_get_params(fss_mlp* m, float* params);
/* Training set: n rows of 16 features, 12 targets and an optional 0/1 mask. */
int fss_mlp_set_data(fss_mlp* m, int64_t n, const float* x, const float* t, const float* mask);
/* Loss = mean over rows of sum_o mask (y - t)^2 and its gradient (no update). */
int fss_mlp_gradient(fss_mlp* m, float* grad, double* loss);
/* Adam (beta 0.9/0.999), shuffled mini-batches (multiples of 128); mean
 * batch loss per epoch into losses[epochs]. */
int fss_mlp_train(fss_mlp* m, int32_t epochs, int32_t batch, double lr, uint64_t seed, double* losses);
int fss_mlp_predict(fss_mlp* m, int64_t n, const float* x, float* y);
/* The 12 classes (degree, theta) of class c = 3 i + j: with clusters = 0
 * (far sources summed at the target particles) n = 4 + 2i, theta = 0.5 +
 * 0.1j; with clusters = 1 (target clusters, cp/cc) n = 6 + 2i, theta = 0.7 +
 * 0.1j.  Host only. */
int fss_selector_class_table(int32_t clusters, int32_t* degree, double* theta);
/* Features (16 per leaf) and exact interaction counts (12 per leaf, one per
 * class of the context's mode) of the current tree and state, and the RMS
 * speed U. */
int fss_selector_features(fss_ctx* ctx, float* features, double* costs, double* u_rms);
/* Per leaf the class minimising cost + mu * 10^(2 y) with mu chosen by
 * bisection so that sum_l 10^(2 y_l) <= budget (host only). */
int fss_select_classes(int64_t nleaf, int32_t nclass, const double* pred_log_err, const double* cost,
                       double budget, int32_t* choice);
/* Predict with `m` (features standardised with mean/std), choose classes
 * for a relative L2 tolerance tol (budget (tol/safety)^2 N), switch the
 * context to per-leaf parameters (FSS_LIST_LEAF; with cluster_targets the
 * per-face dual traversal).  choice_out: nleaf ints (nullable). */
int fss_selector_apply(fss_ctx* ctx, fss_mlp* m, const float* feat_mean, const float* feat_std, double tol,
                       double safety, int32_t* choice_out);

/* Direct sum without any allocation.  No counterpart in the reference.
 *
 * For callers that cannot allocate device memory: real-time loops in which a
 * cudaMalloc or cudaFree could synchronise the device and stall it, and
 * plugins whose host application owns the whole device memory budget.  The
 * caller passes device buffers: state5 (n x 5 doubles, the reference's
 * layout), area (n doubles) and modify5 (n x 5 doubles, overwritten as by
 * rhs_func with the direct sum, mixed precision: FP32 pairs, Kahan-compensated
 * sums).  Kernels go to `stream` (a cudaStream_t, NULL = the default stream)
 * and run asynchronously; the call does not synchronise.
 *
 * Limit: n <= FSS_NOALLOC_MAX_PARTICLES; larger n returns FSS_ERR_CAPACITY
 * with a message in fss_last_error(NULL).  The scratch is a fixed device
 * array of FSS_NOALLOC_MAX_PARTICLES x 16 bytes (4 MiB) that every GPU
 * loading the library holds until the process exits.  Every call looks up
 * that array's device address on the current device (cudaGetSymbolAddress).
 * Under CUDA's lazy module loading (the default) the first call on a device
 * loads the library's module there, 4 MiB array included: make that first
 * call at start-up, before any stream capture (or load modules eagerly with
 * CUDA_MODULE_LOADING=EAGER).  All calls share the array: two calls whose
 * kernels overlap on the GPU race. */
#define FSS_NOALLOC_MAX_PARTICLES 262144
int fss_rhs_direct_noalloc(int64_t n, const double* state5, const double* area, double omega, double* modify5,
                           void* stream);

/* ------------------------------------------------------------ sharding
 * One problem split over several GPUs, one process per GPU.  The reference
 * splits the same work over MPI ranks: fast_sum_mpi.cpp:322-338 gives each
 * rank a range of top-level target faces, direct_sum_mpi.cpp:74-82 a block
 * of target rows, and mpi_utils.h:6-26 replicates the whole state again after
 * every RK stage.  Here every rank holds the whole state and builds the same
 * tree; it evaluates the right-hand side for its own targets only: a
 * contiguous range of units -- the faces of the shallowest level that holds
 * a target cluster, or the leaves (treecode); blocks of target rows (direct
 * sum) -- balanced by their counted interactions, so that every target
 * cluster and its downward pass lie with one rank.  Per RK stage the ranks
 * exchange one device buffer of N x 4 doubles (the context's particle order):
 * a rank writes the velocity sums of its own rows and -0.0 in every other
 * row; the caller sums the buffers over the ranks (an all-reduce, e.g. NCCL
 * through torch.distributed: x + -0.0 = x, so the sum is exact in any order);
 * then every rank advances all particles identically.  One RK4 step:
 *
 *   for stage in 1..4:
 *       fss_shard_stage(ctx, stage, exchange);             this rank's targets
 *       all-reduce (sum) of exchange over the ranks;       the caller's collective
 *       fss_shard_combine(ctx, stage, dt, omega, exchange);
 *
 * Each stage's launches go to the context's stream; the caller orders its
 * collective after them (same stream, or an event).  With the same source
 * split (src_parts) and degrees, the result equals an unsharded context's
 * bit for bit.  No TMA load reads another GPU's memory: the exchange buffer
 * is local and the collective belongs to the caller. */

/* Contiguous unit ranges of near-equal summed cost: bounds[r] ..
 * bounds[r + 1] for rank r (nranks + 1 entries).  Host only. */
int fss_shard_partition(int64_t nunits, const double* cost, int32_t nranks, int64_t* bounds);
/* Make the context rank `rank` of `nranks` (0 ranks: not sharded); applies
 * to the current particles and to later builds. */
int fss_shard_set(fss_ctx* ctx, int32_t rank, int32_t nranks);
typedef struct fss_shard_info {
    int32_t rank, nranks;
    int32_t unit_level;            /* face level of the units (-1: direct-sum row blocks) */
    int32_t pad;
    int64_t units;                 /* units over all ranks */
    int64_t unit_lo, unit_hi;      /* this rank's units */
    int64_t target_lo, target_hi;  /* this rank's leaves (treecode) or rows (direct sum) */
    double cost_total, cost_own;   /* counted interactions per RHS at the build */
} fss_shard_info;
int fss_shard_get_info(fss_ctx* ctx, fss_shard_info* info);
/* Stage `stage` (1..4) of an RK4 step for this rank's targets (stage 1 first
 * re-sorts the particles, as fss_rk4_step does): writes the exchange buffer
 * (device, N x 4 doubles). */
int fss_shard_stage(fss_ctx* ctx, int32_t stage, void* exchange);
/* After the caller summed the exchange buffers of all ranks: the stage's
 * combine and renormalisation for every particle. */
int fss_shard_combine(fss_ctx* ctx, int32_t stage, double dt, double omega, const void* exchange);

/* Test hook for the failure path (no counterpart in the reference, which has
 * no error path): in the next right-hand-side evaluation of this context,
 * block `block` of the target-leaf pair launch neither copies its first
 * source tile nor signals its arrival, so that the block's bounded waits run
 * out.  That call returns FSS_ERR_TIMEOUT; the hook is then cleared and the
 * context stays usable.  No copy is left in flight: the withheld tile was
 * never issued, and a block whose waits ran out waits (bounded) for the
 * copies it did issue before it exits.  block < 0 clears the hook. */
int fss_test_hold_tile(fss_ctx* ctx, int32_t block);

/* Test hook for the batched V^-1 kernels' bounded wait: in the next
 * right-hand-side evaluation, block 0 of the proxy-charge launch (which = 0)
 * or of the cluster-coefficient launch (which = 1) expects the bulk copy of
 * its matrix but does not issue it, so that its wait runs out.  The call
 * returns FSS_ERR_TIMEOUT; the hook is then cleared and the context stays
 * usable.  No copy is left in flight (none was issued).  which < 0 clears
 * the hook. */
int fss_test_hold_stage(fss_ctx* ctx, int32_t which);

/* Test hook for the per-step re-sort (FSS_REBUILD_RESORT): mode 0 (the
 * default) builds the new leaf order by partitioning the old one (particles
 * that stay in their leaf keep their order; the few that move are bucketed
 * by new leaf and ranked by old position), mode 1 by the two-pass radix key
 * sort of the initial tree build.  Both give the unique stable order of the
 * new leaf keys, so every later result is the same to the bit.  Other modes
 * return FSS_ERR_INVALID. */
int fss_test_resort_mode(fss_ctx* ctx, int32_t mode);

/* Library build string (architecture, features). */
const char* fss_version(void);

#ifdef __cplusplus
}
#endif
#endif /* FSS_H */
