// kernels.h -- host-callable launchers of the sm_100a kernels.
#pragma once
#include <cstdint>
#include <vector>
#include <cuda_runtime.h>

#include "dbuf.h"
#include "fss_internal.h"

namespace fss {

enum EpiMode { EPI_RHS = 0, EPI_RK4 = 1 };

struct EpiArgs {
    int64_t n = 0;
    int parts = 1;
    int64_t pstride = 0;
    const double4* partials = nullptr;
    double4* xs = nullptr;          // current stage state (x, y, z, zeta), sorted; updated in RK4 mode
    const double* area = nullptr;   // sorted
    double omega = 0;
    int mode = EPI_RHS;
    // rhs output (caller's order through perm)
    const int32_t* perm = nullptr;
    double* out5 = nullptr;
    double* psi = nullptr;
    const double* wtotal = nullptr;  // device scalar: sum zeta A
    // RK4
    int stage = 1;
    double dt = 0;
    double4* s0 = nullptr;
    double4* acc = nullptr;
    // interaction sources of the next stage
    void* src = nullptr;
    const uint32_t* leaf_of = nullptr;
    const double4* frame = nullptr;
};

// Pair-kernel block: `threads` = one producer warp + consumer warps with one
// target each.
struct PairShape {
    int threads = 160;
    int per_thread = 1;
    int tile = 256;
    int depth = 4;  // ring slots (tiles in flight)
    int targets() const { return (threads - 32) * per_thread; }
};

// k_tree.cu
void launch_assign(cudaStream_t st, int64_t n, const double* in5, const double* verts, const int32_t* tri_verts,
                   const int64_t* lev_off, int tree_levels, int reference_mode, int32_t* loc, uint32_t* key, int* err);
void launch_level_hist(cudaStream_t st, int64_t n, int tree_levels, const int32_t* loc, const int64_t* lev_off,
                       int32_t* counts);
int64_t sort_scratch_words(int64_t n);
// Kernel launches of one launch_sort call.
int sort_launch_count(int64_t n, int bits);
void launch_sort(cudaStream_t st, int64_t n, int bits, uint32_t* keys, uint32_t* keys_tmp, int32_t* vals,
                 int32_t* vals_tmp, uint32_t* hist);
void launch_leaf_bounds(cudaStream_t st, int64_t n, const uint32_t* skey, int32_t nleaf, int32_t* leaf_start);
// Re-sort at the start of an RK4 step: new leaf keys (the previous leaf
// when the particle is still inside it), then, after the key sort gave the
// order q, the state, areas, tracers and caller indices permuted in place
// (through the free stage buffers xs and acc) and the stage-1 sources
// rewritten.
void launch_reassign(cudaStream_t st, int64_t n, const double4* pos, const EnsLeaf* leaves, int leaf_level,
                     const NodeGeom* node, const int64_t* lev_off, uint32_t* key, int* err);
void launch_resort(cudaStream_t st, bool fp64, int64_t n, const int32_t* q, double4* s0, double* area,
                   double* tracer, int32_t* perm, double4* xs, double4* acc, void* src);
// The same re-sort without a key sort: the old order partitioned into the
// new leaves (stayers in place order, movers bucketed and ranked by old
// position), which is the stable sort's order.  key_new and bucket take n
// words each, scratch partition_scratch_words(nleaf).  key and leaf_start
// are updated.
int64_t partition_scratch_words(int64_t nleaf);
void launch_resort_partition(cudaStream_t st, bool fp64, int64_t n, int64_t nleaf, int leaf_level,
                             const NodeGeom* node, const int64_t* lev_off, uint32_t* key, uint32_t* key_new,
                             int32_t* leaf_start, int32_t* bucket, uint32_t* scratch, double4* s0, double* area,
                             double* tracer, int32_t* perm, double4* xs, double4* acc, void* src, int* err);
void launch_gather(cudaStream_t st, bool fp64, int64_t n, const double* in5, const double* area_in, const int32_t* perm,
                   const uint32_t* leaf_of, const double4* frame, double4* s0, double4* xs, double* area_s,
                   double* tracer_s, void* src);

// k_pairs.cu
// Block shapes of the pair kernel the autotuner tries (threads = 32 + targets).
const std::vector<PairShape>& pair_shapes(bool fp64);
// The supported shape with `threads`, or the default (128).
PairShape pairs_shape(bool fp64, int threads, int per_thread);
// Block for work items of k targets (target clusters: their interpolation
// points): the smallest of 64, 96, 128, 160 threads whose consumers hold them.
PairShape cluster_shape(bool fp64, int k);
cudaError_t launch_pairs(cudaStream_t st, bool fp64, bool psi, PairShape shape, int nitems, const void* src,
                         const Segment* segs, const int32_t* leaf_start, const WorkItem* items, double4* partials,
                         int64_t pstride, int* err, PairCtl ctl);
constexpr int kPersistentThreads = 160;
cudaError_t launch_pairs_persistent(cudaStream_t st, int nitems, const void* src, const Segment* segs,
                                    const int32_t* leaf_start, const WorkItem* items, int* queue, double4* partials,
                                    int64_t pstride, int* err, int blocks, PairCtl ctl);
int persistent_blocks_per_sm();

// k_epi.cu
void launch_up_leaf(cudaStream_t st, bool fp64, int nleaf, const void* src, const int32_t* leaf_start,
                    const double4* frame, const NodeGeom* node, const int64_t* lev_off, int leaf_level, int nmax,
                    int level_mask, const int8_t* up_deg, double* part);
// Upward pass, part 2: every proxy face's moments (its rows summed into
// msum, njobs x nproxy(nmax)), then the proxy charges of every (face,
// degree) task, batched by degree (`blocks` of at most batch_tasks() tasks).
// vpad: Vinv of every degree with rows padded to a multiple of 4 doubles
// (vpad_off by degree); a failed wait sets kErrTimeout in err.
void launch_up_proxies(cudaStream_t st, bool fp64, int njobs, const ProxyJob* jobs, const double* part,
                       int leaf_level, int nmax, double* msum, int nblocks, const TaskBlock* blocks,
                       const int32_t* tasks, const double* vpad, const int32_t* vpad_off, const double4* proxy_pos,
                       int64_t n, void* src, int* err, uint64_t wait_ns, int hold_block = -1);
// Tasks per block of the batched V^-1 products (upward proxy charges,
// downward coefficients).
int batch_tasks();
// Allows the batched V^-1 kernels the dynamic shared memory of the largest
// degree (host only; before their first launch).
cudaError_t batch_prepare();
// Downward pass of the target clusters and the faces below them.
struct DownArgs {
    int njobs = 0;                       // target clusters
    const DownJob* jobs = nullptr;
    int ncoef_blocks = 0;                // their coefficient tasks, batched by degree
    int max_deg = 0;                     // highest target-cluster degree
    const TaskBlock* coef_blocks = nullptr;
    const int32_t* coef_tasks = nullptr;
    const double4* partials = nullptr;   // field at the interpolation points: parts slots of stride pstride
    int parts = 1;
    int64_t pstride = 0;
    const double* vtpad = nullptr;       // inverse Vandermonde matrices transposed, rows padded
    const int32_t* vpad_off = nullptr;   // to a multiple of 4 doubles, by degree
    int* err = nullptr;                  // kErrTimeout when a staging wait runs out
    uint64_t wait_ns = 0;
    int hold_block = -1;                 // test hook: coefficient block that withholds its staging copy
    const NodeGeom* node = nullptr;
    double4* coef = nullptr;
    int nleaf = 0;
    const double4* xs = nullptr;
    const int32_t* leaf_start = nullptr;
    const LeafAnc* leaf_anc = nullptr;   // kMaxLevels per leaf
    double4* out = nullptr;              // down-pass partial slot, one per particle
    bool fp32_eval = false;              // mixed precision: interpolants evaluated in FP32 (velocity)
};
void launch_down(cudaStream_t st, bool psi, const DownArgs& d);
int down_launch_count(const DownArgs& d);
void launch_epilogue(cudaStream_t st, bool fp64, const EpiArgs& a);
// Sharded RHS: this rank's rows (leaves [leaf_lo, leaf_hi) through
// leaf_start, or rows [row_lo, row_hi) when leaf_start is null) summed over
// the partial slots into out, -0.0 in the other rows.
void launch_shard_reduce(cudaStream_t st, int64_t n, int parts, int64_t pstride, const double4* partials,
                         const int32_t* leaf_start, int64_t leaf_lo, int64_t leaf_hi, int64_t row_lo, int64_t row_hi,
                         double4* out);
void launch_refresh(cudaStream_t st, bool fp64, int64_t n, const double4* s0, const double* area,
                    const uint32_t* leaf_of, const double4* frame, double4* xs, void* src);
void launch_wsum(cudaStream_t st, int64_t n, const double4* xs, const double* area, double* w);
void launch_scatter_state(cudaStream_t st, int64_t n, const int32_t* perm, const double4* s0, const double* tracer,
                          double* out5);

// k_remesh.cu
// Device scratch of the remesh step, grown on demand and kept by its owner
// between calls.
struct RemeshScratch {
    DBuf failed, counters, adj_cur, caps, box, cells, glist, scal, ent, part;
};
// Vertex -> triangles adjacency of `tris`: off[n + 1] (32-bit), adj[3 ntri]
// holding corner ids 3 t + c, each vertex's list in increasing key order
// (keys[3 t + c]; NULL: increasing triangle order).  *valid = false (nothing
// else usable) when a vertex index is outside [0, n).  Synchronises the
// stream.
cudaError_t launch_remesh_adjacency(cudaStream_t st, int64_t n, int64_t ntri, const int32_t* tris,
                                    const uint64_t* keys, uint32_t* off, int32_t* adj, RemeshScratch& s,
                                    bool* valid);
// Remesh targets (grid points, 5 doubles each, zeta and tracer replaced
// where a moved-mesh triangle contains them); returns the number of points
// that needed the search over all triangles and the number found nowhere.
// Synchronises the stream (the fallback search is sized on the host).
cudaError_t launch_remesh(cudaStream_t st, int64_t n, const double* moved5, double* target5, int64_t ntri,
                          const int32_t* tris, const uint32_t* off, const int32_t* adj, double omega,
                          RemeshScratch& s, int64_t* n_fallback, int64_t* n_not_found);
void launch_remesh_targets(cudaStream_t st, int64_t n, const double* grid3, const double* moved5, double* target5);
// k_amr.cu: one generation of the AMR pass at a time (see k_amr.cu).
cudaError_t amr_seed_parents(cudaStream_t st, int64_t n, const int32_t* parent, unsigned long long* hkeys,
                             long long* hvals, int64_t hmask, int* err);
void amr_test(cudaStream_t st, int64_t q0, int64_t m, const int32_t* tris, const double* state5, double vtol,
              double ctol, uint32_t* flag, uint32_t* rank, double* tarea);
void amr_edges(cudaStream_t st, int64_t q0, int64_t m, const uint32_t* flag, const uint32_t* rank,
               const int32_t* tris, int32_t* refined, int64_t* occ_slot, unsigned long long* hkeys, long long* hvals,
               int64_t hmask, int* err);
void amr_creators(cudaStream_t st, int64_t nocc, const int64_t* occ_slot, const long long* hvals, uint32_t* cflag,
                  uint32_t* crank);
void amr_newpts(cudaStream_t st, int64_t nocc, int64_t n, const int32_t* refined, const int32_t* tris,
                const int64_t* occ_slot, const uint32_t* cflag, const uint32_t* crank, long long* hvals,
                double* state5, int32_t* parent);
void amr_split(cudaStream_t st, int64_t nref, int64_t q0, int64_t q1, uint64_t seq0, const int32_t* refined,
               const int64_t* occ_slot, const long long* hvals, const uint32_t* cflag, const double* tarea,
               int32_t* tris, uint64_t* keys, uint32_t* rec_v, double* rec_d, uint8_t* rec_k);
void amr_areas(cudaStream_t st, int64_t nrec, const uint32_t* sv, const int32_t* perm, const double* rec_d,
               const uint8_t* rec_k, double* area);
void amr_project(cudaStream_t st, int64_t i0, int64_t i1, double* state5, double omega);

// In-place exclusive prefix sum of m 32-bit counts; `part` holds
// scan_part_words(m) words of scratch (NULL: one block scans all).
int64_t scan_part_words(int64_t m);
void launch_scan_u32(cudaStream_t st, uint32_t* a, int64_t m, uint32_t* part);

// k_ensemble.cu
void launch_up_leaf_batch(cudaStream_t st, int nleaf, const void* src, const EnsLeaf* leaves,
                          const int32_t* leaf_start, const NodeGeom* node, const int64_t* lev_off, int nmax,
                          int max_leaf_level, double* part);
void launch_up_combine_batch(cudaStream_t st, int njobs, const ProxyJob* jobs, const EnsLeaf* leaves,
                             const double* part, int nmax, const double* vinv, const int32_t* vinv_off,
                             const double4* proxy_pos, int64_t n, void* src);

}  // namespace fss
