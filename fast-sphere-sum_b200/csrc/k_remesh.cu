// k_remesh.cu -- the remesh step (remesh.h:109-178 regrid_points2 with
// helpers.h:251-265 tri_interp): particles that moved with the flow are put
// back on the regular grid.  Every grid point keeps its position and takes
// the absolute vorticity (zeta + 2 omega z) and the tracer interpolated with
// normalised barycentric coordinates from the first triangle of the moved
// mesh that contains it: first among the triangles adjacent to its own
// vertex (in increasing index order), then among all triangles (index
// order).  The containment test and the coordinates use the explicitly
// rounded LU of the tree assignment, so results are bit-identical to the
// reference's FP64 arithmetic with the same adjacency.
#include <cuda_runtime.h>

#include "device_common.cuh"
#include "exact_lu.cuh"
#include "kernels.h"

namespace fss {

__device__ __forceinline__ bool tri_contains(const double* __restrict__ moved5, const int32_t* tv, const double* p,
                                             double* c) {
    cone_coords_exact(moved5 + 5 * int64_t(tv[0]), moved5 + 5 * int64_t(tv[1]), moved5 + 5 * int64_t(tv[2]), p, c);
    return c[0] >= 0 && c[1] >= 0 && c[2] >= 0;
}

// helpers.h:152-157 norm_barycoords, then helpers.h:251-265 tri_interp.
__device__ __forceinline__ void tri_interp_exact(const double* __restrict__ moved5, const int32_t* tv, double* t,
                                                 double omega, const double* c) {
    const double r = __ddiv_rn(1.0, __dadd_rn(__dadd_rn(c[0], c[1]), c[2]));
    const double b0 = __dmul_rn(c[0], r), b1 = __dmul_rn(c[1], r), b2 = __dmul_rn(c[2], r);
    const double* v1 = moved5 + 5 * int64_t(tv[0]);
    const double* v2 = moved5 + 5 * int64_t(tv[1]);
    const double* v3 = moved5 + 5 * int64_t(tv[2]);
    const double w = __dmul_rn(2.0, omega);
    const double a1 = __dadd_rn(v1[3], __dmul_rn(w, v1[2]));
    const double a2 = __dadd_rn(v2[3], __dmul_rn(w, v2[2]));
    const double a3 = __dadd_rn(v3[3], __dmul_rn(w, v3[2]));
    const double av = __dadd_rn(__dadd_rn(__dmul_rn(b0, a1), __dmul_rn(b1, a2)), __dmul_rn(b2, a3));
    t[3] = __dsub_rn(av, __dmul_rn(w, t[2]));
    t[4] = __dadd_rn(__dadd_rn(__dmul_rn(b0, v1[4]), __dmul_rn(b1, v2[4])), __dmul_rn(b2, v3[4]));
}

// One thread per grid point: the triangles adjacent to its vertex
// (adjacency adj[off[i] .. off[i+1]): corner ids 3 t + c in list order).
// Points found in none are listed in `failed`.
__global__ void k_remesh_adjacent(int64_t n, const double* __restrict__ moved5, double* __restrict__ target5,
                                  const int32_t* __restrict__ tris, const uint32_t* __restrict__ off,
                                  const int32_t* __restrict__ adj, double omega, int32_t* __restrict__ failed,
                                  int32_t* __restrict__ nfailed) {
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double* t = target5 + 5 * i;
    const double p[3] = {t[0], t[1], t[2]};
    double c[3];
    for (uint32_t a = off[i]; a < off[i + 1]; a++) {
        const int32_t* tv = tris + 3 * int64_t(adj[a] / 3);
        if (tri_contains(moved5, tv, p, c)) {
            tri_interp_exact(moved5, tv, t, omega, c);
            return;
        }
    }
    failed[atomicAdd(nfailed, 1)] = int32_t(i);
}

// ---- vertex -> triangles adjacency (count, scan, fill, per-vertex sort)
__global__ void k_adj_count(int64_t n, int64_t ntri, const int32_t* __restrict__ tris, uint32_t* __restrict__ cnt,
                            uint32_t* __restrict__ bad) {
    const int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (j >= 3 * ntri) return;
    const int32_t v = tris[j];
    if (v < 0 || int64_t(v) >= n)
        atomicOr(bad, 1u);
    else
        atomicAdd(cnt + v, 1u);
}

__global__ void k_adj_fill(int64_t n, int64_t ntri, const int32_t* __restrict__ tris, uint32_t* __restrict__ cur,
                           int32_t* __restrict__ adj) {
    const int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (j >= 3 * ntri) return;
    const int32_t v = tris[j];
    if (v >= 0 && int64_t(v) < n) adj[atomicAdd(cur + v, 1u)] = int32_t(j);
}

// Each vertex's list into list order: increasing corner key, or increasing
// corner id (= triangle order) without keys (insertion sort: a few entries
// per vertex on a triangulated sphere).
__global__ void k_adj_sort(int64_t n, const uint32_t* __restrict__ off, const uint64_t* __restrict__ keys,
                           int32_t* __restrict__ adj) {
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t a = off[i], b = off[i + 1];
    for (uint32_t k = a + 1; k < b; k++) {
        const int32_t x = adj[k];
        const uint64_t kx = keys ? keys[x] : uint64_t(x);
        uint32_t q = k;
        while (q > a && (keys ? keys[adj[q - 1]] : uint64_t(adj[q - 1])) > kx) {
            adj[q] = adj[q - 1];
            q--;
        }
        adj[q] = x;
    }
}

cudaError_t launch_remesh_adjacency(cudaStream_t st, int64_t n, int64_t ntri, const int32_t* tris,
                                    const uint64_t* keys, uint32_t* off, int32_t* adj, RemeshScratch& s,
                                    bool* valid) {
    cudaError_t e;
    *valid = false;
    if ((e = s.scal.ensure(2 * sizeof(uint32_t))) != cudaSuccess ||
        (e = s.adj_cur.ensure(size_t(n + 1) * sizeof(uint32_t))) != cudaSuccess ||
        (e = s.part.ensure(size_t(scan_part_words(n + 1)) * sizeof(uint32_t))) != cudaSuccess)
        return e;
    uint32_t* flag = s.scal.as<uint32_t>();
    uint32_t* cur = s.adj_cur.as<uint32_t>();
    if ((e = cudaMemsetAsync(off, 0, size_t(n + 1) * sizeof(uint32_t), st)) != cudaSuccess ||
        (e = cudaMemsetAsync(flag, 0, sizeof(uint32_t), st)) != cudaSuccess)
        return e;
    const unsigned g3 = unsigned((3 * ntri + 255) / 256);
    k_adj_count<<<g3, 256, 0, st>>>(n, ntri, tris, off, flag);
    uint32_t hbad = 1;
    if ((e = cudaMemcpyAsync(&hbad, flag, sizeof(uint32_t), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return e;
    if (hbad) return cudaGetLastError();
    launch_scan_u32(st, off, n + 1, s.part.as<uint32_t>());
    if ((e = cudaMemcpyAsync(cur, off, size_t(n + 1) * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st)) !=
        cudaSuccess)
        return e;
    k_adj_fill<<<g3, 256, 0, st>>>(n, ntri, tris, cur, adj);
    k_adj_sort<<<unsigned((n + 255) / 256), 256, 0, st>>>(n, off, keys, adj);
    *valid = true;
    return cudaGetLastError();
}

// One block per listed point: the first triangle (lowest index) of the whole
// moved mesh that contains it (few listed points).  Points in no triangle
// keep their values and are counted in `bad`.
constexpr int kSearchThreads = 256;
__global__ void __launch_bounds__(kSearchThreads) k_remesh_search(int32_t nfail, const int32_t* __restrict__ failed,
                                                                  const double* __restrict__ moved5,
                                                                  double* __restrict__ target5, int64_t ntri,
                                                                  const int32_t* __restrict__ tris, double omega,
                                                                  int32_t* __restrict__ bad) {
    __shared__ int64_t first;
    for (int32_t f = blockIdx.x; f < nfail; f += gridDim.x) {
        const int64_t i = failed[f];
        double* t = target5 + 5 * i;
        const double p[3] = {t[0], t[1], t[2]};
        if (threadIdx.x == 0) first = ntri;
        __syncthreads();
        int64_t mine = ntri;
        double c[3];
        for (int64_t j = threadIdx.x; j < ntri; j += kSearchThreads)
            if (tri_contains(moved5, tris + 3 * j, p, c)) {
                mine = j;
                break;
            }
        if (mine < ntri) atomicMin(reinterpret_cast<unsigned long long*>(&first), (unsigned long long)mine);
        __syncthreads();
        if (threadIdx.x == 0) {
            if (first < ntri) {
                tri_contains(moved5, tris + 3 * first, p, c);
                tri_interp_exact(moved5, tris + 3 * first, t, omega, c);
            } else {
                atomicAdd(bad, 1);
            }
        }
        __syncthreads();
    }
}

// ---- search over all triangles on a cell grid (many listed points)
//
// Cap of a triangle: with u_k = v_k/|v_k|, c = (u_1+u_2+u_3)/|u_1+u_2+u_3|
// and m = min_k u_k.c, every point p of the cone {sum a_k v_k, a_k >= 0}
// satisfies (p/|p|).c >= m, since |sum b_k u_k| <= sum b_k.  The LU test is
// backward stable (partial pivoting: it decides for vertices perturbed by
// ~1e-15), so a point it places inside still has (p/|p|).c >= m - 1e-13 when
// m >= 1/2 (then |u_1+u_2+u_3| >= 3/2).  Such a cap, widened by 1e-10, lies
// in the ball of chord radius sqrt(2 - 2 cos r) about c, so the triangle can
// contain only points whose unit vector falls in the cells that ball's box
// covers on a G^3 grid over [-1, 1]^3.  Triangles with m < 1/2, a zero pivot
// (tested for every point, as the LU then returns b = p), non-finite values,
// or a box of more than kMaxCells cells go to a list tested for every point.
// A point takes the lowest index that passes the exact test among its
// cell's triangles and that list: the same triangle as a scan in index
// order.  Points whose direction is undefined (zero or non-finite) scan all
// triangles.
constexpr int kMaxCells = 64;
constexpr double kCapSlack = 1e-10;

__device__ __forceinline__ int cell_of(double x, int G) {
    const double f = floor(__dmul_rn(__dadd_rn(x, 1.0), 0.5 * G));  // G a power of two: 0.5 * G exact
    return f < 0 ? 0 : (f > G - 1 ? G - 1 : int(f));
}

// Cap (c, cos r) of triangle j and its cell box; false when the triangle
// belongs to the list tested for every point.
__device__ __forceinline__ bool tri_cap(const double* __restrict__ moved5, const int32_t* tv, int G, double4* cap,
                                        int lo[3], int hi[3]) {
    const double* v[3] = {moved5 + 5 * int64_t(tv[0]), moved5 + 5 * int64_t(tv[1]), moved5 + 5 * int64_t(tv[2])};
    double u[3][3], c[3] = {0, 0, 0};
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const double r = sqrt(v[k][0] * v[k][0] + v[k][1] * v[k][1] + v[k][2] * v[k][2]);
#pragma unroll
        for (int d = 0; d < 3; d++) {
            u[k][d] = v[k][d] / r;
            c[d] += u[k][d];
        }
    }
    const double cn = sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
#pragma unroll
    for (int d = 0; d < 3; d++) c[d] /= cn;
    double m = 1.0;
#pragma unroll
    for (int k = 0; k < 3; k++) m = fmin(m, u[k][0] * c[0] + u[k][1] * c[1] + u[k][2] * c[2]);
    const double cosr = m - kCapSlack;
    *cap = make_double4(c[0], c[1], c[2], cosr);
    if (!(m >= 0.5) || !isfinite(c[0]) || !isfinite(c[1]) || !isfinite(c[2])) return false;
    double b[3];
    const double q[3] = {c[0], c[1], c[2]};
    if (cone_coords_exact(v[0], v[1], v[2], q, b)) return false;  // zero pivot
    const double rho = __dadd_rn(__dsqrt_rn(__dsub_rn(2.0, __dmul_rn(2.0, cosr))), 1e-9);
    int ncell = 1;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        lo[d] = cell_of(__dsub_rn(c[d], rho), G);
        hi[d] = cell_of(__dadd_rn(c[d], rho), G);
        ncell *= hi[d] - lo[d] + 1;
    }
    return ncell <= kMaxCells;
}

// Cell box packed 8 bits per bound (G <= 128); kNoBox marks the list
// tested for every point.
constexpr uint64_t kNoBox = ~uint64_t(0);
__device__ __forceinline__ void unpack_box(uint64_t b, int lo[3], int hi[3]) {
#pragma unroll
    for (int d = 0; d < 3; d++) {
        lo[d] = int((b >> (16 * d)) & 255u);
        hi[d] = int((b >> (16 * d + 8)) & 255u);
    }
}

// Caps, cell boxes, per-cell counts, the list tested for every point and
// the entry total.
__global__ void k_grid_count(int64_t ntri, const double* __restrict__ moved5, const int32_t* __restrict__ tris, int G,
                             double4* __restrict__ caps, uint64_t* __restrict__ box, uint32_t* __restrict__ cnt,
                             int32_t* __restrict__ glist, uint32_t* __restrict__ scal) {
    const int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (j >= ntri) return;
    double4 cap;
    int lo[3], hi[3];
    if (!tri_cap(moved5, tris + 3 * j, G, &cap, lo, hi)) {
        caps[j] = make_double4(0.0, 0.0, 0.0, -2.0);  // passes every cap test
        box[j] = kNoBox;
        glist[atomicAdd(scal + 1, 1u)] = int32_t(j);
        return;
    }
    caps[j] = cap;
    uint64_t b = 0;
#pragma unroll
    for (int d = 0; d < 3; d++) b |= (uint64_t(lo[d]) | (uint64_t(hi[d]) << 8)) << (16 * d);
    box[j] = b;
    uint32_t k = 0;
    for (int x = lo[0]; x <= hi[0]; x++)
        for (int y = lo[1]; y <= hi[1]; y++)
            for (int z = lo[2]; z <= hi[2]; z++, k++) atomicAdd(cnt + (int64_t(x) * G + y) * G + z, 1u);
    atomicAdd(scal, k);
}

// After the exclusive scan cnt[cell] = start of the cell; each entry takes
// cnt[cell]++, leaving cnt[cell] = end of the cell (= start of cell + 1).
__global__ void k_grid_fill(int64_t ntri, const uint64_t* __restrict__ box, int G, uint32_t* __restrict__ cnt,
                            int32_t* __restrict__ ent) {
    const int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (j >= ntri) return;
    const uint64_t b = box[j];
    if (b == kNoBox) return;
    int lo[3], hi[3];
    unpack_box(b, lo, hi);
    for (int x = lo[0]; x <= hi[0]; x++)
        for (int y = lo[1]; y <= hi[1]; y++)
            for (int z = lo[2]; z <= hi[2]; z++) ent[atomicAdd(cnt + (int64_t(x) * G + y) * G + z, 1u)] = int32_t(j);
}

// One warp per listed point.
constexpr int kGridWarps = 8;
__global__ void __launch_bounds__(32 * kGridWarps)
    k_remesh_grid_search(int32_t nfail, const int32_t* __restrict__ failed, const double* __restrict__ moved5,
                         double* __restrict__ target5, int64_t ntri, const int32_t* __restrict__ tris,
                         const double4* __restrict__ caps, int G, const uint32_t* __restrict__ cend,
                         const int32_t* __restrict__ ent, const int32_t* __restrict__ glist, int32_t nglob,
                         double omega, int32_t* __restrict__ bad) {
    const int lane = threadIdx.x & 31;
    const int32_t nwarp = gridDim.x * kGridWarps;
    for (int32_t f = blockIdx.x * kGridWarps + (threadIdx.x >> 5); f < nfail; f += nwarp) {
        const int64_t i = failed[f];
        double* t = target5 + 5 * i;
        const double p[3] = {t[0], t[1], t[2]};
        uint32_t best = uint32_t(ntri);
        double c[3];
        const double r = sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
        if (!(r > 0) || !isfinite(r)) {
            for (int64_t j = lane; j < ntri; j += 32)
                if (tri_contains(moved5, tris + 3 * j, p, c)) {
                    best = uint32_t(j);
                    break;
                }
        } else {
            const double q[3] = {p[0] / r, p[1] / r, p[2] / r};
            const int64_t cell = (int64_t(cell_of(q[0], G)) * G + cell_of(q[1], G)) * G + cell_of(q[2], G);
            const uint32_t e0 = cell ? cend[cell - 1] : 0u, e1 = cend[cell];
            for (uint32_t k = e0 + lane; k < e1; k += 32) {
                const int32_t j = ent[k];
                if (uint32_t(j) >= best) continue;
                const double4 cp = caps[j];
                if (q[0] * cp.x + q[1] * cp.y + q[2] * cp.z < cp.w) continue;
                if (tri_contains(moved5, tris + 3 * int64_t(j), p, c)) best = uint32_t(j);
            }
            for (int32_t k = lane; k < nglob; k += 32) {
                const int32_t j = glist[k];
                if (uint32_t(j) < best && tri_contains(moved5, tris + 3 * int64_t(j), p, c)) best = uint32_t(j);
            }
        }
        best = __reduce_min_sync(0xffffffffu, best);
        if (lane == 0) {
            if (best < uint32_t(ntri)) {
                const int32_t* tv = tris + 3 * int64_t(best);
                tri_contains(moved5, tv, p, c);
                tri_interp_exact(moved5, tv, t, omega, c);
            } else {
                atomicAdd(bad, 1);
            }
        }
        __syncwarp();
    }
}

// Power-of-two grid side with cells about three mean triangle edges wide.
static int grid_side(int64_t ntri) {
    const double edge = sqrt(4.0 * (4.0 * 3.141592653589793 / double(ntri)) / sqrt(3.0));
    int G = 4;
    while (G < 128 && 2.0 / (2 * G) > 3.0 * edge) G *= 2;
    return G;
}

static cudaError_t grid_search(cudaStream_t st, int32_t nfail, const int32_t* failed, const double* moved5,
                               double* target5, int64_t ntri, const int32_t* tris, double omega, int32_t* bad,
                               RemeshScratch& s) {
    const int G = grid_side(ntri);
    const int64_t ncell = int64_t(G) * G * G;
    cudaError_t e;
    if ((e = s.caps.ensure(size_t(ntri) * sizeof(double4))) != cudaSuccess ||
        (e = s.box.ensure(size_t(ntri) * sizeof(uint64_t))) != cudaSuccess ||
        (e = s.cells.ensure(size_t(ncell) * sizeof(uint32_t))) != cudaSuccess ||
        (e = s.glist.ensure(size_t(ntri) * sizeof(int32_t))) != cudaSuccess ||
        (e = s.scal.ensure(2 * sizeof(uint32_t))) != cudaSuccess ||
        (e = s.part.ensure(size_t(scan_part_words(ncell)) * sizeof(uint32_t))) != cudaSuccess)
        return e;
    double4* caps = s.caps.as<double4>();
    uint64_t* box = s.box.as<uint64_t>();
    uint32_t* cnt = s.cells.as<uint32_t>();
    int32_t* glist = s.glist.as<int32_t>();
    uint32_t* scal = s.scal.as<uint32_t>();
    if ((e = cudaMemsetAsync(cnt, 0, size_t(ncell) * sizeof(uint32_t), st)) != cudaSuccess ||
        (e = cudaMemsetAsync(scal, 0, 2 * sizeof(uint32_t), st)) != cudaSuccess)
        return e;
    const unsigned tb = unsigned((ntri + 255) / 256);
    k_grid_count<<<tb, 256, 0, st>>>(ntri, moved5, tris, G, caps, box, cnt, glist, scal);
    launch_scan_u32(st, cnt, ncell, s.part.as<uint32_t>());
    uint32_t hs[2];
    if ((e = cudaMemcpyAsync(hs, scal, sizeof(hs), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return e;
    // every triangle adds at most kMaxCells entries: the total fits 32 bits
    if ((e = s.ent.ensure(size_t(hs[0] ? hs[0] : 1) * sizeof(int32_t))) != cudaSuccess) return e;
    int32_t* ent = s.ent.as<int32_t>();
    k_grid_fill<<<tb, 256, 0, st>>>(ntri, box, G, cnt, ent);
    const int32_t blocks = (nfail + kGridWarps - 1) / kGridWarps < 8 * 148 ? (nfail + kGridWarps - 1) / kGridWarps
                                                                           : 8 * 148;
    k_remesh_grid_search<<<blocks, 32 * kGridWarps, 0, st>>>(nfail, failed, moved5, target5, ntri, tris, caps, G, cnt,
                                                             ent, glist, int32_t(hs[1]), omega, bad);
    return cudaGetLastError();
}

// Grid positions with the moved state's zeta and tracer (the values kept by
// a point found in no triangle).
__global__ void k_remesh_targets(int64_t n, const double* __restrict__ grid3, const double* __restrict__ moved5,
                                 double* __restrict__ target5) {
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double* t = target5 + 5 * i;
    t[0] = grid3[3 * i];
    t[1] = grid3[3 * i + 1];
    t[2] = grid3[3 * i + 2];
    t[3] = moved5[5 * i + 3];
    t[4] = moved5[5 * i + 4];
}

// Up to this many listed points a block scans all triangles per point.
constexpr int32_t kDirectSearchMax = 64;

cudaError_t launch_remesh(cudaStream_t st, int64_t n, const double* moved5, double* target5, int64_t ntri,
                          const int32_t* tris, const uint32_t* off, const int32_t* adj, double omega,
                          RemeshScratch& s, int64_t* n_fallback, int64_t* n_not_found) {
    if (n == 0) return cudaSuccess;
    cudaError_t e;
    if ((e = s.failed.ensure(size_t(n) * sizeof(int32_t))) != cudaSuccess ||
        (e = s.counters.ensure(2 * sizeof(int32_t))) != cudaSuccess)
        return e;
    int32_t* failed = s.failed.as<int32_t>();
    int32_t* counters = s.counters.as<int32_t>();
    if ((e = cudaMemsetAsync(counters, 0, 2 * sizeof(int32_t), st)) != cudaSuccess) return e;
    k_remesh_adjacent<<<unsigned((n + 127) / 128), 128, 0, st>>>(n, moved5, target5, tris, off, adj, omega, failed,
                                                                 counters);
    int32_t nfail = 0;
    if ((e = cudaMemcpyAsync(&nfail, counters, sizeof(int32_t), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return e;
    int32_t nbad = 0;
    if (nfail > 0) {
        if (nfail <= kDirectSearchMax || ntri == 0) {
            k_remesh_search<<<nfail, kSearchThreads, 0, st>>>(nfail, failed, moved5, target5, ntri, tris, omega,
                                                              counters + 1);
        } else if ((e = grid_search(st, nfail, failed, moved5, target5, ntri, tris, omega, counters + 1, s)) !=
                   cudaSuccess) {
            return e;
        }
        if ((e = cudaMemcpyAsync(&nbad, counters + 1, sizeof(int32_t), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
            (e = cudaStreamSynchronize(st)) != cudaSuccess)
            return e;
    }
    if (n_fallback) *n_fallback = nfail;
    if (n_not_found) *n_not_found = nbad;
    return cudaGetLastError();
}

void launch_remesh_targets(cudaStream_t st, int64_t n, const double* grid3, const double* moved5, double* target5) {
    if (n == 0) return;
    k_remesh_targets<<<unsigned((n + 255) / 256), 256, 0, st>>>(n, grid3, moved5, target5);
}

}  // namespace fss
