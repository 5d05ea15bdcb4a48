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
// (adjacency adj[off[i] .. off[i+1]) in increasing triangle order).  Points
// found in none are listed in `failed`.
__global__ void k_remesh_adjacent(int64_t n, const double* __restrict__ moved5, double* __restrict__ target5,
                                  const int32_t* __restrict__ tris, const int32_t* __restrict__ off,
                                  const int32_t* __restrict__ adj, double omega, int32_t* __restrict__ failed,
                                  int32_t* __restrict__ nfailed) {
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double* t = target5 + 5 * i;
    const double p[3] = {t[0], t[1], t[2]};
    double c[3];
    for (int32_t a = off[i]; a < off[i + 1]; a++) {
        const int32_t* tv = tris + 3 * int64_t(adj[a]);
        if (tri_contains(moved5, tv, p, c)) {
            tri_interp_exact(moved5, tv, t, omega, c);
            return;
        }
    }
    failed[atomicAdd(nfailed, 1)] = int32_t(i);
}

// One block per listed point: the first triangle (lowest index) of the whole
// moved mesh that contains it.  Points in no triangle keep their values and
// are counted in `bad`.
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

cudaError_t launch_remesh(cudaStream_t st, int64_t n, const double* moved5, double* target5, int64_t ntri,
                          const int32_t* tris, const int32_t* off, const int32_t* adj, double omega,
                          int32_t* failed, int32_t* counters, int64_t* n_fallback, int64_t* n_not_found) {
    if (n == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(counters, 0, 2 * sizeof(int32_t), st);
    if (e != cudaSuccess) return e;
    k_remesh_adjacent<<<unsigned((n + 127) / 128), 128, 0, st>>>(n, moved5, target5, tris, off, adj, omega, failed,
                                                                 counters);
    int32_t nfail = 0;
    if ((e = cudaMemcpyAsync(&nfail, counters, sizeof(int32_t), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return e;
    int32_t nbad = 0;
    if (nfail > 0) {
        const int blocks = nfail < 4 * 148 ? nfail : 4 * 148;
        k_remesh_search<<<blocks, kSearchThreads, 0, st>>>(nfail, failed, moved5, target5, ntri, tris, omega,
                                                           counters + 1);
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
