// k_ensemble.cu -- the upward pass over the leaves of all members of an
// ensemble (many independent problems advanced together); their pair work
// runs in the persistent pair kernel of k_pairs.cu.
#include <cuda_runtime.h>

#include "device_common.cuh"
#include "kernels.h"
#include "moments.cuh"

namespace fss {

// Upward pass over the leaves of every member.  Leaf i: particles
// [leaf_start[g], leaf_start[g+1]) of the concatenated arrays (g = its
// gleaf, current after each re-sort), its member's leaf level LL, index on
// that level, and the start of its moment slots (LL + 1 levels x KM).
// Every member has 20 * 4^LL leaves and starts at a multiple of four, so
// entries 4 b .. 4 b + 3 are one member's sibling group; block (b, level)
// forms its rows as the single problem's k_up_leaf does (up_row_step).
__global__ void __launch_bounds__(kUpThreads) k_up_leaf_batch(const float4* __restrict__ src, const EnsLeaf* __restrict__ leaves,
                                                       const int32_t* __restrict__ leaf_start,
                                                       const NodeGeom* __restrict__ node,
                                                       const int64_t* __restrict__ lev_off, int nmax, int nleaf,
                                                       double* __restrict__ part) {
    __shared__ double W[kUpLeaves][kUpRows][kUpLd];
    __shared__ double V[kUpLeaves][kUpRows][kUpLd];
    __shared__ double O[kUpLeaves][kMaxK];
    const int l = blockIdx.y;
    const int w = threadIdx.x >> 5;
    const int i = blockIdx.x * kUpLeaves + w;
    const EnsLeaf lf = leaves[min(i, nleaf - 1)];
    // block-uniform: the group's member (its leaf level and level mask)
    if (l > lf.leaf_level || !((lf.level_mask >> l) & 1)) return;
    const int KM = nproxy(nmax);
    const NodeGeom& ng = node[lev_off[l] + (lf.local >> (2 * (lf.leaf_level - l)))];
    if (l == lf.leaf_level) {
        if (i >= nleaf) return;
        leaf_moments<float>(src, leaf_start[lf.gleaf], leaf_start[lf.gleaf + 1], 0.0, 0.0, 0.0, ng, nmax, W[w], V[w],
                            part + lf.part_base + int64_t(l) * KM);
        return;
    }
    if (i < nleaf) {
        leaf_moments<float>(src, leaf_start[lf.gleaf], leaf_start[lf.gleaf + 1], 0.0, 0.0, 0.0, ng, nmax, W[w], V[w],
                            O[w]);
    } else {
        for (int m = threadIdx.x & 31; m < KM; m += 32) O[w][m] = 0.0;
    }
    __syncthreads();
    double* out = part + leaves[blockIdx.x * kUpLeaves].part_base + int64_t(l) * KM;
    for (int m = threadIdx.x; m < KM; m += kUpThreads) out[m] = (O[0][m] + O[1][m]) + (O[2][m] + O[3][m]);
}

// Proxy charges of every member's far clusters: job j sums the rows of its
// leaves (global leaf indices, slots through EnsLeaf::part_base) as the
// single problem's k_up_proxies does (each q_k the same FMA chain).
__global__ void __launch_bounds__(128) k_up_combine_batch(const ProxyJob* __restrict__ jobs,
                                                          const EnsLeaf* __restrict__ leaves,
                                                          const double* __restrict__ part, int nmax,
                                                          const double* __restrict__ vinv,
                                                          const int32_t* __restrict__ vinv_off,
                                                          const double4* __restrict__ proxy_pos, int64_t n,
                                                          float4* __restrict__ src) {
    __shared__ double M[kMaxK];
    // read in place: a copy indexed by a run-time degree (job.off[d]) would sit in local memory
    const ProxyJob& job = jobs[blockIdx.x];
    const int tid = threadIdx.x;
    const int KM = nproxy(nmax);
    if (tid < KM) {
        const int step = up_row_step(job.level, leaves[job.leaf_lo].leaf_level);
        const int64_t off = int64_t(job.level) * KM + tid;
        M[tid] = sum_rows4([&](int r) { return part[leaves[job.leaf_lo + r * step].part_base + off]; },
                           (job.leaf_hi - job.leaf_lo) / step);
    }
    __syncthreads();
    for (int d = 0; d <= nmax; d++) {
        if (!((job.degmask >> d) & 1)) continue;
        const int K = nproxy(d);
        const double* V = vinv + vinv_off[d];
        for (int k = tid; k < K; k += 128) {
            double q = 0;
            for (int m = 0; m < K; m++) q = fma(V[m * K + k], M[m], q);
            const int64_t slot = int64_t(job.off[d]) + k;
            const double4 y = proxy_pos[slot - n];
            src[slot] = make_float4(float(y.x), float(y.y), float(y.z), float(q));
        }
    }
}

void launch_up_leaf_batch(cudaStream_t st, int nleaf, const void* src, const EnsLeaf* leaves,
                          const int32_t* leaf_start, const NodeGeom* node, const int64_t* lev_off, int nmax,
                          int max_leaf_level, double* part) {
    if (nleaf == 0) return;
    const dim3 grid(unsigned((nleaf + kUpLeaves - 1) / kUpLeaves), unsigned(max_leaf_level + 1));
    k_up_leaf_batch<<<grid, kUpThreads, 0, st>>>(
        static_cast<const float4*>(src), leaves, leaf_start, node, lev_off, nmax, nleaf, part);
}

void launch_up_combine_batch(cudaStream_t st, int njobs, const ProxyJob* jobs, const EnsLeaf* leaves,
                             const double* part, int nmax, const double* vinv, const int32_t* vinv_off,
                             const double4* proxy_pos, int64_t n, void* src) {
    if (njobs == 0) return;
    k_up_combine_batch<<<njobs, 128, 0, st>>>(jobs, leaves, part, nmax, vinv, vinv_off, proxy_pos, n,
                                             static_cast<float4*>(src));
}

}  // namespace fss
