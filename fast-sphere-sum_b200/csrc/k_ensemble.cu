// k_ensemble.cu -- the upward pass over the leaves of all members of an
// ensemble (many independent problems advanced together); their pair work
// runs in the persistent pair kernel of k_pairs.cu.
#include <cuda_runtime.h>

#include "device_common.cuh"
#include "kernels.h"
#include "moments.cuh"

namespace fss {

// Upward pass over the leaves of every member.  Leaf g: particles
// [leaf_start[g], leaf_start[g+1]) of the concatenated arrays (current after
// each re-sort), leaf level LL, index within its member's leaf level, and
// the start of its moment slots (LL + 1 levels x KM); moments as for one
// problem (leaf_moments).
__global__ void __launch_bounds__(kUpThreads) k_up_leaf_batch(const float4* __restrict__ src, const EnsLeaf* __restrict__ leaves,
                                                       const int32_t* __restrict__ leaf_start,
                                                       const NodeGeom* __restrict__ node,
                                                       const int64_t* __restrict__ lev_off, int nmax, int nleaf,
                                                       double* __restrict__ part) {
    __shared__ double W[kUpLeaves][kUpRows][kUpLd];
    __shared__ double V[kUpLeaves][kUpRows][kUpLd];
    const int w = threadIdx.x >> 5;
    const int i = blockIdx.x * kUpLeaves + w;
    if (i >= nleaf) return;  // whole warps; no block-wide barrier follows
    const EnsLeaf lf = leaves[i];
    const int a0 = leaf_start[lf.gleaf], a1 = leaf_start[lf.gleaf + 1];
    const int KM = nproxy(nmax);
    for (int l = 0; l <= lf.leaf_level; l++) {
        if (!((lf.level_mask >> l) & 1)) continue;
        const NodeGeom ng = node[lev_off[l] + (lf.local >> (2 * (lf.leaf_level - l)))];
        leaf_moments<float>(src, a0, a1, 0.0, 0.0, 0.0, ng, nmax, W[w], V[w], part + lf.part_base + int64_t(l) * KM);
    }
}

// Proxy charges of every member's far clusters: job j sums the moments of
// its leaves (global leaf indices, slots through EnsLeaf::part_base).
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
        // four independent sums over the face's leaves, as the single
        // problem's combine forms them (same order, same result)
        const int64_t off = int64_t(job.level) * KM + tid;
        const int nl = job.leaf_hi - job.leaf_lo;
        double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
        int lf = 0;
        for (; lf + 4 <= nl; lf += 4) {
            s0 += part[leaves[job.leaf_lo + lf + 0].part_base + off];
            s1 += part[leaves[job.leaf_lo + lf + 1].part_base + off];
            s2 += part[leaves[job.leaf_lo + lf + 2].part_base + off];
            s3 += part[leaves[job.leaf_lo + lf + 3].part_base + off];
        }
        for (; lf < nl; lf++) s0 += part[leaves[job.leaf_lo + lf].part_base + off];
        M[tid] = (s0 + s1) + (s2 + s3);
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
                          double* part) {
    if (nleaf == 0) return;
    k_up_leaf_batch<<<unsigned((nleaf + kUpLeaves - 1) / kUpLeaves), kUpThreads, 0, st>>>(
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
