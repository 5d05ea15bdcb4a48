// k_amr.cu -- adaptive mesh refinement (amr.h:13-178 amr) on the GPU.
//
// The reference visits triangles in index order while their count grows:
// a split triangle keeps its first child at its own index (not visited
// again) and appends the other three, which the same pass visits later.  A
// triangle's decision reads only its corners' state, and corners exist
// before the triangle does, so the pass is a sequence of generations: the
// triangles [q0, q1) are tested together, the r-th split one (in index
// order) appends children q1 + 3r .. q1 + 3r + 2, and those form the next
// generation.  What depends on the order is made explicit:
//   * a shared edge's midpoint is created by its first occurrence (position
//     3r + e, edges 12, 23, 31) among edges without a midpoint yet: an
//     atomicMin over positions in a hash of parent pairs (check_in_vec3);
//     new points are numbered by a scan over those positions;
//   * area updates (-A/6 at the corners, +A/6 or = A/6 at the midpoints)
//     are recorded in processing order and applied per point in that order
//     after the pass (decisions never read areas);
//   * the reference's vert_tris lists become one ordering key per triangle
//     corner (replace() keeps the parent's key, push_back appends
//     2^40 + 9 s + slot, s the running refinement number).
// The area formula (helpers.h:94-115 sphere_tri_area) uses explicitly
// rounded arithmetic around CUDA's acos, tan and atan.
#include <cuda_runtime.h>

#include "device_common.cuh"
#include "kernels.h"

namespace fss {

constexpr uint64_t kAmrKeyAppend = uint64_t(1) << 40;
constexpr long long kAmrPending = 1ll << 62;
constexpr unsigned long long kHashEmpty = ~0ull;

__device__ __forceinline__ double dot_self(const double* x) {
    double s = __dmul_rn(x[0], x[0]);
    s = __dadd_rn(s, __dmul_rn(x[1], x[1]));
    return __dadd_rn(s, __dmul_rn(x[2], x[2]));
}

// helpers.h:94-115 sphere_tri_area on the unit sphere.
__device__ double amr_tri_area(const double* p1, const double* p2, const double* p3) {
    double d23[3], d31[3], d12[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        d23[i] = __dsub_rn(p2[i], p3[i]);
        d31[i] = __dsub_rn(p3[i], p1[i]);
        d12[i] = __dsub_rn(p1[i], p2[i]);
    }
    const double a = acos(__dsub_rn(1.0, __dmul_rn(0.5, dot_self(d23))));
    const double b = acos(__dsub_rn(1.0, __dmul_rn(0.5, dot_self(d31))));
    const double c = acos(__dsub_rn(1.0, __dmul_rn(0.5, dot_self(d12))));
    const double s = __ddiv_rn(__dadd_rn(__dadd_rn(a, b), c), 2.0);
    double z = __dmul_rn(tan(__ddiv_rn(s, 2.0)), tan(__ddiv_rn(__dsub_rn(s, a), 2.0)));
    z = __dmul_rn(z, tan(__ddiv_rn(__dsub_rn(s, b), 2.0)));
    z = __dmul_rn(z, tan(__ddiv_rn(__dsub_rn(s, c), 2.0)));
    return __dmul_rn(4.0, atan(__dsqrt_rn(z)));
}

__device__ __forceinline__ uint64_t hash_mix(uint64_t x) {
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ull;
    x ^= x >> 33;
    return x;
}

// Slot of `key` (inserted when absent); -1 when the table is full.
__device__ int64_t hash_slot(unsigned long long* hkeys, int64_t hmask, uint64_t key) {
    int64_t h = int64_t(hash_mix(key) & uint64_t(hmask));
    for (int64_t probe = 0; probe <= hmask; probe++) {
        const unsigned long long k = hkeys[h];
        if (k == key) return h;
        if (k == kHashEmpty) {
            const unsigned long long prev = atomicCAS(hkeys + h, kHashEmpty, (unsigned long long)key);
            if (prev == kHashEmpty || prev == key) return h;
        }
        h = (h + 1) & hmask;
    }
    return -1;
}

__device__ __forceinline__ uint64_t edge_key(int32_t a, int32_t b) {
    const uint32_t lo = uint32_t(a < b ? a : b), hi = uint32_t(a < b ? b : a);
    return (uint64_t(lo) << 32) | hi;
}

// Parent pairs given at creation: the smallest index of each pair wins
// (check_in_vec3 returns the first); (0, 0) marks a primitive point.
__global__ void k_amr_seed_parents(int64_t n, const int32_t* __restrict__ parent, unsigned long long* hkeys,
                                   long long* hvals, int64_t hmask, int* err) {
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t a = parent[2 * i], b = parent[2 * i + 1];
    if (a == 0 && b == 0) return;
    const int64_t h = hash_slot(hkeys, hmask, (uint64_t(uint32_t(a)) << 32) | uint32_t(b));
    if (h < 0) {
        atomicExch(err, 1);
        return;
    }
    atomicMin(hvals + h, (long long)i);
}

// Generation test: flag and area of triangles q0 .. q0 + m - 1.
__global__ void k_amr_test(int64_t q0, int64_t m, const int32_t* __restrict__ tris, const double* __restrict__ state5,
                           double vtol, double ctol, uint32_t* __restrict__ flag, uint32_t* __restrict__ rank,
                           double* __restrict__ tarea) {
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= m) return;
    const int32_t* tv = tris + 3 * (q0 + t);
    const double* p1 = state5 + 5 * int64_t(tv[0]);
    const double* p2 = state5 + 5 * int64_t(tv[1]);
    const double* p3 = state5 + 5 * int64_t(tv[2]);
    const double vor1 = p1[3], vor2 = p2[3], vor3 = p3[3];
    double mx = (vor2 < vor3) ? vor3 : vor2;  // std::max(vor1, std::max(vor2, vor3))
    mx = (vor1 < mx) ? mx : vor1;
    double mn = (vor3 < vor2) ? vor3 : vor2;  // std::min
    mn = (mn < vor1) ? mn : vor1;
    const double A = amr_tri_area(p1, p2, p3);
    const double circ = __ddiv_rn(__dmul_rn(A, fabs(__dadd_rn(__dadd_rn(vor1, vor2), vor3))), 3.0);
    const uint32_t f = (__dsub_rn(mx, mn) > vtol || circ > ctol) ? 1u : 0u;
    flag[t] = f;
    rank[t] = f;
    tarea[t] = A;
}

// Split triangles: their list, and each edge's first position in the hash.
__global__ void k_amr_edges(int64_t q0, int64_t m, const uint32_t* __restrict__ flag, const uint32_t* __restrict__ rank,
                            const int32_t* __restrict__ tris, int32_t* __restrict__ refined,
                            int64_t* __restrict__ occ_slot, unsigned long long* hkeys, long long* hvals,
                            int64_t hmask, int* err) {
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= m || !flag[t]) return;
    const int64_t r = rank[t], j = q0 + t;
    refined[r] = int32_t(j);
    const int32_t v[3] = {tris[3 * j], tris[3 * j + 1], tris[3 * j + 2]};
#pragma unroll
    for (int e = 0; e < 3; e++) {
        const int64_t h = hash_slot(hkeys, hmask, edge_key(v[e], v[(e + 1) % 3]));
        occ_slot[3 * r + e] = h;
        if (h < 0) {
            atomicExch(err, 1);
            continue;
        }
        atomicMin(hvals + h, kAmrPending + (long long)(3 * r + e));
    }
}

// First occurrences of edges without a midpoint.
__global__ void k_amr_creators(int64_t nocc, const int64_t* __restrict__ occ_slot, const long long* __restrict__ hvals,
                               uint32_t* __restrict__ cflag, uint32_t* __restrict__ crank) {
    const int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= nocc) return;
    const int64_t h = occ_slot[p];
    const uint32_t f = (h >= 0 && hvals[h] == kAmrPending + (long long)p) ? 1u : 0u;
    cflag[p] = f;
    crank[p] = f;
}

// New midpoints n + crank: state (v_a + v_b) / 2 over all five components
// (v12 = v1 + v2, v23 = v2 + v3, v31 = v3 + v1), parent pair, hash entry.
__global__ void k_amr_newpts(int64_t nocc, int64_t n, const int32_t* __restrict__ refined,
                             const int32_t* __restrict__ tris, const int64_t* __restrict__ occ_slot,
                             const uint32_t* __restrict__ cflag, const uint32_t* __restrict__ crank,
                             long long* __restrict__ hvals, double* __restrict__ state5, int32_t* __restrict__ parent) {
    const int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= nocc || !cflag[p]) return;
    const int64_t idx = n + crank[p];
    const int64_t j = refined[p / 3];
    const int e = int(p % 3);
    const int32_t a = tris[3 * j + e], b = tris[3 * j + (e + 1) % 3];
#pragma unroll
    for (int c = 0; c < 5; c++)
        state5[5 * idx + c] = __dmul_rn(__dadd_rn(state5[5 * int64_t(a) + c], state5[5 * int64_t(b) + c]), 0.5);
    parent[2 * idx] = a < b ? a : b;
    parent[2 * idx + 1] = a < b ? b : a;
    hvals[occ_slot[p]] = (long long)idx;
}

enum AmrRec : uint8_t { kRecSub = 0, kRecAdd = 1, kRecInit = 2 };

// The split itself: children, corner keys, area records 6 r .. 6 r + 5.
__global__ void k_amr_split(int64_t nref, int64_t q0, int64_t q1, uint64_t seq0, const int32_t* __restrict__ refined,
                            const int64_t* __restrict__ occ_slot, const long long* __restrict__ hvals,
                            const uint32_t* __restrict__ cflag, const double* __restrict__ tarea,
                            int32_t* __restrict__ tris, uint64_t* __restrict__ keys, uint32_t* __restrict__ rec_v,
                            double* __restrict__ rec_d, uint8_t* __restrict__ rec_k) {
    const int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (r >= nref) return;
    const int64_t j = refined[r];
    const int32_t iv1 = tris[3 * j], iv2 = tris[3 * j + 1], iv3 = tris[3 * j + 2];
    const uint64_t k1 = keys[3 * j], k2 = keys[3 * j + 1], k3 = keys[3 * j + 2];
    const int32_t m12 = int32_t(hvals[occ_slot[3 * r]]), m23 = int32_t(hvals[occ_slot[3 * r + 1]]),
                  m31 = int32_t(hvals[occ_slot[3 * r + 2]]);
    const uint64_t b = kAmrKeyAppend + 9 * (seq0 + uint64_t(r));
    const int64_t t2 = q1 + 3 * r, t3 = t2 + 1, t4 = t2 + 2;
    tris[3 * j] = iv1; tris[3 * j + 1] = m12; tris[3 * j + 2] = m31;
    keys[3 * j] = k1; keys[3 * j + 1] = b + 0; keys[3 * j + 2] = b + 6;
    tris[3 * t2] = iv2; tris[3 * t2 + 1] = m12; tris[3 * t2 + 2] = m23;
    keys[3 * t2] = k2; keys[3 * t2 + 1] = b + 1; keys[3 * t2 + 2] = b + 3;
    tris[3 * t3] = iv3; tris[3 * t3 + 1] = m31; tris[3 * t3 + 2] = m23;
    keys[3 * t3] = k3; keys[3 * t3 + 1] = b + 7; keys[3 * t3 + 2] = b + 4;
    tris[3 * t4] = m12; tris[3 * t4 + 1] = m23; tris[3 * t4 + 2] = m31;
    keys[3 * t4] = b + 2; keys[3 * t4 + 1] = b + 5; keys[3 * t4 + 2] = b + 8;
    const double d = __ddiv_rn(tarea[j - q0], 6.0);
    const int32_t v[6] = {iv1, iv2, iv3, m12, m23, m31};
#pragma unroll
    for (int k = 0; k < 6; k++) {
        rec_v[6 * r + k] = uint32_t(v[k]);
        rec_d[6 * r + k] = d;
        rec_k[6 * r + k] = k < 3 ? kRecSub : (cflag[3 * r + (k - 3)] ? kRecInit : kRecAdd);
    }
}

// Area records sorted by point (stable: processing order kept within a
// point): the first record of each point applies that point's records in
// order.
__global__ void k_amr_areas(int64_t nrec, const uint32_t* __restrict__ sv, const int32_t* __restrict__ perm,
                            const double* __restrict__ rec_d, const uint8_t* __restrict__ rec_k,
                            double* __restrict__ area) {
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= nrec || (i > 0 && sv[i] == sv[i - 1])) return;
    const uint32_t v = sv[i];
    double a = area[v];
    for (int64_t k = i; k < nrec && sv[k] == v; k++) {
        const int32_t q = perm[k];
        const double d = rec_d[q];
        a = rec_k[q] == kRecInit ? d : (rec_k[q] == kRecSub ? __dsub_rn(a, d) : __dadd_rn(a, d));
    }
    area[v] = a;
}

// helpers.h:362-372 project_points on points [i0, i1): x *= 1/|x| (|x|
// summed from 0, helpers.h:82-85 project_to_sphere), zeta += -2 omega dz.
__global__ void k_amr_project(int64_t i0, int64_t i1, double* __restrict__ state5, double omega) {
    const int64_t i = i0 + int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= i1) return;
    double* s = state5 + 5 * i;
    const double z_old = s[2];
    const double r = __ddiv_rn(1.0, __dsqrt_rn(dot_self(s)));
    s[0] = __dmul_rn(s[0], r);
    s[1] = __dmul_rn(s[1], r);
    s[2] = __dmul_rn(s[2], r);
    s[3] = __dadd_rn(s[3], __dmul_rn(__dmul_rn(-2.0, omega), __dsub_rn(s[2], z_old)));
}

// ---------------------------------------------------------------- launchers

void amr_project(cudaStream_t st, int64_t i0, int64_t i1, double* state5, double omega) {
    if (i1 > i0) k_amr_project<<<unsigned((i1 - i0 + 255) / 256), 256, 0, st>>>(i0, i1, state5, omega);
}

cudaError_t amr_seed_parents(cudaStream_t st, int64_t n, const int32_t* parent, unsigned long long* hkeys,
                             long long* hvals, int64_t hmask, int* err) {
    if (n > 0)
        k_amr_seed_parents<<<unsigned((n + 255) / 256), 256, 0, st>>>(n, parent, hkeys, hvals, hmask, err);
    return cudaGetLastError();
}

void amr_test(cudaStream_t st, int64_t q0, int64_t m, const int32_t* tris, const double* state5, double vtol,
              double ctol, uint32_t* flag, uint32_t* rank, double* tarea) {
    k_amr_test<<<unsigned((m + 255) / 256), 256, 0, st>>>(q0, m, tris, state5, vtol, ctol, flag, rank, tarea);
}

void amr_edges(cudaStream_t st, int64_t q0, int64_t m, const uint32_t* flag, const uint32_t* rank,
               const int32_t* tris, int32_t* refined, int64_t* occ_slot, unsigned long long* hkeys, long long* hvals,
               int64_t hmask, int* err) {
    k_amr_edges<<<unsigned((m + 255) / 256), 256, 0, st>>>(q0, m, flag, rank, tris, refined, occ_slot, hkeys, hvals,
                                                           hmask, err);
}

void amr_creators(cudaStream_t st, int64_t nocc, const int64_t* occ_slot, const long long* hvals, uint32_t* cflag,
                  uint32_t* crank) {
    k_amr_creators<<<unsigned((nocc + 255) / 256), 256, 0, st>>>(nocc, occ_slot, hvals, cflag, crank);
}

void amr_newpts(cudaStream_t st, int64_t nocc, int64_t n, const int32_t* refined, const int32_t* tris,
                const int64_t* occ_slot, const uint32_t* cflag, const uint32_t* crank, long long* hvals,
                double* state5, int32_t* parent) {
    k_amr_newpts<<<unsigned((nocc + 255) / 256), 256, 0, st>>>(nocc, n, refined, tris, occ_slot, cflag, crank, hvals,
                                                               state5, parent);
}

void amr_split(cudaStream_t st, int64_t nref, int64_t q0, int64_t q1, uint64_t seq0, const int32_t* refined,
               const int64_t* occ_slot, const long long* hvals, const uint32_t* cflag, const double* tarea,
               int32_t* tris, uint64_t* keys, uint32_t* rec_v, double* rec_d, uint8_t* rec_k) {
    k_amr_split<<<unsigned((nref + 255) / 256), 256, 0, st>>>(nref, q0, q1, seq0, refined, occ_slot, hvals, cflag,
                                                              tarea, tris, keys, rec_v, rec_d, rec_k);
}

void amr_areas(cudaStream_t st, int64_t nrec, const uint32_t* sv, const int32_t* perm, const double* rec_d,
               const uint8_t* rec_k, double* area) {
    if (nrec > 0) k_amr_areas<<<unsigned((nrec + 255) / 256), 256, 0, st>>>(nrec, sv, perm, rec_d, rec_k, area);
}

}  // namespace fss
