// k_epi.cu -- upward pass (proxy charges), epilogue (velocity, stream
// function, fused RK4 stage combine + renormalisation) and the total charge.
#include <cuda_runtime.h>

#include "device_common.cuh"
#include "kernels.h"
#include "moments.cuh"

namespace fss {

// ---------------------------------------------------------------- upward pass
// Proxy charges of a source face S of degree n (BLTC upward pass):
//   q_k = sum_{j in S} w_j l_k(b_j),   l_k = sum_m Vinv[m][k] phi_m
// with b_j the barycentric coordinates of the central projection of x_j on
// S's plane and phi_m = T_a(2 b1 - 1) T_b(2 b2 - 1), a + b <= n.  The moments
// M_m = sum_j w_j phi_m(b_j) are formed per leaf for every ancestor frame
// (kernel 1, one block per leaf, a small FP64 tensor-core contraction per
// level), summed over the leaves of each face and contracted with Vinv
// (kernel 2).  FP64.

// Block (group g of four sibling leaves, level l = blockIdx.y): warp w takes
// leaf 4 g + w, its moments in the frame of its ancestor on level l (levels
// outside level_mask: no work), up to the degree up_deg[face] its proxies
// need (none when -1; nmax everywhere without up_deg).  Rows as described
// at up_row_step; slots keep the stride nproxy(nmax), and moments above a
// face's degree are neither written nor read.  Five blocks per SM: the
// per-lane moment sums of degrees 8-11 need 96 registers (80, for six
// blocks, spilled 320 bytes; 118, for four, ran 0.7% slower in the step).
template <typename T>
__global__ void __launch_bounds__(kUpThreads, 5) k_up_leaf(const typename Vec4<T>::type* __restrict__ src,
                                                        const int32_t* __restrict__ leaf_start,
                                                        const double4* __restrict__ frame,
                                                        const NodeGeom* __restrict__ node,
                                                        const int64_t* __restrict__ lev_off, int leaf_level,
                                                        int nmax, int level_mask, const int8_t* __restrict__ up_deg,
                                                        int nleaf, double* __restrict__ part) {
    __shared__ double W[kUpLeaves][kUpRows][kUpLd];
    __shared__ double V[kUpLeaves][kUpRows][kUpLd];
    __shared__ double O[kUpLeaves][kMaxK];
    const int l = blockIdx.y;
    if (!((level_mask >> l) & 1)) return;  // block-uniform
    const int w = threadIdx.x >> 5;
    const int leaf = blockIdx.x * kUpLeaves + w;
    const int KM = nproxy(nmax);
    const int64_t gi = lev_off[l] + (min(leaf, nleaf - 1) >> (2 * (leaf_level - l)));
    const int nm = up_deg ? int(up_deg[gi]) : nmax;  // block-uniform above the leaf level
    double fx = 0, fy = 0, fz = 0;
    if (frame && leaf < nleaf) {
        const double4 f = frame[leaf];
        fx = f.x; fy = f.y; fz = f.z;
    }
    if (l == leaf_level) {  // one row per leaf; warps independent
        if (leaf >= nleaf || nm < 0) return;
        leaf_moments<T>(src, leaf_start[leaf], leaf_start[leaf + 1], fx, fy, fz, node[gi], nm, W[w], V[w],
                        part + (int64_t(leaf) * (leaf_level + 1) + l) * KM);
        return;
    }
    if (nm < 0) return;  // the group's common ancestor takes no proxies
    const int KJ = nproxy(nm);
    if (leaf < nleaf) {
        leaf_moments<T>(src, leaf_start[leaf], leaf_start[leaf + 1], fx, fy, fz, node[gi], nm, W[w], V[w], O[w]);
    } else {
        for (int m = threadIdx.x & 31; m < KJ; m += 32) O[w][m] = 0.0;
    }
    __syncthreads();
    double* out = part + (int64_t(blockIdx.x) * kUpLeaves * (leaf_level + 1) + l) * KM;
    for (int m = threadIdx.x; m < KJ; m += kUpThreads) out[m] = (O[0][m] + O[1][m]) + (O[2][m] + O[3][m]);
}

// Batched V^-1 products.  A block takes up to kBatchTasks tasks (faces or
// clusters) of one degree, K = nproxy(deg): it stages the K x K matrix, its
// rows padded to Kp = 4 ceil(K / 4) doubles, and the tasks' inputs in shared
// memory, and gives each thread a tile of 2 outputs x 4 tasks, so that every
// staged value it reads feeds several FMA chains.  Each output is the chain
// of FMAs over the inner index in order, as a per-task product forms it (so
// the single problem and the ensemble stay bit-identical).
constexpr int kBatchThreads = 192;
constexpr int kBatchTasks = 16;
__host__ __device__ constexpr int batch_pad(int K) { return (K + 3) & ~3; }
static_assert((batch_pad(kMaxK) / 2) * (kBatchTasks / 4) <= kBatchThreads, "one tile per thread at the largest degree");

// Upward pass, part 2a: the moments of every proxy face, its rows summed
// (up_row_step, sum_rows4), one thread per (face, moment) over a flat grid
// of njobs x nproxy(nmax) items: msum[j][m].
constexpr int kSumThreads = 256;
__global__ void __launch_bounds__(kSumThreads) k_up_sums(const ProxyJob* __restrict__ jobs, int njobs,
                                                         const double* __restrict__ part, int leaf_level, int nmax,
                                                         double* __restrict__ msum) {
    const int KM = nproxy(nmax);
    const int64_t item = int64_t(blockIdx.x) * kSumThreads + threadIdx.x;
    if (item >= int64_t(njobs) * KM) return;
    const int j = int(item / KM), m = int(item - int64_t(j) * KM);
    const ProxyJob& job = jobs[j];
    if (m >= nproxy(31 - __clz(job.degmask))) return;  // moments this face's degrees use
    const int step = up_row_step(job.level, leaf_level);
    const int64_t stride = int64_t(step) * (leaf_level + 1) * KM;
    const double* pr = part + (int64_t(job.leaf_lo) * (leaf_level + 1) + job.level) * KM + m;
    msum[item] = sum_rows4([&](int r) { return pr[r * stride]; }, (job.leaf_hi - job.leaf_lo) / step);
}

// Upward pass, part 2b: proxy charges q_k = sum_m Vinv[m][k] M_m of every
// (face, degree) task, written with the proxy positions at the face's slots
// of the unified source array (absolute coordinates).  Shared memory:
// A[m][k] = Vinv[m][k] (K rows of Kp; one bulk copy of the padded matrix
// `vpad`), then X[t][m] = the task's moments.
template <typename T>
__global__ void __launch_bounds__(kBatchThreads) k_up_proxies(const TaskBlock* __restrict__ blocks,
                                                              const int32_t* __restrict__ tasks,
                                                              const ProxyJob* __restrict__ jobs,
                                                              const double* __restrict__ msum, int nmax,
                                                              const double* __restrict__ vpad,
                                                              const int32_t* __restrict__ vpad_off,
                                                              const double4* __restrict__ proxy_pos, int64_t n,
                                                              typename Vec4<T>::type* __restrict__ src, int* err,
                                                              uint64_t wait_ns, int hold_block) {
    extern __shared__ __align__(32) double bsm[];
    __shared__ __align__(8) uint64_t bar;
    const TaskBlock tb = blocks[blockIdx.x];
    const int d = tb.deg, K = nproxy(d), Kp = batch_pad(K), nt = tb.count;
    const int KM = nproxy(nmax);
    double* A = bsm;
    double* X = bsm + K * Kp;
    stage_issue(A, vpad + vpad_off[d], uint32_t(sizeof(double)) * K * Kp, &bar, int(blockIdx.x) == hold_block);
    for (int i = threadIdx.x; i < nt * K; i += kBatchThreads) {
        const int t = i / K, m = i - t * K;
        X[i] = msum[int64_t(tasks[tb.first + t]) * KM + m];
    }
    __syncthreads();
    if (!stage_wait(&bar, wait_ns)) {
        if (threadIdx.x == 0) set_error(err, kErrTimeout);
        return;
    }
    const int npair = Kp / 2, tid = threadIdx.x;
    if (tid >= npair * ((nt + 3) / 4)) return;  // no barrier follows
    const int k0 = 2 * (tid % npair), t0 = 4 * (tid / npair);
    double q[4][2];
#pragma unroll
    for (int j = 0; j < 4; j++) q[j][0] = q[j][1] = 0.0;
    const double* Xt = X + t0 * K;
    for (int m = 0; m < K; m++) {
        const double2 a = *reinterpret_cast<const double2*>(A + m * Kp + k0);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const double x = (t0 + j < nt) ? Xt[j * K + m] : 0.0;
            q[j][0] = fma(a.x, x, q[j][0]);
            q[j][1] = fma(a.y, x, q[j][1]);
        }
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
        if (t0 + j >= nt) break;
        const ProxyJob& job = jobs[tasks[tb.first + t0 + j]];
#pragma unroll
        for (int r = 0; r < 2; r++) {
            if (k0 + r >= K) break;
            const int64_t slot = int64_t(job.off[d]) + k0 + r;
            const double4 y = proxy_pos[slot - n];
            typename Vec4<T>::type o;
            o.x = T(y.x);
            o.y = T(y.y);
            o.z = T(y.z);
            o.w = T(q[j][r]);
            src[slot] = o;
        }
    }
}

size_t up_proxies_smem(int K) { return sizeof(double) * size_t(K * batch_pad(K) + kBatchTasks * K); }

// ---------------------------------------------------------------- epilogue

// Sum the partial slots of each target, form the velocity (and stream
// function), then either write the reference's modify layout (rhs_func) or
// advance the RK4 stage:
//   stage 1..3: acc (+)= c k;  x_next = project(s0 + h k), h = dt/2, dt/2, dt
//   stage 4:    acc += k;      s0 = project(s0 + (dt/6) acc)
// with project(x) = x/|x| and zeta += -2 omega (z_new - z_old)
// (new_dynamics.cpp:281-340, helpers.h:362-372 project_points), and refresh
// the interaction sources of the next stage.
template <typename T>
__global__ void k_epilogue(EpiArgs a) {
    const int64_t s = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (s >= a.n) return;
    double Ax = 0, Ay = 0, Az = 0, Ap = 0;
    for (int p = 0; p < a.parts; p++) {
        const double4 v = a.partials[int64_t(p) * a.pstride + s];
        Ax += v.x; Ay += v.y; Az += v.z; Ap += v.w;
    }
    const double4 x = a.xs[s];
    const double c = -1.0 / (2.0 * M_PI);
    const double ux = c * (x.y * Az - x.z * Ay);
    const double uy = c * (x.z * Ax - x.x * Az);
    const double uz = c * (x.x * Ay - x.y * Ax);
    const double dzeta = -2 * a.omega * uz;
    if (a.mode == EPI_RHS) {
        const int64_t i = a.perm ? a.perm[s] : s;
        double* m = a.out5 + 5 * i;
        m[0] = ux; m[1] = uy; m[2] = uz; m[3] = dzeta; m[4] = 0.0 * (-1.0 / (4.0 * M_PI));
        if (a.psi) {
            const double wself = x.w * a.area[s];
            a.psi[i] = -(M_LN2 / (4.0 * M_PI)) * (Ap - (a.wtotal[0] - wself));
        }
        return;
    }
    const double4 s0 = a.s0[s];
    double4 acc;
    if (a.stage == 1) {
        acc = make_double4(ux, uy, uz, dzeta);
    } else {
        const double f = (a.stage == 4) ? 1.0 : 2.0;
        acc = a.acc[s];
        acc.x += ux * f; acc.y += uy * f; acc.z += uz * f; acc.w += dzeta * f;
    }
    double t[4];
    if (a.stage < 4) {
        a.acc[s] = acc;
        const double h = (a.stage == 3) ? a.dt : a.dt / 2;
        t[0] = ux * h; t[1] = uy * h; t[2] = uz * h; t[3] = dzeta * h;
        t[0] += s0.x; t[1] += s0.y; t[2] += s0.z; t[3] += s0.w;
    } else {
        const double h = a.dt / 6;
        t[0] = acc.x * h; t[1] = acc.y * h; t[2] = acc.z * h; t[3] = acc.w * h;
        t[0] += s0.x; t[1] += s0.y; t[2] += s0.z; t[3] += s0.w;
    }
    double nn = 0;
    nn += t[0] * t[0];
    nn += t[1] * t[1];
    nn += t[2] * t[2];
    const double sc = 1.0 / sqrt(nn);
    const double px = t[0] * sc, py = t[1] * sc, pz = t[2] * sc;
    const double zeta = t[3] + (-2 * a.omega) * (pz - t[2]);
    const double4 nx = make_double4(px, py, pz, zeta);
    if (a.stage == 4) a.s0[s] = nx;
    a.xs[s] = nx;
    double fx = 0, fy = 0, fz = 0;
    if (a.frame && a.leaf_of) {
        const double4 f = a.frame[a.leaf_of[s]];
        fx = f.x; fy = f.y; fz = f.z;
    }
    typename Vec4<T>::type o;
    o.x = T(px - fx);
    o.y = T(py - fy);
    o.z = T(pz - fz);
    o.w = T(zeta * a.area[s]);
    static_cast<typename Vec4<T>::type*>(a.src)[s] = o;
}

// One rank's share of a sharded right-hand side: the partial slots of its own
// targets -- rows [lo, hi) of the sorted order, read through leaf_start when
// given (leaves [leaf_lo, leaf_hi): particles are re-sorted every step) --
// summed in the epilogue's order, and -0.0 in every other row.  Summing the
// buffers of all ranks then gives every row exactly, in any order
// (x + -0.0 = x, and a sum started from +0.0 is never -0.0).
__global__ void k_shard_reduce(int64_t n, int parts, int64_t pstride, const double4* __restrict__ partials,
                               const int32_t* __restrict__ leaf_start, int64_t leaf_lo, int64_t leaf_hi,
                               int64_t row_lo, int64_t row_hi, double4* __restrict__ out) {
    const int64_t s = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (s >= n) return;
    int64_t lo = row_lo, hi = row_hi;
    if (leaf_start) {
        lo = leaf_start[leaf_lo];
        hi = leaf_start[leaf_hi];
    }
    if (s < lo || s >= hi) {
        out[s] = make_double4(-0.0, -0.0, -0.0, -0.0);
        return;
    }
    double Ax = 0, Ay = 0, Az = 0, Ap = 0;
    for (int p = 0; p < parts; p++) {
        const double4 v = partials[int64_t(p) * pstride + s];
        Ax += v.x; Ay += v.y; Az += v.z; Ap += v.w;
    }
    out[s] = make_double4(Ax, Ay, Az, Ap);
}

// Stage state and interaction sources from the step state (after a
// stand-alone right-hand side overwrote them).
template <typename T>
__global__ void k_refresh(int64_t n, const double4* __restrict__ s0, const double* __restrict__ area,
                          const uint32_t* __restrict__ leaf_of, const double4* __restrict__ frame,
                          double4* __restrict__ xs, typename Vec4<T>::type* __restrict__ src) {
    const int64_t s = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const double4 v = s0[s];
    xs[s] = v;
    double fx = 0, fy = 0, fz = 0;
    if (frame && leaf_of) {
        const double4 f = frame[leaf_of[s]];
        fx = f.x; fy = f.y; fz = f.z;
    }
    typename Vec4<T>::type o;
    o.x = T(v.x - fx);
    o.y = T(v.y - fy);
    o.z = T(v.z - fz);
    o.w = T(v.w * area[s]);
    src[s] = o;
}

// Total charge W = sum zeta_j A_j (deterministic single-block reduction).
__global__ void __launch_bounds__(1024) k_wsum(int64_t n, const double4* __restrict__ xs, const double* __restrict__ area,
                                               double* __restrict__ w) {
    __shared__ double red[1024];
    double s = 0;
    for (int64_t i = threadIdx.x; i < n; i += 1024) s += xs[i].w * area[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int off = 512; off > 0; off >>= 1) {
        if (threadIdx.x < off) red[threadIdx.x] += red[threadIdx.x + off];
        __syncthreads();
    }
    if (threadIdx.x == 0) w[0] = red[0];
}

// Scatter the device state back to the caller's AoS order.
__global__ void k_scatter_state(int64_t n, const int32_t* __restrict__ perm, const double4* __restrict__ s0,
                                const double* __restrict__ tracer, double* __restrict__ out5) {
    const int64_t s = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int64_t i = perm ? perm[s] : s;
    const double4 v = s0[s];
    double* o = out5 + 5 * i;
    o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w; o[4] = tracer[s];
}

// ---------------------------------------------------------------- downward pass
// Target clusters (fast_rhs.h cp and cc): the sum A of a face's far
// sources at its interpolation points y_k becomes the interpolant
//   A(x) = sum_k A(y_k) l_k(b(x)) = sum_m c_m phi_m(b(x)),   c_m = sum_k Vinv[m][k] A(y_k),
// with b(x) the barycentric coordinates of the central projection of x on
// the face's plane and phi_m the Chebyshev product basis of the upward
// pass.  Level by level from the top, a face's coefficients interpolate
// its own far field at its points plus its parent's interpolant there (a
// face below a target cluster inherits this way); then, one block per
// leaf, the leaf face's interpolant is evaluated at its particles into the
// down-pass partial slot.  x, y, z and, when the stream function is wanted,
// its log term.  FP64.

// Downward pass, part 1: the coefficients of every target cluster at once,
// batched by degree (kBatchThreads above): y_k = the cluster's field at its
// K interpolation points (its partial slots summed, in slot order), c_m =
// sum_k Vinv[m][k] y_k over k in order.  Shared memory: A[k][m] =
// Vinv[m][k] (K rows of Kp; one bulk copy of the padded transpose `vtpad`),
// then Y[t][k].
template <bool PSI>
__global__ void __launch_bounds__(kBatchThreads) k_down_coef(const TaskBlock* __restrict__ blocks,
                                                             const int32_t* __restrict__ tasks,
                                                             const DownJob* __restrict__ jobs,
                                                             const double4* __restrict__ partials, int parts,
                                                             int64_t pstride, const double* __restrict__ vtpad,
                                                             const int32_t* __restrict__ vpad_off,
                                                             double4* __restrict__ coef, int* err, uint64_t wait_ns,
                                                             int hold_block) {
    extern __shared__ __align__(32) double bsm[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ int32_t slot_of[kBatchTasks];
    __shared__ int64_t coef_of[kBatchTasks];
    const TaskBlock tb = blocks[blockIdx.x];
    const int d = tb.deg, K = nproxy(d), Kp = batch_pad(K), nt = tb.count;
    double* A = bsm;
    double4* Y = reinterpret_cast<double4*>(bsm + K * Kp);  // K * Kp is a multiple of 4
    stage_issue(A, vtpad + vpad_off[d], uint32_t(sizeof(double)) * K * Kp, &bar, int(blockIdx.x) == hold_block);
    // the block's jobs looked up once (their point slots and coefficient rows)
    if (threadIdx.x < nt) {
        const DownJob jb = jobs[tasks[tb.first + threadIdx.x]];
        slot_of[threadIdx.x] = jb.slot;
        coef_of[threadIdx.x] = jb.coef;
    }
    __syncthreads();
    // unrolled: the partial-slot loads of several points in flight at once
#pragma unroll 4
    for (int i = threadIdx.x; i < nt * K; i += kBatchThreads) {
        const int t = i / K, k = i - t * K;
        const int32_t slot = slot_of[t];
        double4 v = make_double4(0.0, 0.0, 0.0, 0.0);
        for (int q = 0; q < parts; q++) {
            const double4 y = partials[int64_t(q) * pstride + slot + k];
            v.x += y.x; v.y += y.y; v.z += y.z; v.w += y.w;
        }
        Y[i] = v;
    }
    __syncthreads();
    if (!stage_wait(&bar, wait_ns)) {
        if (threadIdx.x == 0) set_error(err, kErrTimeout);
        return;
    }
    const int npair = Kp / 2, tid = threadIdx.x;
    if (tid >= npair * ((nt + 3) / 4)) return;  // no barrier follows
    const int m0 = 2 * (tid % npair), t0 = 4 * (tid / npair);
    double4 c[4][2];
#pragma unroll
    for (int j = 0; j < 4; j++) c[j][0] = c[j][1] = make_double4(0.0, 0.0, 0.0, 0.0);
    const double4* Yt = Y + t0 * K;
    for (int k = 0; k < K; k++) {
        const double2 a = *reinterpret_cast<const double2*>(A + k * Kp + m0);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const double4 y = (t0 + j < nt) ? Yt[j * K + k] : make_double4(0.0, 0.0, 0.0, 0.0);
            c[j][0].x = fma(a.x, y.x, c[j][0].x);
            c[j][0].y = fma(a.x, y.y, c[j][0].y);
            c[j][0].z = fma(a.x, y.z, c[j][0].z);
            c[j][1].x = fma(a.y, y.x, c[j][1].x);
            c[j][1].y = fma(a.y, y.y, c[j][1].y);
            c[j][1].z = fma(a.y, y.z, c[j][1].z);
            if (PSI) {
                c[j][0].w = fma(a.x, y.w, c[j][0].w);
                c[j][1].w = fma(a.y, y.w, c[j][1].w);
            }
        }
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
        if (t0 + j >= nt) break;
        double4* out = coef + coef_of[t0 + j];
        if (m0 < K) out[m0] = c[j][0];
        if (m0 + 1 < K) out[m0 + 1] = c[j][1];
    }
}

size_t down_coef_smem(int K) { return sizeof(double) * size_t(K * batch_pad(K)) + sizeof(double4) * size_t(kBatchTasks * K); }

// The interpolant of degree D with coefficients C at barycentric (u, v)
// (both mapped to [-1, 1]): sum_a T_a(u) sum_b C[m(a, b)] T_b(v), a + b <= D,
// m(a, b) = (a + b)(a + b + 1)/2 + b, both Chebyshev families by their
// three-term recurrences; the degree is known at compile time, so that the
// loops unroll and C is read at fixed offsets.
template <int D, bool PSI>
__device__ __forceinline__ double4 eval_deg(double u, double v, const double4* __restrict__ C) {
    double tv[D + 1];
    tv[0] = 1.0;
    if (D >= 1) tv[1] = v;
    const double v2 = 2.0 * v, u2 = 2.0 * u;
#pragma unroll
    for (int b = 2; b <= D; b++) tv[b] = fma(v2, tv[b - 1], -tv[b - 2]);
    double4 acc = make_double4(0.0, 0.0, 0.0, 0.0);
    double ta = 1.0, ta_prev = u;  // T_a(u), T_{a-1}(u) (T_{-1} = T_1)
#pragma unroll
    for (int a = 0; a <= D; a++) {
        double4 s = make_double4(0.0, 0.0, 0.0, 0.0);
#pragma unroll
        for (int b = 0; a + b <= D; b++) {
            const double4 cm = C[(a + b) * (a + b + 1) / 2 + b];
            s.x = fma(tv[b], cm.x, s.x);
            s.y = fma(tv[b], cm.y, s.y);
            s.z = fma(tv[b], cm.z, s.z);
            if (PSI) s.w = fma(tv[b], cm.w, s.w);
        }
        acc.x = fma(ta, s.x, acc.x);
        acc.y = fma(ta, s.y, acc.y);
        acc.z = fma(ta, s.z, acc.z);
        if (PSI) acc.w = fma(ta, s.w, acc.w);
        const double tn = fma(u2, ta, -ta_prev);
        ta_prev = ta;
        ta = tn;
    }
    return acc;
}

template <bool PSI>
__device__ __forceinline__ double4 eval_any(int deg, double u, double v, const double4* C) {
    switch (deg) {
#define FSS_DEG(D) \
    case D: return eval_deg<D, PSI>(u, v, C);
        FSS_DEG(0) FSS_DEG(1) FSS_DEG(2) FSS_DEG(3) FSS_DEG(4) FSS_DEG(5) FSS_DEG(6)
        FSS_DEG(7) FSS_DEG(8) FSS_DEG(9) FSS_DEG(10) FSS_DEG(11) FSS_DEG(12)
#undef FSS_DEG
    }
    return make_double4(0.0, 0.0, 0.0, 0.0);
}
static_assert(kMaxDegree == 12, "eval_any instantiates degrees 0..12");

// FP32 form of eval_deg for the mixed-precision path (velocity only): the
// recurrences and the K x 3 contraction in FP32 on coefficients rounded to
// FP32; the caller adds the result in FP64.
template <int D>
__device__ __forceinline__ float3 eval_deg_f(float u, float v, const float4* __restrict__ C) {
    float tv[D + 1];
    tv[0] = 1.f;
    if (D >= 1) tv[1] = v;
    const float v2 = 2.f * v, u2 = 2.f * u;
#pragma unroll
    for (int b = 2; b <= D; b++) tv[b] = fmaf(v2, tv[b - 1], -tv[b - 2]);
    float3 acc = make_float3(0.f, 0.f, 0.f);
    float ta = 1.f, ta_prev = u;  // T_a(u), T_{a-1}(u) (T_{-1} = T_1)
#pragma unroll
    for (int a = 0; a <= D; a++) {
        float3 sa = make_float3(0.f, 0.f, 0.f);
#pragma unroll
        for (int b = 0; a + b <= D; b++) {
            const float4 cm = C[(a + b) * (a + b + 1) / 2 + b];
            sa.x = fmaf(tv[b], cm.x, sa.x);
            sa.y = fmaf(tv[b], cm.y, sa.y);
            sa.z = fmaf(tv[b], cm.z, sa.z);
        }
        acc.x = fmaf(ta, sa.x, acc.x);
        acc.y = fmaf(ta, sa.y, acc.y);
        acc.z = fmaf(ta, sa.z, acc.z);
        const float tn = fmaf(u2, ta, -ta_prev);
        ta_prev = ta;
        ta = tn;
    }
    return acc;
}

__device__ __forceinline__ float3 eval_any_f(int deg, float u, float v, const float4* C) {
    switch (deg) {
#define FSS_DEG(D) \
    case D: return eval_deg_f<D>(u, v, C);
        FSS_DEG(0) FSS_DEG(1) FSS_DEG(2) FSS_DEG(3) FSS_DEG(4) FSS_DEG(5) FSS_DEG(6)
        FSS_DEG(7) FSS_DEG(8) FSS_DEG(9) FSS_DEG(10) FSS_DEG(11) FSS_DEG(12)
#undef FSS_DEG
    }
    return make_float3(0.f, 0.f, 0.f);
}

// Downward pass, part 2: one block per leaf; every particle sums the
// interpolants of the target clusters above its leaf (coarse to fine),
// evaluated where it is (barycentric coordinates of its central projection
// in each cluster's frame).  A leaf below none writes zeros.  F32 (mixed
// precision, velocity only): the interpolants evaluated in FP32
// (eval_deg_f), the coordinates and the sum over the clusters in FP64.
template <bool PSI, bool F32>
__global__ void __launch_bounds__(kUpThreads) k_down_direct(const double4* __restrict__ xs,
                                                            const int32_t* __restrict__ leaf_start,
                                                            const NodeGeom* __restrict__ node,
                                                            const LeafAnc* __restrict__ leaf_anc,
                                                            const double4* __restrict__ coef,
                                                            double4* __restrict__ out) {
    __shared__ double4 C[kMaxLevels * kMaxK];
    __shared__ LeafAnc A[kMaxLevels];
    __shared__ NodeGeom G[kMaxLevels];
    __shared__ int off[kMaxLevels + 1];
    const int leaf = blockIdx.x, tid = threadIdx.x;
    const int a0 = leaf_start[leaf], a1 = leaf_start[leaf + 1];
    if (a0 == a1) return;
    if (tid < kMaxLevels) A[tid] = leaf_anc[int64_t(leaf) * kMaxLevels + tid];
    __syncthreads();
    int nanc = 0;
    while (nanc < kMaxLevels && A[nanc].coef >= 0) nanc++;
    if (tid < nanc) G[tid] = node[A[tid].node];
    if (tid == 0) {
        int o = 0;
        for (int k = 0; k < nanc; k++) {
            off[k] = o;
            o += nproxy(A[k].deg);
        }
        off[nanc] = o;
    }
    __syncthreads();
    float4* Cf = reinterpret_cast<float4*>(C);  // F32: the same coefficients rounded, 16 B each
    for (int a = 0; a < nanc; a++)
        for (int m = tid; m < off[a + 1] - off[a]; m += kUpThreads) {
            const double4 cd = coef[int64_t(A[a].coef) + m];
            if (F32)
                Cf[off[a] + m] = make_float4(float(cd.x), float(cd.y), float(cd.z), 0.f);
            else
                C[off[a] + m] = cd;
        }
    __syncthreads();
    for (int i = a0 + tid; i < a1; i += kUpThreads) {
        const double4 x = xs[i];
        double4 acc = make_double4(0.0, 0.0, 0.0, 0.0);
        for (int a = 0; a < nanc; a++) {
            const NodeGeom& ng = G[a];
            const double c0 = ng.minv[0] * x.x + ng.minv[1] * x.y + ng.minv[2] * x.z;
            const double c1 = ng.minv[3] * x.x + ng.minv[4] * x.y + ng.minv[5] * x.z;
            const double c2 = ng.minv[6] * x.x + ng.minv[7] * x.y + ng.minv[8] * x.z;
            const double inv = 1.0 / (c0 + c1 + c2);
            const double u = 2.0 * (c0 * inv) - 1.0, v = 2.0 * (c1 * inv) - 1.0;
            if (F32) {
                const float3 e = eval_any_f(A[a].deg, float(u), float(v), Cf + off[a]);
                acc.x += double(e.x); acc.y += double(e.y); acc.z += double(e.z);
            } else {
                const double4 e = eval_any<PSI>(A[a].deg, u, v, C + off[a]);
                acc.x += e.x; acc.y += e.y; acc.z += e.z; acc.w += e.w;
            }
        }
        out[i] = acc;
    }
}

// ---------------------------------------------------------------- launchers

void launch_up_leaf(cudaStream_t st, bool fp64, int nleaf, const void* src, const int32_t* leaf_start,
                    const double4* frame, const NodeGeom* node, const int64_t* lev_off, int leaf_level, int nmax,
                    int level_mask, const int8_t* up_deg, double* part) {
    if (nleaf == 0 || level_mask == 0) return;
    const dim3 nb(unsigned((nleaf + kUpLeaves - 1) / kUpLeaves), unsigned(leaf_level + 1));
    if (fp64)
        k_up_leaf<double><<<nb, kUpThreads, 0, st>>>(static_cast<const double4*>(src), leaf_start, frame, node,
                                                     lev_off, leaf_level, nmax, level_mask, up_deg, nleaf, part);
    else
        k_up_leaf<float><<<nb, kUpThreads, 0, st>>>(static_cast<const float4*>(src), leaf_start, frame, node,
                                                    lev_off, leaf_level, nmax, level_mask, up_deg, nleaf, part);
}

void launch_up_proxies(cudaStream_t st, bool fp64, int njobs, const ProxyJob* jobs, const double* part,
                       int leaf_level, int nmax, double* msum, int nblocks, const TaskBlock* blocks,
                       const int32_t* tasks, const double* vpad, const int32_t* vpad_off, const double4* proxy_pos,
                       int64_t n, void* src, int* err, uint64_t wait_ns, int hold_block) {
    if (njobs == 0) return;
    const int64_t items = int64_t(njobs) * nproxy(nmax);
    k_up_sums<<<unsigned((items + kSumThreads - 1) / kSumThreads), kSumThreads, 0, st>>>(jobs, njobs, part, leaf_level,
                                                                                          nmax, msum);
    const size_t smem = up_proxies_smem(nproxy(nmax));
    if (fp64)
        k_up_proxies<double><<<nblocks, kBatchThreads, smem, st>>>(blocks, tasks, jobs, msum, nmax, vpad, vpad_off,
                                                                   proxy_pos, n, static_cast<double4*>(src), err,
                                                                   wait_ns, hold_block);
    else
        k_up_proxies<float><<<nblocks, kBatchThreads, smem, st>>>(blocks, tasks, jobs, msum, nmax, vpad, vpad_off,
                                                                  proxy_pos, n, static_cast<float4*>(src), err,
                                                                  wait_ns, hold_block);
}

int batch_tasks() { return kBatchTasks; }

cudaError_t batch_prepare() {
    // dynamic shared memory above the default 48 KB, sized for the largest degree
    const int up = int(up_proxies_smem(kMaxK)), dn = int(down_coef_smem(kMaxK));
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(k_up_proxies<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, up)) ||
        (e = cudaFuncSetAttribute(k_up_proxies<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, up)) ||
        (e = cudaFuncSetAttribute(k_down_coef<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, dn)) ||
        (e = cudaFuncSetAttribute(k_down_coef<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, dn)))
        return e;
    return cudaSuccess;
}

void launch_epilogue(cudaStream_t st, bool fp64, const EpiArgs& a) {
    if (a.n == 0) return;
    const unsigned g = unsigned((a.n + 255) / 256);
    if (fp64)
        k_epilogue<double><<<g, 256, 0, st>>>(a);
    else
        k_epilogue<float><<<g, 256, 0, st>>>(a);
}

void launch_shard_reduce(cudaStream_t st, int64_t n, int parts, int64_t pstride, const double4* partials,
                         const int32_t* leaf_start, int64_t leaf_lo, int64_t leaf_hi, int64_t row_lo, int64_t row_hi,
                         double4* out) {
    if (n == 0) return;
    k_shard_reduce<<<unsigned((n + 255) / 256), 256, 0, st>>>(n, parts, pstride, partials, leaf_start, leaf_lo,
                                                              leaf_hi, row_lo, row_hi, out);
}

void launch_refresh(cudaStream_t st, bool fp64, int64_t n, const double4* s0, const double* area,
                    const uint32_t* leaf_of, const double4* frame, double4* xs, void* src) {
    if (n == 0) return;
    const unsigned g = unsigned((n + 255) / 256);
    if (fp64)
        k_refresh<double><<<g, 256, 0, st>>>(n, s0, area, leaf_of, frame, xs, static_cast<double4*>(src));
    else
        k_refresh<float><<<g, 256, 0, st>>>(n, s0, area, leaf_of, frame, xs, static_cast<float4*>(src));
}

void launch_wsum(cudaStream_t st, int64_t n, const double4* xs, const double* area, double* w) {
    k_wsum<<<1, 1024, 0, st>>>(n, xs, area, w);
}

void launch_scatter_state(cudaStream_t st, int64_t n, const int32_t* perm, const double4* s0, const double* tracer,
                          double* out5) {
    if (n == 0) return;
    k_scatter_state<<<unsigned((n + 255) / 256), 256, 0, st>>>(n, perm, s0, tracer, out5);
}

void launch_down(cudaStream_t st, bool psi, const DownArgs& d) {
    if (d.njobs == 0) return;
    const unsigned nb = unsigned(d.ncoef_blocks);
    const size_t smem = down_coef_smem(nproxy(d.max_deg));
    if (psi) {
        k_down_coef<true><<<nb, kBatchThreads, smem, st>>>(d.coef_blocks, d.coef_tasks, d.jobs, d.partials, d.parts,
                                                           d.pstride, d.vtpad, d.vpad_off, d.coef, d.err, d.wait_ns,
                                                           d.hold_block);
        k_down_direct<true, false><<<d.nleaf, kUpThreads, 0, st>>>(d.xs, d.leaf_start, d.node, d.leaf_anc, d.coef,
                                                                   d.out);
    } else {
        k_down_coef<false><<<nb, kBatchThreads, smem, st>>>(d.coef_blocks, d.coef_tasks, d.jobs, d.partials,
                                                            d.parts, d.pstride, d.vtpad, d.vpad_off, d.coef, d.err,
                                                            d.wait_ns, d.hold_block);
        if (d.fp32_eval)
            k_down_direct<false, true><<<d.nleaf, kUpThreads, 0, st>>>(d.xs, d.leaf_start, d.node, d.leaf_anc,
                                                                       d.coef, d.out);
        else
            k_down_direct<false, false><<<d.nleaf, kUpThreads, 0, st>>>(d.xs, d.leaf_start, d.node, d.leaf_anc,
                                                                        d.coef, d.out);
    }
}

int down_launch_count(const DownArgs& d) { return d.njobs == 0 ? 0 : 2; }

}  // namespace fss
