// k_mlp.cu -- the degree/MAC selector network: a 16 -> 64 -> 64 -> 12 MLP
// (ReLU) with BF16 weights and inputs and FP32 accumulation, with its own
// inference and training kernels (forward, backward, Adam).
//
// Parameter vector (FP32 master copy, kMlpParams floats):
//   W1[64][16], b1[64], W2[64][64], b2[64], W3[12][64], b3[12].
// The kernels read the weights as BF16 (rounded from the master copy after
// every update) and the biases as FP32.
//
// Training step on a batch of B samples (a multiple of 128), one block per
// 128 samples: each thread runs forward and backward for its sample keeping
// activations and deltas in shared memory, then the block forms its share of
// every weight gradient as a 128-term sum (dW = delta^T act) and writes it
// to a per-block slot; a second kernel adds the slots in block order
// (deterministic) and applies Adam.  Loss: mean over the batch of the sum
// over outputs of mask * (y - t)^2.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "fss.h"

namespace fss {

void set_last_error(const std::string& msg);

constexpr int kIn = 16, kHid = 64, kOut = 12;
constexpr int oW1 = 0, ob1 = oW1 + kHid * kIn, oW2 = ob1 + kHid, ob2 = oW2 + kHid * kHid, oW3 = ob2 + kHid,
              ob3 = oW3 + kOut * kHid, kMlpParams = ob3 + kOut;
constexpr int kMlpTile = 128;  // samples per block

struct MlpSmemWeights {
    float W1[kHid * kIn], b1[kHid], W2[kHid * kHid], b2[kHid], W3[kOut * kHid], b3[kOut];
};

__device__ __forceinline__ void load_weights(MlpSmemWeights& w, const __nv_bfloat16* __restrict__ wb,
                                             const float* __restrict__ p) {
    for (int k = threadIdx.x; k < kHid * kIn; k += blockDim.x) w.W1[k] = __bfloat162float(wb[oW1 + k]);
    for (int k = threadIdx.x; k < kHid * kHid; k += blockDim.x) w.W2[k] = __bfloat162float(wb[oW2 + k]);
    for (int k = threadIdx.x; k < kOut * kHid; k += blockDim.x) w.W3[k] = __bfloat162float(wb[oW3 + k]);
    for (int k = threadIdx.x; k < kHid; k += blockDim.x) {
        w.b1[k] = p[ob1 + k];
        w.b2[k] = p[ob2 + k];
    }
    for (int k = threadIdx.x; k < kOut; k += blockDim.x) w.b3[k] = p[ob3 + k];
}

// Inference: y = W3 relu(W2 relu(W1 x + b1) + b2) + b3, one thread per sample.
__global__ void __launch_bounds__(kMlpTile) k_mlp_forward(int64_t n, const __nv_bfloat16* __restrict__ X,
                                                          const __nv_bfloat16* __restrict__ wb,
                                                          const float* __restrict__ p, float* __restrict__ Y) {
    __shared__ MlpSmemWeights w;
    load_weights(w, wb, p);
    __syncthreads();
    const int64_t s = int64_t(blockIdx.x) * kMlpTile + threadIdx.x;
    if (s >= n) return;
    float x[kIn], h1[kHid];
#pragma unroll
    for (int i = 0; i < kIn; i++) x[i] = __bfloat162float(X[s * kIn + i]);
#pragma unroll
    for (int j = 0; j < kHid; j++) {
        float a = w.b1[j];
#pragma unroll
        for (int i = 0; i < kIn; i++) a = fmaf(w.W1[j * kIn + i], x[i], a);
        h1[j] = fmaxf(a, 0.f);
    }
    float y[kOut];
#pragma unroll
    for (int o = 0; o < kOut; o++) y[o] = w.b3[o];
    for (int k = 0; k < kHid; k++) {
        float a = w.b2[k];
#pragma unroll
        for (int j = 0; j < kHid; j++) a = fmaf(w.W2[k * kHid + j], h1[j], a);
        a = fmaxf(a, 0.f);
#pragma unroll
        for (int o = 0; o < kOut; o++) y[o] = fmaf(w.W3[o * kHid + k], a, y[o]);
    }
#pragma unroll
    for (int o = 0; o < kOut; o++) Y[s * kOut + o] = y[o];
}

struct MlpTileSmem {
    MlpSmemWeights w;
    float X[kMlpTile][kIn];
    float H1[kMlpTile][kHid];
    float H2[kMlpTile][kHid];
    float D2[kMlpTile][kHid];
    float D1[kMlpTile][kHid];
    float DY[kMlpTile][kOut];
    float loss[kMlpTile];
};

// Forward + backward for one tile of 128 samples (rows idx[base..]); writes
// this block's gradient share G[block][kMlpParams] and its loss sum.
__global__ void __launch_bounds__(kMlpTile) k_mlp_grad_tile(int64_t nbatch, const int64_t* __restrict__ idx,
                                                            const __nv_bfloat16* __restrict__ X,
                                                            const float* __restrict__ T, const float* __restrict__ M,
                                                            const __nv_bfloat16* __restrict__ wb,
                                                            const float* __restrict__ p, float scale,
                                                            float* __restrict__ G, float* __restrict__ L) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    MlpTileSmem& sm = *reinterpret_cast<MlpTileSmem*>(smem_raw);
    load_weights(sm.w, wb, p);
    const int t = threadIdx.x;
    const int64_t b = int64_t(blockIdx.x) * kMlpTile + t;
    const bool valid = b < nbatch;
    const int64_t row = valid ? idx[b] : 0;
#pragma unroll
    for (int i = 0; i < kIn; i++) sm.X[t][i] = valid ? __bfloat162float(X[row * kIn + i]) : 0.f;
    __syncthreads();
    // forward
    for (int j = 0; j < kHid; j++) {
        float a = sm.w.b1[j];
#pragma unroll
        for (int i = 0; i < kIn; i++) a = fmaf(sm.w.W1[j * kIn + i], sm.X[t][i], a);
        sm.H1[t][j] = fmaxf(a, 0.f);
    }
    for (int k = 0; k < kHid; k++) {
        float a = sm.w.b2[k];
        for (int j = 0; j < kHid; j++) a = fmaf(sm.w.W2[k * kHid + j], sm.H1[t][j], a);
        sm.H2[t][k] = fmaxf(a, 0.f);
    }
    float lsum = 0.f;
#pragma unroll
    for (int o = 0; o < kOut; o++) {
        float a = sm.w.b3[o];
        for (int k = 0; k < kHid; k++) a = fmaf(sm.w.W3[o * kHid + k], sm.H2[t][k], a);
        float d = 0.f;
        if (valid) {
            const float m = M ? M[row * kOut + o] : 1.f;
            const float e = a - T[row * kOut + o];
            lsum += m * e * e;
            d = 2.f * m * e * scale;
        }
        sm.DY[t][o] = d;
    }
    sm.loss[t] = lsum;
    // backward through the hidden layers
    for (int k = 0; k < kHid; k++) {
        float a = 0.f;
#pragma unroll
        for (int o = 0; o < kOut; o++) a = fmaf(sm.w.W3[o * kHid + k], sm.DY[t][o], a);
        sm.D2[t][k] = (sm.H2[t][k] > 0.f) ? a : 0.f;
    }
    for (int j = 0; j < kHid; j++) {
        float a = 0.f;
        for (int k = 0; k < kHid; k++) a = fmaf(sm.w.W2[k * kHid + j], sm.D2[t][k], a);
        sm.D1[t][j] = (sm.H1[t][j] > 0.f) ? a : 0.f;
    }
    __syncthreads();
    // weight gradients: 128-term sums over the tile, fixed order
    float* g = G + int64_t(blockIdx.x) * kMlpParams;
    for (int e = t; e < kMlpParams; e += kMlpTile) {
        float a = 0.f;
        if (e < ob1) {  // W1[j][i]
            const int j = (e - oW1) / kIn, i = (e - oW1) % kIn;
            for (int s = 0; s < kMlpTile; s++) a = fmaf(sm.D1[s][j], sm.X[s][i], a);
        } else if (e < oW2) {
            const int j = e - ob1;
            for (int s = 0; s < kMlpTile; s++) a += sm.D1[s][j];
        } else if (e < ob2) {
            const int k = (e - oW2) / kHid, j = (e - oW2) % kHid;
            for (int s = 0; s < kMlpTile; s++) a = fmaf(sm.D2[s][k], sm.H1[s][j], a);
        } else if (e < oW3) {
            const int k = e - ob2;
            for (int s = 0; s < kMlpTile; s++) a += sm.D2[s][k];
        } else if (e < ob3) {
            const int o = (e - oW3) / kHid, k = (e - oW3) % kHid;
            for (int s = 0; s < kMlpTile; s++) a = fmaf(sm.DY[s][o], sm.H2[s][k], a);
        } else {
            const int o = e - ob3;
            for (int s = 0; s < kMlpTile; s++) a += sm.DY[s][o];
        }
        g[e] = a;
    }
    if (t == 0) {
        float l = 0.f;
        for (int s = 0; s < kMlpTile; s++) l += sm.loss[s];
        L[blockIdx.x] = l;
    }
}

// grad[e] = sum over blocks (in order); loss = sum of block losses * scale.
__global__ void k_mlp_reduce(int nblk, const float* __restrict__ G, const float* __restrict__ L, float scale,
                             float* __restrict__ grad, float* __restrict__ loss) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < kMlpParams) {
        float a = 0.f;
        for (int b = 0; b < nblk; b++) a += G[int64_t(b) * kMlpParams + e];
        grad[e] = a;
    }
    if (e == 0) {
        float l = 0.f;
        for (int b = 0; b < nblk; b++) l += L[b];
        loss[0] = l * scale;
    }
}

// Adam on the FP32 master parameters; refresh the BF16 weight mirror.
__global__ void k_mlp_adam(float* __restrict__ p, float* __restrict__ m1, float* __restrict__ m2,
                           const float* __restrict__ grad, float lr, float b1, float b2, float eps, float c1, float c2,
                           __nv_bfloat16* __restrict__ wb) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= kMlpParams) return;
    const float g = grad[e];
    const float a = b1 * m1[e] + (1.f - b1) * g;
    const float v = b2 * m2[e] + (1.f - b2) * g * g;
    m1[e] = a;
    m2[e] = v;
    const float np = p[e] - lr * (a / c1) / (sqrtf(v / c2) + eps);
    p[e] = np;
    wb[e] = __float2bfloat16(np);
}

__global__ void k_to_bf16(int64_t n, const float* __restrict__ a, __nv_bfloat16* __restrict__ b) {
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) b[i] = __float2bfloat16(a[i]);
}

}  // namespace fss

using namespace fss;

struct fss_mlp {
    int dev = 0;
    cudaStream_t st = nullptr;
    float *p = nullptr, *m1 = nullptr, *m2 = nullptr, *grad = nullptr, *loss = nullptr, *G = nullptr, *L = nullptr;
    __nv_bfloat16* wb = nullptr;
    __nv_bfloat16* X = nullptr;
    float *T = nullptr, *M = nullptr;
    int64_t* idx = nullptr;
    int64_t n = 0, cap_blocks = 0;
    int64_t step = 0;
    std::vector<float> host_p;
    ~fss_mlp() {
        for (void* q : {(void*)p, (void*)m1, (void*)m2, (void*)grad, (void*)loss, (void*)G, (void*)L, (void*)wb,
                        (void*)X, (void*)T, (void*)M, (void*)idx})
            if (q) cudaFree(q);
        if (st) cudaStreamDestroy(st);
    }
};

namespace {

int mlp_fail(int code, const std::string& m) {
    set_last_error(m);
    return code;
}

#define MCU(call)                                                                                  \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) return mlp_fail(FSS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

int sync_weights(fss_mlp* m) {
    k_to_bf16<<<(kMlpParams + 255) / 256, 256, 0, m->st>>>(kMlpParams, m->p, m->wb);
    MCU(cudaGetLastError());
    return FSS_OK;
}

int ensure_blocks(fss_mlp* m, int64_t nblk) {
    if (nblk <= m->cap_blocks) return FSS_OK;
    if (m->G) cudaFree(m->G);
    if (m->L) cudaFree(m->L);
    MCU(cudaMalloc(&m->G, sizeof(float) * kMlpParams * nblk));
    MCU(cudaMalloc(&m->L, sizeof(float) * nblk));
    m->cap_blocks = nblk;
    return FSS_OK;
}

int grad_pass(fss_mlp* m, const int64_t* d_idx, int64_t nb) {
    const int64_t nblk = (nb + kMlpTile - 1) / kMlpTile;
    int r = ensure_blocks(m, nblk);
    if (r) return r;
    const size_t smem = sizeof(MlpTileSmem);
    MCU(cudaFuncSetAttribute(k_mlp_grad_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    const float scale = 1.f / float(nb);
    k_mlp_grad_tile<<<unsigned(nblk), kMlpTile, smem, m->st>>>(nb, d_idx, m->X, m->T, m->M, m->wb, m->p, scale, m->G,
                                                                m->L);
    k_mlp_reduce<<<(kMlpParams + 255) / 256, 256, 0, m->st>>>(int(nblk), m->G, m->L, scale, m->grad, m->loss);
    MCU(cudaGetLastError());
    return FSS_OK;
}

}  // namespace

extern "C" {

int fss_mlp_create(int32_t device, fss_mlp** out) {
    if (!out) return mlp_fail(FSS_ERR_INVALID, "null argument");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return mlp_fail(FSS_ERR_UNSUPPORTED, "no CUDA device");
    }
    fss_mlp* m = new fss_mlp();
    m->dev = device;
    auto bad = [&](int code) { delete m; return code; };
    if (cudaSetDevice(device) != cudaSuccess) return bad(mlp_fail(FSS_ERR_INVALID, "bad device"));
    if (cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&m->p, sizeof(float) * kMlpParams) != cudaSuccess ||
        cudaMalloc(&m->m1, sizeof(float) * kMlpParams) != cudaSuccess ||
        cudaMalloc(&m->m2, sizeof(float) * kMlpParams) != cudaSuccess ||
        cudaMalloc(&m->grad, sizeof(float) * kMlpParams) != cudaSuccess ||
        cudaMalloc(&m->loss, sizeof(float)) != cudaSuccess ||
        cudaMalloc(&m->wb, sizeof(__nv_bfloat16) * kMlpParams) != cudaSuccess)
        return bad(mlp_fail(FSS_ERR_NOMEM, "device allocation failed"));
    m->host_p.assign(kMlpParams, 0.f);
    *out = m;
    return fss_mlp_init(m, 1);
}

void fss_mlp_destroy(fss_mlp* m) {
    if (!m) return;
    cudaSetDevice(m->dev);
    cudaStreamSynchronize(m->st);
    delete m;
}

int32_t fss_mlp_param_count(void) { return kMlpParams; }

int fss_mlp_init(fss_mlp* m, uint64_t seed) {
    if (!m) return mlp_fail(FSS_ERR_INVALID, "null mlp");
    std::mt19937_64 rng(seed);
    std::normal_distribution<float> nd(0.f, 1.f);
    std::vector<float> p(kMlpParams, 0.f);
    for (int k = 0; k < kHid * kIn; k++) p[oW1 + k] = nd(rng) * std::sqrt(2.f / kIn);
    for (int k = 0; k < kHid * kHid; k++) p[oW2 + k] = nd(rng) * std::sqrt(2.f / kHid);
    for (int k = 0; k < kOut * kHid; k++) p[oW3 + k] = nd(rng) * std::sqrt(1.f / kHid);
    return fss_mlp_set_params(m, p.data());
}

int fss_mlp_set_params(fss_mlp* m, const float* params) {
    if (!m || !params) return mlp_fail(FSS_ERR_INVALID, "null argument");
    MCU(cudaSetDevice(m->dev));
    MCU(cudaMemcpyAsync(m->p, params, sizeof(float) * kMlpParams, cudaMemcpyHostToDevice, m->st));
    MCU(cudaMemsetAsync(m->m1, 0, sizeof(float) * kMlpParams, m->st));
    MCU(cudaMemsetAsync(m->m2, 0, sizeof(float) * kMlpParams, m->st));
    m->step = 0;
    int r = sync_weights(m);
    if (r) return r;
    MCU(cudaStreamSynchronize(m->st));
    return FSS_OK;
}

int fss_mlp_get_params(fss_mlp* m, float* params) {
    if (!m || !params) return mlp_fail(FSS_ERR_INVALID, "null argument");
    MCU(cudaSetDevice(m->dev));
    MCU(cudaMemcpyAsync(params, m->p, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost, m->st));
    MCU(cudaStreamSynchronize(m->st));
    return FSS_OK;
}

int fss_mlp_set_data(fss_mlp* m, int64_t n, const float* X, const float* T, const float* M) {
    if (!m || !X || !T || n <= 0) return mlp_fail(FSS_ERR_INVALID, "bad training data");
    MCU(cudaSetDevice(m->dev));
    for (void* q : {(void*)m->X, (void*)m->T, (void*)m->M, (void*)m->idx})
        if (q) cudaFree(q);
    m->X = nullptr; m->T = nullptr; m->M = nullptr; m->idx = nullptr;
    std::vector<__nv_bfloat16> xb(size_t(n) * kIn);
    for (size_t i = 0; i < xb.size(); i++) xb[i] = __float2bfloat16(X[i]);
    MCU(cudaMalloc(&m->X, sizeof(__nv_bfloat16) * xb.size()));
    MCU(cudaMalloc(&m->T, sizeof(float) * n * kOut));
    MCU(cudaMalloc(&m->idx, sizeof(int64_t) * n));
    MCU(cudaMemcpyAsync(m->X, xb.data(), sizeof(__nv_bfloat16) * xb.size(), cudaMemcpyHostToDevice, m->st));
    MCU(cudaMemcpyAsync(m->T, T, sizeof(float) * n * kOut, cudaMemcpyHostToDevice, m->st));
    if (M) {
        MCU(cudaMalloc(&m->M, sizeof(float) * n * kOut));
        MCU(cudaMemcpyAsync(m->M, M, sizeof(float) * n * kOut, cudaMemcpyHostToDevice, m->st));
    }
    MCU(cudaStreamSynchronize(m->st));
    m->n = n;
    return FSS_OK;
}

int fss_mlp_gradient(fss_mlp* m, float* grad, double* loss) {
    if (!m || !m->X) return mlp_fail(FSS_ERR_STATE, "no training data");
    MCU(cudaSetDevice(m->dev));
    std::vector<int64_t> id(m->n);
    for (int64_t i = 0; i < m->n; i++) id[i] = i;
    MCU(cudaMemcpyAsync(m->idx, id.data(), sizeof(int64_t) * m->n, cudaMemcpyHostToDevice, m->st));
    int r = grad_pass(m, m->idx, m->n);
    if (r) return r;
    float l = 0;
    if (grad) MCU(cudaMemcpyAsync(grad, m->grad, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost, m->st));
    MCU(cudaMemcpyAsync(&l, m->loss, sizeof(float), cudaMemcpyDeviceToHost, m->st));
    MCU(cudaStreamSynchronize(m->st));
    if (loss) *loss = l;
    return FSS_OK;
}

int fss_mlp_train(fss_mlp* m, int32_t epochs, int32_t batch, double lr, uint64_t seed, double* losses) {
    if (!m || !m->X) return mlp_fail(FSS_ERR_STATE, "no training data");
    if (epochs < 0 || batch < kMlpTile) return mlp_fail(FSS_ERR_INVALID, "bad epochs or batch");
    MCU(cudaSetDevice(m->dev));
    std::mt19937_64 rng(seed);
    std::vector<int64_t> id(m->n);
    for (int64_t i = 0; i < m->n; i++) id[i] = i;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int ep = 0; ep < epochs; ep++) {
        std::shuffle(id.begin(), id.end(), rng);
        MCU(cudaMemcpyAsync(m->idx, id.data(), sizeof(int64_t) * m->n, cudaMemcpyHostToDevice, m->st));
        double lsum = 0;
        int nb = 0;
        for (int64_t s = 0; s < m->n; s += batch) {
            const int64_t nbatch = std::min<int64_t>(batch, m->n - s);
            int r = grad_pass(m, m->idx + s, nbatch);
            if (r) return r;
            m->step++;
            const float c1 = 1.f - std::pow(b1, float(m->step)), c2 = 1.f - std::pow(b2, float(m->step));
            k_mlp_adam<<<(kMlpParams + 255) / 256, 256, 0, m->st>>>(m->p, m->m1, m->m2, m->grad, float(lr), b1, b2,
                                                                     eps, c1, c2, m->wb);
            MCU(cudaGetLastError());
            float l = 0;
            MCU(cudaMemcpyAsync(&l, m->loss, sizeof(float), cudaMemcpyDeviceToHost, m->st));
            MCU(cudaStreamSynchronize(m->st));
            lsum += l;
            nb++;
        }
        if (losses) losses[ep] = nb ? lsum / nb : 0.0;
    }
    return FSS_OK;
}

int fss_mlp_predict(fss_mlp* m, int64_t n, const float* X, float* Y) {
    if (!m || !X || !Y || n < 0) return mlp_fail(FSS_ERR_INVALID, "bad argument");
    if (n == 0) return FSS_OK;
    MCU(cudaSetDevice(m->dev));
    std::vector<__nv_bfloat16> xb(size_t(n) * kIn);
    for (size_t i = 0; i < xb.size(); i++) xb[i] = __float2bfloat16(X[i]);
    __nv_bfloat16* dx = nullptr;
    float* dy = nullptr;
    MCU(cudaMalloc(&dx, sizeof(__nv_bfloat16) * xb.size()));
    if (cudaMalloc(&dy, sizeof(float) * n * kOut) != cudaSuccess) {
        cudaFree(dx);
        return mlp_fail(FSS_ERR_NOMEM, "device allocation failed");
    }
    cudaMemcpyAsync(dx, xb.data(), sizeof(__nv_bfloat16) * xb.size(), cudaMemcpyHostToDevice, m->st);
    k_mlp_forward<<<unsigned((n + kMlpTile - 1) / kMlpTile), kMlpTile, 0, m->st>>>(n, dx, m->wb, m->p, dy);
    cudaMemcpyAsync(Y, dy, sizeof(float) * n * kOut, cudaMemcpyDeviceToHost, m->st);
    const cudaError_t e = cudaStreamSynchronize(m->st);
    cudaFree(dx);
    cudaFree(dy);
    if (e != cudaSuccess) return mlp_fail(FSS_ERR_CUDA, std::string("mlp predict: ") + cudaGetErrorString(e));
    return FSS_OK;
}

}  // extern "C"
