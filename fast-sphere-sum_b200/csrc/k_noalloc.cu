// k_noalloc.cu -- a direct-sum entry point that allocates no memory.
//
// Some callers of this library cannot call cudaMalloc: a real-time loop in
// which an allocation or free could synchronise the device and stall it, or
// a plugin hosted by an application whose memory manager owns the whole
// device budget and forbids allocations from outside.  fss_rhs_direct_noalloc
// serves them: the caller passes device buffers for the inputs and the
// output, and the only scratch this path needs -- the FP32 source array of
// the mixed-precision direct sum -- lives in a fixed file-scope device array.
//
// Costs and limits: every GPU that loads the library holds that array
// (kNoAllocMaxParticles x 16 bytes = 4 MiB) until the process exits; larger
// particle counts are rejected.  With CUDA's lazy module loading (the
// default), the module holding the array -- and so the 4 MiB -- is loaded on
// a device by the first call there; a caller that must not see that happen
// inside its loop makes one call at start-up (before any stream capture).
// All calls share the array, and each call overwrites the entries it uses
// before reading them, so no clearing is needed; but two calls whose kernels
// overlap on the GPU (different streams, or different host threads) race on
// it.
#include <cuda_runtime.h>

#include <string>

#include "device_common.cuh"
#include "fss.h"

namespace fss {

constexpr int64_t kNoAllocMaxParticles = FSS_NOALLOC_MAX_PARTICLES;

void set_last_error(const std::string& msg);  // fss.cpp: message for fss_last_error(NULL)
constexpr int kNaThreads = 128;
constexpr int kNaTile = 256;

// The scratch: one float4 {x, y, z, zeta*A} per particle.
static __device__ __align__(256) float4 g_noalloc_src[kNoAllocMaxParticles];

// Host code must not pass g_noalloc_src itself (on the host it is only a
// stand-in, not a device address): every call looks up the array's device
// address on the current device with cudaGetSymbolAddress (cheap once the
// module is loaded), so no address outlives a device reset or a re-created
// context.

__global__ void k_na_pack(int64_t n, const double* __restrict__ state5, const double* __restrict__ area,
                          float4* __restrict__ src) {
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double* p = state5 + 5 * i;
    src[i] = make_float4(float(p[0]), float(p[1]), float(p[2]), float(p[3] * area[i]));
}

// One block per 128 targets, all sources streamed through shared memory in
// tiles of 256; per pair d = x_j - x_i, A += w_j d / |d|^2 (the self pair,
// d = 0, contributes nothing); u_i = -(1/2pi) x_i x A; per-tile FP32 sums
// folded into a Kahan-compensated total.
__global__ void __launch_bounds__(kNaThreads) k_na_direct(int64_t n, const float4* __restrict__ src,
                                                          const double* __restrict__ state5, double omega,
                                                          double* __restrict__ modify5) {
    __shared__ float4 tile[kNaTile];
    const int64_t i = int64_t(blockIdx.x) * kNaThreads + threadIdx.x;
    const bool valid = i < n;
    const float4 t = src[valid ? i : 0];
    float sx = 0, sy = 0, sz = 0, cx = 0, cy = 0, cz = 0;
    for (int64_t base = 0; base < n; base += kNaTile) {
        const int cnt = int((n - base < kNaTile) ? (n - base) : kNaTile);
        __syncthreads();
        for (int k = threadIdx.x; k < cnt; k += kNaThreads) tile[k] = src[base + k];
        __syncthreads();
        float ax = 0, ay = 0, az = 0;
        for (int j = 0; j < cnt; j++) {
            const float4 q = tile[j];
            const float dx = q.x - t.x, dy = q.y - t.y, dz = q.z - t.z;
            const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
            const float inv = (r2 > 0.f) ? rcp_fast(r2) : 0.f;
            const float sc = q.w * inv;
            ax = fmaf(sc, dx, ax);
            ay = fmaf(sc, dy, ay);
            az = fmaf(sc, dz, az);
        }
        float y, s;
        y = ax - cx; s = sx + y; cx = (s - sx) - y; sx = s;
        y = ay - cy; s = sy + y; cy = (s - sy) - y; sy = s;
        y = az - cz; s = sz + y; cz = (s - sz) - y; sz = s;
    }
    if (!valid) return;
    const double Ax = double(sx) - double(cx), Ay = double(sy) - double(cy), Az = double(sz) - double(cz);
    const double* x = state5 + 5 * i;
    const double c = -1.0 / (2.0 * M_PI);
    const double ux = c * (x[1] * Az - x[2] * Ay);
    const double uy = c * (x[2] * Ax - x[0] * Az);
    const double uz = c * (x[0] * Ay - x[1] * Ax);
    double* m = modify5 + 5 * i;
    m[0] = ux;
    m[1] = uy;
    m[2] = uz;
    m[3] = -2 * omega * uz;
    m[4] = 0.0 * (-1.0 / (4.0 * M_PI));
}

}  // namespace fss

using namespace fss;

extern "C" int fss_rhs_direct_noalloc(int64_t n, const double* state5, const double* area, double omega,
                                      double* modify5, void* stream) {
    if (!state5 || !area || !modify5) {
        set_last_error("fss_rhs_direct_noalloc: null buffer");
        return FSS_ERR_INVALID;
    }
    if (n < 2) {
        set_last_error("fss_rhs_direct_noalloc: need at least 2 particles");
        return FSS_ERR_INVALID;
    }
    if (n > kNoAllocMaxParticles) {
        set_last_error("fss_rhs_direct_noalloc: " + std::to_string(n) + " particles exceed its fixed scratch of " +
                       std::to_string(kNoAllocMaxParticles) + "; use fss_rhs_direct");
        return FSS_ERR_CAPACITY;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        set_last_error("fss_rhs_direct_noalloc: no current CUDA device");
        return FSS_ERR_CUDA;
    }
    // the array's address on the current device (its module is loaded there
    // by the first call under lazy loading)
    void* scratch = nullptr;
    const cudaError_t ge = cudaGetSymbolAddress(&scratch, g_noalloc_src);
    if (ge != cudaSuccess || !scratch) {
        cudaGetLastError();
        set_last_error(std::string("fss_rhs_direct_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(ge));
        return FSS_ERR_CUDA;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    float4* src = static_cast<float4*>(scratch);
    k_na_pack<<<unsigned((n + 255) / 256), 256, 0, st>>>(n, state5, area, src);
    k_na_direct<<<unsigned((n + kNaThreads - 1) / kNaThreads), kNaThreads, 0, st>>>(n, src, state5, omega, modify5);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_last_error(std::string("fss_rhs_direct_noalloc: launch: ") + cudaGetErrorString(e));
        return FSS_ERR_CUDA;
    }
    return FSS_OK;
}
