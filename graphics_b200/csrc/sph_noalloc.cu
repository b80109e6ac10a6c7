// sph_noalloc.cu -- the CFL time step of sphgpu_step (k_cfl in sph_dfsph.cu)
// as a stand-alone entry point that allocates nothing: its block partials and
// its last-block ticket live in file-scope device arrays.
//
// A velocity with a non-finite component makes the maximum NaN (the
// reduction propagates NaN instead of dropping it as fmax would), so the
// caller sees NaN in vmax_out and dt_out rather than a step length computed
// from the remaining particles.
#include <cuda_runtime.h>
#include <math_constants.h>

#include <mutex>

#include "../../include/sphgpu.h"

#define NOALLOC_NT 256
#define NOALLOC_ITEMS 8
#define NOALLOC_BLOCKS (SPHGPU_NOALLOC_MAX_N / (NOALLOC_NT * NOALLOC_ITEMS))  // 4096
#define NOALLOC_MAX_DEVICES 64

// one FP64 partial maximum per block (32 KB) and the last-block ticket; the
// ticket is zero when the module loads and every call leaves it at zero
static __device__ __align__(256) double g_cfl_partial[NOALLOC_BLOCKS];
static __device__ __align__(256) unsigned g_cfl_ticket;

namespace {

// max that keeps NaN: fmax(NaN, x) returns x, which would hide a bad velocity
__device__ __forceinline__ double nan_max(double a, double b) { return (a != a || b != b) ? CUDART_NAN : fmax(a, b); }

__global__ void __launch_bounds__(NOALLOC_NT) k_cfl_noalloc(const float* __restrict__ v, int n, int stride,
                                                            float cfl, float d, float dt_max, float dt_min,
                                                            float* dt_out, double* vmax_out, double* partial,
                                                            unsigned* ticket) {
    double m = 0.0;
    const int base = blockIdx.x * NOALLOC_NT * NOALLOC_ITEMS + threadIdx.x;
#pragma unroll
    for (int k = 0; k < NOALLOC_ITEMS; ++k) {
        const int i = base + k * NOALLOC_NT;
        if (i < n) {
            const float* p = v + (size_t)i * stride;
            const double x = p[0], y = p[1], z = p[2];
            const bool ok = isfinite(x) && isfinite(y) && isfinite(z);
            m = nan_max(m, ok ? sqrt(x * x + y * y + z * z) : CUDART_NAN);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = nan_max(m, __shfl_down_sync(0xffffffffu, m, o));
    __shared__ double sh[NOALLOC_NT / 32];
    __shared__ bool last;
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = 0.0;
        for (int i = 0; i < NOALLOC_NT / 32; ++i) b = nan_max(b, sh[i]);
        partial[blockIdx.x] = b;
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double vm = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += NOALLOC_NT) vm = nan_max(vm, ((volatile double*)partial)[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) vm = nan_max(vm, __shfl_down_sync(0xffffffffu, vm, o));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = vm;
    __syncthreads();
    if (threadIdx.x == 0) {
        double vmax = 0.0;
        for (int i = 0; i < NOALLOC_NT / 32; ++i) vmax = nan_max(vmax, sh[i]);
        // the same rule as the in-step CFL reduction; NaN stays NaN
        double dt = vmax > 0 ? (double)cfl * (double)d / vmax : (double)dt_max;
        if (dt > dt_max) dt = dt_max;
        if (dt < dt_min) dt = dt_min;
        if (vmax != vmax) dt = CUDART_NAN;
        *dt_out = (float)dt;
        if (vmax_out) *vmax_out = vmax;
        *ticket = 0u;
    }
}

std::mutex g_setup_mu;
double* g_partial_ptr[NOALLOC_MAX_DEVICES];
unsigned* g_ticket_ptr[NOALLOC_MAX_DEVICES];

}  // namespace

extern "C" int sphgpu_cfl_dt_noalloc(const float* vel, int n, int stride, float cfl_factor, float d, float dt_max,
                                     float dt_min, float* dt_out, double* vmax_out, void* stream) {
    if (n < 0 || n > SPHGPU_NOALLOC_MAX_N || stride < 3 || !dt_out || (n > 0 && !vel)) return SPHGPU_EINVAL;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return SPHGPU_ECUDA;
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return SPHGPU_EINVAL;
    double* partial;
    unsigned* ticket;
    {
        // set-up, once per device: the device addresses of the static scratch
        std::lock_guard<std::mutex> lock(g_setup_mu);
        if (!g_partial_ptr[dev]) {
            double* p = nullptr;
            unsigned* t = nullptr;
            if (cudaGetSymbolAddress((void**)&p, g_cfl_partial) != cudaSuccess) return SPHGPU_ECUDA;
            if (cudaGetSymbolAddress((void**)&t, g_cfl_ticket) != cudaSuccess) return SPHGPU_ECUDA;
            g_ticket_ptr[dev] = t;
            g_partial_ptr[dev] = p;
        }
        partial = g_partial_ptr[dev];
        ticket = g_ticket_ptr[dev];
    }
    const int per_block = NOALLOC_NT * NOALLOC_ITEMS;
    const int blocks = n > 0 ? (n + per_block - 1) / per_block : 1;
    k_cfl_noalloc<<<blocks, NOALLOC_NT, 0, (cudaStream_t)stream>>>(vel, n, stride, cfl_factor, d, dt_max, dt_min,
                                                                   dt_out, vmax_out, partial, ticket);
    // peek, not get: an earlier asynchronous error belongs to whoever caused
    // it and stays visible to them
    return cudaPeekAtLastError() == cudaSuccess ? 0 : SPHGPU_ECUDA;
}
