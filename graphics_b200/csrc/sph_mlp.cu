// sph_mlp.cu -- learned warm start for the DFSPH constant-density loop.
//
// The network (16 -> 64 -> 64 -> 1, GELU) predicts, per particle, the total
// stiffness kappa_sum that the density loop (DFSPH.cpp:566-700) applies over
// all of its iterations.  kappa ~ p / rho (the loop's velocity update
// dt sum m (k_i/rho_i + k_j/rho_j) gradW is the pressure acceleration with
// p/rho^2 = kappa/rho), so it is set by the flow (about g times depth) and
// does not scale with the step length, which makes it a stable target.  The
// prediction is applied once before the loop as a pressure-velocity
// correction of the same form as DFSPH.cpp:674; the unmodified loop then
// runs to the same tolerance, so the network only changes where the loop
// starts, and the gain is counted in iterations.
//
// GEMMs run on the tensor cores with mma.sync.m16n8k16 (BF16 operands, FP32
// accumulation): a 128-row tile per 4-warp block, each warp owning 32 rows.
// Training (forward + backward of a mini-batch, FP32 gradient atomics) and
// Adam (FP32 master weights, BF16 copies for the GEMMs) are separate
// kernels; inference is fused into the per-particle feature sweep.
#include <cuda_bf16.h>

#include "sph_kernels.cuh"
#include "sph_mlp.cuh"

namespace {

constexpr int TR = 128;  // rows per block tile (4 warps x 32)

// GELU in its tanh form, 0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3))),
// with the hardware tanh (PTX tanh.approx.f32, relative error about 2^-11,
// below the BF16 rounding the activations take next); the same form in
// training, inference and the CPU restatement (oracle/mlp_oracle.py)
__device__ __forceinline__ float tanh_hw(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
// u = sqrt(2/pi) (z + 0.044715 z^3) = z (k0 + k1 z^2), k0 = sqrt(2/pi),
// k1 = 0.044715 sqrt(2/pi); GELU = h + h tanh(u) with h = z / 2 (five FP32
// operations and one tanh per activation: the inference kernel is bound by
// this elementwise work, not by its GEMMs)
__device__ __forceinline__ float gelu(float z) {
    const float u = z * fmaf(0.0356774081f, z * z, 0.7978845608f);
    const float hz = 0.5f * z;
    return fmaf(hz, tanh_hw(u), hz);
}
// GELU of two activations at once with sm_100's packed FP32 operations
// (f32x2: each lane rounded as its scalar form), the same operations in the
// same order as gelu(), so the results are the same bit for bit; in:
// z = acc + bias per lane, out: the pair rounded to BF16 and packed
__device__ __forceinline__ unsigned long long f2(float lo, float hi) {
    unsigned long long r;
    asm("mov.b64 %0, {%1,%2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void gelu_x2(float a0, float a1, float2 bias, float& g0, float& g1) {
    unsigned long long z, zz, k, u, hz, t, g;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(z) : "l"(f2(a0, a1)), "l"(f2(bias.x, bias.y)));
    asm("mul.rn.f32x2 %0, %1, %1;" : "=l"(zz) : "l"(z));
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(k) : "l"(f2(0.0356774081f, 0.0356774081f)), "l"(zz),
        "l"(f2(0.7978845608f, 0.7978845608f)));
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(u) : "l"(z), "l"(k));
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(hz) : "l"(f2(0.5f, 0.5f)), "l"(z));
    float u0, u1;
    asm("mov.b64 {%0,%1}, %2;" : "=f"(u0), "=f"(u1) : "l"(u));
    t = f2(tanh_hw(u0), tanh_hw(u1));
    asm("fma.rn.f32x2 %0, %1, %2, %1;" : "=l"(g) : "l"(hz), "l"(t));
    asm("mov.b64 {%0,%1}, %2;" : "=f"(g0), "=f"(g1) : "l"(g));
}

// d/dz: (1 + t) / 2 + (z / 2) (1 - t^2) (k0 + 3 k1 z^2)
__device__ __forceinline__ float gelu_d(float z) {
    const float z2 = z * z;
    const float t = tanh_hw(z * fmaf(0.0356774081f, z2, 0.7978845608f));
    return fmaf(0.5f, t, 0.5f) + 0.5f * z * fmaf(-t, t, 1.f) * fmaf(0.1070322243f, z2, 0.7978845608f);
}

__device__ __forceinline__ uint32_t pack2(__nv_bfloat16 lo, __nv_bfloat16 hi) {
    return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

__device__ __forceinline__ void mma16816(float c[4], const uint32_t a[4], const uint32_t b[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// One 16x8 output tile accumulated over K (multiple of 16):
//   C(m0.., n0..) += sum_k A(m, k) B(k, n)
// with A(m, k) = A[m*am + k*ak] and B(k, n) = B[k*bk + n*bn] (BF16, shared
// memory).  Fragment layout of m16n8k16 (PTX ISA): g = lane/4, t = lane%4.
__device__ __forceinline__ void tile_mma(float c[4], const __nv_bfloat16* A, int am, int ak, const __nv_bfloat16* B,
                                         int bk, int bn, int m0, int n0, int K) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    for (int k0 = 0; k0 < K; k0 += 16) {
        uint32_t a[4], b[2];
        const int r0 = m0 + g, r1 = m0 + g + 8, ka = k0 + 2 * t;
        a[0] = pack2(A[r0 * am + ka * ak], A[r0 * am + (ka + 1) * ak]);
        a[1] = pack2(A[r1 * am + ka * ak], A[r1 * am + (ka + 1) * ak]);
        a[2] = pack2(A[r0 * am + (ka + 8) * ak], A[r0 * am + (ka + 9) * ak]);
        a[3] = pack2(A[r1 * am + (ka + 8) * ak], A[r1 * am + (ka + 9) * ak]);
        const int n = n0 + g;
        b[0] = pack2(B[ka * bk + n * bn], B[(ka + 1) * bk + n * bn]);
        b[1] = pack2(B[(ka + 8) * bk + n * bn], B[(ka + 9) * bk + n * bn]);
        mma16816(c, a, b);
    }
}

struct FwdSmem {
    __nv_bfloat16 X[TR * MLP_IN];
    __nv_bfloat16 W1[MLP_IN * MLP_H];
    __nv_bfloat16 W2[MLP_H * MLP_H];
    __nv_bfloat16 H1[TR * MLP_H];
    float Z1[TR * MLP_H];
    float Z2[TR * MLP_H];
    float W3[MLP_H], b1[MLP_H], b2[MLP_H];
    float b3;
};

struct TrainSmem {
    FwdSmem f;
    __nv_bfloat16 dZ2[TR * MLP_H];
    __nv_bfloat16 dZ1[TR * MLP_H];
    float g[TR];
    float pw3[TR / 32][MLP_H], pb2[TR / 32][MLP_H];  // per-warp partials
    float pb3[TR / 32], ploss[TR / 32];
};

// weights into shared memory (BF16 GEMM copies, FP32 biases)
__device__ __forceinline__ void load_weights(const MlpDev& m, FwdSmem& S) {
    for (int i = threadIdx.x; i < MLP_IN * MLP_H; i += blockDim.x) S.W1[i] = m.w_bf16[MLP_OFF_W1 + i];
    for (int i = threadIdx.x; i < MLP_H * MLP_H; i += blockDim.x) S.W2[i] = m.w_bf16[MLP_OFF_W2 + i];
    for (int i = threadIdx.x; i < MLP_H; i += blockDim.x) {
        S.W3[i] = __bfloat162float(m.w_bf16[MLP_OFF_W3 + i]);
        S.b1[i] = m.master[MLP_OFF_B1 + i];
        S.b2[i] = m.master[MLP_OFF_B2 + i];
    }
    if (threadIdx.x == 0) S.b3 = m.master[MLP_OFF_B3];
}

// Forward pass of the warp's 32 rows (S.X filled, weights loaded):
// Z1, H1 (BF16), Z2 in shared memory; returns y for row lane of the warp.
__device__ __forceinline__ float forward_rows(FwdSmem& S) {
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int r0 = w * 32;
    // layer 1: Z1 = X W1 + b1   (K = 16)
    for (int mt = 0; mt < 2; ++mt)
        for (int nt = 0; nt < MLP_H / 8; ++nt) {
            float c[4] = {0.f, 0.f, 0.f, 0.f};
            tile_mma(c, S.X, MLP_IN, 1, S.W1, MLP_H, 1, r0 + mt * 16, nt * 8, MLP_IN);
            const int ra = r0 + mt * 16 + g, col = nt * 8 + 2 * t;
            const float z[4] = {c[0] + S.b1[col], c[1] + S.b1[col + 1], c[2] + S.b1[col], c[3] + S.b1[col + 1]};
            S.Z1[ra * MLP_H + col] = z[0];
            S.Z1[ra * MLP_H + col + 1] = z[1];
            S.Z1[(ra + 8) * MLP_H + col] = z[2];
            S.Z1[(ra + 8) * MLP_H + col + 1] = z[3];
            S.H1[ra * MLP_H + col] = __float2bfloat16_rn(gelu(z[0]));
            S.H1[ra * MLP_H + col + 1] = __float2bfloat16_rn(gelu(z[1]));
            S.H1[(ra + 8) * MLP_H + col] = __float2bfloat16_rn(gelu(z[2]));
            S.H1[(ra + 8) * MLP_H + col + 1] = __float2bfloat16_rn(gelu(z[3]));
        }
    __syncwarp();
    // layer 2: Z2 = H1 W2 + b2   (K = 64)
    for (int mt = 0; mt < 2; ++mt)
        for (int nt = 0; nt < MLP_H / 8; ++nt) {
            float c[4] = {0.f, 0.f, 0.f, 0.f};
            tile_mma(c, S.H1, MLP_H, 1, S.W2, MLP_H, 1, r0 + mt * 16, nt * 8, MLP_H);
            const int ra = r0 + mt * 16 + g, col = nt * 8 + 2 * t;
            S.Z2[ra * MLP_H + col] = c[0] + S.b2[col];
            S.Z2[ra * MLP_H + col + 1] = c[1] + S.b2[col + 1];
            S.Z2[(ra + 8) * MLP_H + col] = c[2] + S.b2[col];
            S.Z2[(ra + 8) * MLP_H + col + 1] = c[3] + S.b2[col + 1];
        }
    __syncwarp();
    // layer 3: y = gelu(Z2) W3 + b3 (row = lane), FP32
    const int row = r0 + lane;
    float y = S.b3;
#pragma unroll 8
    for (int j = 0; j < MLP_H; ++j) y = fmaf(gelu(S.Z2[row * MLP_H + j]), S.W3[j], y);
    return y;
}

// ---------------- training ----------------

// one 128-row tile of a mini-batch: forward, MSE gradient, backward; the
// tile's gradient goes to its own slot of m.gpart (k_mlp_reduce sums the
// slots in order).  inv_total = 1 / (rows in the mini-batch).
__global__ void __launch_bounds__(TR) k_mlp_train(MlpDev m, const float* X, const float* y, int n, int b0, int bsz,
                                                 float inv_total) {
    extern __shared__ __align__(16) unsigned char smraw[];
    TrainSmem& S = *reinterpret_cast<TrainSmem*>(smraw);
    const int tile0 = b0 + blockIdx.x * TR;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    load_weights(m, S.f);
    const float* nrm = m.norm;
    for (int i = threadIdx.x; i < TR * MLP_IN; i += TR) {
        const int r = i / MLP_IN, c = i % MLP_IN;
        const int row = tile0 + r;
        float v = 0.f;
        if (row < b0 + bsz && row < n) v = (X[(size_t)row * MLP_IN + c] - nrm[c]) * nrm[MLP_IN + c];
        S.f.X[i] = __float2bfloat16_rn(v);
    }
    __syncthreads();
    const float yhat = forward_rows(S.f);
    const int myrow = tile0 + w * 32 + lane;
    const bool valid = myrow < b0 + bsz && myrow < n;
    const float target = valid ? (y[myrow] - nrm[2 * MLP_IN]) * nrm[2 * MLP_IN + 1] : 0.f;
    const float err = valid ? yhat - target : 0.f;
    const float gr = 2.f * err * inv_total;  // dL/dy, L = mean (y - t)^2
    S.g[w * 32 + lane] = gr;
    float* gp = m.gpart + (size_t)blockIdx.x * MLP_NPARAM_PAD;
    // loss
    float se = err * err;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) se += __shfl_down_sync(0xffffffffu, se, o);
    if (lane == 0) S.ploss[w] = se;
    __syncwarp();
    // output layer: dW3_j = sum_r g_r gelu(Z2_rj), db3 = sum g; dZ2 = g W3_j gelu'(Z2)
    const int r0 = w * 32;
    for (int j = lane; j < MLP_H; j += 32) {
        float s3 = 0.f, sb = 0.f;
        for (int r = 0; r < 32; ++r) {
            const float z = S.f.Z2[(r0 + r) * MLP_H + j];
            const float gg = S.g[r0 + r];
            s3 = fmaf(gg, gelu(z), s3);
            const float dz = gg * S.f.W3[j] * gelu_d(z);
            sb += dz;
            S.dZ2[(r0 + r) * MLP_H + j] = __float2bfloat16_rn(dz);
        }
        S.pw3[w][j] = s3;
        S.pb2[w][j] = sb;
    }
    if (lane == 0) {
        float sg = 0.f;
        for (int r = 0; r < 32; ++r) sg += S.g[r0 + r];
        S.pb3[w] = sg;
    }
    __syncwarp();
    // dH1 = dZ2 W2^T, dZ1 = dH1 * gelu'(Z1)   (B(k=j2, n=j1) = W2[j1][j2])
    for (int mt = 0; mt < 2; ++mt)
        for (int nt = 0; nt < MLP_H / 8; ++nt) {
            float c[4] = {0.f, 0.f, 0.f, 0.f};
            tile_mma(c, S.dZ2, MLP_H, 1, S.f.W2, 1, MLP_H, r0 + mt * 16, nt * 8, MLP_H);
            const int ra = r0 + mt * 16 + g, col = nt * 8 + 2 * t;
            S.dZ1[ra * MLP_H + col] = __float2bfloat16_rn(c[0] * gelu_d(S.f.Z1[ra * MLP_H + col]));
            S.dZ1[ra * MLP_H + col + 1] = __float2bfloat16_rn(c[1] * gelu_d(S.f.Z1[ra * MLP_H + col + 1]));
            S.dZ1[(ra + 8) * MLP_H + col] = __float2bfloat16_rn(c[2] * gelu_d(S.f.Z1[(ra + 8) * MLP_H + col]));
            S.dZ1[(ra + 8) * MLP_H + col + 1] =
                __float2bfloat16_rn(c[3] * gelu_d(S.f.Z1[(ra + 8) * MLP_H + col + 1]));
        }
    __syncthreads();
    // the warps' W3 / b2 / b3 / loss partials, in warp order
    for (int j = threadIdx.x; j < MLP_H; j += TR) {
        float a = 0.f, b = 0.f;
        for (int v = 0; v < TR / 32; ++v) { a += S.pw3[v][j]; b += S.pb2[v][j]; }
        gp[MLP_OFF_W3 + j] = a;
        gp[MLP_OFF_B2 + j] = b;
    }
    if (threadIdx.x == 0) {
        float a = 0.f, l = 0.f;
        for (int v = 0; v < TR / 32; ++v) { a += S.pb3[v]; l += S.ploss[v]; }
        gp[MLP_OFF_B3] = a;
        m.gpart[(size_t)gridDim.x * MLP_NPARAM_PAD + blockIdx.x] = l;
    }
    // db1 (from the BF16 dZ1 the GEMMs use)
    for (int j = threadIdx.x; j < MLP_H; j += TR) {
        float sb = 0.f;
        for (int r = 0; r < TR; ++r) sb += __bfloat162float(S.dZ1[r * MLP_H + j]);
        gp[MLP_OFF_B1 + j] = sb;
    }
    // dW2 = H1^T dZ2 (64 x 64, K = 128 rows): 4 x 8 tiles, 8 per warp
    for (int tt = w; tt < 32; tt += 4) {
        const int mt = tt / 8, nt = tt % 8;
        float c[4] = {0.f, 0.f, 0.f, 0.f};
        tile_mma(c, S.f.H1, 1, MLP_H, S.dZ2, MLP_H, 1, mt * 16, nt * 8, TR);
        const int ra = mt * 16 + g, col = nt * 8 + 2 * t;
        gp[MLP_OFF_W2 + ra * MLP_H + col] = c[0];
        gp[MLP_OFF_W2 + ra * MLP_H + col + 1] = c[1];
        gp[MLP_OFF_W2 + (ra + 8) * MLP_H + col] = c[2];
        gp[MLP_OFF_W2 + (ra + 8) * MLP_H + col + 1] = c[3];
    }
    // dW1 = X^T dZ1 (16 x 64, K = 128): 1 x 8 tiles, 2 per warp
    for (int nt = w; nt < 8; nt += 4) {
        float c[4] = {0.f, 0.f, 0.f, 0.f};
        tile_mma(c, S.f.X, 1, MLP_IN, S.dZ1, MLP_H, 1, 0, nt * 8, TR);
        const int ra = g, col = nt * 8 + 2 * t;
        gp[MLP_OFF_W1 + ra * MLP_H + col] = c[0];
        gp[MLP_OFF_W1 + ra * MLP_H + col + 1] = c[1];
        gp[MLP_OFF_W1 + (ra + 8) * MLP_H + col] = c[2];
        gp[MLP_OFF_W1 + (ra + 8) * MLP_H + col + 1] = c[3];
    }
}

// gradient of the mini-batch = the tiles' gradients summed in tile order;
// the batch's squared error is added to m.loss (one thread, in order)
__global__ void k_mlp_reduce(MlpDev m, int blocks) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < MLP_NPARAM) {
        float a = 0.f;
        for (int b = 0; b < blocks; ++b) a += m.gpart[(size_t)b * MLP_NPARAM_PAD + i];
        m.grad[i] = a;
    }
    if (i == 0) {
        float l = 0.f;
        for (int b = 0; b < blocks; ++b) l += m.gpart[(size_t)blocks * MLP_NPARAM_PAD + b];
        *m.loss += l;
    }
}

// Adam on the FP32 master weights, BF16 copies for the GEMMs, gradient reset
__global__ void k_mlp_adam(MlpDev m, float lr, float bc1, float bc2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= MLP_NPARAM) return;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float gr = m.grad[i];
    const float mm = b1 * m.adam_m[i] + (1.f - b1) * gr;
    const float vv = b2 * m.adam_v[i] + (1.f - b2) * gr * gr;
    m.adam_m[i] = mm;
    m.adam_v[i] = vv;
    const float w = m.master[i] - lr * (mm / bc1) / (sqrtf(vv / bc2) + eps);
    m.master[i] = w;
    m.w_bf16[i] = __float2bfloat16_rn(w);
    m.grad[i] = 0.f;
}

__global__ void k_mlp_sync(MlpDev m) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < MLP_NPARAM) m.w_bf16[i] = __float2bfloat16_rn(m.master[i]);
}

__global__ void __launch_bounds__(TR) k_mlp_predict(MlpDev m, const float* X, float* y, int n) {
    extern __shared__ __align__(16) unsigned char smraw[];
    FwdSmem& S = *reinterpret_cast<FwdSmem*>(smraw);
    const int tile0 = blockIdx.x * TR;
    load_weights(m, S);
    const float* nrm = m.norm;
    for (int i = threadIdx.x; i < TR * MLP_IN; i += TR) {
        const int r = i / MLP_IN, c = i % MLP_IN;
        const int row = tile0 + r;
        const float v = row < n ? (X[(size_t)row * MLP_IN + c] - nrm[c]) * nrm[MLP_IN + c] : 0.f;
        S.X[i] = __float2bfloat16_rn(v);
    }
    __syncthreads();
    const float yh = forward_rows(S);
    const int row = tile0 + threadIdx.x;
    if (row < n) y[row] = yh / nrm[2 * MLP_IN + 1] + nrm[2 * MLP_IN];
}

}  // namespace

static size_t smem_train() { return sizeof(TrainSmem); }
static size_t smem_fwd() { return sizeof(FwdSmem); }

void mlp_init_attributes() {
    cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_train());
    cudaFuncSetAttribute(k_mlp_predict, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_fwd());
}

int mlp_train_blocks(int bsz) { return (bsz + TR - 1) / TR; }

void launch_mlp_train_batch(const MlpDev& m, const float* X, const float* y, int n, int b0, int bsz, float inv_total,
                            cudaStream_t st) {
    const int blocks = mlp_train_blocks(bsz);
    k_mlp_train<<<blocks, TR, smem_train(), st>>>(m, X, y, n, b0, bsz, inv_total);
    k_mlp_reduce<<<(MLP_NPARAM + 255) / 256, 256, 0, st>>>(m, blocks);
}

void launch_mlp_adam(const MlpDev& m, float lr, int t, cudaStream_t st) {
    const float bc1 = 1.f - powf(0.9f, (float)t), bc2 = 1.f - powf(0.999f, (float)t);
    k_mlp_adam<<<(MLP_NPARAM + 255) / 256, 256, 0, st>>>(m, lr, bc1, bc2);
}

void launch_mlp_sync_bf16(const MlpDev& m, cudaStream_t st) { k_mlp_sync<<<(MLP_NPARAM + 255) / 256, 256, 0, st>>>(m); }

void launch_mlp_predict(const MlpDev& m, const float* X, float* y, int n, cudaStream_t st) {
    if (n > 0) k_mlp_predict<<<(n + TR - 1) / TR, TR, smem_fwd(), st>>>(m, X, y, n);
}

// ===================== warm-start kernels on a scene =====================
namespace {

// Per-particle features (16, FP32) from the state after the non-pressure
// forces (v_adv known) and before the density loop, plus the prediction.
//  0 neighbour count / 32             8  |a_adv| dt^2 / d
//  1 (rho - rho0)/rho0 * 100          9  boundary-neighbour fraction
//  2 dt * Drho/Dt / rho0 * 100        10 log(alpha / alpha_ref)
//  3 (max(rho_adv0, rho0) - rho0)/rho0 * 100   11 neighbour mean of feature 4
//  4 kappa_sum of the previous step/10 12 dt / dt_max
//  5 feature 3 of the previous step   13 |sum_j m gradW_ij| d / rho0
//  6 feature 2 of the previous step   14 v_y dt / d
//  7 |v| dt / d                       15 1
__device__ __forceinline__ void ws_features(const DevScene& s, const SolverConst& c, int p, float dt, float dt_max,
                                            float alpha_ref, float x[MLP_IN], float& pred, float& divt) {
    const float4 pa = s.pv[2 * p];
    const float4 va = s.pv[2 * p + 1];
    const int cnt = s.ncount[p];
    const size_t stride = (size_t)c.stride;
    float acc = 0.f, ax = 0.f, ay = 0.f, az = 0.f, kp = 0.f;
    int nb = 0, nfl = 0;
    // four list entries per 16-byte load (the next group's issued before the
    // current group's record gathers); entries past the count read the
    // particle's own record and are masked out
    const int ng = (cnt + 3) >> 2;
    const unsigned long long polL = l2_policy(c.l2pol & 3);  // lists stream through L2
    int4 nxt = ng ? ell_group_pol(s.nbr, stride, p, 0, polL) : make_int4(0, 0, 0, 0);
    for (int gi = 0; gi < ng; ++gi) {
        const int4 cur = nxt;
        if (gi + 1 < ng) nxt = ell_group_pol(s.nbr, stride, p, gi + 1, polL);
        const unsigned e4[4] = {(unsigned)cur.x, (unsigned)cur.y, (unsigned)cur.z, (unsigned)cur.w};
        float4 pb[4], vb[4];
        bool ok[4], bnd[4];
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            ok[t] = gi * 4 + t < cnt;
            const unsigned u = ok[t] ? e4[t] : (unsigned)p;
            bnd[t] = (u & BND_FLAG) != 0u;
            ld_record32((bnd[t] ? s.bpv : s.pv) + 2 * (size_t)(u & BND_MASK), pb[t], vb[t]);
        }
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            if (!ok[t]) continue;
            const float m = bnd[t] ? c.rho0 * pb[t].w : c.fm0;
            const float xx = pa.x - pb[t].x, xy = pa.y - pb[t].y, xz = pa.z - pb[t].z;
            const float f = grad_over_r(c.k, xx * xx + xy * xy + xz * xz);
            acc = fmaf((xx * (va.x - vb[t].x) + xy * (va.y - vb[t].y) + xz * (va.z - vb[t].z)) * f, m, acc);
            ax = fmaf(xx * f, m, ax);
            ay = fmaf(xy * f, m, ay);
            az = fmaf(xz * f, m, az);
            if (bnd[t]) ++nb;
            else { kp += vb[t].w; ++nfl; }  // the neighbour's history, carried in its record (k_df_forces)
        }
    }
    const float rho0 = c.rho0, rho = s.rho[p], d = c.dpart;
    const float4 hp = s.hist[p];
    const float4 a = s.acc[p];
    const float4 v = s.vel[p];
    divt = dt * acc / rho0 * 100.f;
    const float dadv = fmaxf(fmaf(acc, dt, rho), rho0);
    pred = (dadv - rho0) / rho0 * 100.f;
    x[0] = cnt * (1.f / 32.f);
    x[1] = (rho - rho0) / rho0 * 100.f;
    x[2] = divt;
    x[3] = pred;
    x[4] = hp.x * 0.1f;
    x[5] = hp.y;
    x[6] = hp.z;
    x[7] = sqrtf(v.x * v.x + v.y * v.y + v.z * v.z) * dt / d;
    x[8] = sqrtf(a.x * a.x + a.y * a.y + a.z * a.z) * dt * dt / d;
    x[9] = cnt ? (float)nb / (float)cnt : 0.f;
    x[10] = logf(fmaxf(s.alpha[p], 1e-30f) / alpha_ref);
    x[11] = nfl ? 0.1f * kp / (float)nfl : 0.f;
    x[12] = dt / dt_max;
    x[13] = sqrtf(ax * ax + ay * ay + az * az) * d / rho0;
    x[14] = v.y * dt / d;
    x[15] = 1.f;
}

// features of the step (and, when recording, their FP32 copy); INFER 0:
// features only; 1: also the normalised BF16 features the inference kernel
// reads; 2: previous step's stiffness (the classic warm start, as a
// comparison for the network)
template <int INFER>
__global__ void __launch_bounds__(TR) k_ws_features(DevScene s, SolverConst c, MlpDev m, float dt_max,
                                                   float alpha_ref, float* Xout, __nv_bfloat16* xn) {
    const int n = s.st->n_active;
    const int p = blockIdx.x * TR + threadIdx.x;
    if (p >= n) return;
    const float dt = *s.dt;
    float x[MLP_IN];
    float pred = 0.f, divt = 0.f;
    ws_features(s, c, p, dt, dt_max, alpha_ref, x, pred, divt);
    s.wsbuf[p] = make_float2(pred, divt);
    if (Xout)
        for (int i = 0; i < MLP_IN; ++i) Xout[(size_t)p * MLP_IN + i] = x[i];
    if (INFER == 1) {
        const float* nrm = m.norm;
        uint32_t u[MLP_IN / 2];
#pragma unroll
        for (int i = 0; i < MLP_IN / 2; ++i)
            u[i] = pack2(__float2bfloat16_rn((x[2 * i] - nrm[2 * i]) * nrm[MLP_IN + 2 * i]),
                         __float2bfloat16_rn((x[2 * i + 1] - nrm[2 * i + 1]) * nrm[MLP_IN + 2 * i + 1]));
        uint4* dst = reinterpret_cast<uint4*>(xn + (size_t)p * MLP_IN);
        dst[0] = make_uint4(u[0], u[1], u[2], u[3]);
        dst[1] = make_uint4(u[4], u[5], u[6], u[7]);
    } else if (INFER == 2) {
        const float kw = c.ws_scale * fmaxf(s.hist[p].x, 0.f);
        s.kwarm[p] = kw;
        s.pk[p].w = kw / s.rho[p];
    }
}

// Inference of the warm-start network over the normalised features, on the
// tensor cores with every activation in registers: each warp runs 2 x 16
// rows; the layer-1 accumulator fragments (m16n8, FP32) are biased, passed
// through GELU, rounded to BF16 and re-packed as the A fragments of layer 2
// (m16k16: the C tiles of columns 16kk..16kk+7 and 16kk+8..16kk+15 form the
// A fragment of k-step kk); layer 3 (64 -> 1) is a per-thread dot product
// over the thread's accumulator columns, finished with two quad shuffles.
// Weights sit in shared memory as pre-packed per-lane B fragments.
struct InferSmem {
    uint2 w1f[8 * 32];       // [n-tile][lane]
    uint2 w2f[4 * 8 * 32];   // [k-step][n-tile][lane]
    float b1[MLP_H], b2[MLP_H], w3[MLP_H];
    float b3;
    float y[TR];
};

// the weights as per-lane B fragments, the biases and W3 (all threads of the
// block; the caller synchronises)
__device__ __forceinline__ void infer_pack(InferSmem& S, const MlpDev& m) {
    const __nv_bfloat16* W = m.w_bf16;
    for (int i = threadIdx.x; i < 8 * 32; i += TR) {
        const int nt = i >> 5, lane = i & 31, g = lane >> 2, t = lane & 3, col = nt * 8 + g;
        const __nv_bfloat16* w1 = W + MLP_OFF_W1;
        S.w1f[i] = make_uint2(pack2(w1[(2 * t) * MLP_H + col], w1[(2 * t + 1) * MLP_H + col]),
                              pack2(w1[(2 * t + 8) * MLP_H + col], w1[(2 * t + 9) * MLP_H + col]));
    }
    for (int i = threadIdx.x; i < 4 * 8 * 32; i += TR) {
        const int kk = i >> 8, nt = (i >> 5) & 7, lane = i & 31, g = lane >> 2, t = lane & 3;
        const int k = 16 * kk + 2 * t, col = nt * 8 + g;
        const __nv_bfloat16* w2 = W + MLP_OFF_W2;
        S.w2f[i] = make_uint2(pack2(w2[k * MLP_H + col], w2[(k + 1) * MLP_H + col]),
                              pack2(w2[(k + 8) * MLP_H + col], w2[(k + 9) * MLP_H + col]));
    }
    for (int i = threadIdx.x; i < MLP_H; i += TR) {
        S.b1[i] = m.master[MLP_OFF_B1 + i];
        S.b2[i] = m.master[MLP_OFF_B2 + i];
        S.w3[i] = __bfloat162float(W[MLP_OFF_W3 + i]);
    }
    if (threadIdx.x == 0) S.b3 = m.master[MLP_OFF_B3];
}

// The network on the warp's 32 rows [rt, rt + 32) of the block tile:
// row(r) gives the 32-byte BF16 feature row r (the 16 normalised
// features); the outputs (before the label scale) go to S.y[rt + r].
template <class Row>
__device__ __forceinline__ void infer_rows(InferSmem& S, Row row, int rt0) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    for (int mt = 0; mt < 2; ++mt) {
        const int rt = rt0 + mt * 16;
        const uint32_t* x0 = row(rt + g);
        const uint32_t* x1 = row(rt + g + 8);
        const uint32_t a[4] = {x0[t], x1[t], x0[4 + t], x1[4 + t]};
        uint32_t h[4][4];
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            float cc[4] = {0.f, 0.f, 0.f, 0.f};
            const uint2 b = S.w1f[nt * 32 + lane];
            const uint32_t bb[2] = {b.x, b.y};
            mma16816(cc, a, bb);
            const int col = nt * 8 + 2 * t;
            const float2 bb1 = *reinterpret_cast<const float2*>(S.b1 + col);
            float g0, g1, g2, g3;
            gelu_x2(cc[0], cc[1], bb1, g0, g1);
            gelu_x2(cc[2], cc[3], bb1, g2, g3);
            const uint32_t u01 = pack2(__float2bfloat16_rn(g0), __float2bfloat16_rn(g1));
            const uint32_t u23 = pack2(__float2bfloat16_rn(g2), __float2bfloat16_rn(g3));
            h[nt >> 1][(nt & 1) * 2] = u01;
            h[nt >> 1][(nt & 1) * 2 + 1] = u23;
        }
        float y0 = 0.f, y1 = 0.f;
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            float cc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) {
                const uint2 b = S.w2f[(kk * 8 + nt) * 32 + lane];
                const uint32_t bb[2] = {b.x, b.y};
                mma16816(cc, h[kk], bb);
            }
            const int col = nt * 8 + 2 * t;
            const float2 bb2 = *reinterpret_cast<const float2*>(S.b2 + col);
            float g0, g1, g2, g3;
            gelu_x2(cc[0], cc[1], bb2, g0, g1);
            gelu_x2(cc[2], cc[3], bb2, g2, g3);
            y0 = fmaf(g0, S.w3[col], y0);
            y0 = fmaf(g1, S.w3[col + 1], y0);
            y1 = fmaf(g2, S.w3[col], y1);
            y1 = fmaf(g3, S.w3[col + 1], y1);
        }
        y0 += __shfl_xor_sync(0xffffffffu, y0, 1);
        y0 += __shfl_xor_sync(0xffffffffu, y0, 2);
        y1 += __shfl_xor_sync(0xffffffffu, y1, 1);
        y1 += __shfl_xor_sync(0xffffffffu, y1, 2);
        if (t == 0) {
            S.y[rt + g] = y0 + S.b3;
            S.y[rt + g + 8] = y1 + S.b3;
        }
    }
}

// the prediction of particle p from its network output: negative
// predictions are not applied (the loop only adds pressure)
__device__ __forceinline__ void infer_apply(const DevScene& s, const SolverConst& c, const MlpDev& m, int p, float y) {
    const float* nrm = m.norm;
    const float kpred = y / nrm[2 * MLP_IN + 1] + nrm[2 * MLP_IN];
    const float kw = c.ws_scale * fmaxf(kpred, 0.f);
    s.kwarm[p] = kw;
    s.pk[p].w = kw / s.rho[p];  // read by the warm-correction sweep
}

__global__ void __launch_bounds__(TR) k_ws_infer(DevScene s, SolverConst c, MlpDev m, const __nv_bfloat16* xn) {
    __shared__ InferSmem S;
    infer_pack(S, m);
    __syncthreads();
    const int n = s.st->n_active;
    const int w = threadIdx.x >> 5;
    for (int base = blockIdx.x * TR; base < n; base += gridDim.x * TR) {
        infer_rows(S, [&](int r) {
            return reinterpret_cast<const uint32_t*>(xn + (size_t)min(base + r, n - 1) * MLP_IN);
        }, w * 32);
        __syncwarp();
        const int p = base + threadIdx.x;
        if (p < n) infer_apply(s, c, m, p, S.y[threadIdx.x]);
        __syncwarp();
    }
}

// Features and inference in one pass: each thread gathers its particle's
// features (a neighbour sweep, bound by the L1 gathers), writes them
// normalised as a BF16 row into shared memory, and its warp runs the
// network on its 32 rows (bound by the GELUs' issue slots); resident warps
// in the two phases overlap.  Persistent blocks pack the weights once.  The
// rows and the network are those of k_ws_features<1> + k_ws_infer, so the
// predictions are the same bit for bit.  Seven resident blocks per SM
// (at most 73 registers, no spills): 204 -> 192 us at 1 M against six at
// the compiler's own 79 (eight, at 64 registers, spill: 197 us).
struct FusedSmem {
    InferSmem I;
    uint32_t x[TR][MLP_IN / 2];
};
__global__ void __launch_bounds__(TR, 7) k_ws_features_infer(DevScene s, SolverConst c, MlpDev m, float dt_max,
                                                          float alpha_ref, __nv_bfloat16* xn) {
    __shared__ FusedSmem S;
    infer_pack(S.I, m);
    __syncthreads();
    const int n = s.st->n_active;
    const int w = threadIdx.x >> 5;
    const float* nrm = m.norm;
    for (int base = blockIdx.x * TR; base < n; base += gridDim.x * TR) {
        const int p = base + threadIdx.x;
        if (p < n) {
            float x[MLP_IN];
            float pred = 0.f, divt = 0.f;
            ws_features(s, c, p, *s.dt, dt_max, alpha_ref, x, pred, divt);
            s.wsbuf[p] = make_float2(pred, divt);
            uint32_t u[MLP_IN / 2];
#pragma unroll
            for (int i = 0; i < MLP_IN / 2; ++i) {
                u[i] = pack2(__float2bfloat16_rn((x[2 * i] - nrm[2 * i]) * nrm[MLP_IN + 2 * i]),
                             __float2bfloat16_rn((x[2 * i + 1] - nrm[2 * i + 1]) * nrm[MLP_IN + 2 * i + 1]));
                S.x[threadIdx.x][i] = u[i];
            }
            // the normalised row also goes out (the ws_features getter reads it)
            uint4* dst = reinterpret_cast<uint4*>(xn + (size_t)p * MLP_IN);
            dst[0] = make_uint4(u[0], u[1], u[2], u[3]);
            dst[1] = make_uint4(u[4], u[5], u[6], u[7]);
        }
        // (a block-wide barrier: in the last tile a warp past the count reads
        // another warp's row)
        __syncthreads();
        // rows past the count repeat the last particle's row, as k_ws_infer's
        // clamped reads do (their outputs are discarded)
        const int last = min(n - 1 - base, TR - 1);
        infer_rows(S.I, [&](int r) { return S.x[min(r, last)]; }, w * 32);
        __syncwarp();
        if (p < n) infer_apply(s, c, m, p, S.I.y[threadIdx.x]);
        __syncwarp();
    }
}

// after the density loop: the step's total stiffness (warm + loop), history
// for the next step's features, and the training label
__global__ void k_ws_post(DevScene s, SolverConst c, float* yout) {
    const int n = s.st->n_active;
    const int p = blockIdx.x * TR + threadIdx.x;
    if (p >= n) return;
    const float ktot = s.ksum[p] + s.kwarm[p];  // kwarm is 0 unless the warm start ran
    const float2 w = s.wsbuf[p];
    s.hist[p] = make_float4(ktot, w.x, w.y, 0.f);
    if (yout) yout[p] = ktot;
    s.ksum[p] = 0.f;
}

// append every `every`-th particle (from `offset`) of the step to the dataset,
// sample i of the step at slot ds_count + i (the order of the particles, so
// recording is run-to-run deterministic)
__global__ void k_ws_append(const float* X, const float* y, int n_max, const int* n_act, int every, const int* offset,
                            float* dsX, float* dsy, const int* ds_count, int ds_cap) {
    const int n = *n_act;
    const long long i = (long long)blockIdx.x * TR + threadIdx.x;
    const long long pl = (long long)*offset + i * (long long)every;
    if (pl < 0 || pl >= n || pl >= n_max) return;
    const int p = (int)pl;
    const long long slot = (long long)*ds_count + i;
    if (slot >= ds_cap) return;
    for (int k = 0; k < MLP_IN; ++k) dsX[(size_t)slot * MLP_IN + k] = X[(size_t)p * MLP_IN + k];
    dsy[slot] = y[p];
}
// after the append: the dataset count grows by the step's samples and the
// sampling offset advances by one particle per recorded step
__global__ void k_ws_advance(int* offset, int every, const int* n_act, int n_max, int* ds_count, int ds_cap) {
    const int n = min(*n_act, n_max), o = *offset;
    const long long cnt = n > o ? ((long long)n - o + every - 1) / every : 0;
    *ds_count = (int)min((long long)*ds_count + cnt, (long long)ds_cap);
    *offset = (o + 1) % every;
}
}  // namespace

void ws_init_attributes() {}

void launch_ws_features(const DevScene& s, const SolverConst& c, const MlpDev& m, int infer, float dt_max,
                        float alpha_ref, float* Xout, __nv_bfloat16* xn, int n_max, cudaStream_t st) {
    const int blocks = (n_max + TR - 1) / TR;
    if (infer == 1) k_ws_features<1><<<blocks, TR, 0, st>>>(s, c, m, dt_max, alpha_ref, Xout, xn);
    else if (infer == 2) k_ws_features<2><<<blocks, TR, 0, st>>>(s, c, m, dt_max, alpha_ref, Xout, xn);
    else k_ws_features<0><<<blocks, TR, 0, st>>>(s, c, m, dt_max, alpha_ref, Xout, xn);
}

void launch_ws_infer(const DevScene& s, const SolverConst& c, const MlpDev& m, const __nv_bfloat16* xn, int n_max,
                     int sm_count, cudaStream_t st) {
    int blocks = (n_max + TR - 1) / TR;
    const int cap = sm_count * 8;  // persistent: each block packs the weights once
    if (blocks > cap) blocks = cap;
    k_ws_infer<<<blocks, TR, 0, st>>>(s, c, m, xn);
}

void launch_ws_features_infer(const DevScene& s, const SolverConst& c, const MlpDev& m, float dt_max, float alpha_ref,
                              __nv_bfloat16* xn, int n_max, int sm_count, cudaStream_t st) {
    static int per_sm = 0;  // resident blocks per SM (the kernel's registers and shared memory)
    if (!per_sm && cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ws_features_infer, TR, 0) != cudaSuccess)
        per_sm = 4;
    if (per_sm < 1) per_sm = 1;
    int blocks = (n_max + TR - 1) / TR;
    if (blocks > sm_count * per_sm) blocks = sm_count * per_sm;
    k_ws_features_infer<<<blocks, TR, 0, st>>>(s, c, m, dt_max, alpha_ref, xn);
}

void launch_ws_post(const DevScene& s, const SolverConst& c, float* yout, int n_max, cudaStream_t st) {
    k_ws_post<<<(n_max + TR - 1) / TR, TR, 0, st>>>(s, c, yout);
}

void launch_ws_append(const float* X, const float* y, int n_max, const int* n_act, int every, int* offset, float* dsX,
                      float* dsy, int* ds_count, int ds_cap, cudaStream_t st) {
    const long long cnt = ((long long)n_max + every - 1) / every + 1;
    k_ws_append<<<(int)((cnt + TR - 1) / TR), TR, 0, st>>>(X, y, n_max, n_act, every, offset, dsX, dsy, ds_count,
                                                          ds_cap);
    k_ws_advance<<<1, 1, 0, st>>>(offset, every, n_act, n_max, ds_count, ds_cap);
}
