// sph_common.cuh -- device-side definitions shared by the SPH kernels.
//
// Data layout in HBM (all fluid arrays in cell-sorted order, rebuilt every
// neighbour search):
//   pos   float4 (x, y, z, phase | scene << 4 as int bits)   16 B/particle
//   vel   float4 (vx, vy, vz, 0)                16 B/particle
//   gid   int   global fluid index (phase-major insertion order; the
//               reference's m_Fluids[k].fluidParticles[i] order)
//   rho, alpha, ... float per particle
//   nbr   int   ELL neighbour list in groups of four, column-major: entry k
//               of particle p at nbr[((k / 4) * stride + p) * 4 + k % 4], so
//               one 16-byte load gives a thread four entries; fluid
//               neighbour j -> j, boundary neighbour b -> b | BND_FLAG
//   boundary: bpos float4 (x, y, z, volume), bvel float4
//
// Cell keys: the reference's uniform grid (cell = smoothRadius_h,
// SphBase.cpp:963-988) with cells enumerated brick by brick (4x4x4 bricks,
// Morton order inside a brick) so that particles sorted by key are
// spatially local in memory.  The reference's linear cell index
// (SpaceGridStruct::gridOfPos, SphBase.h:700-701) is derived from the same
// integer cell coordinates when a caller asks for it.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define BND_FLAG 0x80000000u
#define BND_MASK 0x7fffffffu

struct GridGeom {
    float min[3];      // SpaceGridStruct::min = spaceMin - 2h
    float divisor;     // 1/h
    int num[3];        // cells per axis
    int nb[3];         // 4x4x4 bricks per axis
    int nkeys;         // keys of the whole key space + 1 (last key: removed particles)
    int key0, key1;    // this grid's keys are [key0, key1) (a batch packs one grid per scene)
    float smin[3], smax[3];  // m_TH.spaceMin / spaceMax (outside-particle removal)
};

// Kernel constants of the reference's single-h cubic spline
// (SphBase::ker_update_numbers, SphBase.h:808-829).
struct KerConst {
    float h, inv_h, theta, thetah;
    float g_in;   // -thetah / h      : -W'(r)/r = g_in * (3 - 2.25 q)     for q <= 1
    float g_out;  // -0.75 * thetah   : -W'(r)/r = g_out * (2 - q)^2 / r   for q > 1
};

struct SolverConst {
    KerConst k;
    float hs;          // smoothRadius_h (viscosity epsilon uses it)
    float h2cut;       // (d + d)^2 neighbour cut (SphBase.cpp:883-886)
    float dpart;       // particle diameter
    float fm0;         // rho0 * spacing_r^3 (phase 0)
    float rho0;        // phase 0 rest density
    float gravity[3];
    float nu;
    float cs;
    float visc_alpha;  // phase 0 artificial viscosity (WCSPH)
    float bvisc;       // boundary viscosity alpha
    float wc_B, wc_gamma;
    float th_h, th_r, th_bt;  // WCSPH surface tension / adhesion (m_TH.h, r, bt)
    float rho0_ph[4];  // per phase rest density
    float fm_ph[4];    // per phase mass
    float alpha_ph[4]; // per phase viscosity alpha
    int nphase;
    float ws_scale;    // applied fraction of the predicted warm-start stiffness
    int cap;           // neighbour cap
    int stride;        // ELL column stride (>= fluid capacity)
    int lanes;         // threads per particle of the WCSPH list build and force pass (1 or 4)
    int l2pol;         // L2 eviction priority of the sweeps' loads: bits 0-1 the
                       // neighbour lists, bits 2-3 the gathered records
                       // (0 normal, 1 evict first, 2 evict last)
    // IISph (volume form, IISph.cpp): spline of the per-pair h = (d_a + d_b)/2
    // (= d, one diameter for all particles), rest volume d^3, per-phase mass
    // rho0 * beta * d^3 (beta = 1), kinematic viscosity of fluid / boundary
    KerConst kd;
    float iv_V;
    float iv_m[4];
    float iv_kv, iv_kvb;
    int iv_multi_solid;  // 1 if the walls hold more than one solid (boundary lists then see the others)
};

// -------- cubic spline, SphBase.h:840-889 (single-h forms) --------
__device__ __forceinline__ float ker_W(const KerConst& k, float r) {
    float q = r / k.h, qm2 = 2.f - q;
    return q <= 1.f ? k.theta * (1.f - 1.5f * q * q + 0.75f * q * q * q)
                    : k.theta * (0.25f * qm2 * qm2 * qm2);
}
__device__ __forceinline__ float ker_Wg(const KerConst& k, float r) {
    float q = r / k.h, qm2 = 2.f - q;
    return q <= 1.f ? k.thetah * (3.f * q - 2.25f * q * q) : k.thetah * 0.75f * qm2 * qm2;
}
// -W'(r)/r from r^2 with one reciprocal square root and no division: the
// fast form of the reference's `-ker_W_grad(dis) / dis` (SphBase.h:876-889),
// used by the Jacobi sweeps (relative error a few ulp).
__device__ __forceinline__ float grad_over_r(const KerConst& k, float len2) {
    const float inv_r = rsqrtf(len2);
    const float q = len2 * inv_r * k.inv_h;
    const float t = 2.f - q;
    const float fin = k.g_in * fmaf(-2.25f, q, 3.f);
    const float fout = k.g_out * t * t * inv_r;
    return q <= 1.f ? fin : fout;
}

// W(r) and -W'(r)/r of the single-h spline from r^2 (one rsqrt, no
// division): the forms of ker_W / ker_W_grad (SphBase.h:840-889) used where
// the result is summed (densities, alpha), relative error a few ulp.
__device__ __forceinline__ void kernel_pair(const KerConst& k, float len2, float& w, float& f) {
    const float inv_r = rsqrtf(len2);
    const float q = len2 * inv_r * k.inv_h;
    const float t = 2.f - q;
    const float win = k.theta * fmaf(q * q, fmaf(0.75f, q, -1.5f), 1.f);
    const float wout = k.theta * 0.25f * t * t * t;
    w = q <= 1.f ? win : wout;
    const float fin = k.g_in * fmaf(-2.25f, q, 3.f);
    const float fout = k.g_out * t * t * inv_r;
    f = q <= 1.f ? fin : fout;
}

// W(r) and -W'(r)/r evaluated as the reference does: r = sqrt(len2) and
// q = r / h correctly rounded, so 2 - q is the reference's.  For sums whose
// result can hinge on a single pair near the cut (a boundary particle with
// one fluid neighbour), where the rsqrt form's few-ulp error in q becomes a
// large relative error in (2 - q)^2.
__device__ __forceinline__ void kernel_pair_rn(const KerConst& k, float len2, float& w, float& f) {
    const float r = __fsqrt_rn(len2);
    const float q = __fdiv_rn(r, k.h), qm2 = 2.f - q;
    w = q <= 1.f ? k.theta * (1.f - 1.5f * q * q + 0.75f * q * q * q) : k.theta * (0.25f * qm2 * qm2 * qm2);
    const float g = q <= 1.f ? k.thetah * (3.f * q - 2.25f * q * q) : k.thetah * 0.75f * qm2 * qm2;
    f = __fdiv_rn(-g, r);
}

// per-pair-h spline with range check, SphBase.h:855-871
__device__ __forceinline__ float ker_W_h(float r, float h) {
    float q = r / h, qm2 = 2.f - q;
    float th = 1.f / 3.14159265358979323846f / (h * h * h);
    if (!(q >= 0.f && q <= 2.f)) return 0.f;
    return q <= 1.f ? th * (1.f - 1.5f * q * q + 0.75f * q * q * q) : th * (0.25f * qm2 * qm2 * qm2);
}

// Squared distance exactly as vec3::dis_square (Vec23.h:170-171) evaluates
// it in float without contraction: ((dx*dx + dy*dy) + dz*dz).
__device__ __forceinline__ float dis_square_rn(float ax, float ay, float az, float bx, float by, float bz) {
    float dx = __fsub_rn(ax, bx), dy = __fsub_rn(ay, by), dz = __fsub_rn(az, bz);
    return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
}

// Integer cell coordinate per axis: int((pos - min) * divisor), SphBase.h:700-701.
__device__ __forceinline__ int cell_coord(float p, float mn, float div) {
    return (int)__fmul_rn(__fsub_rn(p, mn), div);
}

__device__ __forceinline__ int morton2x3(int x, int y, int z) {
    return (x & 1) | ((y & 1) << 1) | ((z & 1) << 2) | ((x & 2) << 2) | ((y & 2) << 3) | ((z & 2) << 4);
}

__device__ __forceinline__ int cell_key(const GridGeom& g, int cx, int cy, int cz) {
    int b = ((cz >> 2) * g.nb[1] + (cy >> 2)) * g.nb[0] + (cx >> 2);
    return g.key0 + b * 64 + morton2x3(cx & 3, cy & 3, cz & 3);
}

__device__ __forceinline__ bool cell_inside(const GridGeom& g, int cx, int cy, int cz) {
    return cx >= 0 && cy >= 0 && cz >= 0 && cx < g.num[0] && cy < g.num[1] && cz < g.num[2];
}

// pos.w holds the fluid phase (4 bits) and, in a batch, the scene index
// above them; the bits travel with the particle through every reorder
__device__ __forceinline__ int phase_of(float4 p) { return __float_as_int(p.w) & 15; }
__device__ __forceinline__ int scene_of(float4 p) { return __float_as_int(p.w) >> 4; }

// One 32-byte record in a single 256-bit load (sm_100 ld.global.v8; the
// address must be 32-byte aligned, which the packed pv/bpv arrays are).
__device__ __forceinline__ void ld_record32(const float4* p, float4& a, float4& b) {
    asm volatile("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
                 : "l"(p));
}

// L2 cache policy (createpolicy) of the given eviction priority: 0 normal,
// 1 evict first, 2 evict last
__device__ __forceinline__ unsigned long long l2_policy(int pri) {
    unsigned long long p;
    if (pri == 1) asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    else if (pri == 2) asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    else asm("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(p));
    return p;
}
// the 32-byte record load under an L2 cache policy
__device__ __forceinline__ void ld_record32_pol(const float4* p, float4& a, float4& b, unsigned long long pol) {
    asm volatile("ld.global.nc.L2::cache_hint.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8], %9;"
                 : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
                 : "l"(p), "l"(pol));
}
__device__ __forceinline__ float4 ld_f4_pol(const float4* p, unsigned long long pol) {
    float4 a;
    asm volatile("ld.global.nc.L2::cache_hint.v4.f32 {%0,%1,%2,%3}, [%4], %5;"
                 : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w)
                 : "l"(p), "l"(pol));
    return a;
}

// ELL4 addressing (see the layout note at the top)
__device__ __forceinline__ size_t ell_index(size_t stride, int p, int k) {
    return ((size_t)(k >> 2) * stride + (size_t)p) * 4 + (k & 3);
}
__device__ __forceinline__ int ell_get(const int* L, size_t stride, int p, int k) { return L[ell_index(stride, p, k)]; }
__device__ __forceinline__ int4 ell_group(const int* L, size_t stride, int p, int g) {
    return __ldg(reinterpret_cast<const int4*>(L) + (size_t)g * stride + p);
}
// one group under an L2 cache policy
__device__ __forceinline__ int4 ell_group_pol(const int* L, size_t stride, int p, int g, unsigned long long pol) {
    int4 v;
    const int4* a = reinterpret_cast<const int4*>(L) + (size_t)g * stride + p;
    asm volatile("ld.global.nc.L2::cache_hint.v4.s32 {%0,%1,%2,%3}, [%4], %5;"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(a), "l"(pol));
    return v;
}

// ---- reductions ----
template <int NT>
__device__ __forceinline__ double block_sum_double(double v, double* sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double r = 0;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int i = 0; i < NT / 32; ++i) r += sh[i];
    }
    __syncthreads();
    return r;  // valid in thread 0
}

template <int NT>
__device__ __forceinline__ int block_sum_int(int v, int* sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sh[w] = v;
    __syncthreads();
    int r = 0;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int i = 0; i < NT / 32; ++i) r += sh[i];
    }
    __syncthreads();
    return r;
}

template <int NT>
__device__ __forceinline__ int block_max_int(int v, int* sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_down_sync(0xffffffffu, v, o));
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sh[w] = v;
    __syncthreads();
    int r = 0;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int i = 0; i < NT / 32; ++i) r = max(r, sh[i]);
    }
    __syncthreads();
    return r;
}
