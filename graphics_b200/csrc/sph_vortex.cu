// sph_vortex.cu -- the DFSPH vorticity options (m_TH.enable_vortex,
// DFSPH.cpp:233-553 at the start of DF_constantDensitySolverSecond, after the
// non-pressure forces; DFSPH.cpp:913-1022 after the divergence loop).
//
//   1  TRRV: omega = curl v (difference form, Bender et al.'s micropolar
//      paper); dOmega = -(diffusion + stretching of omega) dt; every
//      particle's velocity gains sum_b (dOmega_b / 2) x x_ab
//      (spacing_r / 2 / |x_ab|)^2 alpha (a Rankine vortex per neighbour)
//   2  micropolar: vorticity curl v and the Laplacian of the carried angular
//      velocity w give w += (zeta lap w + (curl v - 2 w)(nu + nu_t)) dt / 2,
//      then v += curl w (nu + nu_t) dt
//   3  stream-function correction: the vorticity at the start of the step
//      (n0) against the one after the divergence loop (n1); the loss
//      delta = n0 - n1 (0 where |n0| < |n1| or a boundary particle is a
//      neighbour) is put back through psi = sum_b delta_b V / (4 pi r) and
//      v += curl psi.  (The reference's n0 also gains the TRRV transport of
//      its omega, which only mode 1 computes: 0 here.)
// Per particle in FP32 over the stored neighbour lists, kernel gradient
// x_ab (-W'(r)/r) as the other sweeps compute it.  The carried vector (w for
// mode 2, n0 for mode 3) lives in cA and follows the particle through the
// sort; vA / vB hold the per-step vectors.
#include "sph_kernels.cuh"

namespace {
constexpr int NT = 128;

__device__ __forceinline__ float3 cross3(float ax, float ay, float az, float bx, float by, float bz) {
    return make_float3(ay * bz - az * by, az * bx - ax * bz, ax * by - ay * bx);
}

struct Nb {
    float4 p;   // (x, y, z, rho) fluid / (x, y, z, volume) boundary
    float4 v;   // velocity (fluid) / singleVelocity (bpv) or rigid velocity (bpf)
    bool bnd;
    unsigned j;
};

__device__ __forceinline__ Nb nb_get(const DevScene& s, const SolverConst& c, int p, int k, bool rigid_vel) {
    const unsigned e = (unsigned)ell_get(s.nbr, (size_t)c.stride, p, k);
    Nb n;
    n.bnd = (e & BND_FLAG) != 0u;
    n.j = e & BND_MASK;
    ld_record32((n.bnd ? (rigid_vel ? s.bpf : s.bpv) : s.prv) + 2 * (size_t)n.j, n.p, n.v);
    return n;
}

// the velocity the density loop starts from, v_adv = v + a_adv dt
// (DFSPH.cpp:557-563), after a vorticity option changed v
__device__ __forceinline__ void set_velocity(DevScene& s, int p, float3 v, float dt) {
    const float4 a = s.acc[p];
    s.vel[p] = make_float4(v.x, v.y, v.z, 0.f);
    s.prv[2 * p + 1] = make_float4(v.x, v.y, v.z, 0.f);
    const float w = s.pv[2 * p + 1].w;
    s.pv[2 * p + 1] = make_float4(v.x + a.x * dt, v.y + a.y * dt, v.z + a.z * dt, w);
}

// curl v (difference form) at the start of the step.  TRRV: boundary
// neighbours with singleVelocity and the fluid mass (DFSPH.cpp:312-317);
// stream function: fluid neighbours only (:256-268).  Out: vA (mode 1) or
// cA (mode 3).
template <int MODE>
__global__ void __launch_bounds__(NT) k_vort_curl(DevScene s, SolverConst c) {
    const int n = s.st->n_active;
    const int p = blockIdx.x * NT + threadIdx.x;
    if (p >= n) return;
    const float4 pa = s.prv[2 * p], va = s.prv[2 * p + 1];
    const float sc = 1.f / pa.w * c.fm0;
    float ox = 0.f, oy = 0.f, oz = 0.f;
    const int cnt = s.ncount[p];
    for (int k = 0; k < cnt; ++k) {
        const Nb b = nb_get(s, c, p, k, false);
        if (b.bnd && MODE == 3) continue;
        const float xx = pa.x - b.p.x, xy = pa.y - b.p.y, xz = pa.z - b.p.z;
        const float f = grad_over_r(c.k, xx * xx + xy * xy + xz * xz);
        const float3 cr = cross3((va.x - b.v.x) * sc, (va.y - b.v.y) * sc, (va.z - b.v.z) * sc, xx * f, xy * f, xz * f);
        ox += cr.x;
        oy += cr.y;
        oz += cr.z;
    }
    const float4 o = make_float4(ox, oy, oz, 0.f);
    if (MODE == 3) s.cA[p] = o;
    else s.vA[p] = o;
}

// TRRV, 2nd loop (DFSPH.cpp:352-396): dOmega = -(diffusion + stretching) dt
__global__ void __launch_bounds__(NT) k_trrv_domega(DevScene s, SolverConst c) {
    const int n = s.st->n_active;
    const int p = blockIdx.x * NT + threadIdx.x;
    if (p >= n) return;
    const float dt = *s.dt;
    const float4 pa = s.prv[2 * p], va = s.prv[2 * p + 1], wa = s.vA[p];
    const float ra2 = pa.w * pa.w;
    const float den0 = 0.01f * c.hs * c.hs, visc = 10.f * c.nu;
    float t1x = 0.f, t1y = 0.f, t1z = 0.f, t2x = 0.f, t2y = 0.f, t2z = 0.f;
    const int cnt = s.ncount[p];
    for (int k = 0; k < cnt; ++k) {
        const Nb b = nb_get(s, c, p, k, false);
        if (b.bnd) continue;
        const float4 wb = s.vA[b.j];
        const float xx = pa.x - b.p.x, xy = pa.y - b.p.y, xz = pa.z - b.p.z;
        const float len2 = xx * xx + xy * xy + xz * xz;
        const float f = grad_over_r(c.k, len2);
        const float gx = xx * f, gy = xy * f, gz = xz * f;
        const float pro = (wa.x - wb.x) * xx + (wa.y - wb.y) * xy + (wa.z - wb.z) * xz;
        const float d = pro / (len2 + den0) * c.fm0 / b.p.w * visc;
        t1x += gx * d;
        t1y += gy * d;
        t1z += gz * d;
        const float wg = (wa.x * gx + wa.y * gy + wa.z * gz) * c.fm0;
        const float rb2 = b.p.w * b.p.w;
        t2x += wg * (va.x / ra2 + b.v.x / rb2);
        t2y += wg * (va.y / ra2 + b.v.y / rb2);
        t2z += wg * (va.z / ra2 + b.v.z / rb2);
    }
    s.vB[p] = make_float4(-(t1x + t2x) * dt, -(t1y + t2y) * dt, -(t1z + t2z) * dt, 0.f);
}

// TRRV, 3rd loop (DFSPH.cpp:398-417): v += sum_b (dOmega_b / 2) x x_ab
// (spacing / 2 / |x_ab|)^2 alpha
__global__ void __launch_bounds__(NT) k_trrv_apply(DevScene s, SolverConst c, float alpha, float spacing) {
    const int n = s.st->n_active;
    const int p = blockIdx.x * NT + threadIdx.x;
    if (p >= n) return;
    const float dt = *s.dt;
    const float4 pa = s.prv[2 * p], va = s.prv[2 * p + 1];
    float3 v = make_float3(va.x, va.y, va.z);
    const float hs = spacing / 2.f;
    const int cnt = s.ncount[p];
    for (int k = 0; k < cnt; ++k) {
        const unsigned e = (unsigned)ell_get(s.nbr, (size_t)c.stride, p, k);
        if (e & BND_FLAG) continue;
        const float4 pb = s.prv[2 * (size_t)e];
        const float4 db = s.vB[e];
        const float xx = pa.x - pb.x, xy = pa.y - pb.y, xz = pa.z - pb.z;
        const float l = sqrtf(xx * xx + xy * xy + xz * xz);
        const float q = hs / l;
        const float3 t = cross3(db.x / 2, db.y / 2, db.z / 2, xx, xy, xz);
        const float sc = q * q * alpha;
        v.x += t.x * sc;
        v.y += t.y * sc;
        v.z += t.z * sc;
    }
    set_velocity(s, p, v, dt);
}

// micropolar, loops 1.4-1.6 (DFSPH.cpp:446-511): curl v, the Laplacian of
// the carried angular velocity w (cA), and w's update into vA
__global__ void __launch_bounds__(NT) k_micro_w(DevScene s, SolverConst c, float zeta, float nu_t) {
    const int n = s.st->n_active;
    const int p = blockIdx.x * NT + threadIdx.x;
    if (p >= n) return;
    const float dt = *s.dt;
    const float4 pa = s.prv[2 * p], va = s.prv[2 * p + 1], wa = s.cA[p];
    const float sc = 1.f / pa.w * c.fm0;
    const float den0 = 0.01f * c.hs * c.hs;
    float ox = 0.f, oy = 0.f, oz = 0.f, lx = 0.f, ly = 0.f, lz = 0.f;
    const int cnt = s.ncount[p];
    for (int k = 0; k < cnt; ++k) {
        const Nb b = nb_get(s, c, p, k, true);
        const float xx = pa.x - b.p.x, xy = pa.y - b.p.y, xz = pa.z - b.p.z;
        const float len2 = xx * xx + xy * xy + xz * xz;
        const float f = grad_over_r(c.k, len2);
        const float gx = xx * f, gy = xy * f, gz = xz * f;
        // curl v: a boundary neighbour with its velocity and mass V rho0 (:466-471)
        const float s2 = b.bnd ? 1.f / pa.w * (b.p.w * c.rho0) : sc;
        const float3 cr = cross3((va.x - b.v.x) * s2, (va.y - b.v.y) * s2, (va.z - b.v.z) * s2, gx, gy, gz);
        ox += cr.x;
        oy += cr.y;
        oz += cr.z;
        // Laplacian of w; a boundary particle's angular velocity is 0 (:485-494)
        const float4 wb = b.bnd ? make_float4(0.f, 0.f, 0.f, 0.f) : s.cA[b.j];
        const float pro = (wa.x - wb.x) * xx + (wa.y - wb.y) * xy + (wa.z - wb.z) * xz;
        const float m = b.bnd ? b.p.w * 10.f : c.fm0 / b.p.w * 10.f;
        const float d = pro / (len2 + den0) * m;
        lx += gx * d;
        ly += gy * d;
        lz += gz * d;
    }
    const float nn = c.nu + nu_t;
    s.vA[p] = make_float4(wa.x + (lx * zeta + (ox - wa.x * 2.f) * nn) * 0.5f * dt,
                          wa.y + (ly * zeta + (oy - wa.y * 2.f) * nn) * 0.5f * dt,
                          wa.z + (lz * zeta + (oz - wa.z * 2.f) * nn) * 0.5f * dt, 0.f);
}

// micropolar, loops 1.2-1.3 (DFSPH.cpp:513-552): curl of the new w, v += it
// (nu + nu_t) dt; the new w becomes the carried one
__global__ void __launch_bounds__(NT) k_micro_v(DevScene s, SolverConst c, float nu_t) {
    const int n = s.st->n_active;
    const int p = blockIdx.x * NT + threadIdx.x;
    if (p >= n) return;
    const float dt = *s.dt;
    const float4 pa = s.prv[2 * p], va = s.prv[2 * p + 1], wa = s.vA[p];
    const float sc = 1.f / pa.w * c.fm0;
    float ox = 0.f, oy = 0.f, oz = 0.f;
    const int cnt = s.ncount[p];
    for (int k = 0; k < cnt; ++k) {
        const Nb b = nb_get(s, c, p, k, true);
        const float xx = pa.x - b.p.x, xy = pa.y - b.p.y, xz = pa.z - b.p.z;
        const float f = grad_over_r(c.k, xx * xx + xy * xy + xz * xz);
        const float4 wb = b.bnd ? make_float4(0.f, 0.f, 0.f, 0.f) : s.vA[b.j];
        const float s2 = b.bnd ? 1.f / pa.w * (b.p.w * c.rho0) : sc;
        const float3 cr = cross3((wa.x - wb.x) * s2, (wa.y - wb.y) * s2, (wa.z - wb.z) * s2, xx * f, xy * f, xz * f);
        ox += cr.x;
        oy += cr.y;
        oz += cr.z;
    }
    const float nn = (c.nu + nu_t) * dt;
    set_velocity(s, p, make_float3(va.x + ox * nn, va.y + oy * nn, va.z + oz * nn), dt);
    s.cA[p] = wa;
}

// stream function, 1st loop after the divergence loop (DFSPH.cpp:913-968):
// delta = n0 - n1 into vA
__global__ void __launch_bounds__(NT) k_sfc_delta(DevScene s, SolverConst c) {
    const int n = s.st->n_active;
    const int p = blockIdx.x * NT + threadIdx.x;
    if (p >= n) return;
    const float4 pa = s.prv[2 * p], va = s.prv[2 * p + 1], n0 = s.cA[p];
    const float sc = 1.f / pa.w * c.fm0;
    float ox = 0.f, oy = 0.f, oz = 0.f;
    bool bnd = false;
    const int cnt = s.ncount[p];
    for (int k = 0; k < cnt && !bnd; ++k) {
        const Nb b = nb_get(s, c, p, k, false);
        if (b.bnd) { bnd = true; break; }
        const float xx = pa.x - b.p.x, xy = pa.y - b.p.y, xz = pa.z - b.p.z;
        const float f = grad_over_r(c.k, xx * xx + xy * xy + xz * xz);
        const float3 cr = cross3((va.x - b.v.x) * sc, (va.y - b.v.y) * sc, (va.z - b.v.z) * sc, xx * f, xy * f, xz * f);
        ox += cr.x;
        oy += cr.y;
        oz += cr.z;
    }
    float4 d = make_float4(0.f, 0.f, 0.f, 0.f);
    if (!bnd && !(n0.x * n0.x + n0.y * n0.y + n0.z * n0.z < ox * ox + oy * oy + oz * oz))
        d = make_float4(n0.x - ox, n0.y - oy, n0.z - oz, 0.f);
    s.vA[p] = d;
}

// psi = sum_b delta_b v0 / 4 / pi / r (DFSPH.cpp:970-991) into vB
__global__ void __launch_bounds__(NT) k_sfc_psi(DevScene s, SolverConst c, float v0) {
    const int n = s.st->n_active;
    const int p = blockIdx.x * NT + threadIdx.x;
    if (p >= n) return;
    const float4 pa = s.prv[2 * p];
    float x = 0.f, y = 0.f, z = 0.f;
    const int cnt = s.ncount[p];
    for (int k = 0; k < cnt; ++k) {
        const unsigned e = (unsigned)ell_get(s.nbr, (size_t)c.stride, p, k);
        if (e & BND_FLAG) continue;
        const float4 pb = s.prv[2 * (size_t)e];
        const float4 d = s.vA[e];
        const float xx = pa.x - pb.x, xy = pa.y - pb.y, xz = pa.z - pb.z;
        const float r = sqrtf(xx * xx + xy * xy + xz * xz);
        const float w = v0 / 4.f / 3.1415926f / r;
        x += d.x * w;
        y += d.y * w;
        z += d.z * w;
    }
    s.vB[p] = make_float4(x, y, z, 0.f);
}

// v += curl psi (DFSPH.cpp:992-1019)
__global__ void __launch_bounds__(NT) k_sfc_apply(DevScene s, SolverConst c) {
    const int n = s.st->n_active;
    const int p = blockIdx.x * NT + threadIdx.x;
    if (p >= n) return;
    const float4 pa = s.prv[2 * p], va = s.prv[2 * p + 1], sa = s.vB[p];
    const float sc = 1.f / pa.w * c.fm0;
    float ox = 0.f, oy = 0.f, oz = 0.f;
    const int cnt = s.ncount[p];
    for (int k = 0; k < cnt; ++k) {
        const unsigned e = (unsigned)ell_get(s.nbr, (size_t)c.stride, p, k);
        if (e & BND_FLAG) continue;
        const float4 pb = s.prv[2 * (size_t)e];
        const float4 sb = s.vB[e];
        const float xx = pa.x - pb.x, xy = pa.y - pb.y, xz = pa.z - pb.z;
        const float f = grad_over_r(c.k, xx * xx + xy * xy + xz * xz);
        const float3 cr = cross3((sa.x - sb.x) * sc, (sa.y - sb.y) * sc, (sa.z - sb.z) * sc, xx * f, xy * f, xz * f);
        ox += cr.x;
        oy += cr.y;
        oz += cr.z;
    }
    const float4 v = make_float4(va.x + ox, va.y + oy, va.z + oz, 0.f);
    s.vel[p] = v;
    s.prv[2 * p + 1] = v;
}
}  // namespace

static inline int nblk(int n) { return (n > 0 ? n + NT - 1 : NT) / NT; }

void launch_vortex_second(const DevScene& s, const SolverConst& c, int mode, float alpha, float zeta, float nu_t,
                          float spacing, int n_max, cudaStream_t st) {
    const int nb = nblk(n_max);
    if (mode == 1) {
        k_vort_curl<1><<<nb, NT, 0, st>>>(s, c);
        k_trrv_domega<<<nb, NT, 0, st>>>(s, c);
        k_trrv_apply<<<nb, NT, 0, st>>>(s, c, alpha, spacing);
    } else if (mode == 2) {
        k_micro_w<<<nb, NT, 0, st>>>(s, c, zeta, nu_t);
        k_micro_v<<<nb, NT, 0, st>>>(s, c, nu_t);
    } else if (mode == 3) {
        k_vort_curl<3><<<nb, NT, 0, st>>>(s, c);
    }
}

void launch_vortex_after_div(const DevScene& s, const SolverConst& c, float spacing, int n_max, cudaStream_t st) {
    const int nb = nblk(n_max);
    const float v0 = (float)std::pow((double)spacing, 3.0);
    k_sfc_delta<<<nb, NT, 0, st>>>(s, c);
    k_sfc_psi<<<nb, NT, 0, st>>>(s, c, v0);
    k_sfc_apply<<<nb, NT, 0, st>>>(s, c);
}
