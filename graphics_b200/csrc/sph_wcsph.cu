// sph_wcsph.cu -- WCSPH kernels (reference: WcSph.cpp).
//
// WcSph::sphStep (WcSph.cpp:23-96) is neighbourSearch -> wc_computePressure ->
// wc_computeForce -> updateFluids.  The density + Tait pressure pass is fused
// into the neighbour-list kernel (sph_grid.cu, mode 2); this file holds the
// force pass, fused with the Euler-Cromer update (SphBase.cpp:377-402), which
// writes the new state into the staging arrays that the next neighbour search
// sorts.  Surface tension and adhesion (WcSph.cpp:188-211, 300-311) run when
// m_TH.h, r or bt is set: k_wc_normal computes the surface normals
// n_i = h sum_j m/rho_j gradW_ij over fluid neighbours from this step's
// densities (the reference reads the neighbours' densities in the same loop
// that writes them, WcSph.cpp:129-133, so its values depend on the thread
// schedule), and the force kernel adds cohesion, curvature and adhesion.
#include "sph_kernels.cuh"

namespace {
constexpr int NT = 128;

// wc_computePressure's surface normal (WcSph.cpp:124-137) into vA
__global__ void __launch_bounds__(NT) k_wc_normal(DevScene s, SolverConst c) {
    const int n = s.st->n_active;
    const int p = blockIdx.x * NT + threadIdx.x;
    if (p >= n) return;
    const float4 pa = s.pos[p];
    const float fm0 = c.fm_ph[phase_of(pa)];
    float nx = 0.f, ny = 0.f, nz = 0.f;
    const int cnt = s.ncount[p];
    const size_t stride = (size_t)c.stride;
    for (int k = 0; k < cnt; ++k) {
        const unsigned e = (unsigned)ell_get(s.nbr, stride, p, k);
        if (e & BND_FLAG) continue;
        const float4 pb = s.pos[e];
        const float xx = pa.x - pb.x, xy = pa.y - pb.y, xz = pa.z - pb.z;
        const float dis = sqrtf(xx * xx + xy * xy + xz * xz);
        const float g = -ker_Wg(c.k, dis) / dis * (fm0 / s.rho[e]);
        nx += xx * g;
        ny += xy * g;
        nz += xz * g;
    }
    s.vA[p] = make_float4(nx * c.th_h, ny * c.th_h, nz * c.th_h, 0.f);
}

// Per-particle constants of the force pass.
struct WcOwn {
    float4 pa, va;
    int ph;
    float ra, pra, fma, rho0, alpha, den0, pa_term;
};
__device__ __forceinline__ WcOwn wc_own(const DevScene& s, const SolverConst& c, int p) {
    WcOwn o;
    o.pa = s.pos[p];
    o.va = s.vel[p];
    o.ph = phase_of(o.pa);
    o.ra = s.rho[p];
    o.pra = s.kr[p];
    o.fma = c.fm_ph[o.ph];
    o.rho0 = c.rho0_ph[o.ph];
    o.alpha = c.alpha_ph[o.ph];
    o.den0 = 0.01f * c.hs * c.hs;
    o.pa_term = o.pra / (o.ra * o.ra);
    return o;
}

// One neighbour's contribution to the acceleration (WcSph.cpp:156-311),
// added to (ax, ay, az) in the reference's order of terms; zero-distance
// pairs add nothing and are counted.
template <bool SURF>
__device__ __forceinline__ void wc_pair(const DevScene& s, const SolverConst& c, const WcOwn& o, int p, unsigned e,
                                        float& ax, float& ay, float& az, int& zero) {
    float acce;
    float4 pb;
    float xx, xy, xz, dis;
    if (e & BND_FLAG) {
        // wc_fluidPartForce_bound, WcSph.cpp:262-299
        const unsigned b = e & BND_MASK;
        pb = s.bpos[b];
        const float4 vb = s.bvel[b];
        xx = o.pa.x - pb.x; xy = o.pa.y - pb.y; xz = o.pa.z - pb.z;
        const float len2 = xx * xx + xy * xy + xz * xz;
        if (len2 == 0.f) { ++zero; return; }
        dis = sqrtf(len2);
        const float grad = -ker_Wg(c.k, dis) / dis;
        const float vol = pb.w;
        acce = 0.f;
        if (o.pra > 0.f) acce += grad * (-o.rho0 * vol * (o.pa_term * 2.f));
        const float pro = (o.va.x - vb.x) * xx + (o.va.y - vb.y) * xy + (o.va.z - vb.z) * xz;
        if (pro < 0.f) {
            const float nu = 2.f * c.bvisc * c.hs * c.cs / (o.ra * 2.f);
            const float pi = -nu * pro / (len2 + o.den0);
            acce += grad * (-o.rho0 * vol * pi);
        }
        if (SURF) {
            // adhesion (WcSph.cpp:300-311)
            const float h = c.th_h;
            float A = 0.f;
            if (2.f * dis > h && dis <= h)
                A = 0.007f / powf(h, 3.25f) * powf(-4.f * dis * dis / h + 6.f * dis - 2.f * h, 0.25f);
            acce += -c.th_bt * o.rho0 * vol * A / dis;
        }
    } else {
        pb = s.pos[e];
        const float4 vb = s.vel[e];
        xx = o.pa.x - pb.x; xy = o.pa.y - pb.y; xz = o.pa.z - pb.z;
        const float len2 = xx * xx + xy * xy + xz * xz;
        if (len2 == 0.f) { ++zero; return; }
        dis = sqrtf(len2);
        const float grad = -ker_Wg(c.k, dis) / dis;
        const float rb = s.rho[e], prb = s.kr[e];
        const int phb = phase_of(pb);
        const float pro = (o.va.x - vb.x) * xx + (o.va.y - vb.y) * xy + (o.va.z - vb.z) * xz;
        if (phb == o.ph) {
            // wc_fluidPartForce_fsame, WcSph.cpp:174-187
            acce = grad * (-o.fma * (o.pa_term + prb / (rb * rb)));
            if (pro < 0.f) {
                const float nu = 2.f * o.alpha * c.hs * c.cs / (o.ra + rb);
                const float pi = -nu * pro / (len2 + o.den0);
                acce += grad * (-o.fma * pi);
            }
            if (SURF) {
                // cohesion and curvature (WcSph.cpp:188-210), Kij with the
                // reference's rest density 1000
                const float h = c.th_h;
                const float Kij = 2.f * 1000.0f / (o.ra + rb);
                float C = 0.f;
                const float k9 = 32.0f / (3.14f * powf(h, 9.0f));
                if (2.f * dis > h && dis <= h) C = k9 * powf(h - dis, 3.0f) * powf(dis, 3.0f);
                else if (dis > 0.f && 2.f * dis <= h)
                    C = k9 * (2.f * powf(h - dis, 3.0f) * powf(dis, 3.0f) - powf(h, 6.0f) / 64.0f);
                const float coh = -c.th_r * o.fma * C / dis;
                const float4 na = s.vA[p], nb = s.vA[e];
                ax += (xx * coh + (na.x - nb.x) * -c.th_r) * Kij;
                ay += (xy * coh + (na.y - nb.y) * -c.th_r) * Kij;
                az += (xz * coh + (na.z - nb.z) * -c.th_r) * Kij;
            }
        } else {
            // wc_fluidPartForce_fdiff, WcSph.cpp:239-253
            const float fmb = c.fm_ph[phb];
            const float al = (o.alpha + c.alpha_ph[phb]) / 2.f;
            const float da = o.ra / o.fma, db = rb / fmb;
            acce = grad * (-1.f / o.fma * (o.pra / (da * da) + prb / (db * db)));
            if (pro < 0.f) {
                const float nu = 2.f * al * c.hs * c.cs / (o.ra + rb);
                const float pi = -nu * pro / (len2 + o.den0);
                acce += grad * (-(o.fma + fmb) / 2.f * pi);
            }
        }
    }
    ax += xx * acce;
    ay += xy * acce;
    az += xz * acce;
}

// the acceleration, then Euler-Cromer: v += a dt; x += v dt
// (SphBase.cpp:390-392) into the staging arrays the next sort reads
__device__ __forceinline__ void wc_finish(const DevScene& s, const WcOwn& o, int p, float ax, float ay, float az) {
    const float dt = *s.dt;
    s.acc[p] = make_float4(ax, ay, az, 0.f);
    float4 v, x;
    v.x = __fadd_rn(o.va.x, __fmul_rn(ax, dt));
    v.y = __fadd_rn(o.va.y, __fmul_rn(ay, dt));
    v.z = __fadd_rn(o.va.z, __fmul_rn(az, dt));
    v.w = 0.f;
    x.x = __fadd_rn(o.pa.x, __fmul_rn(v.x, dt));
    x.y = __fadd_rn(o.pa.y, __fmul_rn(v.y, dt));
    x.z = __fadd_rn(o.pa.z, __fmul_rn(v.z, dt));
    x.w = o.pa.w;
    s.pos_s[p] = x;
    s.vel_s[p] = v;
    s.gid_s[p] = s.gid[p];
}

// one thread per particle, neighbours in list order
template <bool SURF>
__global__ void __launch_bounds__(NT) k_wc_force(DevScene s, SolverConst c) {
    const int n = s.st->n_active;
    const int p = blockIdx.x * NT + threadIdx.x;
    int zero = 0;
    if (p < n) {
        const WcOwn o = wc_own(s, c, p);
        float ax = c.gravity[0], ay = c.gravity[1], az = c.gravity[2];
        const int cnt = s.ncount[p];
        const size_t stride = (size_t)c.stride;
        for (int k = 0; k < cnt; ++k) wc_pair<SURF>(s, c, o, p, (unsigned)ell_get(s.nbr, stride, p, k), ax, ay, az, zero);
        wc_finish(s, o, p, ax, ay, az);
    }
    if (__syncthreads_or(zero)) {
        if (zero) atomicAdd(&s.st->zero_dis, zero);
    }
}

// L threads per particle (small scenes, where one thread per particle
// leaves the SMs with too few warps to hide the gathers' latency): lane l
// takes neighbours l, l + L, ...; the lanes' sums are added in a fixed
// shuffle order (deterministic), the group's first lane integrates
template <bool SURF, int L>
__global__ void __launch_bounds__(NT) k_wc_force_lanes(DevScene s, SolverConst c) {
    const int n = s.st->n_active;
    const int t = blockIdx.x * NT + threadIdx.x;
    const int p = t / L, l = t % L;
    int zero = 0;
    float ax = 0.f, ay = 0.f, az = 0.f;
    WcOwn o;
    if (p < n) {
        o = wc_own(s, c, p);
        if (l == 0) { ax = c.gravity[0]; ay = c.gravity[1]; az = c.gravity[2]; }
        const int cnt = s.ncount[p];
        const size_t stride = (size_t)c.stride;
        for (int k = l; k < cnt; k += L) wc_pair<SURF>(s, c, o, p, (unsigned)ell_get(s.nbr, stride, p, k), ax, ay, az, zero);
    }
#pragma unroll
    for (int off = 1; off < L; off <<= 1) {
        ax += __shfl_xor_sync(0xffffffffu, ax, off);
        ay += __shfl_xor_sync(0xffffffffu, ay, off);
        az += __shfl_xor_sync(0xffffffffu, az, off);
    }
    if (p < n && l == 0) wc_finish(s, o, p, ax, ay, az);
    if (__syncthreads_or(zero)) {
        if (zero) atomicAdd(&s.st->zero_dis, zero);
    }
}
}  // namespace

void launch_wc_force(const DevScene& s, const SolverConst& c, int n_max, cudaStream_t st, bool surf, int lanes) {
    if (lanes == 4) {
        const int nb = (int)(((long long)n_max * 4 + NT - 1) / NT);
        if (surf) k_wc_force_lanes<true, 4><<<nb, NT, 0, st>>>(s, c);
        else k_wc_force_lanes<false, 4><<<nb, NT, 0, st>>>(s, c);
        return;
    }
    if (surf) k_wc_force<true><<<(n_max + NT - 1) / NT, NT, 0, st>>>(s, c);
    else k_wc_force<false><<<(n_max + NT - 1) / NT, NT, 0, st>>>(s, c);
}
void launch_wc_normal(const DevScene& s, const SolverConst& c, int n_max, cudaStream_t st) {
    k_wc_normal<<<(n_max + NT - 1) / NT, NT, 0, st>>>(s, c);
}
