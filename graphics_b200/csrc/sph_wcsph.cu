// sph_wcsph.cu -- WCSPH kernels (reference: WcSph.cpp).
//
// WcSph::sphStep (WcSph.cpp:23-96) is neighbourSearch -> wc_computePressure ->
// wc_computeForce -> updateFluids.  The density + Tait pressure pass is fused
// into the neighbour-list kernel (k_build_win, mode 2); this file holds the
// force pass, fused with the Euler-Cromer update (SphBase.cpp:377-402), which
// writes the new state into the staging arrays that the next neighbour search
// sorts.  One block per brick with the window's positions, velocities,
// densities and pressures in shared memory (sph_window.cuh).  Surface tension
// and adhesion (WcSph.cpp:188-211, 300-311) are not on this path: they vanish
// for m_TH.r = m_TH.bt = 0, the plain method.
#include "sph_window.cuh"

namespace {

__global__ void __launch_bounds__(WIN_NT) k_wc_force(DevScene s, GridGeom g, SolverConst c) {
    extern __shared__ float4 sm[];
    float4* sp = sm;
    float4* sv = sm + WIN_MAX;
    float2* srp = (float2*)(sm + 2 * WIN_MAX);  // (rho, pressure) of fluid slots
    __shared__ WinHead H;
    win_setup(s, g, blockIdx.x, H);
    int zero = 0;
    if (H.own_b > H.own_a) {
        const bool wide = H.wide;
        if (!wide) {
            win_stage4(H, s.pos, s.bpos, sp);
            win_stage4(H, s.vel, s.bvel, sv);
            for (int q = threadIdx.x; q < H.nf; q += WIN_NT) {
                const int cc = win_cell_of(H.fstart, q);
                const int j = H.fglob[cc] + (q - H.fstart[cc]);
                srp[q] = make_float2(s.rho[j], s.kr[j]);
            }
        }
        __syncthreads();
        const float dt = *s.dt;
        const float den0 = 0.01f * c.hs * c.hs;
        const size_t stride = (size_t)c.stride;
        const int nf = H.nf;
        for (int p = H.own_a + threadIdx.x; p < H.own_b; p += WIN_NT) {
            const float4 pa = s.pos[p];
            const float4 va = s.vel[p];
            const int ph = phase_of(pa);
            const float ra = s.rho[p], pra = s.kr[p];
            const float fma_ = c.fm_ph[ph], rho0 = c.rho0_ph[ph], alpha = c.alpha_ph[ph];
            const float pa_term = pra / (ra * ra);
            float ax = c.gravity[0], ay = c.gravity[1], az = c.gravity[2];
            const int cnt = s.ncount[p];
            for (int k = 0; k < cnt; ++k) {
                float4 pb, vb;
                bool bnd;
                float rb = 0.f, prb = 0.f;
                if (!wide) {
                    const int q = s.nbr16[k * stride + p];
                    pb = sp[q];
                    vb = sv[q];
                    bnd = q >= nf;
                    if (!bnd) { const float2 t = srp[q]; rb = t.x; prb = t.y; }
                } else {
                    const unsigned e = (unsigned)s.nbr[k * stride + p];
                    bnd = (e & BND_FLAG) != 0u;
                    const unsigned j = e & BND_MASK;
                    pb = (bnd ? s.bpos : s.pos)[j];
                    vb = (bnd ? s.bvel : s.vel)[j];
                    if (!bnd) { rb = s.rho[j]; prb = s.kr[j]; }
                }
                const float xx = pa.x - pb.x, xy = pa.y - pb.y, xz = pa.z - pb.z;
                const float len2 = xx * xx + xy * xy + xz * xz;
                if (len2 == 0.f) { ++zero; continue; }
                const float dis = sqrtf(len2);
                const float grad = -ker_Wg(c.k, dis) / dis;
                const float pro = (va.x - vb.x) * xx + (va.y - vb.y) * xy + (va.z - vb.z) * xz;
                float acce;
                if (bnd) {
                    // wc_fluidPartForce_bound, WcSph.cpp:281-294
                    const float vol = pb.w;
                    acce = 0.f;
                    if (pra > 0.f) acce += grad * (-rho0 * vol * (pa_term * 2.f));
                    if (pro < 0.f) {
                        const float nu = 2.f * c.bvisc * c.hs * c.cs / (ra * 2.f);
                        const float pi = -nu * pro / (len2 + den0);
                        acce += grad * (-rho0 * vol * pi);
                    }
                } else {
                    const int phb = phase_of(pb);
                    if (phb == ph) {
                        // wc_fluidPartForce_fsame, WcSph.cpp:174-187
                        acce = grad * (-fma_ * (pa_term + prb / (rb * rb)));
                        if (pro < 0.f) {
                            const float nu = 2.f * alpha * c.hs * c.cs / (ra + rb);
                            const float pi = -nu * pro / (len2 + den0);
                            acce += grad * (-fma_ * pi);
                        }
                    } else {
                        // wc_fluidPartForce_fdiff, WcSph.cpp:239-253
                        const float fmb = c.fm_ph[phb];
                        const float al = (alpha + c.alpha_ph[phb]) / 2.f;
                        const float da = ra / fma_, db = rb / fmb;
                        acce = grad * (-1.f / fma_ * (pra / (da * da) + prb / (db * db)));
                        if (pro < 0.f) {
                            const float nu = 2.f * al * c.hs * c.cs / (ra + rb);
                            const float pi = -nu * pro / (len2 + den0);
                            acce += grad * (-(fma_ + fmb) / 2.f * pi);
                        }
                    }
                }
                ax += xx * acce;
                ay += xy * acce;
                az += xz * acce;
            }
            s.acc[p] = make_float4(ax, ay, az, 0.f);
            // Euler-Cromer: v += a dt; x += v dt (SphBase.cpp:390-392)
            float4 v, x;
            v.x = __fadd_rn(va.x, __fmul_rn(ax, dt));
            v.y = __fadd_rn(va.y, __fmul_rn(ay, dt));
            v.z = __fadd_rn(va.z, __fmul_rn(az, dt));
            v.w = 0.f;
            x.x = __fadd_rn(pa.x, __fmul_rn(v.x, dt));
            x.y = __fadd_rn(pa.y, __fmul_rn(v.y, dt));
            x.z = __fadd_rn(pa.z, __fmul_rn(v.z, dt));
            x.w = pa.w;
            s.pos_s[p] = x;
            s.vel_s[p] = v;
            s.gid_s[p] = s.gid[p];
        }
    }
    if (__syncthreads_or(zero)) {
        if (zero) atomicAdd(&s.st->zero_dis, zero);
    }
}
}  // namespace

static const size_t SMEM_WC = (size_t)WIN_MAX * 40;

void wcsph_init_attributes() {
    cudaFuncSetAttribute(k_wc_force, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_WC);
}

void launch_wc_force(const DevScene& s, const GridGeom& g, const SolverConst& c, cudaStream_t st) {
    k_wc_force<<<g.nb[0] * g.nb[1] * g.nb[2], WIN_NT, SMEM_WC, st>>>(s, g, c);
}
