// sph_pci_ii.cu -- PCISPH (PciSph.cpp) and IISPH-multiphase (IISph_M.cpp)
// kernels.
//
// PCISPH step (PciSph::sphStep, PciSph.cpp:31-94; pci_computeForce :98-129):
//   neighbour search (lists only, sph_grid.cu)
//   k_pci_force_except  gravity + artificial viscosity (PciSph.cpp:166-274),
//                       pressure := 0, first predicted position (:278-296)
//   loop                k_pci_density: rho* over the stored list at the
//                                      predicted positions, cut at
//                                      smoothRadius_h; p += delta max(rho*-rho0,0);
//                                      max error (:300-352)
//                       k_pci_pressure: pressure acceleration (:356-439), next
//                                      predicted position, loop decision (:123)
//   k_pci_finish        a += a_p; Euler-Cromer into the staging arrays
//                       (:466-478, SphBase.cpp:377-402)
//
// IISPH_M step (IISph_M::sphStep, IISph_M.cpp:10-75):
//   neighbour search (lists only)
//   k_ii_force_except   a_adv for all phases, pressure := 0 (IISph_M.cpp:362-476)
//   per phase k, in order (later phases see the earlier phases' new values,
//   earlier phases see the later phases' values of the previous step, as the
//   reference's phase loop does):
//     k_ii_density      rho (own-phase mass times number density), d_ii, v_adv (:94-136)
//     k_ii_aii          a_ii, rho_adv, p_l = p/2 (:243-278)
//     loop              k_ii_sum: sum_j d_ij p_j (:290-313)
//                       k_ii_press: relaxed Jacobi update, clamp, FP64 error
//                                   sum and loop decision (:315-358)
//   k_ii_force          pressure acceleration (:480-571, 609-647) and the
//                       integration into the staging arrays
//
// The per-particle state that the reference keeps across steps and reads in
// the next step (the density of the previous step in the non-pressure forces;
// for IISPH_M also v_adv, p_l, d_ii, sum d_ij p_j of the other phases) travels
// through the cell reorder in three float4 arrays:
//   cA = (v_adv, p_l), cB = (d_ii, rho), cC = (sum_j d_ij p_j, a_ii)
// (PCISPH uses cB.w only).
#include "sph_kernels.cuh"

namespace {
constexpr int NT = 128;

__device__ __forceinline__ void nbr_fetch(const DevScene& s, unsigned e, bool& bnd, unsigned& j) {
    bnd = (e & BND_FLAG) != 0u;
    j = e & BND_MASK;
}

// x + (v + a dt) dt in the reference's operation order (PciSph.cpp:287-291)
__device__ __forceinline__ float4 predict(float4 x, float4 v, float ax, float ay, float az, float dt) {
    float4 r = x;
    r.x = __fadd_rn(__fmul_rn(__fadd_rn(__fmul_rn(ax, dt), v.x), dt), x.x);
    r.y = __fadd_rn(__fmul_rn(__fadd_rn(__fmul_rn(ay, dt), v.y), dt), x.y);
    r.z = __fadd_rn(__fmul_rn(__fadd_rn(__fmul_rn(az, dt), v.z), dt), x.z);
    return r;
}

// last-block reduction of two FP64 per-block values (sum, count)
__device__ __forceinline__ bool finish_sum2(double* partial, unsigned* ticket, double a, double b, double* ta,
                                            double* tb) {
    __shared__ bool last;
    if (threadIdx.x == 0) {
        partial[2 * blockIdx.x] = a;
        partial[2 * blockIdx.x + 1] = b;
        __threadfence();
        unsigned t = atomicAdd(ticket, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    __shared__ double sh[NT / 32];
    double x = 0, y = 0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += NT) {
        x += ((volatile double*)partial)[2 * i];
        y += ((volatile double*)partial)[2 * i + 1];
    }
    double tx = block_sum_double<NT>(x, sh);
    double ty = block_sum_double<NT>(y, sh);
    if (threadIdx.x == 0) {
        *ta = tx;
        *tb = ty;
        *ticket = 0u;
    }
    return threadIdx.x == 0;
}

// ============================== PCISPH ==============================

__global__ void __launch_bounds__(NT) k_pci_force_except(DevScene s, SolverConst c) {
    const int n = s.st->n_active;
    const int p = blockIdx.x * NT + threadIdx.x;
    int zero = 0;
    if (p < n) {
        const float dt = *s.dt;
        const float4 pa = s.pos[p], va = s.vel[p];
        const int ph = phase_of(pa);
        const float fm0 = c.fm_ph[ph], rho0 = c.rho0_ph[ph], alpha = c.alpha_ph[ph];
        const float ra = s.cB[p].w;  // density of the previous step
        const float den0 = 0.01f * c.hs * c.hs;
        const float hscs = c.hs * c.cs;
        float ax = c.gravity[0], ay = c.gravity[1], az = c.gravity[2];
        const int cnt = s.ncount[p];
        const size_t stride = (size_t)c.stride;
        for (int k = 0; k < cnt; ++k) {
            bool bnd;
            unsigned j;
            nbr_fetch(s, (unsigned)ell_get(s.nbr, stride, p, k), bnd, j);
            const float4 pb = bnd ? s.bpos[j] : s.pos[j];
            const float4 vb = bnd ? s.bvel[j] : s.vel[j];
            const float xx = pa.x - pb.x, xy = pa.y - pb.y, xz = pa.z - pb.z;
            const float len2 = xx * xx + xy * xy + xz * xz;
            if (len2 == 0.f) { ++zero; continue; }
            const float pro = (va.x - vb.x) * xx + (va.y - vb.y) * xy + (va.z - vb.z) * xz;
            if (!(pro < 0.f)) continue;
            const float f = grad_over_r(c.k, len2);
            float acce;
            if (bnd) {
                // PciSph.cpp:218-224
                const float nu = 2.f * c.bvisc * hscs / (ra * 2.f);
                const float pi = -nu * pro / (len2 + den0);
                acce = f * (-rho0 * pb.w * pi);
            } else {
                const float rb = s.cB[j].w;
                const int phb = phase_of(pb);
                if (phb == ph) {  // PciSph.cpp:178-184
                    const float nu = 2.f * alpha * hscs / (ra + rb);
                    const float pi = -nu * pro / (len2 + den0);
                    acce = f * (-fm0 * pi);
                } else {          // PciSph.cpp:198-204
                    const float al = (alpha + c.alpha_ph[phb]) / 2.f;
                    const float nu = 2.f * al * hscs / (ra + rb);
                    const float pi = -nu * pro / (len2 + den0);
                    acce = f * (-(fm0 + c.fm_ph[phb]) / 2.f * pi);
                }
            }
            ax = fmaf(xx, acce, ax);
            ay = fmaf(xy, acce, ay);
            az = fmaf(xz, acce, az);
        }
        s.acc[p] = make_float4(ax, ay, az, 0.f);
        s.ap[p] = make_float4(0.f, 0.f, 0.f, 0.f);
        s.kr[p] = 0.f;
        s.aux4[p] = predict(pa, va, ax, ay, az, dt);
    }
    if (__syncthreads_or(zero)) {
        if (zero) atomicAdd(&s.st->zero_dis, zero);
    }
}

// predicted density over the stored list with distances from the predicted
// positions, cut at smoothRadius_h (PciSph.cpp:318-333)
__global__ void __launch_bounds__(NT) k_pci_density(DevScene s, SolverConst c, float delta) {
    const int n = s.st->n_active;
    const int p = blockIdx.x * NT + threadIdx.x;
    float mine = 0.f;
    if (p < n) {
        const float4 xa = s.aux4[p];
        const float4 pa = s.pos[p];
        const int ph = phase_of(pa);
        const float fm0 = c.fm_ph[ph], rho0 = c.rho0_ph[ph];
        float density = ker_W(c.k, 0.f) * fm0;
        const int cnt = s.ncount[p];
        const int ng = (cnt + 3) >> 2;
        const size_t stride = (size_t)c.stride;
        const unsigned long long polL = l2_policy(c.l2pol & 3);  // lists stream through L2
        // four list entries per 16-byte load, the next group's issued before
        // the current group's gathers; the sum stays in list order
        int4 nxt = ng ? ell_group_pol(s.nbr, stride, p, 0, polL) : make_int4(0, 0, 0, 0);
        for (int gi = 0; gi < ng; ++gi) {
            const int4 cur = nxt;
            if (gi + 1 < ng) nxt = ell_group_pol(s.nbr, stride, p, gi + 1, polL);
            const unsigned e[4] = {(unsigned)cur.x, (unsigned)cur.y, (unsigned)cur.z, (unsigned)cur.w};
            float4 xb[4];
            bool bnd[4];
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                const unsigned u = gi * 4 + t < cnt ? e[t] : (unsigned)p;
                unsigned j;
                nbr_fetch(s, u, bnd[t], j);
                xb[t] = __ldg(bnd[t] ? s.bpos + j : s.aux4 + j);
            }
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                if (gi * 4 + t >= cnt) break;
                const float dis = sqrtf(dis_square_rn(xa.x, xa.y, xa.z, xb[t].x, xb[t].y, xb[t].z));
                if (dis < c.hs) density += (bnd[t] ? rho0 * xb[t].w : fm0) * ker_W(c.k, dis);
            }
        }
        s.rho[p] = density;
        float e = density - rho0;
        if (e < 0.f) e = 0.f;  // NEGLECT_NEGATIVE_PRESSURE (SphBase.h:32)
        const float pr = s.kr[p] + delta * e;
        s.kr[p] = pr;
        // the record the pressure sweep gathers per fluid neighbour:
        // {position (w: phase bits), (p/rho^2, p/(rho/m)^2)} -- the
        // neighbour's factors of PciSph.cpp:383-420, each a function of the
        // neighbour alone, computed once here instead of once per pair
        const float db = density / fm0;
        s.prv[2 * p] = pa;
        s.prv[2 * p + 1] = make_float4(pr / (density * density), pr / (db * db), 0.f, 0.f);
        mine = e / rho0;
    }
    // max of non-negative floats: their bit patterns order as ints (NaN and
    // inf order above every finite value, so they are reported)
    int b = __float_as_int(mine);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) b = max(b, __shfl_down_sync(0xffffffffu, b, o));
    if ((threadIdx.x & 31) == 0 && b > 0) atomicMax(&s.st->pci_emax_bits, b);
}

// pressure acceleration (PciSph.cpp:356-439), next predicted position, and
// the decision of PciSph.cpp:123.  Nine resident blocks per SM declared (56
// registers instead of 62 at eight): 69.9 -> 68 us on the 500k column.
__global__ void __launch_bounds__(NT, 9) k_pci_pressure(DevScene s, SolverConst c, float eta, int min_it, int max_it,
                                                     cudaGraphConditionalHandle h, int use_handle) {
    const int n = s.st->n_active;
    const int p = blockIdx.x * NT + threadIdx.x;
    int zero = 0;
    if (p < n) {
        const float dt = *s.dt;
        const float4 pa = s.pos[p];
        const int ph = phase_of(pa);
        const float fm0 = c.fm_ph[ph], rho0 = c.rho0_ph[ph];
        const float ra = s.rho[p], pra = s.kr[p];
        const float sa = pra / (ra * ra);
        float px = 0.f, py = 0.f, pz = 0.f;
        const int cnt = s.ncount[p];
        const int ng = (cnt + 3) >> 2;
        const size_t stride = (size_t)c.stride;
        const unsigned long long polL = l2_policy(c.l2pol & 3);  // lists stream through L2
        // one 32-byte record per fluid neighbour ({position, (rho, p)}, written
        // by this iteration's density sweep); boundary neighbours: position
        // and volume
        int4 nxt = ng ? ell_group_pol(s.nbr, stride, p, 0, polL) : make_int4(0, 0, 0, 0);
        for (int gi = 0; gi < ng; ++gi) {
            const int4 cur = nxt;
            if (gi + 1 < ng) nxt = ell_group_pol(s.nbr, stride, p, gi + 1, polL);
            const unsigned e[4] = {(unsigned)cur.x, (unsigned)cur.y, (unsigned)cur.z, (unsigned)cur.w};
            float4 pbs[4], rps[4];
            bool bnd[4];
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                const unsigned u = gi * 4 + t < cnt ? e[t] : (unsigned)p;
                unsigned j;
                nbr_fetch(s, u, bnd[t], j);
                ld_record32(bnd[t] ? s.bpv + 2 * (size_t)j : s.prv + 2 * (size_t)j, pbs[t], rps[t]);
            }
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                if (gi * 4 + t >= cnt) break;
                const float4 pb = pbs[t];
                const float xx = pa.x - pb.x, xy = pa.y - pb.y, xz = pa.z - pb.z;
                const float len2 = xx * xx + xy * xy + xz * xz;
                if (len2 == 0.f) { ++zero; continue; }
                const float f = grad_over_r(c.k, len2);
                float acce;
                if (bnd[t]) {
                    if (!(pra > 0.f)) continue;
                    acce = f * (-rho0 * pb.w * (2.f * pra / (ra * ra)));
                } else {
                    // rps: (p_j / rho_j^2, p_j / (rho_j / m_j)^2)
                    const int phb = phase_of(pb);
                    if (phb == ph) {
                        acce = f * (-fm0 * (sa + rps[t].x));
                    } else {
                        const float da = ra / fm0;
                        acce = f * (-1.f / fm0 * (pra / (da * da) + rps[t].y));
                    }
                }
                px = fmaf(xx, acce, px);
                py = fmaf(xy, acce, py);
                pz = fmaf(xz, acce, pz);
            }
        }
        s.ap[p] = make_float4(px, py, pz, 0.f);
        const float4 a = s.acc[p];
        s.aux4[p] = predict(pa, s.vel[p], __fadd_rn(a.x, px), __fadd_rn(a.y, py), __fadd_rn(a.z, pz), dt);
    }
    if (__syncthreads_or(zero)) {
        if (zero) atomicAdd(&s.st->zero_dis, zero);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        // the density kernel of this iteration has finished: its maximum is final
        const int it = ++s.st->it_density;
        ++s.st->total_it_density;
        const float emax = __int_as_float(s.st->pci_emax_bits);
        s.st->pci_emax_bits = 0;
        s.st->err_density = (double)emax;
        const bool crit = !(emax < eta);
        int cont = (crit || it < min_it) && it < max_it;
        if (!cont && crit) atomicOr(&s.st->status, 1u);
        if (!(emax == emax) || isinf(emax)) {
            cont = 0;
            atomicOr(&s.st->status, 4u);
        }
        s.st->cont = cont;
        if (use_handle) cudaGraphSetConditional(h, cont ? 1u : 0u);
    }
}

// a += a_p (PciSph.cpp:466-478); v += a dt; x += v dt (SphBase.cpp:390-392)
// into the staging arrays; the density rides along for the next step
__global__ void __launch_bounds__(NT) k_pci_finish(DevScene s) {
    const int n = s.st->n_active;
    const int p = blockIdx.x * NT + threadIdx.x;
    if (p >= n) return;
    const float dt = *s.dt;
    float4 a = s.acc[p];
    const float4 ap = s.ap[p];
    a.x = __fadd_rn(a.x, ap.x);
    a.y = __fadd_rn(a.y, ap.y);
    a.z = __fadd_rn(a.z, ap.z);
    float4 v = s.vel[p], x = s.pos[p];
    v.x = __fadd_rn(v.x, __fmul_rn(a.x, dt));
    v.y = __fadd_rn(v.y, __fmul_rn(a.y, dt));
    v.z = __fadd_rn(v.z, __fmul_rn(a.z, dt));
    x.x = __fadd_rn(x.x, __fmul_rn(v.x, dt));
    x.y = __fadd_rn(x.y, __fmul_rn(v.y, dt));
    x.z = __fadd_rn(x.z, __fmul_rn(v.z, dt));
    s.acc[p] = a;
    s.pos_s[p] = x;
    s.vel_s[p] = v;
    s.gid_s[p] = s.gid[p];
    s.cB_s[p] = make_float4(0.f, 0.f, 0.f, s.rho[p]);
}

// ============================== IISPH_M ==============================

// IISph_M::ii_forceExceptPressure (IISph_M.cpp:430-476): the same-phase and
// boundary viscosity terms have no sign guard (:362-381, 407-428), the
// different-phase term is the guarded Monaghan form (:384-404)
__global__ void __launch_bounds__(NT) k_ii_force_except(DevScene s, SolverConst c) {
    const int n = s.st->n_active;
    const int p = blockIdx.x * NT + threadIdx.x;
    int zero = 0;
    if (p < n) {
        const float4 pa = s.pos[p], va = s.vel[p];
        const int ph = phase_of(pa);
        const float fm0 = c.fm_ph[ph], rho0 = c.rho0_ph[ph], alpha = c.alpha_ph[ph];
        const float ra = s.cB[p].w;  // density of the previous step
        const float den0 = 0.01f * c.hs * c.hs;
        const float visc = 10.f * c.nu;
        float ax = c.gravity[0], ay = c.gravity[1], az = c.gravity[2];
        const int cnt = s.ncount[p];
        const size_t stride = (size_t)c.stride;
        for (int k = 0; k < cnt; ++k) {
            bool bnd;
            unsigned j;
            nbr_fetch(s, (unsigned)ell_get(s.nbr, stride, p, k), bnd, j);
            const float4 pb = bnd ? s.bpos[j] : s.pos[j];
            const float4 vb = bnd ? s.bvel[j] : s.vel[j];
            const float xx = pa.x - pb.x, xy = pa.y - pb.y, xz = pa.z - pb.z;
            const float len2 = xx * xx + xy * xy + xz * xz;
            if (len2 == 0.f) { ++zero; continue; }
            const float pro = (va.x - vb.x) * xx + (va.y - vb.y) * xy + (va.z - vb.z) * xz;
            const float f = grad_over_r(c.k, len2);
            float t;
            if (bnd) {
                t = f * pro / (len2 + den0) * (rho0 * pb.w) / ra * visc;
            } else {
                const int phb = phase_of(pb);
                const float rb = s.cB[j].w;
                if (phb == ph) {
                    t = f * pro / (len2 + den0) * fm0 / rb * visc;
                } else {
                    if (!(pro < 0.f)) continue;
                    const float al = (alpha + c.alpha_ph[phb]) / 2.f;
                    const float nu = 2.f * al * c.hs * c.cs / (ra + rb);
                    const float pi = -nu * pro / (len2 + den0);
                    t = f * (-(fm0 + c.fm_ph[phb]) / 2.f * pi);
                }
            }
            ax = fmaf(xx, t, ax);
            ay = fmaf(xy, t, ay);
            az = fmaf(xz, t, az);
        }
        s.acc[p] = make_float4(ax, ay, az, 0.f);
        s.kr[p] = 0.f;
    }
    if (__syncthreads_or(zero)) {
        if (zero) atomicAdd(&s.st->zero_dis, zero);
    }
}

__global__ void k_ii_phase_begin(DevScene s) {
    DevStats* st = s.st;
    st->ii_iter = 0;
    st->ii_num = 0;
    st->ii_sum_cum = 0.0;
    st->ii_nb_cum = 0.0;
    st->cont = 1;
}

// rho = m_k (W(0) + sum_f W) + sum_b rho0_k V_b W; d_ii = -dt^2 sum m_j/rho^2 gradW;
// v_adv = v + a_adv dt (IISph_M.cpp:94-136)
__global__ void __launch_bounds__(NT) k_ii_density(DevScene s, SolverConst c, int phase) {
    const int n = s.st->n_active;
    const int p = blockIdx.x * NT + threadIdx.x;
    int mine = 0;
    if (p < n) {
        const float4 pa = s.pos[p];
        if (phase_of(pa) == phase) {
            mine = 1;
            const float dt = *s.dt;
            const float fm0 = c.fm_ph[phase], rho0 = c.rho0_ph[phase];
            float density = ker_W(c.k, 0.f) * fm0;
            float gx = 0.f, gy = 0.f, gz = 0.f;
            const int cnt = s.ncount[p];
            const size_t stride = (size_t)c.stride;
            for (int k = 0; k < cnt; ++k) {
                bool bnd;
                unsigned j;
                nbr_fetch(s, (unsigned)ell_get(s.nbr, stride, p, k), bnd, j);
                const float4 pb = bnd ? s.bpos[j] : s.pos[j];
                const float xx = pa.x - pb.x, xy = pa.y - pb.y, xz = pa.z - pb.z;
                const float len2 = xx * xx + xy * xy + xz * xz;
                float w, f;
                kernel_pair(c.k, len2, w, f);
                const float m = bnd ? rho0 * pb.w : fm0;
                density = fmaf(m, w, density);
                const float fm = f * m;
                gx = fmaf(xx, fm, gx);
                gy = fmaf(xy, fm, gy);
                gz = fmaf(xz, fm, gz);
            }
            const float q = -(dt * dt) / (density * density);
            s.cB[p] = make_float4(gx * q, gy * q, gz * q, density);
            s.rho[p] = density;
            const float4 v = s.vel[p], a = s.acc[p];
            float4 ca = s.cA[p];
            ca.x = __fadd_rn(v.x, __fmul_rn(a.x, dt));
            ca.y = __fadd_rn(v.y, __fmul_rn(a.y, dt));
            ca.z = __fadd_rn(v.z, __fmul_rn(a.z, dt));
            s.cA[p] = ca;
        }
    }
    __shared__ int sh[NT / 32];
    const int cntb = block_sum_int<NT>(mine, sh);
    if (threadIdx.x == 0 && cntb) atomicAdd(&s.st->ii_num, cntb);
}

// a_ii, rho_adv, p_l = p/2 (IISph_M.cpp:243-278)
__global__ void __launch_bounds__(NT) k_ii_aii(DevScene s, SolverConst c, int phase) {
    const int n = s.st->n_active;
    const int p = blockIdx.x * NT + threadIdx.x;
    if (p >= n) return;
    const float4 pa = s.pos[p];
    // every particle's record for the sum sweep of this phase's loop:
    // {position, (p_l, rho)} (the other phases keep their carried values)
    s.prv[2 * p] = pa;
    if (phase_of(pa) != phase) {
        s.prv[2 * p + 1] = make_float4(s.cA[p].w, s.cB[p].w, 0.f, 0.f);
        return;
    }
    const float dt = *s.dt;
    const float fm0 = c.fm_ph[phase], rho0 = c.rho0_ph[phase];
    const float4 da = s.cB[p];  // (d_ii, rho)
    const float ra = da.w;
    const float4 va = s.vel[p];
    const float4 wa = s.cA[p];  // (v_adv, p_l)
    const float qd = fm0 * dt * dt / (ra * ra);
    float tv1 = 0.f, tv2 = 0.f;
    const int cnt = s.ncount[p];
    const size_t stride = (size_t)c.stride;
    for (int k = 0; k < cnt; ++k) {
        bool bnd;
        unsigned j;
        nbr_fetch(s, (unsigned)ell_get(s.nbr, stride, p, k), bnd, j);
        const float4 pb = bnd ? s.bpos[j] : s.pos[j];
        const float xx = pa.x - pb.x, xy = pa.y - pb.y, xz = pa.z - pb.z;
        const float f = grad_over_r(c.k, xx * xx + xy * xy + xz * xz);
        const float g0 = xx * f, g1 = xy * f, g2 = xz * f;
        if (bnd) {
            const float4 vb = s.bvel[j];
            const float m = rho0 * pb.w;
            tv1 += (g0 * (va.x - vb.x) + g1 * (va.y - vb.y) + g2 * (va.z - vb.z)) * m * dt;
            tv2 += (da.x * g0 + da.y * g1 + da.z * g2) * m;
        } else {
            const float4 wb = s.cA[j];
            tv1 += (g0 * (wa.x - wb.x) + g1 * (wa.y - wb.y) + g2 * (wa.z - wb.z)) * fm0 * dt;
            tv2 += ((da.x - g0 * qd) * g0 + (da.y - g1 * qd) * g1 + (da.z - g2 * qd) * g2) * fm0;
        }
    }
    if (tv2 == 0.f) tv2 = 1.f;
    reinterpret_cast<float*>(s.cC + p)[3] = tv2;
    s.aux1[p] = ra + tv1;
    const float pl = (float)(0.5 * (double)s.kr[p]);
    reinterpret_cast<float*>(s.cA + p)[3] = pl;
    s.prv[2 * p + 1] = make_float4(pl, ra, 0.f, 0.f);
}

// sum_j d_ij p_j = -dt^2 sum_f m_k p_j / rho_j^2 gradW (IISph_M.cpp:290-313);
// every particle also saves its p_l as the previous iterate
// Records: prv = {position, (p_l, rho)} (written by k_ii_aii for every
// particle, p_l updated by k_ii_press), read here per fluid neighbour in one
// 32-byte load; this kernel writes every particle's record for k_ii_press,
// pv = {(d_ii, previous iterate p_l), (sum_j d_ij p_j, 0)}.
__global__ void __launch_bounds__(NT) k_ii_sum(DevScene s, SolverConst c, int phase) {
    const int n = s.st->n_active;
    const int p = blockIdx.x * NT + threadIdx.x;
    if (p >= n) return;
    const float4 pa = s.pos[p];
    const float pla = s.cA[p].w;
    s.pl2[p] = pla;
    const float4 db = s.cB[p];
    float4 cc = s.cC[p];
    if (phase_of(pa) == phase) {
        const float dt = *s.dt;
        const float fm0 = c.fm_ph[phase];
        float tx = 0.f, ty = 0.f, tz = 0.f;
        const int cnt = s.ncount[p];
        const int ng = (cnt + 3) >> 2;
        const size_t stride = (size_t)c.stride;
        const unsigned long long polL = l2_policy(c.l2pol & 3);  // lists stream through L2
        int4 nxt = ng ? ell_group_pol(s.nbr, stride, p, 0, polL) : make_int4(0, 0, 0, 0);
        for (int gi = 0; gi < ng; ++gi) {
            const int4 cur = nxt;
            if (gi + 1 < ng) nxt = ell_group_pol(s.nbr, stride, p, gi + 1, polL);
            const unsigned e[4] = {(unsigned)cur.x, (unsigned)cur.y, (unsigned)cur.z, (unsigned)cur.w};
            float4 pb[4], rb[4];
            bool use[4];
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                // boundary neighbours add nothing here: they read the own record
                use[t] = gi * 4 + t < cnt && !(e[t] & BND_FLAG);
                ld_record32(s.prv + 2 * (size_t)(use[t] ? e[t] : (unsigned)p), pb[t], rb[t]);
            }
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                if (!use[t]) continue;
                const float xx = pa.x - pb[t].x, xy = pa.y - pb[t].y, xz = pa.z - pb[t].z;
                const float f = grad_over_r(c.k, xx * xx + xy * xy + xz * xz);
                const float q = -(fm0 * rb[t].x) / (rb[t].y * rb[t].y) * f;
                tx = fmaf(xx, q, tx);
                ty = fmaf(xy, q, ty);
                tz = fmaf(xz, q, tz);
            }
        }
        const float dt2 = dt * dt;
        cc = make_float4(tx * dt2, ty * dt2, tz * dt2, cc.w);
        s.cC[p] = cc;
    }
    s.pv[2 * p] = make_float4(db.x, db.y, db.z, pla);
    s.pv[2 * p + 1] = make_float4(cc.x, cc.y, cc.z, 0.f);
}

// relaxed Jacobi update (IISph_M.cpp:315-351) and the loop decision (:352-358)
__global__ void __launch_bounds__(NT) k_ii_press(DevScene s, SolverConst c, int phase, double omega, double eta_rel,
                                                 int min_it, int max_it, int compat, cudaGraphConditionalHandle h,
                                                 int use_handle) {
    const int n = s.st->n_active;
    const int p = blockIdx.x * NT + threadIdx.x;
    const float fm0 = c.fm_ph[phase], rho0 = c.rho0_ph[phase];
    double msum = 0.0, mnb = 0.0;
    if (p < n) {
        const float4 pa = s.pos[p];
        if (phase_of(pa) == phase) {
            const float dt = *s.dt;
            const float4 ca = s.cC[p];  // (sum d_ij p_j, a_ii)
            const float ra = s.cB[p].w;
            const float pla = s.pl2[p];
            const float qd = dt * dt * fm0 / (ra * ra);
            float ft = 0.f;
            const int cnt = s.ncount[p];
            const int ng = (cnt + 3) >> 2;
            const size_t stride = (size_t)c.stride;
            const unsigned long long polL = l2_policy(c.l2pol & 3);  // lists stream through L2
            // per fluid neighbour: its position and its k_ii_sum record
            // {(d_jj, previous p_l), (sum_k d_jk p_k, 0)}; boundary: position
            // and volume
            int4 nxt = ng ? ell_group_pol(s.nbr, stride, p, 0, polL) : make_int4(0, 0, 0, 0);
            for (int gi = 0; gi < ng; ++gi) {
                const int4 cur = nxt;
                if (gi + 1 < ng) nxt = ell_group_pol(s.nbr, stride, p, gi + 1, polL);
                const unsigned e[4] = {(unsigned)cur.x, (unsigned)cur.y, (unsigned)cur.z, (unsigned)cur.w};
                float4 pb[4], db[4], sb[4];
                bool bnd[4];
#pragma unroll
                for (int t = 0; t < 4; ++t) {
                    const unsigned u = gi * 4 + t < cnt ? e[t] : (unsigned)p;
                    unsigned j;
                    nbr_fetch(s, u, bnd[t], j);
                    pb[t] = __ldg(bnd[t] ? s.bpos + j : s.pos + j);
                    ld_record32(s.pv + 2 * (size_t)(bnd[t] ? (unsigned)p : j), db[t], sb[t]);
                }
#pragma unroll
                for (int t = 0; t < 4; ++t) {
                    if (gi * 4 + t >= cnt) break;
                    const float xx = pa.x - pb[t].x, xy = pa.y - pb[t].y, xz = pa.z - pb[t].z;
                    const float f = grad_over_r(c.k, xx * xx + xy * xy + xz * xz);
                    const float g0 = xx * f, g1 = xy * f, g2 = xz * f;
                    if (bnd[t]) {
                        ft += (rho0 * pb[t].w) * (ca.x * g0 + ca.y * g1 + ca.z * g2);
                    } else {
                        const float plb = db[t].w;
                        const float t0 = (ca.x - db[t].x * plb) - (sb[t].x - g0 * qd * pla);
                        const float t1 = (ca.y - db[t].y * plb) - (sb[t].y - g1 * qd * pla);
                        const float t2 = (ca.z - db[t].z * plb) - (sb[t].z - g2 * qd * pla);
                        ft += fm0 * (t0 * g0 + t1 * g1 + t2 * g2);
                    }
                }
            }
            const float aii = ca.w, radv = s.aux1[p];
            float t = (float)((1.0 - omega) * (double)pla + (omega / (double)aii) * (double)(rho0 - radv - ft));
            if (t < 0.f) {
                t = 0.f;
            } else {
                const float dn = radv + aii * pla + ft;
                msum = (compat & 1) ? (double)dn : (double)dn - (double)rho0;
                mnb = 1.0;
            }
            reinterpret_cast<float*>(s.cA + p)[3] = t;
            s.kr[p] = t;
            s.prv[2 * p + 1] = make_float4(t, ra, 0.f, 0.f);  // the next sum sweep's p_l
        }
    }
    __shared__ double sh[NT / 32];
    const double bs = block_sum_double<NT>(msum, sh);
    const double bn = block_sum_double<NT>(mnb, sh);
    double tot, nb;
    if (finish_sum2(s.partial, &s.st->ticket[3], bs, bn, &tot, &nb)) {
        DevStats* st = s.st;
        const int it = ++st->ii_iter;
        ++st->it_density;
        ++st->total_it_density;
        const double num = (double)st->ii_num;
        const double eta = eta_rel * (double)rho0;
        double err;
        bool crit;
        int cont;
        if (compat & 1) {
            // IISph_M.cpp:283-284, 350, 353-358: running sums over all
            // iterations, l counts particle updates
            st->ii_sum_cum += tot;
            st->ii_nb_cum += nb;
            err = st->ii_nb_cum > 0 ? (float)((float)st->ii_sum_cum / (float)num - rho0) : 0.0;
            crit = err > eta;
            cont = (crit || (double)it * num < 2.0) && it < max_it;
        } else {
            err = num > 0 ? tot / num : 0.0;
            crit = err > eta;
            cont = (crit || it < min_it) && it < max_it;
        }
        st->err_density = err / (double)rho0;
        if (!cont && crit) atomicOr(&st->status, 1u);
        if (!(err == err)) {
            cont = 0;
            atomicOr(&st->status, 4u);
        }
        st->cont = cont;
        if (use_handle) cudaGraphSetConditional(h, cont ? 1u : 0u);
    }
}

// pressure acceleration (IISph_M.cpp:480-571, 609-647) and the integration
// v = v_adv + a_p dt (or, with compat bit 2, v + a_p dt as SphBase.cpp:387-389
// under -DIISPH); x += v dt; into the staging arrays with the carried state
__global__ void __launch_bounds__(NT) k_ii_force(DevScene s, SolverConst c, int compat) {
    const int n = s.st->n_active;
    const int p = blockIdx.x * NT + threadIdx.x;
    int zero = 0;
    if (p < n) {
        const float dt = *s.dt;
        const float4 pa = s.pos[p], va = s.vel[p];
        const int ph = phase_of(pa);
        const float fm0 = c.fm_ph[ph], rho0 = c.rho0_ph[ph], alpha = c.alpha_ph[ph];
        const float4 cb = s.cB[p];
        const float ra = cb.w, pra = s.kr[p];
        const float den0 = 0.01f * c.hs * c.hs;
        float px = 0.f, py = 0.f, pz = 0.f;
        const int cnt = s.ncount[p];
        const size_t stride = (size_t)c.stride;
        for (int k = 0; k < cnt; ++k) {
            bool bnd;
            unsigned j;
            nbr_fetch(s, (unsigned)ell_get(s.nbr, stride, p, k), bnd, j);
            const float4 pb = bnd ? s.bpos[j] : s.pos[j];
            const float xx = pa.x - pb.x, xy = pa.y - pb.y, xz = pa.z - pb.z;
            const float len2 = xx * xx + xy * xy + xz * xz;
            if (len2 == 0.f) { ++zero; continue; }
            const float f = grad_over_r(c.k, len2);
            float acce;
            if (bnd) {
                if (!(pra > 0.f)) continue;
                acce = f * (-rho0 * pb.w * (pra / (ra * ra) * 2.f));
            } else {
                const float rb = s.cB[j].w, prb = s.kr[j];
                const int phb = phase_of(pb);
                if (phb == ph) {
                    acce = f * (-fm0 * (pra / (ra * ra) + prb / (rb * rb)));
                } else {
                    const float fmb = c.fm_ph[phb];
                    const float da = ra / fm0, db = rb / fmb;
                    acce = f * (-1.f / fm0 * (pra / (da * da) + prb / (db * db)));
                    const float4 vb = s.vel[j];
                    const float pro = (va.x - vb.x) * xx + (va.y - vb.y) * xy + (va.z - vb.z) * xz;
                    if (pro < 0.f) {
                        const float al = (alpha + c.alpha_ph[phb]) / 2.f;
                        const float nu = 2.f * al * c.hs * c.cs / (ra + rb);
                        const float pi = -nu * pro / (len2 + den0);
                        acce += f * (-(fm0 + fmb) / 2.f * pi);
                    }
                }
            }
            px = fmaf(xx, acce, px);
            py = fmaf(xy, acce, py);
            pz = fmaf(xz, acce, pz);
        }
        s.acc[p] = make_float4(px, py, pz, 0.f);
        const float4 ca = s.cA[p];
        float4 v = (compat & 2) ? va : make_float4(ca.x, ca.y, ca.z, 0.f);
        float4 x = pa;
        v.x = __fadd_rn(v.x, __fmul_rn(px, dt));
        v.y = __fadd_rn(v.y, __fmul_rn(py, dt));
        v.z = __fadd_rn(v.z, __fmul_rn(pz, dt));
        v.w = 0.f;
        x.x = __fadd_rn(x.x, __fmul_rn(v.x, dt));
        x.y = __fadd_rn(x.y, __fmul_rn(v.y, dt));
        x.z = __fadd_rn(x.z, __fmul_rn(v.z, dt));
        s.pos_s[p] = x;
        s.vel_s[p] = v;
        s.gid_s[p] = s.gid[p];
        s.cA_s[p] = ca;
        s.cB_s[p] = cb;
        s.cC_s[p] = s.cC[p];
    }
    if (__syncthreads_or(zero)) {
        if (zero) atomicAdd(&s.st->zero_dis, zero);
    }
}
// carried state for particles that arrive from another solver: sorted
// arrays take the last computed density, staging arrays the rest density
__global__ void k_carry_init(DevScene s, SolverConst c, int staging) {
    const int n = s.st->n_active;
    const int p = blockIdx.x * NT + threadIdx.x;
    if (p >= n) return;
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    if (staging) {
        s.cA_s[p] = z;
        s.cB_s[p] = make_float4(0.f, 0.f, 0.f, c.rho0_ph[phase_of(s.pos_s[p])]);
        s.cC_s[p] = z;
    } else {
        s.cA[p] = z;
        s.cB[p] = make_float4(0.f, 0.f, 0.f, s.rho[p]);
        s.cC[p] = z;
    }
}
}  // namespace

static inline int nblk(int n) { return (n > 0 ? n + NT - 1 : NT) / NT; }

void launch_carry_init(const DevScene& s, const SolverConst& c, int staging, int n_max, cudaStream_t st) {
    k_carry_init<<<nblk(n_max), NT, 0, st>>>(s, c, staging);
}

void launch_pci_force_except(const DevScene& s, const SolverConst& c, int n_max, cudaStream_t st) {
    k_pci_force_except<<<nblk(n_max), NT, 0, st>>>(s, c);
}
void launch_pci_density(const DevScene& s, const SolverConst& c, float delta, int n_max, cudaStream_t st) {
    k_pci_density<<<nblk(n_max), NT, 0, st>>>(s, c, delta);
}
void launch_pci_pressure(const DevScene& s, const SolverConst& c, float eta, int min_it, int max_it,
                         unsigned long long cond_handle, int use_handle, int n_max, cudaStream_t st) {
    k_pci_pressure<<<nblk(n_max), NT, 0, st>>>(s, c, eta, min_it, max_it, (cudaGraphConditionalHandle)cond_handle,
                                                use_handle);
}
void launch_pci_finish(const DevScene& s, int n_max, cudaStream_t st) { k_pci_finish<<<nblk(n_max), NT, 0, st>>>(s); }

void launch_ii_force_except(const DevScene& s, const SolverConst& c, int n_max, cudaStream_t st) {
    k_ii_force_except<<<nblk(n_max), NT, 0, st>>>(s, c);
}
void launch_ii_phase_begin(const DevScene& s, cudaStream_t st) { k_ii_phase_begin<<<1, 1, 0, st>>>(s); }
void launch_ii_density(const DevScene& s, const SolverConst& c, int phase, int n_max, cudaStream_t st) {
    k_ii_density<<<nblk(n_max), NT, 0, st>>>(s, c, phase);
}
void launch_ii_aii(const DevScene& s, const SolverConst& c, int phase, int n_max, cudaStream_t st) {
    k_ii_aii<<<nblk(n_max), NT, 0, st>>>(s, c, phase);
}
void launch_ii_sum(const DevScene& s, const SolverConst& c, int phase, int n_max, cudaStream_t st) {
    k_ii_sum<<<nblk(n_max), NT, 0, st>>>(s, c, phase);
}
void launch_ii_press(const DevScene& s, const SolverConst& c, int phase, double omega, double eta_rel, int min_it,
                     int max_it, int compat, unsigned long long cond_handle, int use_handle, int n_max,
                     cudaStream_t st) {
    k_ii_press<<<nblk(n_max), NT, 0, st>>>(s, c, phase, omega, eta_rel, min_it, max_it, compat,
                                            (cudaGraphConditionalHandle)cond_handle, use_handle);
}
void launch_ii_force(const DevScene& s, const SolverConst& c, int compat, int n_max, cudaStream_t st) {
    k_ii_force<<<nblk(n_max), NT, 0, st>>>(s, c, compat);
}
