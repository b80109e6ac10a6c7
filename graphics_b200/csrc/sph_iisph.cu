// sph_iisph.cu -- IISph, the volume form of the implicit solver (reference:
// IISph.cpp, class IISph; the solver the reference's demo scene derives from,
// Demo-mySPH.h:21).
//
// One step (IISph::sphStep, IISph.cpp:14-99, temperature update off):
//   neighbour search + k_build mode 3   sphDensity, VF_gamma, VF_sphVolume,
//                                       VF_alpha per fluid particle (sph_grid.cu)
//   k_iv_boundary_build                 each boundary particle's own list of
//                                       fluid neighbours and its gamma,
//                                       sphVolume, alpha (IISph.cpp:452-543)
//   k_iv_forces                         advectionStep: gravity + viscosity with
//                                       the kinematic viscosity (:1458-1570)
//   divergence-free loop per phase      k_iv_boundary_sweep, k_iv_sweep_a,
//                                       k_iv_sweep_b (:1219-1456)
//   constant-volume loop per phase      the same three kernels (:546-815)
//   k_iv_integrate                      acce_presure = (v_adv - v)/dt,
//                                       v += acce_presure dt, x += v dt
//                                       (SphBase.cpp:377-402 with -DIISPH)
//
// Carried between steps (through the reorder): the loop velocity v_adv
// (cA) and the last stiffnesses (kappa, kappaV) (cC), which the other
// phases' loops read as the reference reads them from the particle.
//
// In every iteration the boundary particles first compute their own volume
// change (or divergence) from their fluid neighbours' loop velocities and
// from it a stiffness kappa_b; the fluid sweep A computes kappa_i; sweep B
// updates the loop velocity with both:
//   v_i -= dt/m_i sum_j gradW_ij (V_i^2 V_j kappa_i/gamma_i + V_j^2 V_i kappa_j/gamma_j).
// Per-particle arithmetic is FP32; the error sums are FP64 block partials
// reduced in a fixed order by the last block.  Phases are solved in turn,
// as the reference does; the loop velocities of the other phases are the
// carried ones (the reference keeps advectionVelocity in the particle).
//
// Records gathered per neighbour: sweep A and the boundary sweep read
// {position, loop velocity} (pv / bpv, 32 B, one 256-bit load); sweep B
// reads (x, y, z, kappa/gamma) (pk, 16 B) for fluid neighbours and
// (x, y, z, V_b) plus kappa_b/gamma_b for boundary ones.
#include "sph_kernels.cuh"

namespace {
constexpr int NT = 128;

// Boundary particle p: its neighbour list in the reference's order (27 cells,
// per cell the fluid range then the boundary range; same-solid neighbours
// skipped for rigid solids, SphBase.cpp:922), capped at c.cap entries of
// which only the fluid ones are stored, and VF_prepareAttribute's boundary
// terms (IISph.cpp:452-543).  Walls are static, so boundary-boundary pairs
// only enter gamma and sphVolume.
template <int BS>
__global__ void __launch_bounds__(BS) k_iv_boundary_build(DevScene s, GridGeom g, SolverConst c) {
    const int p = blockIdx.x * BS + threadIdx.x;
    int over = 0;
    if (p < s.nb) {
        const float4 pa = s.bpos[p];
        const int sid = s.bsid[p];
        const float Va = pa.w;
        const float w0 = c.kd.theta;
        float gamma = Va * w0;
        float sphv = (float)((double)w0 * (double)Va * (double)Va);
        float a2 = 0.f;
        int all = 0, nf = 0;
        const size_t bstride = (size_t)s.bstride;
        const int cx = cell_coord(pa.x, g.min[0], g.divisor);
        const int cy = cell_coord(pa.y, g.min[1], g.divisor);
        const int cz = cell_coord(pa.z, g.min[2], g.divisor);
        const float hc = 1.f / g.divisor;
        const float lo_x = pa.x - (g.min[0] + cx * hc), hi_x = (g.min[0] + (cx + 1) * hc) - pa.x;
        const float lo_y = pa.y - (g.min[1] + cy * hc), hi_y = (g.min[1] + (cy + 1) * hc) - pa.y;
        const float lo_z = pa.z - (g.min[2] + cz * hc), hi_z = (g.min[2] + (cz + 1) * hc) - pa.z;
        const float cull = c.h2cut * 1.001f + 1e-12f;
        for (int dz = -1; dz <= 1; ++dz) {
            const float gz = dz < 0 ? fmaxf(lo_z, 0.f) : (dz > 0 ? fmaxf(hi_z, 0.f) : 0.f);
            for (int dy = -1; dy <= 1; ++dy) {
                const float gy = dy < 0 ? fmaxf(lo_y, 0.f) : (dy > 0 ? fmaxf(hi_y, 0.f) : 0.f);
                for (int dx = -1; dx <= 1; ++dx) {
                    const float gx = dx < 0 ? fmaxf(lo_x, 0.f) : (dx > 0 ? fmaxf(hi_x, 0.f) : 0.f);
                    if (gx * gx + gy * gy + gz * gz > cull) continue;
                    const int x = cx + dx, y = cy + dy, z = cz + dz;
                    if (!cell_inside(g, x, y, z)) continue;
                    const int key = cell_key(g, x, y, z);
                    const int2 s0 = __ldg(s.cstart2 + key), s1 = __ldg(s.cstart2 + key + 1);
                    for (int q = s0.x; q < s1.x; ++q) {
                        const float4 pb = __ldg(s.pos + q);
                        const float len2 = dis_square_rn(pa.x, pa.y, pa.z, pb.x, pb.y, pb.z);
                        if (!(len2 < c.h2cut)) continue;
                        if (all >= c.cap) { ++over; continue; }
                        ++all;
                        s.bnbr[ell_index(bstride, p, nf++)] = q;
                        float w, f;
                        kernel_pair_rn(c.kd, len2, w, f);
                        const float Vb = c.iv_V;
                        gamma = fmaf(Vb, w, gamma);
                        sphv = fmaf(Va * Vb, w, sphv);
                        const float fv = f * Vb;
                        a2 = fmaf(fv * fv, len2 / c.iv_m[phase_of(pb)], a2);
                    }
                    if (!c.iv_multi_solid) continue;
                    for (int q = s0.y; q < s1.y; ++q) {
                        if (q == p || __ldg(s.bsid + q) == sid) continue;
                        const float4 pb = __ldg(s.bpos + q);
                        const float len2 = dis_square_rn(pa.x, pa.y, pa.z, pb.x, pb.y, pb.z);
                        if (!(len2 < c.h2cut)) continue;
                        if (all >= c.cap) { ++over; continue; }
                        ++all;
                        float w, f;
                        kernel_pair_rn(c.kd, len2, w, f);
                        gamma = fmaf(pb.w, w, gamma);
                        sphv = fmaf(Va * pb.w, w, sphv);
                    }
                }
            }
        }
        s.bncount[p] = nf;
        float al = a2 / gamma;
        if (al < 1.0e-10f) al = 1.0e-10f;
        s.bivs[p] = make_float4(gamma, sphv, 1.f / al, 0.f);
    }
    if (__syncthreads_or(over)) {
        if (over) {
            atomicAdd(&s.st->overflow, over);
            atomicOr(&s.st->status, 8u);
        }
    }
}

// advectionStep (IISph.cpp:1505-1570): a = g + viscosity.  Same phase
// (f2fAdvection, :1458-1470) and boundary (b2fAdvection, :1490-1503):
//   a += gradW * 2 (dim + 2) nu_k (V_j / gamma_j) (v_ij . x_ij) / (r^2 + 1e-6)
// with nu_k the mean kinematic viscosity of the pair; other phases
// (ii_fluidPartForceExceptPressure_fdiff, :1472-1488): Monaghan's term with
// the single-h kernel, only for approaching pairs.  The loop velocities
// start from the carried ones (other phases keep them through the first
// phase's loops, as in the reference).
template <int BS>
__global__ void __launch_bounds__(BS) k_iv_forces(DevScene s, SolverConst c) {
    const int n = s.st->n_active;
    const int p = blockIdx.x * BS + threadIdx.x;
    int zero = 0;
    if (p < n) {
        const float4 pa = s.pos[p];
        const float4 va = s.vel[p];
        const int ph = phase_of(pa);
        const float Va = c.iv_V, ma = c.iv_m[ph], alpha = c.alpha_ph[ph];
        const float rhoa = s.ivs[p].w;
        const float kvf = (c.iv_kv + c.iv_kv) / 2, kvb = (c.iv_kv + c.iv_kvb) / 2;
        const float den0 = 0.01f * c.hs * c.hs;
        float ax = c.gravity[0], ay = c.gravity[1], az = c.gravity[2];
        const int cnt = s.ncount[p];
        const size_t stride = (size_t)c.stride;
        for (int k = 0; k < cnt; ++k) {
            const unsigned e = (unsigned)ell_get(s.nbr, stride, p, k);
            const bool bnd = (e & BND_FLAG) != 0u;
            const unsigned j = e & BND_MASK;
            const float4 pb = bnd ? s.bpos[j] : s.pos[j];
            const float4 vb = bnd ? s.bvel[j] : s.vel[j];
            const float xx = pa.x - pb.x, xy = pa.y - pb.y, xz = pa.z - pb.z;
            const float len2 = xx * xx + xy * xy + xz * xz;
            if (len2 == 0.f) { ++zero; continue; }
            const float pro = (va.x - vb.x) * xx + (va.y - vb.y) * xy + (va.z - vb.z) * xz;
            float t;
            if (bnd || phase_of(pb) == ph) {
                const float vg = bnd ? pb.w / s.bivs[j].x : Va / s.ivs[j].x;
                const float f = grad_over_r(c.kd, len2);
                t = f * 10.f * (bnd ? kvb : kvf) * vg * pro / (len2 + 1e-6f);
            } else {
                if (!(pro < 0.f)) continue;
                const int phb = phase_of(pb);
                const float fmb = Va * c.rho0_ph[phb];
                const float al = (alpha + c.alpha_ph[phb]) / 2.f;
                const float nu = 2.f * al * c.hs * c.cs / (rhoa + s.ivs[j].w);
                const float pi = -nu * pro / (len2 + den0);
                t = grad_over_r(c.k, len2) * (-(ma + fmb) / 2.f * pi);
            }
            ax = fmaf(xx, t, ax);
            ay = fmaf(xy, t, ay);
            az = fmaf(xz, t, az);
        }
        s.acc[p] = make_float4(ax, ay, az, 0.f);
        const float4 ca = s.cA[p], cc = s.cC[p];
        s.pv[2 * p + 1] = make_float4(ca.x, ca.y, ca.z, 0.f);
        s.kappa[p] = cc.x;
        s.kappav[p] = cc.y;
    }
    if (__syncthreads_or(zero)) {
        if (zero) atomicAdd(&s.st->zero_dis, zero);
    }
}

__global__ void k_iv_phase_begin(DevScene s) {
    s.st->ii_iter = 0;
    s.st->ii_num = 0;
    s.st->cont = 1;
}

// loop velocity of the phase: v (IISph.cpp:1232) or v + a dt (:560).
// Particles of the other phases enter this phase's velocity updates with
// their own last stiffness of the same loop kind (VF_kappaV or VF_kappa,
// carried between steps as the reference keeps them in the particle).
__global__ void __launch_bounds__(NT) k_iv_loop_init(DevScene s, int phase, int div) {
    const int n = s.st->n_active;
    const int p = blockIdx.x * NT + threadIdx.x;
    int mine = 0;
    if (p < n && phase_of(s.pos[p]) != phase) {
        s.pk[p].w = (div ? s.kappav[p] : s.kappa[p]) / s.ivs[p].x;
    } else if (p < n) {
        mine = 1;
        float4 v = s.vel[p];
        if (!div) {
            const float dt = *s.dt;
            const float4 a = s.acc[p];
            v.x = __fadd_rn(v.x, __fmul_rn(a.x, dt));
            v.y = __fadd_rn(v.y, __fmul_rn(a.y, dt));
            v.z = __fadd_rn(v.z, __fmul_rn(a.z, dt));
        }
        v.w = 0.f;
        s.pv[2 * p + 1] = v;
    }
    __shared__ int sh[NT / 32];
    const int c = block_sum_int<NT>(mine, sh);
    if (threadIdx.x == 0 && c) atomicAdd(&s.st->ii_num, c);
}

// sum over the stored list of V_j gradW_ij . (v_i - v_j), gradW with the
// per-pair h; fluid neighbours read {position, loop velocity} (pv), boundary
// ones {(x, y, z, V_b), velocity} (bpv)
__device__ __forceinline__ float iv_div_sum(const DevScene& s, const SolverConst& c, int p, float4 pa, float4 va) {
    const int cnt = s.ncount[p];
    const int ng = (cnt + 3) >> 2;
    const size_t stride = (size_t)c.stride;
    const float Vf = c.iv_V;
    float acc = 0.f;
    const unsigned long long polL = l2_policy(c.l2pol & 3);  // lists stream through L2
    int4 nxt = ng ? ell_group_pol(s.nbr, stride, p, 0, polL) : make_int4(0, 0, 0, 0);
    for (int gi = 0; gi < ng; ++gi) {
        const int4 cur = nxt;
        if (gi + 1 < ng) nxt = ell_group_pol(s.nbr, stride, p, gi + 1, polL);
        const unsigned e[4] = {(unsigned)cur.x, (unsigned)cur.y, (unsigned)cur.z, (unsigned)cur.w};
        float4 pb[4], vb[4];
        bool ok[4], bnd[4];
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            ok[t] = gi * 4 + t < cnt;
            const unsigned u = ok[t] ? e[t] : (unsigned)p;
            bnd[t] = (u & BND_FLAG) != 0u;
            const float4* rec = (bnd[t] ? s.bpv : s.pv) + 2 * (size_t)(u & BND_MASK);
            ld_record32(rec, pb[t], vb[t]);
        }
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            const float Vb = bnd[t] ? pb[t].w : Vf;
            const float xx = pa.x - pb[t].x, xy = pa.y - pb[t].y, xz = pa.z - pb[t].z;
            const float f = grad_over_r(c.kd, xx * xx + xy * xy + xz * xz);
            const float dot = xx * (va.x - vb[t].x) + xy * (va.y - vb[t].y) + xz * (va.z - vb[t].z);
            const float nacc = fmaf(dot * f, Vb, acc);
            acc = ok[t] ? nacc : acc;
        }
    }
    return acc;
}

// Boundary particles, one iteration (IISph.cpp:566-606 / 1237-1275): volume
// change (constant volume) or divergence from the fluid neighbours' loop
// velocities, clamped as the reference does, and the stiffness
//   kappa_b  = (V_adv - V_b) / dt^2 / V_b^3 * alpha_b
//   kappaV_b = div * alpha_b / dt / V_b^3.
// Boundary-boundary pairs of static walls add exactly zero and are skipped.
template <int BS, int DIV>
__global__ void __launch_bounds__(BS) k_iv_boundary_sweep(DevScene s, SolverConst c) {
    const int p = blockIdx.x * BS + threadIdx.x;
    if (p >= s.nb) return;
    const float4 pa = s.bpos[p], vb0 = s.bvel[p];
    const float4 iv = s.bivs[p];
    const float Va = pa.w, dt = *s.dt;
    const int cnt = s.bncount[p];
    const size_t bstride = (size_t)s.bstride;
    float acc = 0.f;
    for (int k = 0; k < cnt; ++k) {
        const int j = s.bnbr[ell_index(bstride, p, k)];
        float4 pb, vb;
        ld_record32(s.pv + 2 * (size_t)j, pb, vb);
        const float xx = pa.x - pb.x, xy = pa.y - pb.y, xz = pa.z - pb.z;
        const float f = grad_over_r(c.kd, xx * xx + xy * xy + xz * xz);
        const float dot = xx * (vb0.x - vb.x) + xy * (vb0.y - vb.y) + xz * (vb0.z - vb.z);
        acc = fmaf(dot * f, c.iv_V, acc);
    }
    float4 o = s.bivo[p];
    float kap;
    if (DIV) {
        float dd = acc * Va;
        if (dd < 0.f || (iv.y + dd * dt) < Va) dd = 0.f;
        kap = (float)((double)(dd * iv.z / dt) / ((double)Va * (double)Va * (double)Va));
        o.y = kap;
        o.w = dd;
    } else {
        float vadv = fmaf(acc * Va, dt, iv.y);
        if (vadv < Va) vadv = Va;
        kap = (float)((double)(vadv - Va) / ((double)dt * (double)dt) / ((double)Va * (double)Va * (double)Va) *
                      (double)iv.z);
        o.x = kap;
        o.z = vadv;
    }
    s.bivo[p] = o;
    s.bivs[p].w = kap / iv.x;
}

// Fluid sweep A of phase `phase` (IISph.cpp:1278-1317 / 607-650): volume
// change or divergence, clamp, stiffness kappa (pk.w = kappa/gamma), FP64
// sum of the error term: (V_adv - V)/V (constant volume) or the divergence.
template <int BS, int DIV>
__global__ void __launch_bounds__(BS) k_iv_sweep_a(DevScene s, SolverConst c, int phase) {
    const int n = s.st->n_active;
    const int p = blockIdx.x * BS + threadIdx.x;
    double mine = 0.0;
    if (p < n) {
        const float4 pa = s.pv[2 * p];
        if (phase_of(pa) == phase) {
            const float4 va = s.pv[2 * p + 1];
            const float4 iv = s.ivs[p];
            const float Va = c.iv_V, dt = *s.dt;
            const float acc = iv_div_sum(s, c, p, pa, va);
            float kap;
            if (DIV) {
                float dd = acc * Va;
                if (dd < 0.f || (iv.y + dd * dt) < Va) dd = 0.f;
                kap = (float)((double)(dd * iv.z / dt) / ((double)Va * (double)Va * (double)Va));
                s.kappav[p] = kap;
                s.aux1[p] = dd;
                mine = (double)dd;
            } else {
                float vadv = fmaf(acc * Va, dt, iv.y);
                if (vadv < Va) vadv = Va;
                kap = (float)((double)(vadv - Va) / ((double)dt * (double)dt) /
                              ((double)Va * (double)Va * (double)Va) * (double)iv.z);
                s.kappa[p] = kap;
                s.aux0[p] = vadv;
                mine = (double)((vadv - Va) / Va);
            }
            s.pk[p].w = kap / iv.x;
        }
    }
    __shared__ double sh[BS / 32];
    double bsum = block_sum_double<BS>(mine, sh);
    double tot;
    if (finish_sum<BS>(s.partial, &s.st->ticket[DIV ? 1 : 0], bsum, &tot)) {
        const double num = (double)s.st->ii_num;
        const double e = num > 0 ? tot / num : 0.0;
        if (DIV) s.st->err_div = e * (double)*s.dt;
        else s.st->err_density = e;
    }
}

// Fluid sweep B of phase `phase` (IISph.cpp:1360-1437 / 692-786):
//   v_i -= dt/m_i sum_j gradW_ij (V_i^2 V_j k_i + V_j^2 V_i k_j),  k = kappa/gamma,
// then (one thread) the loop decision: continue while the error is above
// the goal or fewer than min_it iterations ran, and stop once the count
// exceeds max_it (the reference breaks when it > max, :558,1234).
template <int BS, int DIV>
__global__ void __launch_bounds__(BS) k_iv_sweep_b(DevScene s, SolverConst c, int phase, double goal, int min_it,
                                                   int max_it, cudaGraphConditionalHandle h, int use_handle) {
    const int n = s.st->n_active;
    const int p = blockIdx.x * BS + threadIdx.x;
    if (p < n) {
        const float4 pa = s.pk[p];
        if (phase_of(s.pos[p]) == phase) {
            const float dt = *s.dt;
            const float Va = c.iv_V, ka = pa.w;
            const float fa = Va * Va * Va * ka;  // V_a^2 V_j k_a for fluid j (V_j = V_a)
            float4 va = s.pv[2 * p + 1];
            float dx = 0.f, dy = 0.f, dz = 0.f;
            const int cnt = s.ncount[p];
            const int ng = (cnt + 3) >> 2;
            const size_t stride = (size_t)c.stride;
            const unsigned long long polL = l2_policy(c.l2pol & 3);  // lists stream through L2
            int4 nxt = ng ? ell_group_pol(s.nbr, stride, p, 0, polL) : make_int4(0, 0, 0, 0);
            for (int gi = 0; gi < ng; ++gi) {
                const int4 cur = nxt;
                if (gi + 1 < ng) nxt = ell_group_pol(s.nbr, stride, p, gi + 1, polL);
                const unsigned e[4] = {(unsigned)cur.x, (unsigned)cur.y, (unsigned)cur.z, (unsigned)cur.w};
                float4 pb[4];
                float kb[4];
                bool ok[4], bnd[4];
#pragma unroll
                for (int t = 0; t < 4; ++t) {
                    ok[t] = gi * 4 + t < cnt;
                    const unsigned u = ok[t] ? e[t] : (unsigned)p;
                    bnd[t] = (u & BND_FLAG) != 0u;
                    const unsigned j = u & BND_MASK;
                    pb[t] = __ldg(bnd[t] ? s.bpos + j : s.pk + j);
                    kb[t] = bnd[t] ? __ldg(&s.bivs[j].w) : pb[t].w;
                }
#pragma unroll
                for (int t = 0; t < 4; ++t) {
                    const float Vb = pb[t].w;  // boundary: V_b
                    const float coef = bnd[t] ? Va * Va * Vb * ka + Vb * Vb * Va * kb[t]
                                              : fmaf(Va * Va * Va, kb[t], fa);
                    const float xx = pa.x - pb[t].x, xy = pa.y - pb[t].y, xz = pa.z - pb[t].z;
                    const float f = ok[t] ? grad_over_r(c.kd, xx * xx + xy * xy + xz * xz) * coef : 0.f;
                    dx = fmaf(xx, f, dx);
                    dy = fmaf(xy, f, dy);
                    dz = fmaf(xz, f, dz);
                }
            }
            const float sc = dt / c.iv_m[phase];
            va.x = fmaf(-dx, sc, va.x);
            va.y = fmaf(-dy, sc, va.y);
            va.z = fmaf(-dz, sc, va.z);
            s.pv[2 * p + 1] = va;
            if (DIV) s.vel[p] = va;  // velocity = advectionVelocity (IISph.cpp:1452-1455)
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        DevStats* st = s.st;
        const int it = ++st->ii_iter;
        const double err = DIV ? st->err_div : st->err_density;
        if (DIV) { ++st->it_div; ++st->total_it_div; }
        else { ++st->it_density; ++st->total_it_density; }
        const bool crit = err > goal;
        int cont = (crit || it < min_it) && it <= max_it;
        if (!cont && crit) atomicOr(&st->status, DIV ? 2u : 1u);
        if (!(err == err)) {
            cont = 0;
            atomicOr(&st->status, 4u);
        }
        st->cont = cont;
        if (use_handle) cudaGraphSetConditional(h, cont ? 1u : 0u);
    }
}

// acce_presure = (v_adv - v)/dt (IISph.cpp:797-800), then updateFluids with
// -DIISPH (SphBase.cpp:387-392): v = v + acce_presure dt, x += v dt, in
// round-to-nearest float ops, into the staging arrays; v_adv is carried
__global__ void __launch_bounds__(NT) k_iv_integrate(DevScene s) {
    const int n = s.st->n_active;
    const int p = blockIdx.x * NT + threadIdx.x;
    if (p >= n) return;
    const float dt = *s.dt;
    const float4 va = s.vel[p], vadv = s.pv[2 * p + 1];
    float4 ap, v, x = s.pos[p];
    ap.x = __fdiv_rn(__fsub_rn(vadv.x, va.x), dt);
    ap.y = __fdiv_rn(__fsub_rn(vadv.y, va.y), dt);
    ap.z = __fdiv_rn(__fsub_rn(vadv.z, va.z), dt);
    ap.w = 0.f;
    v.x = __fadd_rn(va.x, __fmul_rn(ap.x, dt));
    v.y = __fadd_rn(va.y, __fmul_rn(ap.y, dt));
    v.z = __fadd_rn(va.z, __fmul_rn(ap.z, dt));
    v.w = 0.f;
    x.x = __fadd_rn(x.x, __fmul_rn(v.x, dt));
    x.y = __fadd_rn(x.y, __fmul_rn(v.y, dt));
    x.z = __fadd_rn(x.z, __fmul_rn(v.z, dt));
    s.ap[p] = ap;
    s.pos_s[p] = x;
    s.vel_s[p] = v;
    s.gid_s[p] = s.gid[p];
    s.cA_s[p] = make_float4(vadv.x, vadv.y, vadv.z, 0.f);
    s.cC_s[p] = make_float4(s.kappa[p], s.kappav[p], 0.f, 0.f);
}
}  // namespace

static inline int nblk(int n, int bs = NT) { return (n > 0 ? n + bs - 1 : bs) / bs; }

#define IV_DISPATCH_BS(bs, CALL)                          \
    switch (bs) {                                         \
        case 64: { constexpr int B = 64; CALL; break; }   \
        case 256: { constexpr int B = 256; CALL; break; } \
        default: { constexpr int B = 128; CALL; break; }  \
    }

void launch_iv_boundary_build(const DevScene& s, const GridGeom& g, const SolverConst& c, int bs, cudaStream_t st) {
    if (s.nb <= 0) return;
    IV_DISPATCH_BS(bs, (k_iv_boundary_build<B><<<nblk(s.nb, B), B, 0, st>>>(s, g, c)));
}
void launch_iv_forces(const DevScene& s, const SolverConst& c, int n_max, int bs, cudaStream_t st) {
    IV_DISPATCH_BS(bs, (k_iv_forces<B><<<nblk(n_max, B), B, 0, st>>>(s, c)));
}
void launch_iv_phase_begin(const DevScene& s, cudaStream_t st) { k_iv_phase_begin<<<1, 1, 0, st>>>(s); }
void launch_iv_loop_init(const DevScene& s, int phase, int div, int n_max, cudaStream_t st) {
    k_iv_loop_init<<<nblk(n_max), NT, 0, st>>>(s, phase, div);
}
void launch_iv_boundary_sweep(const DevScene& s, const SolverConst& c, int div, int bs, cudaStream_t st) {
    if (s.nb <= 0) return;
    if (div) IV_DISPATCH_BS(bs, (k_iv_boundary_sweep<B, 1><<<nblk(s.nb, B), B, 0, st>>>(s, c)))
    else IV_DISPATCH_BS(bs, (k_iv_boundary_sweep<B, 0><<<nblk(s.nb, B), B, 0, st>>>(s, c)))
}
void launch_iv_sweep_a(const DevScene& s, const SolverConst& c, int phase, int div, int n_max, int bs,
                       cudaStream_t st) {
    if (div) IV_DISPATCH_BS(bs, (k_iv_sweep_a<B, 1><<<nblk(n_max, B), B, 0, st>>>(s, c, phase)))
    else IV_DISPATCH_BS(bs, (k_iv_sweep_a<B, 0><<<nblk(n_max, B), B, 0, st>>>(s, c, phase)))
}
void launch_iv_sweep_b(const DevScene& s, const SolverConst& c, int phase, int div, double goal, int min_it,
                       int max_it, unsigned long long cond_handle, int use_handle, int n_max, int bs,
                       cudaStream_t st) {
    const cudaGraphConditionalHandle hd = (cudaGraphConditionalHandle)cond_handle;
    if (div)
        IV_DISPATCH_BS(bs, (k_iv_sweep_b<B, 1><<<nblk(n_max, B), B, 0, st>>>(s, c, phase, goal, min_it, max_it, hd,
                                                                           use_handle)))
    else
        IV_DISPATCH_BS(bs, (k_iv_sweep_b<B, 0><<<nblk(n_max, B), B, 0, st>>>(s, c, phase, goal, min_it, max_it, hd,
                                                                           use_handle)))
}
void launch_iv_integrate(const DevScene& s, int n_max, cudaStream_t st) {
    k_iv_integrate<<<nblk(n_max), NT, 0, st>>>(s);
}
