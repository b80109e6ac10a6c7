// sph_dfsph.cu -- DFSPH kernels (reference: DFSPH.cpp) and the brick-window
// neighbour-list build they share with the other solvers.
//
// Per step (DFSPH::sphStep, DFSPH.cpp:45-62):
//   k_df_forces       DF_forceExceptPressure + v_adv = v + a_adv dt
//                     (DFSPH.cpp:1419-1475, 1246-1359, 557-563)
//   density loop      k_df_sweep_a<0>: rho_adv, clamp, kappa = (rho_adv-rho0)/dt^2 alpha,
//                                      FP64 sum of rho_adv      (DFSPH.cpp:574-643)
//                     k_df_vupdate<0>: v_adv -= dt sum m gradW (k_i/rho_i + k_j/rho_j),
//                                      convergence decision     (DFSPH.cpp:647-698)
//   integrate + neighbour search + rho/alpha (sph_grid.cu, k_build_win here)
//   divergence loop   k_df_sweep_a<1> / k_df_vupdate<1>        (DFSPH.cpp:769-900)
//
// Every sweep runs one block per 4x4x4-cell brick with the brick's 6x6x6-cell
// window staged in shared memory (sph_window.cuh) and reads the 16-bit
// window-slot neighbour lists; wide windows fall back to 32-bit global lists.
// The kernel gradient is recomputed from positions (-W'(r)/r with one rsqrt),
// per-particle arithmetic is FP32, and the convergence sums are FP64 block
// partials reduced in block order by the last block, so results are
// run-to-run deterministic.
//
// Loop control: k_df_vupdate decides whether another iteration runs.  Inside
// a CUDA graph the loop is a conditional WHILE node and the decision is
// written with cudaGraphSetConditional; host-driven loops read st->cont.
#include "sph_window.cuh"

namespace {
constexpr int NT = 128;

// last-block FP64 reduction of per-block partials; returns true in the
// thread that holds the total (thread 0 of the last block).  Every block of
// the grid must call it exactly once.
template <int BT>
__device__ __forceinline__ bool finish_sum(double* partial, unsigned* ticket, double v, double* total) {
    __shared__ bool last;
    if (threadIdx.x == 0) {
        partial[blockIdx.x] = v;
        __threadfence();
        unsigned t = atomicAdd(ticket, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    __shared__ double sh[BT / 32];
    double acc = 0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += BT) acc += ((volatile double*)partial)[i];
    double tot = block_sum_double<BT>(acc, sh);
    if (threadIdx.x == 0) {
        *total = tot;
        *ticket = 0u;
    }
    return threadIdx.x == 0;
}

__global__ void k_step_begin(DevScene s) {
    DevStats* st = s.st;
    st->max_nbrs = 0;
    st->nbr_total = 0ull;
    st->it_density = 0;
    st->it_div = 0;
    st->err_density = 0;
    st->err_div = 0;
}

__global__ void k_call_begin(DevScene s) {
    DevStats* st = s.st;
    st->removed = 0;
    st->overflow = 0;
    st->zero_dis = 0;
    st->status = 0u;
    st->total_it_density = 0;
    st->total_it_div = 0;
    st->wide_bricks = 0;
}

__global__ void k_loop_reset(DevScene s, int which) {
    if (which == 0) s.st->it_density = 0;
    else s.st->it_div = 0;
    s.st->cont = 1;
}

// ---------------------------------------------------------------------------
// neighbour lists + rho/alpha (mode 1) or + rho/Tait pressure (mode 2)
// ---------------------------------------------------------------------------
template <int MODE>
__global__ void __launch_bounds__(WIN_NT) k_build_win(DevScene s, GridGeom g, SolverConst c) {
    extern __shared__ float4 sp[];
    __shared__ WinHead H;
    const int brick = blockIdx.x;
    win_setup(s, g, brick, H);
    int cntsum = 0, over = 0, mx = 0;
    if (H.own_b > H.own_a) {
        const bool wide = H.wide;
        if (!wide) win_stage4(H, s.pos, s.bpos, sp);
        if (threadIdx.x == 0) s.brick_wide[brick] = wide;
        __syncthreads();
        const int x0 = H.bx * 4 - 1, y0 = H.by * 4 - 1, z0 = H.bz * 4 - 1;
        const size_t stride = (size_t)c.stride;
        const int cap = c.cap;
        for (int p = H.own_a + threadIdx.x; p < H.own_b; p += WIN_NT) {
            const float4 pa = s.pos[p];
            const int ph = phase_of(pa);
            const float fm0 = c.fm_ph[ph], rho0 = c.rho0_ph[ph];
            const int lx = cell_coord(pa.x, g.min[0], g.divisor) - x0;
            const int ly = cell_coord(pa.y, g.min[1], g.divisor) - y0;
            const int lz = cell_coord(pa.z, g.min[2], g.divisor) - z0;
            const int wc = (lz * 6 + ly) * 6 + lx;
            const int myslot = H.fstart[wc] + (p - H.fglob[wc]);
            float density = ker_W(c.k, 0.f) * fm0;
            float a1x = 0.f, a1y = 0.f, a1z = 0.f, a2 = 0.f;
            int cnt = 0;
            unsigned short* out16 = s.nbr16 + p;
            int* out32 = s.nbr + p;
            for (int dz = -1; dz <= 1; ++dz)
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dx = -1; dx <= 1; ++dx) {
                        const int w = ((lz + dz) * 6 + (ly + dy)) * 6 + (lx + dx);
                        // fluid range of the cell, then its boundary range
                        for (int pass = 0; pass < 2; ++pass) {
                            const int qa = pass ? H.nf + H.bstart[w] : H.fstart[w];
                            const int qb = pass ? H.nf + H.bstart[w + 1] : H.fstart[w + 1];
                            const int gbase = pass ? H.bglob[w] - (H.nf + H.bstart[w]) : H.fglob[w] - H.fstart[w];
                            for (int q = qa; q < qb; ++q) {
                                if (!pass && q == myslot) continue;
                                const float4 pb = wide ? (pass ? s.bpos[gbase + q] : s.pos[gbase + q]) : sp[q];
                                const float len2 = dis_square_rn(pa.x, pa.y, pa.z, pb.x, pb.y, pb.z);
                                if (len2 < c.h2cut) {
                                    if (cnt < cap) {
                                        if (wide) out32[(size_t)cnt * stride] = pass ? (int)((gbase + q) | BND_FLAG) : gbase + q;
                                        else out16[(size_t)cnt * stride] = (unsigned short)q;
                                        ++cnt;
                                        if (MODE != 0) {
                                            const float dis = sqrtf(len2);
                                            const float m = pass ? rho0 * pb.w : fm0;
                                            density += m * ker_W(c.k, dis);
                                            if (MODE == 1) {
                                                const float gs = -ker_Wg(c.k, dis);
                                                const float f = gs / dis;
                                                a1x += (pa.x - pb.x) * f * m;
                                                a1y += (pa.y - pb.y) * f * m;
                                                a1z += (pa.z - pb.z) * f * m;
                                                if (!pass) {
                                                    const float t = gs * fm0;
                                                    a2 = (float)((double)a2 + (double)t * (double)t);
                                                }
                                            }
                                        }
                                    } else {
                                        ++over;
                                    }
                                }
                            }
                        }
                    }
            s.ncount[p] = cnt;
            cntsum += cnt;
            mx = max(mx, cnt);
            if (MODE == 1) {
                s.rho[p] = density;
                float al = a1x * a1x + a1y * a1y + a1z * a1z + a2;
                if (al < 1.0e-6f) al = 1.0e-6f;
                s.alpha[p] = density / al;
            } else if (MODE == 2) {
                s.rho[p] = density;
                // Tait, WcSph.cpp:142-146 (NEGLECT_NEGATIVE_PRESSURE)
                float pr = c.wc_B * (powf(density / rho0, c.wc_gamma) - 1.f);
                if (pr < 0.f) pr = 0.f;
                s.kr[p] = pr;
            }
        }
        if (wide && threadIdx.x == 0) atomicAdd(&s.st->wide_bricks, 1);
    }
    __shared__ int shi[WIN_NT / 32];
    int tot = block_sum_int<WIN_NT>(cntsum, shi);
    int ov = block_sum_int<WIN_NT>(over, shi);
    int m2 = block_max_int<WIN_NT>(mx, shi);
    if (threadIdx.x == 0) {
        if (tot) atomicAdd(&s.st->nbr_total, (unsigned long long)tot);
        if (ov) { atomicAdd(&s.st->overflow, ov); atomicOr(&s.st->status, 8u); }
        if (m2) atomicMax(&s.st->max_nbrs, m2);
    }
}

// 16-bit window lists -> 32-bit global lists (for callers that read lists)
__global__ void __launch_bounds__(WIN_NT) k_expand_lists(DevScene s, GridGeom g, SolverConst c) {
    __shared__ WinHead H;
    win_setup(s, g, blockIdx.x, H);
    if (H.own_b <= H.own_a || H.wide) return;
    const size_t stride = (size_t)c.stride;
    for (int p = H.own_a + threadIdx.x; p < H.own_b; p += WIN_NT) {
        const int cnt = s.ncount[p];
        for (int k = 0; k < cnt; ++k) s.nbr[k * stride + p] = (int)win_global(H, s.nbr16[k * stride + p]);
    }
}

// ---------------------------------------------------------------------------
// Jacobi sweeps
// ---------------------------------------------------------------------------

// A sweep: sum_j m_j gradW_ij . (v_i - v_j), then
//   DIV = 0: rho_adv = max(rho + dt*sum, rho0), kappa  (DFSPH.cpp:574-643)
//   DIV = 1: Drho/Dt clamp, kappa_v                    (DFSPH.cpp:780-836)
// V = v_adv (density loop) or v (divergence loop, which updates v in place).
template <int DIV>
__global__ void __launch_bounds__(WIN_NT) k_df_sweep_a(DevScene s, GridGeom g, SolverConst c, int record) {
    extern __shared__ float4 sm[];
    float4* sp = sm;
    float4* sv = sm + WIN_MAX;
    __shared__ WinHead H;
    win_setup(s, g, blockIdx.x, H);
    const float4* V = DIV ? s.vel : s.vadv;
    double mine = 0.0;
    if (H.own_b > H.own_a) {
        const bool wide = H.wide;
        if (!wide) {
            win_stage4(H, s.pos, s.bpos, sp);
            win_stage4(H, V, s.bvel, sv);
        }
        __syncthreads();
        const float dt = *s.dt;
        const float rho0 = c.rho0, fm0 = c.fm0;
        const size_t stride = (size_t)c.stride;
        const int nf = H.nf;
        for (int p = H.own_a + threadIdx.x; p < H.own_b; p += WIN_NT) {
            const float4 pa = s.pos[p];
            const float4 va = V[p];
            const int cnt = s.ncount[p];
            float acc = 0.f;
            if (!wide) {
                const unsigned short* L = s.nbr16 + p;
#pragma unroll 4
                for (int k = 0; k < cnt; ++k) {
                    const int q = L[k * stride];
                    const float4 pb = sp[q];
                    const float4 vb = sv[q];
                    const float m = q >= nf ? rho0 * pb.w : fm0;
                    const float xx = pa.x - pb.x, xy = pa.y - pb.y, xz = pa.z - pb.z;
                    const float f = grad_over_r(c.k, xx * xx + xy * xy + xz * xz);
                    const float dot = xx * (va.x - vb.x) + xy * (va.y - vb.y) + xz * (va.z - vb.z);
                    acc = fmaf(dot * f, m, acc);
                }
            } else {
                const int* L = s.nbr + p;
                for (int k = 0; k < cnt; ++k) {
                    const unsigned e = (unsigned)L[k * stride];
                    const bool bnd = (e & BND_FLAG) != 0u;
                    const unsigned j = e & BND_MASK;
                    const float4 pb = (bnd ? s.bpos : s.pos)[j];
                    const float4 vb = (bnd ? s.bvel : V)[j];
                    const float m = bnd ? rho0 * pb.w : fm0;
                    const float xx = pa.x - pb.x, xy = pa.y - pb.y, xz = pa.z - pb.z;
                    const float f = grad_over_r(c.k, xx * xx + xy * xy + xz * xz);
                    const float dot = xx * (va.x - vb.x) + xy * (va.y - vb.y) + xz * (va.z - vb.z);
                    acc = fmaf(dot * f, m, acc);
                }
            }
            const float rho = s.rho[p];
            if (DIV == 0) {
                float dadv = fmaf(acc, dt, rho);
                if (dadv < rho0) dadv = rho0;
                // kappa = (rho_adv - rho0) / pow(dt,2) * alpha  (DFSPH.cpp:641)
                const float kap = (float)((double)(dadv - rho0) / ((double)dt * (double)dt) * (double)s.alpha[p]);
                s.kr[p] = kap / rho;
                s.kappa[p] = kap;
                if (record) s.ksum[p] += kap;
                s.aux0[p] = dadv;
                mine += (double)dadv;
            } else {
                float dd = acc;
                if (dd < 0.f || (rho + dd * dt) < rho0) dd = 0.f;  // DFSPH.cpp:829-832
                const float kv = dd * s.alpha[p] / dt;              // DFSPH.cpp:835
                s.kr[p] = kv / rho;
                s.kappav[p] = kv;
                s.aux1[p] = dd;
                mine += (double)dd;
            }
        }
    }
    __shared__ double sh[WIN_NT / 32];
    const double bs = block_sum_double<WIN_NT>(mine, sh);
    double tot;
    if (finish_sum<WIN_NT>(s.partial, &s.st->ticket[DIV], bs, &tot)) {
        const int n = s.st->n_active;
        if (DIV == 0) s.st->err_density = (tot / (double)n - (double)c.rho0) / (double)c.rho0;
        else s.st->err_div = tot / (double)n;
    }
}

// B sweep: v -= dt sum_j m_j (k_i + k_j) gradW_ij, k = kappa/rho
// (DFSPH.cpp:647-693 / 840-883); then the loop decision.
template <int DIV, int DECIDE>
__global__ void __launch_bounds__(WIN_NT) k_df_vupdate(DevScene s, GridGeom g, SolverConst c, double goal_abs,
                                                       double goal_rel, int min_it, int max_it,
                                                       cudaGraphConditionalHandle h, int use_handle) {
    extern __shared__ float4 sm[];
    float4* sp = sm;
    float* sk = (float*)(sm + WIN_MAX);
    __shared__ WinHead H;
    win_setup(s, g, blockIdx.x, H);
    if (H.own_b > H.own_a) {
        const bool wide = H.wide;
        if (!wide) {
            win_stage4(H, s.pos, s.bpos, sp);
            for (int q = threadIdx.x; q < H.nf; q += WIN_NT) {
                const int cc = win_cell_of(H.fstart, q);
                sk[q] = s.kr[H.fglob[cc] + (q - H.fstart[cc])];
            }
        }
        __syncthreads();
        const float dt = *s.dt;
        const size_t stride = (size_t)c.stride;
        const int nf = H.nf;
        float4* V = DIV ? s.vel : s.vadv;
        for (int p = H.own_a + threadIdx.x; p < H.own_b; p += WIN_NT) {
            const float4 pa = s.pos[p];
            float4 va = V[p];
            const float ka = s.kr[p];
            const float fa = c.fm0 * ka, ba = c.rho0 * ka;
            const int cnt = s.ncount[p];
            float dx = 0.f, dy = 0.f, dz = 0.f;
            if (!wide) {
                const unsigned short* L = s.nbr16 + p;
#pragma unroll 4
                for (int k = 0; k < cnt; ++k) {
                    const int q = L[k * stride];
                    const float4 pb = sp[q];
                    const bool bnd = q >= nf;
                    const float w = bnd ? ba * pb.w : fmaf(c.fm0, sk[bnd ? 0 : q], fa);
                    const float xx = pa.x - pb.x, xy = pa.y - pb.y, xz = pa.z - pb.z;
                    const float f = grad_over_r(c.k, xx * xx + xy * xy + xz * xz) * w;
                    dx = fmaf(xx, f, dx);
                    dy = fmaf(xy, f, dy);
                    dz = fmaf(xz, f, dz);
                }
            } else {
                const int* L = s.nbr + p;
                for (int k = 0; k < cnt; ++k) {
                    const unsigned e = (unsigned)L[k * stride];
                    const bool bnd = (e & BND_FLAG) != 0u;
                    const unsigned j = e & BND_MASK;
                    const float4 pb = (bnd ? s.bpos : s.pos)[j];
                    const float w = bnd ? ba * pb.w : fmaf(c.fm0, s.kr[j], fa);
                    const float xx = pa.x - pb.x, xy = pa.y - pb.y, xz = pa.z - pb.z;
                    const float f = grad_over_r(c.k, xx * xx + xy * xy + xz * xz) * w;
                    dx = fmaf(xx, f, dx);
                    dy = fmaf(xy, f, dy);
                    dz = fmaf(xz, f, dz);
                }
            }
            va.x = fmaf(-dx, dt, va.x);
            va.y = fmaf(-dy, dt, va.y);
            va.z = fmaf(-dz, dt, va.z);
            V[p] = va;
        }
    }
    if (DECIDE && blockIdx.x == 0 && threadIdx.x == 0) {
        // convergence decision of the iteration that just finished
        int it, cont;
        if (DIV) {
            it = ++s.st->it_div;
            ++s.st->total_it_div;
            const double avg = s.st->err_div;  // mean Drho/Dt of this iteration
            const double dtd = (double)*s.dt;
            const bool crit = goal_abs > 0 ? (avg > goal_abs) : (avg * dtd / (double)c.rho0 > goal_rel);
            cont = (crit || it < min_it) && it <= max_it;
            if (!cont && crit) atomicOr(&s.st->status, 2u);
        } else {
            it = ++s.st->it_density;
            ++s.st->total_it_density;
            const double err = s.st->err_density;
            const bool crit = err > goal_rel;
            cont = (crit || it < min_it) && it < max_it;
            if (!cont && crit) atomicOr(&s.st->status, 1u);
            if (!(err == err)) { cont = 0; atomicOr(&s.st->status, 4u); }
        }
        s.st->cont = cont;
        if (use_handle) cudaGraphSetConditional(h, cont ? 1u : 0u);
    }
}

// non-pressure accelerations (gravity + viscosity) and v_adv
// (DF_forceExceptPressure, DFSPH.cpp:1246-1359, 1419-1475)
__global__ void __launch_bounds__(WIN_NT) k_df_forces(DevScene s, GridGeom g, SolverConst c, int warm) {
    extern __shared__ float4 sm[];
    float4* sp = sm;
    float4* sv = sm + WIN_MAX;
    float* sr = (float*)(sm + 2 * WIN_MAX);
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
                sr[q] = s.rho[H.fglob[cc] + (q - H.fstart[cc])];
            }
        }
        __syncthreads();
        const float dt = *s.dt;
        const float den0 = 0.01f * c.hs * c.hs;
        const float visc = 10.f * c.nu;
        const size_t stride = (size_t)c.stride;
        const int nf = H.nf;
        for (int p = H.own_a + threadIdx.x; p < H.own_b; p += WIN_NT) {
            const float4 pa = s.pos[p];
            const float4 va = s.vel[p];
            const float rhoa = s.rho[p];
            float ax = c.gravity[0], ay = c.gravity[1], az = c.gravity[2];
            const int cnt = s.ncount[p];
            for (int k = 0; k < cnt; ++k) {
                float4 pb, vb;
                float m;
                if (!wide) {
                    const int q = s.nbr16[k * stride + p];
                    pb = sp[q];
                    vb = sv[q];
                    // (frho0*volume)/fa.density, DFSPH.cpp:1353 ; fm0/fb.density, :1265
                    m = q >= nf ? c.rho0 * pb.w / rhoa : c.fm0 / sr[q];
                } else {
                    const unsigned e = (unsigned)s.nbr[k * stride + p];
                    const bool bnd = (e & BND_FLAG) != 0u;
                    const unsigned j = e & BND_MASK;
                    pb = (bnd ? s.bpos : s.pos)[j];
                    vb = (bnd ? s.bvel : s.vel)[j];
                    m = bnd ? c.rho0 * pb.w / rhoa : c.fm0 / s.rho[j];
                }
                const float xx = pa.x - pb.x, xy = pa.y - pb.y, xz = pa.z - pb.z;
                const float len2 = xx * xx + xy * xy + xz * xz;
                if (len2 == 0.f) { ++zero; continue; }
                const float pro = (va.x - vb.x) * xx + (va.y - vb.y) * xy + (va.z - vb.z) * xz;
                if (pro < 0.f) {
                    const float f = grad_over_r(c.k, len2);
                    const float t = f * pro / (len2 + den0) * m * visc;
                    ax += xx * t;
                    ay += xy * t;
                    az += xz * t;
                }
            }
            s.acc[p] = make_float4(ax, ay, az, 0.f);
            s.vadv[p] = make_float4(va.x + ax * dt, va.y + ay * dt, va.z + az * dt, 0.f);
            // learned warm start: the predicted stiffness is applied once
            // before the loop by a k_df_vupdate sweep with kr = kwarm/rho
            if (warm) s.kr[p] = s.kwarm[p] / rhoa;
        }
    }
    if (__syncthreads_or(zero)) {
        if (zero) atomicAdd(&s.st->zero_dis, zero);
    }
}

// FP64 max |v| and the CFL step dt = clamp(cfl * d / vmax, dt_min, dt_max)
__global__ void __launch_bounds__(NT) k_cfl(DevScene s, float cfl, float d, float dt_max, float dt_min) {
    const int n = s.st->n_active;
    const int p = blockIdx.x * NT + threadIdx.x;
    double m = 0.0;
    if (p < n) {
        float4 v = s.vel[p];
        double x = v.x, y = v.y, z = v.z;
        m = sqrt(x * x + y * y + z * z);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    __shared__ double sh[NT / 32];
    __shared__ bool last;
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = 0;
        for (int i = 0; i < NT / 32; ++i) b = fmax(b, sh[i]);
        s.partial[blockIdx.x] = b;
        __threadfence();
        last = atomicAdd(&s.st->ticket[2], 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        double vmax = 0;
        for (int i = 0; i < (int)gridDim.x; ++i) vmax = fmax(vmax, ((volatile double*)s.partial)[i]);
        double dt = vmax > 0 ? (double)cfl * (double)d / vmax : (double)dt_max;
        if (dt > dt_max) dt = dt_max;
        if (dt < dt_min) dt = dt_min;
        s.st->vmax = vmax;
        *s.dt = (float)dt;
        s.st->ticket[2] = 0u;
    }
}
}  // namespace

static inline int nblk(int n) { return (n > 0 ? n + NT - 1 : NT) / NT; }
static inline int nbricks(const GridGeom& g) { return g.nb[0] * g.nb[1] * g.nb[2]; }
static const size_t SMEM_A = (size_t)WIN_MAX * 32;
static const size_t SMEM_B = (size_t)WIN_MAX * 20;
static const size_t SMEM_F = (size_t)WIN_MAX * 36;
static const size_t SMEM_BUILD = (size_t)WIN_MAX * 16;

void dfsph_init_attributes() {
    cudaFuncSetAttribute(k_df_sweep_a<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_A);
    cudaFuncSetAttribute(k_df_sweep_a<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_A);
    cudaFuncSetAttribute(k_df_vupdate<0, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_B);
    cudaFuncSetAttribute(k_df_vupdate<0, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_B);
    cudaFuncSetAttribute(k_df_vupdate<1, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_B);
    cudaFuncSetAttribute(k_df_forces, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_F);
    cudaFuncSetAttribute(k_build_win<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BUILD);
    cudaFuncSetAttribute(k_build_win<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BUILD);
    cudaFuncSetAttribute(k_build_win<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BUILD);
}

void launch_step_begin(const DevScene& s, cudaStream_t st) { k_step_begin<<<1, 1, 0, st>>>(s); }
void launch_call_begin(const DevScene& s, cudaStream_t st) { k_call_begin<<<1, 1, 0, st>>>(s); }
void launch_df_loop_reset(const DevScene& s, int which, cudaStream_t st) { k_loop_reset<<<1, 1, 0, st>>>(s, which); }

void launch_build(const DevScene& s, const GridGeom& g, const SolverConst& c, int mode, int n_max, cudaStream_t st) {
    (void)n_max;
    const int nbk = nbricks(g);
    if (mode == 0) k_build_win<0><<<nbk, WIN_NT, SMEM_BUILD, st>>>(s, g, c);
    else if (mode == 1) k_build_win<1><<<nbk, WIN_NT, SMEM_BUILD, st>>>(s, g, c);
    else k_build_win<2><<<nbk, WIN_NT, SMEM_BUILD, st>>>(s, g, c);
}
void launch_expand_lists(const DevScene& s, const GridGeom& g, const SolverConst& c, cudaStream_t st) {
    k_expand_lists<<<nbricks(g), WIN_NT, 0, st>>>(s, g, c);
}
void launch_df_forces(const DevScene& s, const GridGeom& g, const SolverConst& c, int warm, cudaStream_t st) {
    k_df_forces<<<nbricks(g), WIN_NT, SMEM_F, st>>>(s, g, c, warm);
}
void launch_df_dens_a(const DevScene& s, const GridGeom& g, const SolverConst& c, int record, cudaStream_t st) {
    k_df_sweep_a<0><<<nbricks(g), WIN_NT, SMEM_A, st>>>(s, g, c, record);
}
void launch_df_dens_b(const DevScene& s, const GridGeom& g, const SolverConst& c, double goal, int min_it,
                      int max_it, unsigned long long cond_handle, int use_handle, cudaStream_t st) {
    k_df_vupdate<0, 1><<<nbricks(g), WIN_NT, SMEM_B, st>>>(s, g, c, 0.0, goal, min_it, max_it,
                                                           (cudaGraphConditionalHandle)cond_handle, use_handle);
}
void launch_df_warm_correction(const DevScene& s, const GridGeom& g, const SolverConst& c, cudaStream_t st) {
    k_df_vupdate<0, 0><<<nbricks(g), WIN_NT, SMEM_B, st>>>(s, g, c, 0.0, 0.0, 0, 0, (cudaGraphConditionalHandle)0, 0);
}
void launch_df_div_a(const DevScene& s, const GridGeom& g, const SolverConst& c, cudaStream_t st) {
    k_df_sweep_a<1><<<nbricks(g), WIN_NT, SMEM_A, st>>>(s, g, c, 0);
}
void launch_df_div_b(const DevScene& s, const GridGeom& g, const SolverConst& c, double goal_abs, double goal_rel,
                     int min_it, int max_it, unsigned long long cond_handle, int use_handle, cudaStream_t st) {
    k_df_vupdate<1, 1><<<nbricks(g), WIN_NT, SMEM_B, st>>>(s, g, c, goal_abs, goal_rel, min_it, max_it,
                                                           (cudaGraphConditionalHandle)cond_handle, use_handle);
}
void launch_cfl(const DevScene& s, int n_max, float cfl, float d, float dt_max, float dt_min, cudaStream_t st) {
    k_cfl<<<nblk(n_max), NT, 0, st>>>(s, cfl, d, dt_max, dt_min);
}
