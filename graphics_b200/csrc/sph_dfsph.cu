// sph_dfsph.cu -- DFSPH kernels (reference: DFSPH.cpp).
//
// Per step (DFSPH::sphStep, DFSPH.cpp:45-62):
//   k_df_forces       DF_forceExceptPressure + v_adv = v + a_adv dt
//                     (DFSPH.cpp:1419-1475, 1246-1359, 557-563)
//   density loop      k_df_dens_a: rho_adv, clamp, kappa = (rho_adv-rho0)/dt^2 alpha,
//                                  FP64 sum of rho_adv      (DFSPH.cpp:574-643)
//                     k_df_dens_b: v_adv -= dt sum m gradW (k_i/rho_i + k_j/rho_j),
//                                  convergence decision     (DFSPH.cpp:647-698)
//   integrate + neighbour search + rho/alpha (sph_grid.cu)
//   divergence loop   k_df_div_a / k_df_div_b             (DFSPH.cpp:769-900)
//
// The loop kernels read neighbour indices from the ELL lists and recompute
// the kernel gradient from positions (-W'(r)/r with one rsqrt; the reference
// stores the distance per pair, recomputing saves 4 bytes per pair of HBM
// traffic in every sweep).  Neighbour state is gathered as one packed record
// per neighbour: {position, loop velocity} (32 B) in the A sweeps and
// (x, y, z, kappa/rho) (16 B) in the B sweeps.  Per-particle arithmetic is
// FP32; the convergence sums are FP64 block partials reduced in a fixed order
// by the last block, so results are run-to-run deterministic.
//
// Loop control: k_*_b decides whether another iteration runs.  Inside a CUDA
// graph the loop is a conditional WHILE node and the decision is written with
// cudaGraphSetConditional; in host-driven mode it is written to st->cont.
#include "sph_kernels.cuh"

namespace {
constexpr int NT = 128;

// per-step counters (the last step's values are reported)
__global__ void k_step_begin(DevScene s) {
    DevStats* st = s.st;
    st->max_nbrs = 0;
    st->nbr_total = 0ull;
    st->it_density = 0;
    st->it_div = 0;
    st->err_density = 0;
    st->err_div = 0;
}

// per-call counters: status bits are OR-ed and removals / dropped pairs
// summed over all steps of one API call
__global__ void k_call_begin(DevScene s) {
    DevStats* st = s.st;
    st->removed = 0;
    st->overflow = 0;
    st->zero_dis = 0;
    st->status = 0u;
    st->total_it_density = 0;
    st->total_it_div = 0;
}

__global__ void k_loop_reset(DevScene s, int which) {
    if (which == 0) s.st->it_density = 0;
    else s.st->it_div = 0;
    s.st->cont = 1;
}

// non-pressure accelerations (gravity + viscosity) and v_adv.  The list is
// read four entries at a time (one 16-byte load, the next group's issued
// before the current group's record gathers) and each neighbour costs one
// 32-byte record; the per-pair divisions become reciprocals (1/rho_i once
// per particle, 1/rho_j and 1/(r^2 + 0.01 h^2) per pair).
template <int BS>
__global__ void __launch_bounds__(BS) k_df_forces(DevScene s, SolverConst c, int warm) {
    const int n = s.st->n_active;
    const int p = blockIdx.x * BS + threadIdx.x;
    int zero = 0;
    if (p < n) {
        const float4 pa = s.pos[p];
        const float dt = dt_of(s, pa);
        const float4 va = s.vel[p];
        const float rhoa = s.rho[p];
        const float fm0 = c.fm0;
        const float bm = c.rho0 * __frcp_rn(rhoa);  // (frho0*volume)/fa.density = bm * volume, DFSPH.cpp:1353
        const float den0 = 0.01f * c.hs * c.hs;
        const float visc = 10.f * c.nu;
        float ax = c.gravity[0], ay = c.gravity[1], az = c.gravity[2];
        const int cnt = s.ncount[p];
        const int ng = (cnt + 3) >> 2;
        const size_t stride = (size_t)c.stride;
        const unsigned long long polL = l2_policy(c.l2pol & 3);  // lists stream through L2
        int4 nxt = ng ? ell_group_pol(s.nbr, stride, p, 0, polL) : make_int4(0, 0, 0, 0);
        for (int gi = 0; gi < ng; ++gi) {
            const int4 cur = nxt;
            if (gi + 1 < ng) nxt = ell_group_pol(s.nbr, stride, p, gi + 1, polL);
            const unsigned e[4] = {(unsigned)cur.x, (unsigned)cur.y, (unsigned)cur.z, (unsigned)cur.w};
            // one 32-byte record per neighbour: {(x, y, z, rho), v} or, for a
            // boundary particle, {(x, y, z, volume), singleVelocity + velocity}
            // (DFSPH.cpp:1349); entries past the count read the particle's own
            // record and are masked out
            float4 pb[4], vb[4];
            bool ok[4], bnd[4];
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                ok[t] = gi * 4 + t < cnt;
                const unsigned u = ok[t] ? e[t] : (unsigned)p;
                bnd[t] = (u & BND_FLAG) != 0u;
                ld_record32((bnd[t] ? s.bpf : s.prv) + 2 * (size_t)(u & BND_MASK), pb[t], vb[t]);
            }
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                const float m = bnd[t] ? bm * pb[t].w              // DFSPH.cpp:1353
                                       : fm0 * __frcp_rn(pb[t].w);  // fm0/fb.density, DFSPH.cpp:1265
                const float xx = pa.x - pb[t].x, xy = pa.y - pb[t].y, xz = pa.z - pb[t].z;
                const float len2 = xx * xx + xy * xy + xz * xz;
                const bool z0 = len2 == 0.f;  // zero distance: counted, no force (m_EC.zeroDis)
                zero += ok[t] && z0;
                const float pro = (va.x - vb[t].x) * xx + (va.y - vb[t].y) * xy + (va.z - vb[t].z) * xz;
                if (ok[t] && !z0 && pro < 0.f) {
                    const float f = grad_over_r(c.k, len2);
                    const float tt = f * pro * __frcp_rn(len2 + den0) * m * visc;
                    ax = fmaf(xx, tt, ax);
                    ay = fmaf(xy, tt, ay);
                    az = fmaf(xz, tt, az);
                }
            }
        }
        s.acc[p] = make_float4(ax, ay, az, 0.f);
        // w: the previous step's predicted stiffness (warm-start history),
        // which the feature sweep then reads with the neighbour's record
        s.pv[2 * p + 1] = make_float4(va.x + ax * dt, va.y + ay * dt, va.z + az * dt, s.hist[p].x);
        if (warm) {
            // learned warm start: the predicted stiffness is applied once before
            // the Jacobi loop as a pressure-velocity correction of the form of
            // DFSPH.cpp:674 (launch_df_warm_correction with kappa/rho =
            // kwarm/rho); the unmodified loop then runs to the same tolerance.
            s.pk[p].w = s.kwarm[p] / rhoa;
        }
    }
    if (__syncthreads_or(zero)) {
        if (zero) atomicAdd(&s.st->zero_dis, zero);
    }
}

// Neighbour-sum of m_j gradW_ij . (v_i - v_j) over the stored list: the
// common sweep of the density loop (DFSPH.cpp:589-617) and of the divergence
// loop (DFSPH.cpp:795-825).  Indices come four at a time (one 16-byte load),
// the next group's load is issued before the current group's four record
// gathers, and each neighbour costs one 32-byte record {position, loop
// velocity} (pv / bpv) fetched by one 256-bit load.  Entries past the count read the particle's own
// record and are masked out.
__device__ __forceinline__ float div_sweep(const DevScene& s, const SolverConst& c, int p, float4 pa, float4 va) {
    const int cnt = s.ncount[p];
    const int ng = (cnt + 3) >> 2;
    const size_t stride = (size_t)c.stride;
    const unsigned long long polL = l2_policy(c.l2pol & 3), polR = l2_policy((c.l2pol >> 2) & 3);
    float acc = 0.f;
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
            ld_record32_pol(rec, pb[t], vb[t], polR);
        }
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            const float nacc = div_term(c, pa, va, pb[t], vb[t], bnd[t], acc);
            acc = ok[t] ? nacc : acc;
        }
    }
    return acc;
}

// density loop, part A: rho_adv, kappa, FP64 sum of rho_adv
template <int BS>
__global__ void __launch_bounds__(BS) k_df_dens_a(DevScene s, SolverConst c, int record) {
    const int n = s.st->n_active;
    const int p = blockIdx.x * BS + threadIdx.x;
    double mine = 0.0;
    if (p < n && scene_active(s, s.pv[2 * p])) {
        const float4 pa = s.pv[2 * p];
        const float dt = dt_of(s, pa);
        const float4 va = s.pv[2 * p + 1];
        const float rho0 = c.rho0;
        const float acc = div_sweep(s, c, p, pa, va);
        const float rho = s.rho[p];
        float dadv = fmaf(acc, dt, rho);
        if (dadv < rho0) dadv = rho0;
        // kappa = (rho_adv - rho0) / pow(dt,2) * alpha  (DFSPH.cpp:641)
        const float kap = (float)((double)(dadv - rho0) / ((double)dt * (double)dt) * (double)s.alpha[p]);
        s.pk[p].w = kap / rho;
        s.kappa[p] = kap;
        if (record) s.ksum[p] += kap;
        s.aux0[p] = dadv;
        mine = (double)dadv;
    }
    if (s.nscenes > 1) return;  // a batch reduces per scene (k_batch_decide)
    __shared__ double sh[BS / 32];
    double bs = block_sum_double<BS>(mine, sh);
    double tot;
    if (finish_sum<BS>(s.partial, &s.st->ticket[0], bs, &tot)) {
        // no particle left (all removed): nothing to solve
        s.st->err_density = n > 0 ? (tot / (double)n - (double)c.rho0) / (double)c.rho0 : 0.0;
    }
}

// density/divergence loop, part B: v_adv update with k = kappa/rho
// (DFSPH.cpp:647-693 / 840-883); then the loop decision.  Each neighbour
// costs one 16-byte record (x, y, z, k) (pk; boundary: (x, y, z, volume)).
template <int BS, int DIV, int DECIDE>
__global__ void __launch_bounds__(BS) k_df_vupdate(DevScene s, SolverConst c, double goal_abs, double goal_rel,
                                                   int min_it, int max_it, cudaGraphConditionalHandle h,
                                                   int use_handle) {
    const int n = s.st->n_active;
    const int p = blockIdx.x * BS + threadIdx.x;
    if (p < n && scene_active(s, s.pv[2 * p])) {
        const float dt = dt_of(s, s.pv[2 * p]);
        const float4 pa = s.pk[p];
        float4 va = s.pv[2 * p + 1];
        const float ka = pa.w;
        const float fa = c.fm0 * ka, ba = c.rho0 * ka;
        float dx = 0.f, dy = 0.f, dz = 0.f;
        const int cnt = s.ncount[p];
        const int ng = (cnt + 3) >> 2;
        const size_t stride = (size_t)c.stride;
        const unsigned long long polL = l2_policy(c.l2pol & 3), polR = l2_policy((c.l2pol >> 2) & 3);
        int4 nxt = ng ? ell_group_pol(s.nbr, stride, p, 0, polL) : make_int4(0, 0, 0, 0);
        for (int gi = 0; gi < ng; ++gi) {
            const int4 cur = nxt;
            if (gi + 1 < ng) nxt = ell_group_pol(s.nbr, stride, p, gi + 1, polL);
            const unsigned e[4] = {(unsigned)cur.x, (unsigned)cur.y, (unsigned)cur.z, (unsigned)cur.w};
            float4 pb[4];
            bool ok[4], bnd[4];
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                ok[t] = gi * 4 + t < cnt;
                const unsigned u = ok[t] ? e[t] : (unsigned)p;
                bnd[t] = (u & BND_FLAG) != 0u;
                const unsigned j = u & BND_MASK;
                pb[t] = ld_f4_pol(bnd[t] ? s.bpv + 2 * (size_t)j : s.pk + j, polR);
            }
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                const float w = bnd[t] ? ba * pb[t].w : fmaf(c.fm0, pb[t].w, fa);
                const float xx = pa.x - pb[t].x, xy = pa.y - pb[t].y, xz = pa.z - pb[t].z;
                const float f = ok[t] ? grad_over_r(c.k, xx * xx + xy * xy + xz * xz) * w : 0.f;
                dx = fmaf(xx, f, dx);
                dy = fmaf(xy, f, dy);
                dz = fmaf(xz, f, dz);
            }
        }
        va.x = fmaf(-dx, dt, va.x);
        va.y = fmaf(-dy, dt, va.y);
        va.z = fmaf(-dz, dt, va.z);
        s.pv[2 * p + 1] = va;
        if (DIV) {
            s.vel[p] = va;  // velocity = vel_adv (DFSPH.cpp:909)
            s.prv[2 * p + 1] = va;
        }
    }
    if (DECIDE && s.nscenes <= 1 && blockIdx.x == 0 && threadIdx.x == 0) {
        // convergence decision of the iteration that just finished
        int it;
        int cont;
        if (DIV) {
            it = ++s.st->it_div;
            ++s.st->total_it_div;
            const double avg = s.st->err_div;  // mean Drho/Dt of this iteration
            const double dtd = (double)*s.dt;
            bool crit = goal_abs > 0 ? (avg > goal_abs) : (avg * dtd / (double)c.rho0 > goal_rel);
            cont = (crit || it < min_it) && it <= max_it;
            if (!cont && crit) atomicOr(&s.st->status, 2u);
        } else {
            it = ++s.st->it_density;
            ++s.st->total_it_density;
            const double err = s.st->err_density;
            bool crit = err > goal_rel;
            cont = (crit || it < min_it) && it < max_it;
            if (!cont && crit) atomicOr(&s.st->status, 1u);
            if (!(err == err)) { cont = 0; atomicOr(&s.st->status, 4u); }
        }
        s.st->cont = cont;
        if (use_handle) cudaGraphSetConditional(h, cont ? 1u : 0u);
    }
}

// divergence loop, part A: Drho/Dt, clamp, kappa_v, FP64 sum
template <int BS>
__global__ void __launch_bounds__(BS) k_df_div_a(DevScene s, SolverConst c) {
    const int n = s.st->n_active;
    const int p = blockIdx.x * BS + threadIdx.x;
    double mine = 0.0;
    if (p < n && scene_active(s, s.pv[2 * p])) {
        const float4 pa = s.pv[2 * p];
        const float dt = dt_of(s, pa);
        const float4 va = s.pv[2 * p + 1];
        float dd = div_sweep(s, c, p, pa, va);
        const float rho = s.rho[p];
        if (dd < 0.f || (rho + dd * dt) < c.rho0) dd = 0.f;  // DFSPH.cpp:829-832
        const float kv = dd * s.alpha[p] / dt;              // DFSPH.cpp:835
        s.pk[p].w = kv / rho;
        s.kappav[p] = kv;
        s.aux1[p] = dd;
        mine = (double)dd;
    }
    if (s.nscenes > 1) return;  // a batch reduces per scene (k_batch_decide)
    __shared__ double sh[BS / 32];
    double bs = block_sum_double<BS>(mine, sh);
    double tot;
    if (finish_sum<BS>(s.partial, &s.st->ticket[1], bs, &tot)) s.st->err_div = n > 0 ? tot / (double)n : 0.0;
}

// FP64 max |v| and the CFL step dt = clamp(cfl * d / vmax, dt_min, dt_max).
// Each thread takes CFL_ITEMS velocities and the maximum is taken over the
// squared speeds, with one square root at the end: sqrt is correctly rounded
// and monotone, so this is the maximum of the per-particle speeds exactly.
constexpr int CFL_ITEMS = 8;
__global__ void __launch_bounds__(NT) k_cfl(DevScene s, float cfl, float d, float dt_max, float dt_min) {
    const int n = s.st->n_active;
    double m = 0.0;
#pragma unroll
    for (int k = 0; k < CFL_ITEMS; ++k) {
        const int p = (blockIdx.x * CFL_ITEMS + k) * NT + threadIdx.x;
        if (p < n) {
            const float4 v = s.vel[p];
            const double x = v.x, y = v.y, z = v.z;
            m = fmax(m, x * x + y * y + z * z);
        }
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
    if (!last) return;
    __threadfence();
    // the last block reduces the block maxima with all its threads
    double vm = 0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += NT) vm = fmax(vm, ((volatile double*)s.partial)[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) vm = fmax(vm, __shfl_down_sync(0xffffffffu, vm, o));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = vm;
    __syncthreads();
    if (threadIdx.x == 0) {
        double vmax = 0;
        for (int i = 0; i < NT / 32; ++i) vmax = fmax(vmax, sh[i]);
        vmax = sqrt(vmax);
        double dt = vmax > 0 ? (double)cfl * (double)d / vmax : (double)dt_max;
        if (dt > dt_max) dt = dt_max;
        if (dt < dt_min) dt = dt_min;
        s.st->vmax = vmax;
        *s.dt = (float)dt;
        s.st->ticket[2] = 0u;
    }
}
}  // namespace

static inline int nblk(int n, int bs = NT) { return (n > 0 ? n + bs - 1 : bs) / bs; }

// block size chosen at run time (the autotuner picks it per kernel class)
#define DISPATCH_BS(bs, CALL)                       \
    switch (bs) {                                   \
        case 64: { constexpr int B = 64; CALL; break; }   \
        case 256: { constexpr int B = 256; CALL; break; } \
        default: { constexpr int B = 128; CALL; break; }  \
    }

void launch_step_begin(const DevScene& s, cudaStream_t st) { k_step_begin<<<1, 1, 0, st>>>(s); }
void launch_call_begin(const DevScene& s, cudaStream_t st) { k_call_begin<<<1, 1, 0, st>>>(s); }
void launch_df_loop_reset(const DevScene& s, int which, cudaStream_t st) { k_loop_reset<<<1, 1, 0, st>>>(s, which); }

void launch_df_forces(const DevScene& s, const SolverConst& c, int n_max, int warm, cudaStream_t st, int bs) {
    DISPATCH_BS(bs, (k_df_forces<B><<<nblk(n_max, B), B, 0, st>>>(s, c, warm)));
}
void launch_df_dens_a(const DevScene& s, const SolverConst& c, int n_max, int record, cudaStream_t st, int bs) {
    DISPATCH_BS(bs, (k_df_dens_a<B><<<nblk(n_max, B), B, 0, st>>>(s, c, record)));
}
void launch_df_dens_b(const DevScene& s, const SolverConst& c, int n_max, double goal, int min_it, int max_it,
                      unsigned long long cond_handle, int use_handle, cudaStream_t st, int bs) {
    DISPATCH_BS(bs, (k_df_vupdate<B, 0, 1><<<nblk(n_max, B), B, 0, st>>>(
                        s, c, 0.0, goal, min_it, max_it, (cudaGraphConditionalHandle)cond_handle, use_handle)));
}
void launch_df_warm_correction(const DevScene& s, const SolverConst& c, int n_max, cudaStream_t st, int bs) {
    DISPATCH_BS(bs, (k_df_vupdate<B, 0, 0><<<nblk(n_max, B), B, 0, st>>>(s, c, 0.0, 0.0, 0, 0,
                                                                         (cudaGraphConditionalHandle)0, 0)));
}
void launch_df_div_a(const DevScene& s, const SolverConst& c, int n_max, cudaStream_t st, int bs) {
    DISPATCH_BS(bs, (k_df_div_a<B><<<nblk(n_max, B), B, 0, st>>>(s, c)));
}
void launch_df_div_b(const DevScene& s, const SolverConst& c, int n_max, double goal_abs, double goal_rel,
                     int min_it, int max_it, unsigned long long cond_handle, int use_handle, cudaStream_t st, int bs) {
    DISPATCH_BS(bs, (k_df_vupdate<B, 1, 1><<<nblk(n_max, B), B, 0, st>>>(
                        s, c, goal_abs, goal_rel, min_it, max_it, (cudaGraphConditionalHandle)cond_handle, use_handle)));
}
// every block-size instantiation of the per-neighbour sweep kernels
template <int B, class F>
static void each_sweep_kernel_bs(F f) {
    f((const void*)k_df_forces<B>);
    f((const void*)k_df_dens_a<B>);
    f((const void*)k_df_div_a<B>);
    f((const void*)k_df_vupdate<B, 0, 1>);
    f((const void*)k_df_vupdate<B, 0, 0>);
    f((const void*)k_df_vupdate<B, 1, 1>);
}
template <class F>
static void each_sweep_kernel(F f) {
    each_sweep_kernel_bs<64>(f);
    each_sweep_kernel_bs<128>(f);
    each_sweep_kernel_bs<256>(f);
}
// preferred shared-memory carveout (percent of the unified L1/shared
// storage; -1 = the driver's choice) of the per-neighbour sweep kernels
void set_sweep_carveout(int pct) {
    each_sweep_kernel([&](const void* k) { cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, pct); });
}
// loads every instantiation now (the runtime loads a kernel at its first
// launch, which would land inside the autotuner's first timed candidate)
void preload_sweep_kernels() {
    each_sweep_kernel([](const void* k) {
        cudaFuncAttributes a;
        cudaFuncGetAttributes(&a, k);
    });
}
void launch_cfl(const DevScene& s, int n_max, float cfl, float d, float dt_max, float dt_min, cudaStream_t st) {
    k_cfl<<<nblk(n_max, NT * CFL_ITEMS), NT, 0, st>>>(s, cfl, d, dt_max, dt_min);
}
