// sph_engine.cu -- host engine behind the C ABI in include/sphgpu.h.
//
// One sphgpu_scene owns the device buffers of one SPH scene, one CUDA stream
// and the step graphs.  A DFSPH step is one CUDA graph: its two Jacobi loops
// are conditional WHILE nodes whose bodies (two kernels each) decide on the
// device whether another iteration runs, so a step needs no host round trip.
// Profiling mode runs the same kernels as individual launches bracketed by
// CUDA events (host-driven loops) to time each kernel class.
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/sphgpu.h"
#include "sph_kernels.cuh"
#include "sph_mlp.cuh"
#include "sph_sync.cuh"

// warm-start kernels (sph_mlp.cu)
void mlp_init_attributes();
int mlp_train_blocks(int rows);
void ws_init_attributes();
void launch_ws_features(const DevScene& s, const SolverConst& c, const MlpDev& m, int infer, float dt_max,
                        float alpha_ref, float* Xout, __nv_bfloat16* xn, int n_max, cudaStream_t st);
void launch_ws_infer(const DevScene& s, const SolverConst& c, const MlpDev& m, const __nv_bfloat16* xn, int n_max,
                     int sm_count, cudaStream_t st);
void launch_ws_post(const DevScene& s, const SolverConst& c, float* yout, int n_max, cudaStream_t st);
void launch_ws_features_infer(const DevScene& s, const SolverConst& c, const MlpDev& m, float dt_max, float alpha_ref,
                              __nv_bfloat16* xn, int n_max, int sm_count, cudaStream_t st);
void launch_ws_append(const float* X, const float* y, int n_max, const int* n_act, int every, int* offset, float* dsX,
                      float* dsy, int* ds_count, int ds_cap, cudaStream_t st);

namespace {

struct EvPair {
    const char* name;
    cudaEvent_t a, b;
};

struct Prof {
    bool on = false;
    std::vector<cudaEvent_t> pool;
    size_t used = 0;
    std::vector<EvPair> pending;
    std::map<std::string, std::pair<double, int>> acc;
};

}  // namespace

// Warm-start network + its training set (one per sphgpu_mlp handle).
struct sphgpu_mlp {
    int device = 0;
    cudaStream_t stream = nullptr;
    MlpDev m{};
    float* dsX = nullptr;
    float* dsy = nullptr;
    int* ds_count = nullptr;
    int ds_cap = 0;
    int adam_t = 0;
    int gpart_blocks = 0;  // capacity of m.gpart in training tiles
    std::string err;
};

struct sphgpu_scene {
    SphParams P;
    int device = 0;
    cudaStream_t stream = nullptr, stream2 = nullptr;
    // host-buffer step: the integrated positions leave on stream3 while the
    // neighbour search and the divergence loop run (sphgpu_step_host)
    cudaStream_t stream3 = nullptr;
    cudaEvent_t ev_out[2] = {nullptr, nullptr};
    float* out_xyz = nullptr;
    int out_n = 0;
    bool out_xyz_done = false;
    // host-buffer step, speculative: the step's first part runs on the
    // device state while stream4 copies the host inputs in and checks them
    // against that state (in_xyz / in_vel, d_diff -> h_diff); the second part
    // starts only if they were equal
    cudaStream_t stream4 = nullptr;
    cudaEvent_t ev_in[2] = {nullptr, nullptr};
    float* in_xyz = nullptr;
    float* in_vel = nullptr;
    int* d_diff = nullptr;
    int* h_diff = nullptr;
    bool spec_pending = false, spec_failed = false;
    int spec = 1;  // debug knob "speculative_host_step"
    int cap = 0, stride = 0, ncap = 48;
    GridGeom g{};
    SolverConst c{};
    DevScene d{};
    std::vector<float> rho0_ph, alpha_ph;
    std::vector<int> phase_n;
    int n_total = 0;  // particles known to the host (before removals)
    bool ns_valid = false, in_staging = true;
    // Sort bookkeeping for the getters.  A DFSPH step writes the
    // non-pressure acceleration (and the vorticity vectors) and the density
    // loop's per-particle results before its neighbour search re-sorts the
    // particles, so after the step those arrays are in the previous sorted
    // order -- the order the integration copied into the staging arrays
    // (gid_s).  sorts counts the sorts enqueued; ep_acc / ep_loop / ep_vort
    // hold the count at which each group was last written (the vorticity
    // vectors of options 1 and 2 come before the sort, those of option 3
    // after the divergence loop).
    long sorts = 0, ep_acc = -2, ep_loop = -2, ep_vort = -2;
    int frame = 0;
    double time = 0;
    void* cub_tmp = nullptr;
    size_t cub_bytes = 0;
    DevStats* h_stats = nullptr;
    int* h_cont = nullptr;
    // graphs: key -> exec
    std::map<int, cudaGraphExec_t> graphs;
    bool use_graphs = true;
    Prof prof;
    std::string err;
    std::vector<int> bgid_h;
    std::vector<int> bsolid_h;
    int nb = 0;
    int iv_multi_solid = 0;  // walls hold more than one solid id
    int record_ksum = 0;
    // SolverConst::l2pol: the neighbour lists stream through L2 with evict-first
    // priority, so the records the sweeps gather stay resident (measured at
    // 1 M: density sweeps A/B 135/74 -> 129/72 us; records evict-last: no gain)
    int l2pol = 1;
    int fuse_div = 1;  // DFSPH: the list build performs the divergence loop's first sweep A
    int fuse_ws = 1;   // warm start: features and inference in one kernel
    // set while a step that is not its call's last is enqueued: the step's
    // statistics stay on the device (the call's last step copies them)
    bool skip_stats = false;
    // WCSPH threads per particle: 0 = by size (4 up to 262,144 particles of
    // capacity, 1 above), else 1 or 4 (debug knob "wc_lanes")
    int wc_lanes = 0;
    // learned warm start: 0 off, 1 apply the network, 2 record training data
    sphgpu_mlp* mlp = nullptr;
    int ws_mode = 0;
    int ws_every = 10;
    int ws_offset = 0;
    float* recX = nullptr;  // [cap][16] features of the step being recorded
    float* recY = nullptr;  // [cap] labels
    __nv_bfloat16* xn = nullptr;  // [cap][16] normalised features for the network (mode 1)
    int sm_count = 148;
    float alpha_ref = 1.f;
    long long total_removed = 0;  // gid stays a permutation of [0, n) while 0
    int last_solver = -1;         // solver of the last step (carried-state validity)
    // block sizes per kernel class (sphgpu_autotune picks them by measurement)
    struct Tune {
        int forces = 128, sweep_a = 128, sweep_b = 128, build = 128;
    } tune;
    // batch of independent scenes (nscenes > 1): one grid per scene in one key space
    int nscenes = 1;
    std::vector<GridGeom> sgeom;  // per scene (key ranges, boxes)
    int last_scene = 0;           // scenes receive their fluid in order
    GridGeom* d_geom = nullptr;
    void* d_batch = nullptr;      // one allocation holding the BatchDev arrays
    // dynamic rigid solids (DFSPH): device data, the dense list of dynamic
    // solids with their reference ranges, pinned exchange buffers
    RigidDev R{};
    std::vector<int> dyn_ids, dyn_r0, dyn_r1;
    float* h_rstate = nullptr;    // [cap * 25] states (SphRigidState layout)
    double* h_rout = nullptr;     // [cap * 6 + 1] joined force, torque; dt
    int rigid_cap = 0;            // capacity of the per-solid arrays
    int vort_last = 0;            // vorticity option of the last DFSPH step (its carried state in cA)
    sphgpu_rigid_fn rigid_fn = nullptr;
    void* rigid_user = nullptr;
    int rigid_fail = 0;
};

namespace {

#define CK(x)                                                                                 \
    do {                                                                                      \
        cudaError_t e_ = (x);                                                                 \
        if (e_ != cudaSuccess) {                                                              \
            h->err = std::string(#x) + ": " + cudaGetErrorString(e_);                         \
            return SPHGPU_ECUDA;                                                              \
        }                                                                                     \
    } while (0)

#define CKV(x)                                                                                \
    do {                                                                                      \
        cudaError_t e_ = (x);                                                                 \
        if (e_ != cudaSuccess && h->err.empty()) h->err = std::string(#x) + ": " + cudaGetErrorString(e_); \
    } while (0)

inline int roundup(int a, int b) { return (a + b - 1) / b * b; }

inline float int_bits_as_float(int v) {
    float f;
    memcpy(&f, &v, sizeof f);
    return f;
}

// ---- profiling launch wrapper ----
template <class F>
void launch(sphgpu_scene* h, const char* name, cudaStream_t st, F&& f) {
    if (h->prof.on) {
        if (h->prof.used + 2 > h->prof.pool.size()) {
            for (int i = 0; i < 64; ++i) {
                cudaEvent_t e;
                cudaEventCreate(&e);
                h->prof.pool.push_back(e);
            }
        }
        cudaEvent_t a = h->prof.pool[h->prof.used++], b = h->prof.pool[h->prof.used++];
        cudaEventRecord(a, st);
        f();
        cudaEventRecord(b, st);
        h->prof.pending.push_back({name, a, b});
    } else {
        f();
    }
}

void prof_collect(sphgpu_scene* h) {
    if (!h->prof.on) return;
    cudaStreamSynchronize(h->stream);
    for (auto& p : h->prof.pending) {
        float ms = 0;
        cudaEventElapsedTime(&ms, p.a, p.b);
        auto& e = h->prof.acc[p.name];
        e.first += ms;
        e.second += 1;
    }
    h->prof.pending.clear();
    h->prof.used = 0;
}

// Grid geometry exactly as SpaceGridStruct::initialize computes it in float
// (SphBase.cpp:963-988), plus the brick enumeration of the cell keys.
GridGeom make_grid(const SphParams& P) {
    GridGeom g{};
    float hr = P.smoothRadius_h;
    for (int i = 0; i < 3; ++i) g.min[i] = P.spaceMin[i] - hr * 2;
    g.divisor = 1 / hr;
    for (int i = 0; i < 3; ++i) {
        float t = (P.spaceMax[i] - P.spaceMin[i]) + hr * 2;
        g.num[i] = (int)(t * g.divisor) + 2;
        g.nb[i] = (g.num[i] + 3) / 4;
    }
    g.nkeys = g.nb[0] * g.nb[1] * g.nb[2] * 64 + 1;
    g.key0 = 0;
    g.key1 = g.nkeys - 1;
    for (int i = 0; i < 3; ++i) { g.smin[i] = P.spaceMin[i]; g.smax[i] = P.spaceMax[i]; }
    return g;
}

void fill_solver_const(sphgpu_scene* h) {
    const SphParams& P = h->P;
    SolverConst& c = h->c;
    // ker_update_numbers, SphBase.h:808-829 (float arithmetic)
    float kh = P.smoothRadius_h / 2;
    c.k.h = kh;
    c.k.inv_h = 1.f / kh;
    c.k.theta = 1 / (float)M_PI / (kh * kh * kh);
    c.k.thetah = 1 / (float)M_PI / (kh * kh * kh) / kh;
    c.k.g_in = -c.k.thetah / kh;
    c.k.g_out = -0.75f * c.k.thetah;
    c.hs = P.smoothRadius_h;
    float dd = P.particle_d + P.particle_d;
    c.h2cut = (float)std::pow((double)dd, 2);
    c.dpart = P.particle_d;
    float v0 = (float)std::pow((double)P.spacing_r, 3);
    c.nphase = (int)h->rho0_ph.size();
    for (int i = 0; i < 4; ++i) {
        float r0 = i < c.nphase ? h->rho0_ph[i] : 1000.f;
        c.rho0_ph[i] = r0;
        c.fm_ph[i] = r0 * v0;
        c.alpha_ph[i] = i < c.nphase ? h->alpha_ph[i] : 0.f;
    }
    c.rho0 = c.rho0_ph[0];
    c.fm0 = c.fm_ph[0];
    for (int i = 0; i < 3; ++i) c.gravity[i] = P.gravity[i];
    c.nu = P.nu;
    c.cs = P.soundSpeed_cs;
    c.visc_alpha = c.alpha_ph[0];
    c.bvisc = P.boundary_visc;
    c.wc_gamma = P.wc_gamma;
    c.wc_B = c.rho0 * P.soundSpeed_cs * P.soundSpeed_cs / P.wc_gamma;
    c.th_h = P.th_h;
    c.th_r = P.th_r;
    c.th_bt = P.th_bt;
    c.cap = h->ncap;
    c.stride = h->stride;
    c.l2pol = h->l2pol;
    c.lanes = h->wc_lanes ? h->wc_lanes : (h->cap <= (1 << 18) ? 4 : 1);
    c.ws_scale = P.ws_scale;
    // IISph: per-pair h = (d + d)/2 = d (SphBase.h:855-915 with one diameter)
    {
        const float hd = (P.particle_d + P.particle_d) / 2;
        c.kd.h = hd;
        c.kd.inv_h = 1.f / hd;
        c.kd.theta = 1 / (float)M_PI / (hd * hd * hd);
        c.kd.thetah = 1 / (float)M_PI / (hd * hd * hd) / hd;
        c.kd.g_in = -c.kd.thetah / hd;
        c.kd.g_out = -0.75f * c.kd.thetah;
        c.iv_V = (float)std::pow((double)P.particle_d, 3);  // std::pow(d, vec_t::dim), IISph.cpp:109
        for (int i = 0; i < 4; ++i) c.iv_m[i] = c.rho0_ph[i] * c.iv_V;  // rho0 * beta * V, beta = 1
        c.iv_kv = P.iv_kvisc;
        c.iv_kvb = P.iv_kvisc_b;
        c.iv_multi_solid = h->iv_multi_solid;
    }
    // alpha of an interior particle of the ideal cubic lattice (spacing d),
    // the normalisation of the warm-start feature log(alpha / alpha_ref)
    {
        double hk = kh, th = c.k.theta, thh = c.k.thetah, d = P.particle_d, rho = 0, s2 = 0;
        auto W = [&](double r) { double q = r / hk, t = 2 - q; return q <= 1 ? th * (1 - 1.5 * q * q + 0.75 * q * q * q) : th * 0.25 * t * t * t; };
        auto Wg = [&](double r) { double q = r / hk, t = 2 - q; return q <= 1 ? thh * (3 * q - 2.25 * q * q) : thh * 0.75 * t * t; };
        rho = W(0);
        for (int i = -2; i <= 2; ++i)
            for (int j = -2; j <= 2; ++j)
                for (int k = -2; k <= 2; ++k) {
                    double r = d * std::sqrt((double)(i * i + j * j + k * k));
                    if (r <= 0 || r >= 2 * d) continue;
                    rho += W(r);
                    s2 += (c.fm0 * Wg(r)) * (c.fm0 * Wg(r));
                }
        rho *= c.fm0;
        h->alpha_ref = s2 > 0 ? (float)(rho / s2) : 1.f;
    }
}

template <class T>
int dalloc(sphgpu_scene* h, T** p, size_t n) {
    cudaError_t e = cudaMalloc((void**)p, std::max<size_t>(n, 1) * sizeof(T));
    if (e != cudaSuccess) {
        h->err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
        return SPHGPU_ENOMEM;
    }
    return 0;
}

int alloc_scene(sphgpu_scene* h) {
    const int n = h->cap;
    DevScene& d = h->d;
    int r = 0;
    r |= dalloc(h, &d.pos, n); r |= dalloc(h, &d.vel, n); r |= dalloc(h, &d.gid, n);
    r |= dalloc(h, &d.rho, n); r |= dalloc(h, &d.alpha, n); r |= dalloc(h, &d.vadv, n);
    r |= dalloc(h, &d.acc, n); r |= dalloc(h, &d.kr, n); r |= dalloc(h, &d.kappa, n); r |= dalloc(h, &d.kappav, n);
    r |= dalloc(h, &d.pv, 2 * (size_t)n); r |= dalloc(h, &d.pk, n); r |= dalloc(h, &d.prv, 2 * (size_t)n);
    r |= dalloc(h, &d.ksum, n); r |= dalloc(h, &d.aux0, n); r |= dalloc(h, &d.aux1, n);
    r |= dalloc(h, &d.vA, n); r |= dalloc(h, &d.vB, n);
    r |= dalloc(h, &d.aux4, n); r |= dalloc(h, &d.kwarm, n); r |= dalloc(h, &d.hist, n); r |= dalloc(h, &d.wsbuf, n);
    r |= dalloc(h, &d.pos_s, n); r |= dalloc(h, &d.vel_s, n); r |= dalloc(h, &d.gid_s, n);
    r |= dalloc(h, &d.hist_s, n);
    r |= dalloc(h, &d.cA, n); r |= dalloc(h, &d.cB, n); r |= dalloc(h, &d.cC, n);
    r |= dalloc(h, &d.cA_s, n); r |= dalloc(h, &d.cB_s, n); r |= dalloc(h, &d.cC_s, n);
    r |= dalloc(h, &d.ap, n); r |= dalloc(h, &d.pl2, n); r |= dalloc(h, &d.ivs, n);
    r |= dalloc(h, &d.key, n); r |= dalloc(h, &d.slot, n); r |= dalloc(h, &d.tmp, n);
    r |= dalloc(h, &d.cell_count, (size_t)h->g.nkeys + 1);
    r |= dalloc(h, &d.cell_start, (size_t)h->g.nkeys + 1);
    r |= dalloc(h, &d.cstart2, (size_t)h->g.nkeys + 1);
    r |= dalloc(h, &d.bcell_start, (size_t)h->g.nkeys + 1);
    r |= dalloc(h, &d.nbr, (size_t)h->stride * ((h->ncap + 3) / 4) * 4);
    r |= dalloc(h, &d.ncount, n);
    r |= dalloc(h, &d.partial, (size_t)n / 64 + 4096);
    r |= dalloc(h, &d.st, 1);
    if (r) return SPHGPU_ENOMEM;
    d.cap_fluid = n;
    d.dt = &d.st->dt;
    d.nb = 0;
    cudaMemsetAsync(d.st, 0, sizeof(DevStats), h->stream);
    cudaMemsetAsync(d.bcell_start, 0, sizeof(int) * ((size_t)h->g.nkeys + 1), h->stream);
    cudaMemsetAsync(d.ksum, 0, sizeof(float) * n, h->stream);
    cudaMemsetAsync(d.kwarm, 0, sizeof(float) * n, h->stream);
    cudaMemsetAsync(d.hist, 0, sizeof(float4) * n, h->stream);
    cudaMemsetAsync(d.hist_s, 0, sizeof(float4) * n, h->stream);
    for (float4* c4 : {d.cA, d.cB, d.cC, d.cA_s, d.cB_s, d.cC_s, d.ap}) cudaMemsetAsync(c4, 0, sizeof(float4) * n, h->stream);
    // CUB scan scratch
    cub::DeviceScan::ExclusiveSum(nullptr, h->cub_bytes, d.cell_count, d.cell_start, h->g.nkeys + 1, h->stream);
    if (cudaMalloc(&h->cub_tmp, h->cub_bytes + 16) != cudaSuccess) return SPHGPU_ENOMEM;
    if (cudaMallocHost((void**)&h->h_stats, sizeof(DevStats)) != cudaSuccess) return SPHGPU_ENOMEM;
    if (cudaMallocHost((void**)&h->h_cont, sizeof(int)) != cudaSuccess) return SPHGPU_ENOMEM;
    memset(h->h_stats, 0, sizeof(DevStats));
    float dt = h->P.dt;
    cudaMemcpyAsync(d.dt, &dt, sizeof(float), cudaMemcpyHostToDevice, h->stream);
    return cudaStreamSynchronize(h->stream) == cudaSuccess ? 0 : SPHGPU_ECUDA;
}

// dynamic-solid state (the boundary returns to static walls)
void free_rigid(sphgpu_scene* h) {
    RigidDev& R = h->R;
    DevScene& d = h->d;
    void* ptrs[] = {R.x0, R.vol, R.dyn, R.sid, R.state, R.wpos, R.wvel, R.key, R.slot, R.tmp, R.cnt,
                    R.binv, R.out, R.partial, R.ticket, d.bforce, d.bks};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (d.bpf && d.bpf != d.bpv) cudaFree(d.bpf);
    d.bpf = d.bpv;
    d.bforce = nullptr;
    d.bks = nullptr;
    if (h->h_rstate) cudaFreeHost(h->h_rstate);
    if (h->h_rout) cudaFreeHost(h->h_rout);
    h->h_rstate = nullptr;
    h->h_rout = nullptr;
    h->rigid_cap = 0;
    R = RigidDev{};
    h->dyn_ids.clear();
    h->dyn_r0.clear();
    h->dyn_r1.clear();
}

void free_scene(sphgpu_scene* h) {
    DevScene& d = h->d;
    void* ptrs[] = {d.pos, d.vel, d.gid, d.rho, d.alpha, d.vadv, d.pv, d.pk, d.prv, d.bpv, d.kappav, d.acc, d.kr, d.kappa, d.ksum, d.vA, d.vB, d.aux0,
                    d.aux1, d.aux4, d.kwarm, d.hist, d.wsbuf, d.pos_s, d.vel_s, d.gid_s, d.hist_s, d.key, d.slot, d.tmp,
                    d.cA, d.cB, d.cC, d.cA_s, d.cB_s, d.cC_s, d.ap, d.pl2, d.ivs,
                    d.bsid, d.bnbr, d.bncount, d.bivs, d.bivo,
                    h->recX, h->recY, h->xn,
                    d.cell_count, d.cell_start, d.bcell_start, d.cstart2, d.nbr, d.ncount, d.partial, d.st,
                    d.bpos, d.bvel, d.bgid, h->cub_tmp};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    free_rigid(h);
    if (h->d_geom) cudaFree(h->d_geom);
    if (h->d_batch) cudaFree(h->d_batch);
    if (h->h_stats) cudaFreeHost(h->h_stats);
    if (h->h_cont) cudaFreeHost(h->h_cont);
    if (h->h_diff) cudaFreeHost(h->h_diff);
    for (void* q : {(void*)h->in_xyz, (void*)h->in_vel, (void*)h->d_diff})
        if (q) cudaFree(q);
    for (auto& kv : h->graphs) cudaGraphExecDestroy(kv.second);
    for (auto e : h->prof.pool) cudaEventDestroy(e);
}

// ---------------- step building blocks ----------------

// updatePaticles of every dynamic solid with the states in h_rstate, and the
// re-sort of the whole boundary (SphWithBullet.cpp:212-221)
void enq_boundary_update(sphgpu_scene* h, cudaStream_t st) {
    if (!h->R.nd) return;
    cudaMemcpyAsync(h->R.state, h->h_rstate, sizeof(float) * 25 * h->R.nd, cudaMemcpyHostToDevice, st);
    launch(h, "rigid_place", st, [&] {
        launch_rigid_place_sort(h->d, h->R, h->g, h->cub_tmp, h->cub_bytes, st);
    });
}

void enq_ns(sphgpu_scene* h, int integrate, int build_mode, cudaStream_t st, int carry = 1) {
    DevScene& d = h->d;
    cudaMemsetAsync(d.cell_count, 0, sizeof(int) * ((size_t)h->g.nkeys + 1), st);
    launch(h, "hash", st, [&] { launch_hash(d, h->g, integrate, h->cap, st); });
    launch(h, "scan", st, [&] {
        size_t b = h->cub_bytes;
        cub::DeviceScan::ExclusiveSum(h->cub_tmp, b, d.cell_count, d.cell_start, h->g.nkeys + 1, st);
    });
    launch(h, "reorder", st, [&] { launch_scatter_reorder(d, h->g, h->cap, carry, st); });
    launch_count_active(d, h->g, st);
    if (h->nscenes > 1) launch_batch_count(d, h->nscenes, st);
    if (h->R.nd)
        launch(h, "rigid_volume", st,
               [&] { launch_rigid_volume(d, h->R, h->g, h->P.particle_d, h->c.h2cut, h->ncap, st); });
    launch(h,
           build_mode == 1   ? "build_first"
           : build_mode == 4 ? "build_first_div"
           : build_mode == 2 ? "build_pressure"
                             : "build",
           st, [&] { launch_build(d, h->g, h->c, build_mode, h->cap, st, h->tune.build); });
}

// Jacobi loop: a conditional WHILE node while capturing, host-driven otherwise.
// `pre`, when given, is the tail of a first iteration whose other kernels
// ran earlier: it runs once on the main stream and decides (through the
// handle, or st->cont) whether the loop body runs at all.
struct NoPre {
    void operator()(cudaStream_t, unsigned long long, int) const {}
};
template <class Body, class Pre = NoPre>
int enq_loop(sphgpu_scene* h, bool capturing, Body&& body, Pre&& pre = NoPre(), bool has_pre = false) {
    if (capturing) {
        cudaStreamCaptureStatus cs;
        cudaGraph_t cg;
        const cudaGraphNode_t* deps = nullptr;
        size_t ndeps = 0;
        CK(cudaStreamGetCaptureInfo(h->stream, &cs, nullptr, &cg, &deps, &ndeps));
        cudaGraphConditionalHandle handle;
        CK(cudaGraphConditionalHandleCreate(&handle, cg, 1, cudaGraphCondAssignDefault));
        if (has_pre) {
            pre(h->stream, (unsigned long long)handle, 1);
            CK(cudaStreamGetCaptureInfo(h->stream, &cs, nullptr, &cg, &deps, &ndeps));
        }
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = handle;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        CK(cudaGraphAddNode(&node, cg, deps, ndeps, &cp));
        CK(cudaStreamUpdateCaptureDependencies(h->stream, &node, 1, cudaStreamSetCaptureDependencies));
        cudaGraph_t bodyg = cp.conditional.phGraph_out[0];
        CK(cudaStreamBeginCaptureToGraph(h->stream2, bodyg, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
        body(h->stream2, (unsigned long long)handle, 1);
        CK(cudaStreamEndCapture(h->stream2, &bodyg));
        return 0;
    }
    if (has_pre) {
        pre(h->stream, 0ull, 0);
        CK(cudaMemcpyAsync(h->h_cont, &h->d.st->cont, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        if (!*h->h_cont) return 0;
    }
    for (int guard = 0; guard < 100000; ++guard) {
        body(h->stream, 0ull, 0);
        CK(cudaMemcpyAsync(h->h_cont, &h->d.st->cont, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        if (!*h->h_cont) break;
    }
    return 0;
}

int enq_df_density_loop(sphgpu_scene* h, bool capturing) {
    DevScene& d = h->d;
    const SphParams& P = h->P;
    launch_df_loop_reset(d, 0, h->stream);
    if (h->nscenes > 1) launch_batch_loop_reset(d, h->nscenes, 0, h->stream);
    return enq_loop(h, capturing, [&](cudaStream_t st, unsigned long long hd, int use) {
        launch(h, "df_density_a", st,
               [&] { launch_df_dens_a(d, h->c, h->cap, h->record_ksum, st, h->tune.sweep_a); });
        launch(h, "df_density_b", st, [&] {
            launch_df_dens_b(d, h->c, h->cap, P.df_density_goal, P.df_density_min_iter, P.df_density_max_iter, hd,
                             use, st, h->tune.sweep_b);
        });
        if (h->nscenes > 1)
            launch(h, "batch_decide", st, [&] {
                launch_batch_decide(d, h->c, 0, h->nscenes, h->cap, 0.0, P.df_density_goal, P.df_density_min_iter,
                                    P.df_density_max_iter, hd, use, st);
            });
    });
}

// fused: the list build (mode 4) already ran the first iteration's sweep A
int enq_df_div_loop(sphgpu_scene* h, bool capturing, bool fused = false) {
    DevScene& d = h->d;
    const SphParams& P = h->P;
    launch_df_loop_reset(d, 1, h->stream);
    if (h->nscenes > 1) launch_batch_loop_reset(d, h->nscenes, 1, h->stream);
    // the velocity update and, for a batch, the per-scene decisions
    auto div_b = [&](cudaStream_t st, unsigned long long hd, int use) {
        launch(h, "df_div_b", st, [&] {
            launch_df_div_b(d, h->c, h->cap, P.df_div_goal_abs, P.df_div_goal_rel, P.df_div_min_iter,
                            P.df_div_max_iter, hd, use, st, h->tune.sweep_b);
        });
        if (h->nscenes > 1)
            launch(h, "batch_decide", st, [&] {
                launch_batch_decide(d, h->c, 1, h->nscenes, h->cap, P.df_div_goal_abs, P.df_div_goal_rel, P.df_div_min_iter,
                                    P.df_div_max_iter, hd, use, st);
            });
    };
    auto body = [&](cudaStream_t st, unsigned long long hd, int use) {
        launch(h, "df_div_a", st, [&] { launch_df_div_a(d, h->c, h->cap, st, h->tune.sweep_a); });
        div_b(st, hd, use);
    };
    return enq_loop(h, capturing, body, div_b, fused);
}

// the list build runs the divergence loop's first sweep A
bool fused_div(const sphgpu_scene* h) { return h->fuse_div != 0; }

// The body of one DFSPH step after the first neighbour search
// (DFSPH::sphStep, DFSPH.cpp:52-62), with the learned warm start when a
// network is attached (ws_mode 1) or training-data recording (ws_mode 2).
// Part 1: forces, the density loop and, with dynamic solids, their boundary
// forces (copied to h_rout); part 2: updateSolids' particle update, the
// neighbour search with rho/alpha, the divergence loop.  Without dynamic
// solids one graph holds both; with them the rigid-body world runs on the
// host between the two.
int enq_df_part1(sphgpu_scene* h, bool capturing);
int enq_df_part2(sphgpu_scene* h, bool capturing);

int enq_df_step(sphgpu_scene* h, bool capturing) {
    int r = enq_df_part1(h, capturing);
    return r ? r : enq_df_part2(h, capturing);
}

// boundary forces of every dynamic solid and their FP64 joins -> h_rout
void enq_rigid_forces(sphgpu_scene* h, cudaStream_t st) {
    const int nd = h->R.nd;
    if (!nd) return;
    for (int i = 0; i < nd; ++i)
        launch(h, "rigid_force", st, [&] {
            launch_rigid_force(h->d, h->R, h->c, h->g, h->dyn_r0[i], h->dyn_r1[i], i, st);
        });
    cudaMemcpyAsync(h->h_rout, h->R.out, sizeof(double) * 6 * nd, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(h->h_rout + 6 * nd, h->d.dt, sizeof(float), cudaMemcpyDeviceToHost, st);
}

int enq_df_part1(sphgpu_scene* h, bool capturing) {
    DevScene& d = h->d;
    cudaStream_t st = h->stream;
    launch_step_begin(d, st);
    // the boundary forces read the loop's summed stiffness; without the
    // warm start (whose post-processing clears the sum) it restarts here
    const bool dyn = h->R.nd > 0;
    if (dyn && !(h->mlp && h->ws_mode)) cudaMemsetAsync(d.ksum, 0, sizeof(float) * h->cap, st);
    if (h->P.cfl && h->nscenes > 1)
        launch(h, "cfl", st, [&] {
            launch_batch_cfl(d, h->nscenes, h->cap, h->P.cfl_factor, h->P.particle_d, h->P.dt_max, h->P.dt_min, st);
        });
    else if (h->P.cfl)
        launch(h, "cfl", st, [&] { launch_cfl(d, h->cap, h->P.cfl_factor, h->P.particle_d, h->P.dt_max, h->P.dt_min, st); });
    const int ws = h->mlp ? h->ws_mode : 0;
    launch(h, "df_forces", st, [&] { launch_df_forces(d, h->c, h->cap, 0, st, h->tune.forces); });
    if (h->P.enable_vortex)
        launch(h, "vortex", st, [&] {
            launch_vortex_second(d, h->c, h->P.enable_vortex, h->P.vort_alpha, h->P.vort_zeta, h->P.vort_nu_t,
                                 h->P.spacing_r, h->cap, st);
        });
    if (ws == 1 && h->fuse_ws) {
        launch(h, "ws_features_infer", st, [&] {
            launch_ws_features_infer(d, h->c, h->mlp->m, h->P.dt_max, h->alpha_ref, h->xn, h->cap, h->sm_count, st);
        });
        launch(h, "df_warm", st, [&] { launch_df_warm_correction(d, h->c, h->cap, st, h->tune.sweep_b); });
    } else if (ws == 1 || ws == 3) {
        launch(h, "ws_features", st, [&] {
            launch_ws_features(d, h->c, h->mlp->m, ws == 1 ? 1 : 2, h->P.dt_max, h->alpha_ref, nullptr, h->xn, h->cap,
                               st);
        });
        if (ws == 1)
            launch(h, "ws_infer", st, [&] { launch_ws_infer(d, h->c, h->mlp->m, h->xn, h->cap, h->sm_count, st); });
        launch(h, "df_warm", st, [&] { launch_df_warm_correction(d, h->c, h->cap, st, h->tune.sweep_b); });
    } else if (ws == 2) {
        launch(h, "ws_features", st, [&] {
            launch_ws_features(d, h->c, h->mlp->m, 0, h->P.dt_max, h->alpha_ref, h->recX, nullptr, h->cap, st);
        });
    }
    const int rec = h->record_ksum;
    h->record_ksum = rec || ws != 0 || dyn;
    int r = enq_df_density_loop(h, capturing);
    h->record_ksum = rec;
    if (r) return r;
    enq_rigid_forces(h, st);
    return 0;
}

int enq_df_part2(sphgpu_scene* h, bool capturing) {
    DevScene& d = h->d;
    cudaStream_t st = h->stream;
    // the warm start's history and training label (part 2, so that part 1
    // leaves every carried per-particle array as it found it: a speculative
    // host step may run part 1 again)
    const int ws = h->mlp ? h->ws_mode : 0;
    // with a network applied (no recording) the hash kernel writes the history
    const int ws_in_hash = ws == 1 ? 4 : 0;
    if (ws && !ws_in_hash) {
        launch(h, "ws_post", st, [&] { launch_ws_post(d, h->c, ws == 2 ? h->recY : nullptr, h->cap, st); });
        if (ws == 2) {
            sphgpu_mlp* m = h->mlp;
            launch_ws_append(h->recX, h->recY, h->cap, &d.st->n_active, h->ws_every, &d.st->pad2, m->dsX, m->dsy,
                             m->ds_count, m->ds_cap, st);
        }
    }
    enq_boundary_update(h, st);
    const int vort = h->P.enable_vortex ? 2 : 0;  // carry cA (w or n0) through the sort
    const bool fused = fused_div(h);
    enq_ns(h, 1 | vort | ws_in_hash, fused ? 4 : 1, st, 1 | vort);
    int r = enq_df_div_loop(h, capturing, fused);
    if (r) return r;
    if (h->P.enable_vortex == 3)
        launch(h, "vortex", st, [&] { launch_vortex_after_div(d, h->c, h->P.spacing_r, h->cap, st); });
    if (!h->skip_stats) CK(cudaMemcpyAsync(h->h_stats, d.st, sizeof(DevStats), cudaMemcpyDeviceToHost, st));
    return 0;
}

// The sorted arrays hold the state: copy it, with the carried per-particle
// state, into the staging arrays the next sort reads.
void stage_from_sorted(sphgpu_scene* h, int n) {
    DevScene& d = h->d;
    cudaStream_t st = h->stream;
    cudaMemcpyAsync(d.pos_s, d.pos, sizeof(float4) * n, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(d.vel_s, d.vel, sizeof(float4) * n, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(d.gid_s, d.gid, sizeof(int) * n, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(d.hist_s, d.hist, sizeof(float4) * n, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(d.cA_s, d.cA, sizeof(float4) * n, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(d.cB_s, d.cB, sizeof(float4) * n, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(d.cC_s, d.cC, sizeof(float4) * n, cudaMemcpyDeviceToDevice, st);
}

// PciSph::pci_updateDelta (PciSph.cpp:133-162), in float as the reference
// evaluates it: delta of a prototype particle with a full neighbourhood on
// the lattice of spacing spacing_r, divided by dt^2.
float pci_delta(const SphParams& P, const KerConst& k) {
    const float sp = P.spacing_r, hs = P.smoothRadius_h, dt = P.dt;
    const int n = (int)std::ceil(hs / sp);
    float gs[3] = {0.f, 0.f, 0.f}, g2 = 0.f;
    auto wg = [&](float r) {
        float q = r / k.h, qm2 = 2 - q;
        return q <= 1 ? k.thetah * (3 * q - 2.25f * q * q) : k.thetah * 0.75f * qm2 * qm2;
    };
    for (int z = -n; z <= n; ++z)
        for (int y = -n; y <= n; ++y)
            for (int x = -n; x <= n; ++x) {
                if (!x && !y && !z) continue;
                const float vf[3] = {(float)x * sp, (float)y * sp, (float)z * sp};
                const float dis = std::sqrt(vf[0] * vf[0] + vf[1] * vf[1] + vf[2] * vf[2]);
                if (dis < hs) {
                    const float grad = -wg(dis);
                    for (int c = 0; c < 3; ++c) gs[c] += vf[c] * (grad / dis);
                    g2 += grad * grad;
                }
            }
    const float v0 = (float)std::pow((double)sp, 3);
    const float beta = 2 * v0 * v0;
    const float delta = -1 / (beta * (-(gs[0] * gs[0] + gs[1] * gs[1] + gs[2] * gs[2]) - g2));
    return delta / (dt * dt);
}

// One PCISPH step (PciSph::sphStep, PciSph.cpp:31-94): the state enters and
// leaves in the staging arrays, like WCSPH.
int enq_pci_step(sphgpu_scene* h, bool capturing) {
    DevScene& d = h->d;
    cudaStream_t st = h->stream;
    const SphParams& P = h->P;
    launch_step_begin(d, st);
    enq_ns(h, 0, 0, st, 4);
    const float delta = pci_delta(P, h->c.k);
    launch(h, "pci_force_except", st, [&] { launch_pci_force_except(d, h->c, h->cap, st); });
    launch_df_loop_reset(d, 0, st);
    int r = enq_loop(h, capturing, [&](cudaStream_t s2, unsigned long long hd, int use) {
        launch(h, "pci_density", s2, [&] { launch_pci_density(d, h->c, delta, h->cap, s2); });
        launch(h, "pci_pressure", s2, [&] {
            launch_pci_pressure(d, h->c, P.densityErro_eta, P.pci_min_iter, P.pci_max_iter, hd, use, h->cap, s2);
        });
    });
    if (r) return r;
    launch(h, "pci_finish", st, [&] { launch_pci_finish(d, h->cap, st); });
    CK(cudaMemcpyAsync(h->h_stats, d.st, sizeof(DevStats), cudaMemcpyDeviceToHost, st));
    return 0;
}

// One IISPH_M step (IISph_M::sphStep, IISph_M.cpp:10-75): phases solved in
// turn, each with its own Jacobi loop.
int enq_ii_step(sphgpu_scene* h, bool capturing) {
    DevScene& d = h->d;
    cudaStream_t st = h->stream;
    const SphParams& P = h->P;
    launch_step_begin(d, st);
    enq_ns(h, 0, 0, st, 2 | 4 | 8);
    launch(h, "ii_force_except", st, [&] { launch_ii_force_except(d, h->c, h->cap, st); });
    const int nph = (int)h->rho0_ph.size();
    for (int ph = 0; ph < nph; ++ph) {
        launch_ii_phase_begin(d, st);
        launch(h, "ii_density", st, [&] { launch_ii_density(d, h->c, ph, h->cap, st); });
        launch(h, "ii_aii", st, [&] { launch_ii_aii(d, h->c, ph, h->cap, st); });
        int r = enq_loop(h, capturing, [&](cudaStream_t s2, unsigned long long hd, int use) {
            launch(h, "ii_sum", s2, [&] { launch_ii_sum(d, h->c, ph, h->cap, s2); });
            launch(h, "ii_press", s2, [&] {
                launch_ii_press(d, h->c, ph, (double)P.ii_omega, (double)P.ii_eta_rel, P.ii_min_iter, P.ii_max_iter,
                                P.ii_compat, hd, use, h->cap, s2);
            });
        });
        if (r) return r;
    }
    launch(h, "ii_force", st, [&] { launch_ii_force(d, h->c, P.ii_compat, h->cap, st); });
    CK(cudaMemcpyAsync(h->h_stats, d.st, sizeof(DevStats), cudaMemcpyDeviceToHost, st));
    return 0;
}

void invalidate_graphs(sphgpu_scene* h);

// IISph boundary state (allocated on first use: other solvers never need it)
int ensure_iv_boundary(sphgpu_scene* h) {
    DevScene& d = h->d;
    if (d.bivs || h->nb == 0) return 0;
    const int nb = h->nb;
    d.bstride = roundup(nb, 32);
    int r = dalloc(h, &d.bsid, nb) | dalloc(h, &d.bncount, nb) | dalloc(h, &d.bivs, nb) | dalloc(h, &d.bivo, nb) |
            dalloc(h, &d.bnbr, (size_t)d.bstride * ((h->ncap + 3) / 4) * 4);
    if (r) return SPHGPU_ENOMEM;
    CK(copy_sync(d.bsid, h->bsolid_h.data(), sizeof(int) * nb, cudaMemcpyHostToDevice));
    CK(memset_sync(d.bivs, 0, sizeof(float4) * nb));
    CK(memset_sync(d.bivo, 0, sizeof(float4) * nb));
    CK(memset_sync(d.bncount, 0, sizeof(int) * nb));
    invalidate_graphs(h);
    return 0;
}

// neighbour lists of fluid and boundary particles with IISph's
// DF_prepareAttribute / VF_prepareAttribute terms (IISph.cpp:100-545); the
// carried loop velocity (cA) and stiffnesses (cC) follow the reorder
void enq_iv_prepare(sphgpu_scene* h, bool from_staging, cudaStream_t st) {
    DevScene& d = h->d;
    if (from_staging) enq_ns(h, 0, 3, st, 2 | 8);
    else launch(h, "build_iisph", st, [&] { launch_build(d, h->g, h->c, 3, h->cap, st, h->tune.build); });
    launch(h, "iv_boundary_build", st, [&] { launch_iv_boundary_build(d, h->g, h->c, h->tune.build, st); });
}

// the divergence-free (div = 1, IISph.cpp:1219-1456) or constant-volume
// (div = 0, :546-815) loops, phase by phase
int enq_iv_loops(sphgpu_scene* h, bool capturing, int div) {
    DevScene& d = h->d;
    const SphParams& P = h->P;
    const double goal = (double)(div ? P.iv_div_goal : P.iv_cv_goal);  // real_t goals (float)
    const int mn = div ? P.iv_div_min_iter : P.iv_cv_min_iter, mx = div ? P.iv_div_max_iter : P.iv_cv_max_iter;
    const int nph = (int)h->rho0_ph.size();
    for (int ph = 0; ph < nph; ++ph) {
        launch_iv_phase_begin(d, h->stream);
        launch(h, "iv_loop_init", h->stream, [&] { launch_iv_loop_init(d, ph, div, h->cap, h->stream); });
        int r = enq_loop(h, capturing, [&](cudaStream_t s2, unsigned long long hd, int use) {
            launch(h, div ? "iv_div_boundary" : "iv_cv_boundary", s2,
                   [&] { launch_iv_boundary_sweep(d, h->c, div, h->tune.sweep_a, s2); });
            launch(h, div ? "iv_div_a" : "iv_cv_a", s2,
                   [&] { launch_iv_sweep_a(d, h->c, ph, div, h->cap, h->tune.sweep_a, s2); });
            launch(h, div ? "iv_div_b" : "iv_cv_b", s2, [&] {
                launch_iv_sweep_b(d, h->c, ph, div, goal, mn, mx, hd, use, h->cap, h->tune.sweep_b, s2);
            });
        });
        if (r) return r;
    }
    return 0;
}

// One IISph step (IISph::sphStep, IISph.cpp:14-99): the state enters and
// leaves in the staging arrays, like PCISPH and IISPH_M.
int enq_iv_step(sphgpu_scene* h, bool capturing) {
    DevScene& d = h->d;
    cudaStream_t st = h->stream;
    launch_step_begin(d, st);
    enq_iv_prepare(h, true, st);
    launch(h, "iv_forces", st, [&] { launch_iv_forces(d, h->c, h->cap, h->tune.forces, st); });
    int r = enq_iv_loops(h, capturing, 1);
    if (r) return r;
    r = enq_iv_loops(h, capturing, 0);
    if (r) return r;
    launch(h, "iv_integrate", st, [&] { launch_iv_integrate(d, h->cap, st); });
    CK(cudaMemcpyAsync(h->h_stats, d.st, sizeof(DevStats), cudaMemcpyDeviceToHost, st));
    return 0;
}

// WCSPH step from the staged state: neighbour search with density and
// pressure, (surface normals,) forces and the integration into staging;
// the statistics go to the host after the last step of a call only (each
// copy sits on the step's critical path: 75 -> 69 us per step at 27 k)
int enq_wc_step(sphgpu_scene* h, bool, bool copy_stats = true) {
    cudaStream_t st = h->stream;
    launch_step_begin(h->d, st);
    enq_ns(h, 0, 2, st);
    const bool surf = h->P.th_h != 0.f || h->P.th_r != 0.f || h->P.th_bt != 0.f;
    if (surf) launch(h, "wc_normal", st, [&] { launch_wc_normal(h->d, h->c, h->cap, st); });
    launch(h, "wc_force", st, [&] { launch_wc_force(h->d, h->c, h->cap, st, surf, h->c.lanes); });
    if (copy_stats) CK(cudaMemcpyAsync(h->h_stats, h->d.st, sizeof(DevStats), cudaMemcpyDeviceToHost, st));
    return 0;
}

int wc_graph_build(sphgpu_scene* h, bool cap) { return enq_wc_step(h, cap); }
int wc_graph_build_nostats(sphgpu_scene* h, bool cap) { return enq_wc_step(h, cap, false); }
int pci_graph_build(sphgpu_scene* h, bool cap) { return enq_pci_step(h, cap); }
int ii_graph_build(sphgpu_scene* h, bool cap) { return enq_ii_step(h, cap); }
int iv_graph_build(sphgpu_scene* h, bool cap) { return enq_iv_step(h, cap); }

int run_initial_ns(sphgpu_scene* h, int build_mode) {
    if (!h->in_staging) stage_from_sorted(h, h->h_stats->n_active);  // the sort reads staging
    enq_boundary_update(h, h->stream);
    enq_ns(h, 0, build_mode, h->stream, 1 | 2 | 4 | 8);
    ++h->sorts;
    h->in_staging = false;
    h->ns_valid = build_mode == 1;
    CK(cudaMemcpyAsync(h->h_stats, h->d.st, sizeof(DevStats), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return 0;
}

int graph_for(sphgpu_scene* h, int key, cudaGraphExec_t* out, int (*build)(sphgpu_scene*, bool)) {
    auto it = h->graphs.find(key);
    if (it != h->graphs.end()) {
        *out = it->second;
        return 0;
    }
    cudaGraph_t gph;
    CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeRelaxed));
    int r = build(h, true);
    cudaError_t e = cudaStreamEndCapture(h->stream, &gph);
    if (r) return r;
    if (e != cudaSuccess) {
        h->err = std::string("graph capture: ") + cudaGetErrorString(e);
        return SPHGPU_ECUDA;
    }
    cudaGraphExec_t ex;
    e = cudaGraphInstantiate(&ex, gph, 0);
    cudaGraphDestroy(gph);
    if (e != cudaSuccess) {
        h->err = std::string("graph instantiate: ") + cudaGetErrorString(e);
        return SPHGPU_ECUDA;
    }
    h->graphs[key] = ex;
    *out = ex;
    return 0;
}

int df_graph_build(sphgpu_scene* h, bool cap) { return enq_df_step(h, cap); }
int df1_graph_build(sphgpu_scene* h, bool cap) { return enq_df_part1(h, cap); }
// part 1 and the positions the integration will write, in reference order
// (d.aux4 as 3 floats per particle), for a host-buffer step
int df1o_graph_build(sphgpu_scene* h, bool cap) {
    int r = enq_df_part1(h, cap);
    if (!r) launch_integrated_to_ref(h->d, h->cap, (float*)h->d.aux4, h->stream);
    return r;
}
int df2_graph_build(sphgpu_scene* h, bool cap) { return enq_df_part2(h, cap); }

// SphWithBullet::updateSolids' exchange with the rigid-body world: the
// joined forces of the last step (h_rout, on the host once the stream is
// synchronised) in, the new states (h_rstate) out
int run_rigid_callback(sphgpu_scene* h) {
    const int nd = h->R.nd;
    if (!nd || !h->rigid_fn) return 0;
    const double* f = h->h_rout;
    std::vector<double> force(3 * nd), torque(3 * nd);
    for (int i = 0; i < nd; ++i)
        for (int c = 0; c < 3; ++c) {
            force[3 * i + c] = f[6 * i + c];
            torque[3 * i + c] = f[6 * i + 3 + c];
        }
    float dt;
    memcpy(&dt, h->h_rout + 6 * nd, sizeof(float));
    static_assert(sizeof(SphRigidState) == 25 * sizeof(float), "SphRigidState is 25 floats");
    if (h->rigid_fn(h->rigid_user, nd, h->dyn_ids.data(), force.data(), torque.data(), (double)dt,
                    reinterpret_cast<SphRigidState*>(h->h_rstate)))
        h->rigid_fail = 1;
    return 0;
}

void invalidate_graphs(sphgpu_scene* h) {
    for (auto& kv : h->graphs) cudaGraphExecDestroy(kv.second);
    h->graphs.clear();
}

int status_to_rc(unsigned s) {
    if (s & SPHGPU_STATUS_NAN) return SPHGPU_ENAN;
    if (s & SPHGPU_STATUS_SOLID_OUTSIDE) return SPHGPU_EOUT_OF_DOMAIN;
    if (s & (SPHGPU_STATUS_MAXITER_DENSITY | SPHGPU_STATUS_MAXITER_DIVERGENCE)) return SPHGPU_EMAXITER;
    return 0;
}

void fill_stats(sphgpu_scene* h, SphStepStats* o, int steps) {
    if (!o) return;
    const DevStats& s = *h->h_stats;
    memset(o, 0, sizeof(*o));
    o->n_fluid = s.n_active;
    o->iter_density = s.it_density;
    o->iter_divergence = s.it_div;
    o->removed = s.removed;
    o->err_density = s.err_density;
    o->err_divergence = s.err_div;
    o->dt = s.dt;
    o->status = s.status;
    o->neighbour_overflow = s.overflow;
    o->zero_distance = s.zero_dis;
    o->max_neighbours_seen = s.max_nbrs;
    o->mean_neighbours = s.n_active ? (double)s.nbr_total / s.n_active : 0.0;
    o->total_iter_density = s.total_it_density;
    o->total_iter_divergence = s.total_it_div;
    o->steps = steps;
}

int enq_steps(sphgpu_scene* h, int solver, int nsteps) {
    if (solver != SPHGPU_DFSPH && solver != SPHGPU_WCSPH && solver != SPHGPU_PCISPH && solver != SPHGPU_IISPH_M &&
        solver != SPHGPU_IISPH) {
        h->err = "unknown solver";
        return SPHGPU_EINVAL;
    }
    if (h->h_stats->n_active <= 0 && h->n_total <= 0) {
        h->err = "no fluid particles";
        return SPHGPU_EINVAL;
    }
    if (solver == SPHGPU_DFSPH && h->rho0_ph.size() != 1) {
        h->err = "DFSPH path supports one fluid phase";
        return SPHGPU_ENOTIMPL;
    }
    if (h->nscenes > 1 && (solver != SPHGPU_DFSPH || (h->mlp && h->ws_mode))) {
        h->err = "a batch of scenes runs the plain DFSPH solver";
        return SPHGPU_ENOTIMPL;
    }
    if (h->R.nd && solver != SPHGPU_DFSPH) {
        h->err = "dynamic solids are coupled in the DFSPH step";
        return SPHGPU_ENOTIMPL;
    }
    if (solver == SPHGPU_DFSPH && h->P.enable_vortex) {
        if (h->P.enable_vortex < 0 || h->P.enable_vortex > 3) { h->err = "enable_vortex is 0..3"; return SPHGPU_EINVAL; }
        if (h->nscenes > 1 || (h->mlp && h->ws_mode)) {
            h->err = "the vorticity options run in the plain single-scene DFSPH step";
            return SPHGPU_ENOTIMPL;
        }
    }
    if (h->R.nd && h->record_ksum) {
        h->err = "record_kappa_sum cannot be combined with dynamic solids";
        return SPHGPU_EINVAL;
    }
    launch_call_begin(h->d, h->stream);
    if (h->nscenes > 1) launch_batch_call_begin(h->d, h->nscenes, h->stream);
    if (solver == SPHGPU_PCISPH || solver == SPHGPU_IISPH_M || solver == SPHGPU_IISPH) {
        if (solver == SPHGPU_IISPH) {
            int r = ensure_iv_boundary(h);
            if (r) return r;
        }
        if (h->last_solver != solver && h->last_solver >= 0) {
            // entering from another solver: the carried state starts as the
            // reference's fresh particles (the last density, zeros)
            launch_carry_init(h->d, h->c, h->in_staging ? 1 : 0, h->cap, h->stream);
        }
        if (!h->in_staging) stage_from_sorted(h, h->cap);
        h->last_solver = solver;
        for (int s = 0; s < nsteps; ++s) {
            if (h->use_graphs && !h->prof.on) {
                cudaGraphExec_t ex;
                // DFSPH keys use bits 0-8; these sit above them
                const int key = (solver == SPHGPU_PCISPH ? 1 : (solver == SPHGPU_IISPH_M ? 2 : 3)) << 12;
                int r = graph_for(h, key, &ex,
                                  solver == SPHGPU_PCISPH ? pci_graph_build
                                                          : (solver == SPHGPU_IISPH_M ? ii_graph_build : iv_graph_build));
                if (r) return r;
                CK(cudaGraphLaunch(ex, h->stream));
            } else {
                int r = solver == SPHGPU_PCISPH ? enq_pci_step(h, false)
                                                : (solver == SPHGPU_IISPH_M ? enq_ii_step(h, false) : enq_iv_step(h, false));
                if (r) return r;
                prof_collect(h);
            }
            // the step sorts first, then writes every per-particle result
            h->ep_acc = h->ep_loop = ++h->sorts;
            h->frame++;
        }
        h->in_staging = true;
        h->ns_valid = false;
        return 0;
    }
    const bool entering = h->last_solver != solver;
    h->last_solver = solver;
    if (solver == SPHGPU_DFSPH) {
        if (!h->ns_valid) {
            int r = run_initial_ns(h, 1);
            if (r) return r;
        }
        const bool dyn = h->R.nd > 0;
        if (h->P.enable_vortex != h->vort_last || (h->P.enable_vortex && entering)) {
            // a vorticity option starts from zero carried vectors
            CK(cudaMemsetAsync(h->d.cA, 0, sizeof(float4) * h->cap, h->stream));
            CK(cudaMemsetAsync(h->d.cA_s, 0, sizeof(float4) * h->cap, h->stream));
            h->vort_last = h->P.enable_vortex;
        }
        for (int s = 0; s < nsteps; ++s) {
            const int key = (h->mlp ? h->ws_mode : 0) | (h->record_ksum ? 4 : 0) | (h->P.cfl ? 8 : 0) |
                            (h->P.enable_vortex << 6);
            if (h->out_xyz && nsteps == 1 && !dyn && h->use_graphs && !h->prof.on) {
                // the step as two graphs with the output of the integrated
                // positions between them, on stream3, joined at the end
                cudaGraphExec_t ex1, ex2;
                int r = graph_for(h, key | 16 | 256, &ex1, df1o_graph_build);
                if (!r) r = graph_for(h, key | 32, &ex2, df2_graph_build);
                if (r) return r;
                CK(cudaGraphLaunch(ex1, h->stream));
                CK(cudaEventRecord(h->ev_out[0], h->stream));
                CK(cudaStreamWaitEvent(h->stream3, h->ev_out[0], 0));
                // the output may be the input buffer: after the input copy
                if (h->spec_pending) CK(cudaStreamWaitEvent(h->stream3, h->ev_in[1], 0));
                CK(cudaMemcpyAsync(h->out_xyz, h->d.aux4, sizeof(float) * 3 * (size_t)h->out_n,
                                   cudaMemcpyDeviceToHost, h->stream3));
                CK(cudaEventRecord(h->ev_out[1], h->stream3));
                if (h->spec_pending) {
                    // part 1 ran ahead of the check of the host inputs
                    // (sphgpu_step_host): part 2, which re-sorts the state,
                    // starts only if they equal the state part 1 read
                    h->spec_pending = false;
                    CK(cudaEventSynchronize(h->ev_in[1]));
                    if (*h->h_diff) {
                        h->spec_failed = true;
                        return 0;
                    }
                }
                CK(cudaGraphLaunch(ex2, h->stream));
                CK(cudaStreamWaitEvent(h->stream, h->ev_out[1], 0));
                h->out_xyz_done = true;
            } else if (h->use_graphs && !h->prof.on) {
                cudaGraphExec_t ex;
                int r;
                if (dyn) {
                    r = graph_for(h, key | 16, &ex, df1_graph_build);
                } else {
                    // steps before the call's last leave the statistics on the device
                    h->skip_stats = s < nsteps - 1;
                    r = graph_for(h, key | (h->skip_stats ? 512 : 0), &ex, df_graph_build);
                    h->skip_stats = false;
                }
                if (r) return r;
                CK(cudaGraphLaunch(ex, h->stream));
            } else {
                int r = dyn ? enq_df_part1(h, false) : enq_df_step(h, false);
                if (r) return r;
                prof_collect(h);
            }
            if (dyn) {
                // the rigid-body world between the density loop and the
                // neighbour search (DFSPH.cpp:52-56)
                CK(cudaStreamSynchronize(h->stream));
                run_rigid_callback(h);
                if (h->use_graphs && !h->prof.on) {
                    cudaGraphExec_t ex;
                    int r = graph_for(h, key | 32, &ex, df2_graph_build);
                    if (r) return r;
                    CK(cudaGraphLaunch(ex, h->stream));
                } else {
                    int r = enq_df_part2(h, false);
                    if (r) return r;
                    prof_collect(h);
                }
            }
            // forces and the density loop ran before the step's sort
            h->ep_acc = h->ep_loop = h->sorts++;
            h->ep_vort = h->P.enable_vortex == 3 ? h->sorts : h->sorts - 1;
            h->frame++;
        }
        return 0;
    }
    // WCSPH: NS + density/pressure (fused), forces + integrate into staging;
    // one graph per step (at 27 k particles the step is launch-bound)
    for (int s = 0; s < nsteps; ++s) {
        if (!h->in_staging) stage_from_sorted(h, h->cap);
        const bool last = s == nsteps - 1;
        if (h->use_graphs && !h->prof.on) {
            cudaGraphExec_t ex;
            int r = last ? graph_for(h, 4 << 12, &ex, wc_graph_build)
                         : graph_for(h, (4 << 12) | 1, &ex, wc_graph_build_nostats);
            if (r) return r;
            CK(cudaGraphLaunch(ex, h->stream));
        } else {
            int r = enq_wc_step(h, false, last);
            if (r) return r;
            prof_collect(h);
        }
        h->ep_acc = h->ep_loop = ++h->sorts;
        h->in_staging = true;
        h->ns_valid = false;
        h->frame++;
    }
    return 0;
}

// host-order gather helpers
int download_gid(sphgpu_scene* h, std::vector<int>& gid, int& n, bool staging) {
    CK(cudaStreamSynchronize(h->stream));
    n = h->h_stats->n_active;
    gid.resize(n);
    if (n) CK(copy_sync(gid.data(), staging ? h->d.gid_s : h->d.gid, sizeof(int) * n, cudaMemcpyDeviceToHost));
    return 0;
}

// order[k] = sorted slot holding the k-th particle in reference order
void ref_order(const std::vector<int>& gid, std::vector<int>& order) {
    order.resize(gid.size());
    std::iota(order.begin(), order.end(), 0);
    std::sort(order.begin(), order.end(), [&](int a, int b) { return gid[a] < gid[b]; });
}

}  // namespace

// ---- dynamic rigid solids ----
namespace {
// with a dynamic solid the boundary is re-sorted every step: refresh the
// host copies of its order (reference index and solid of each sorted slot)
int sync_boundary_order(sphgpu_scene* h) {
    if (!h->R.nd || !h->nb) return 0;
    CK(cudaStreamSynchronize(h->stream));
    CK(copy_sync(h->bgid_h.data(), h->d.bgid, sizeof(int) * h->nb, cudaMemcpyDeviceToHost));
    CK(copy_sync(h->bsolid_h.data(), h->d.bsid, sizeof(int) * h->nb, cudaMemcpyDeviceToHost));
    return 0;
}

int dyn_index(sphgpu_scene* h, int solid_id) {
    for (size_t i = 0; i < h->dyn_ids.size(); ++i)
        if (h->dyn_ids[i] == solid_id) return (int)i;
    return -1;
}

// device arrays for the dynamic-solid path, on first use: the boundary in
// reference order (world positions, static volumes), sort scratch, records
int rigid_init(sphgpu_scene* h) {
    CK(cudaStreamSynchronize(h->stream));
    if (h->R.x0) return 0;
    DevScene& d = h->d;
    RigidDev& R = h->R;
    const int nb = h->nb;
    R.nb = nb;
    int r = dalloc(h, &R.x0, nb) | dalloc(h, &R.vol, nb) | dalloc(h, &R.dyn, nb) | dalloc(h, &R.sid, nb) |
            dalloc(h, &R.wpos, nb) | dalloc(h, &R.wvel, nb) | dalloc(h, &R.key, nb) | dalloc(h, &R.slot, nb) |
            dalloc(h, &R.tmp, nb) | dalloc(h, &R.cnt, (size_t)h->g.nkeys + 1) | dalloc(h, &R.binv, nb) |
            dalloc(h, &R.partial, 6 * ((size_t)nb / 4 + 2)) | dalloc(h, &d.bforce, nb) | dalloc(h, &d.bks, nb);
    float4* bpf = nullptr;
    r |= dalloc(h, &bpf, 2 * (size_t)nb);
    if (!d.bsid) r |= dalloc(h, &d.bsid, nb);
    if (r) return SPHGPU_ENOMEM;
    d.bpf = bpf;
    // reference order from the sorted walls
    std::vector<float4> bp(nb), x0(nb);
    std::vector<float> vol(nb);
    std::vector<int> dyn(nb, -1), sid(nb);
    CK(copy_sync(bp.data(), d.bpos, sizeof(float4) * nb, cudaMemcpyDeviceToHost));
    for (int q = 0; q < nb; ++q) {
        const int k = h->bgid_h[q];
        x0[k] = make_float4(bp[q].x, bp[q].y, bp[q].z, 0.f);
        vol[k] = bp[q].w;
        sid[k] = h->bsolid_h[q];
    }
    CK(copy_sync(R.x0, x0.data(), sizeof(float4) * nb, cudaMemcpyHostToDevice));
    CK(copy_sync(R.vol, vol.data(), sizeof(float) * nb, cudaMemcpyHostToDevice));
    CK(copy_sync(R.dyn, dyn.data(), sizeof(int) * nb, cudaMemcpyHostToDevice));
    CK(copy_sync(R.sid, sid.data(), sizeof(int) * nb, cudaMemcpyHostToDevice));
    CK(copy_sync(d.bsid, h->bsolid_h.data(), sizeof(int) * nb, cudaMemcpyHostToDevice));
    CK(memset_sync(d.bforce, 0, sizeof(float4) * nb));
    return 0;
}

// per-solid arrays with room for n dynamic solids
int rigid_reserve(sphgpu_scene* h, int n) {
    if (n <= h->rigid_cap) return 0;
    const int cap = std::max(n, std::max(8, 2 * h->rigid_cap));
    RigidDev& R = h->R;
    float* st = nullptr;
    double* out = nullptr;
    unsigned* tk = nullptr;
    float* hst = nullptr;
    double* hout = nullptr;
    if (dalloc(h, &st, 25 * (size_t)cap) || dalloc(h, &out, 6 * (size_t)cap) || dalloc(h, &tk, cap))
        return SPHGPU_ENOMEM;
    if (cudaMallocHost((void**)&hst, sizeof(float) * 25 * cap) != cudaSuccess ||
        cudaMallocHost((void**)&hout, sizeof(double) * (6 * cap + 1)) != cudaSuccess)
        return SPHGPU_ENOMEM;
    memset(hst, 0, sizeof(float) * 25 * cap);
    memset(hout, 0, sizeof(double) * (6 * cap + 1));
    CK(memset_sync(tk, 0, sizeof(unsigned) * cap));
    CK(memset_sync(out, 0, sizeof(double) * 6 * cap));
    if (h->h_rstate) memcpy(hst, h->h_rstate, sizeof(float) * 25 * h->rigid_cap);
    if (h->h_rout) memcpy(hout, h->h_rout, sizeof(double) * 6 * h->rigid_cap);
    if (R.state) cudaFree(R.state);
    if (R.out) cudaFree(R.out);
    if (R.ticket) cudaFree(R.ticket);
    if (h->h_rstate) cudaFreeHost(h->h_rstate);
    if (h->h_rout) cudaFreeHost(h->h_rout);
    R.state = st;
    R.out = out;
    R.ticket = tk;
    h->h_rstate = hst;
    h->h_rout = hout;
    h->rigid_cap = cap;
    return 0;
}
}  // namespace

// ======================= C ABI =======================
extern "C" {

int sphgpu_abi_version(void) { return SPHGPU_ABI_VERSION; }

int sphgpu_params_default(SphParams* p) {
    if (!p) return SPHGPU_EINVAL;
    memset(p, 0, sizeof(*p));
    // SphBase::SphBase (SphBase.cpp:214-225), DFSPH/WcSph constructors
    p->spacing_r = 0.1f;
    p->smoothRadius_h = 0.2f;
    p->particle_d = 0.1f;
    p->dt = 0.001f;
    p->gravity[1] = -9.8f;
    for (int i = 0; i < 3; ++i) { p->spaceMin[i] = 0.f; p->spaceMax[i] = 1.f; }
    p->soundSpeed_cs = 100.f;
    p->nu = 0.f;
    p->densityErro_eta = 0.01f;
    p->boundary_visc = 0.f;
    p->max_neighbours = 48;
    p->df_density_goal = 1e-4;
    p->df_density_min_iter = 2;
    p->df_density_max_iter = 100;
    p->df_div_goal_abs = 2.5;
    p->df_div_goal_rel = 1e-3;
    p->df_div_min_iter = 1;
    p->df_div_max_iter = 30;
    p->cfl = 0;
    p->cfl_factor = 0.4f;
    p->dt_max = 5e-3f;
    p->dt_min = 1e-6f;
    p->wc_gamma = 7.f;
    p->pci_min_iter = 3;
    p->pci_max_iter = 10;
    p->ii_omega = 0.5f;
    p->ii_eta_rel = 1e-3f;
    p->ii_min_iter = 2;
    p->ii_max_iter = 100;
    p->warm_start = 0;
    p->ws_scale = 1.0f;
    p->iv_kvisc = 0.1f;
    p->iv_kvisc_b = 0.1f;
    p->iv_cv_goal = 1e-4f;
    p->iv_div_goal = 1e-3f;
    p->iv_cv_min_iter = 3;
    p->iv_cv_max_iter = 100;
    p->iv_div_min_iter = 2;
    p->iv_div_max_iter = 50;
    return 0;
}

// One scene (nscenes == 1, box from p) or a batch of nscenes scenes with
// boxes smin/smax[3 * scene]: one grid per scene, key ranges back to back.
static int create_impl(const SphParams* p, int device, int max_fluid, int nscenes, const float* smin,
                       const float* smax, sphgpu_t* out) {
    if (!p || !out || max_fluid <= 0 || nscenes <= 0) return SPHGPU_EINVAL;
    if (p->max_neighbours <= 0 || p->max_neighbours > 128) return SPHGPU_EINVAL;
    if (!(p->smoothRadius_h > 0) || !(p->particle_d > 0) || !(p->spacing_r > 0)) return SPHGPU_EINVAL;
    for (int sc = 0; sc < nscenes; ++sc)
        for (int i = 0; i < 3; ++i) {
            const float lo = nscenes > 1 ? smin[3 * sc + i] : p->spaceMin[i];
            const float hi = nscenes > 1 ? smax[3 * sc + i] : p->spaceMax[i];
            if (!(hi > lo)) return SPHGPU_EINVAL;
        }
    *out = nullptr;
    sphgpu_scene* h = new sphgpu_scene();
    h->P = *p;
    h->device = device;
    if (cudaSetDevice(device) != cudaSuccess) {
        delete h;
        return SPHGPU_ECUDA;
    }
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&h->stream2, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&h->stream3, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&h->stream4, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_out[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_out[1], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_in[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_in[1], cudaEventDisableTiming) != cudaSuccess) {
        delete h;
        return SPHGPU_ECUDA;
    }
    h->cap = max_fluid;
    cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, device);
    h->stride = roundup(max_fluid, 32);
    h->ncap = p->max_neighbours;
    h->nscenes = nscenes;
    if (nscenes == 1) {
        h->g = make_grid(*p);
    } else {
        int off = 0;
        for (int sc = 0; sc < nscenes; ++sc) {
            SphParams q = *p;
            for (int i = 0; i < 3; ++i) { q.spaceMin[i] = smin[3 * sc + i]; q.spaceMax[i] = smax[3 * sc + i]; }
            GridGeom g = make_grid(q);
            g.key0 = off;
            g.key1 = off + g.nkeys - 1;
            off = g.key1;
            h->sgeom.push_back(g);
        }
        h->g = h->sgeom[0];
        h->g.key0 = 0;
        h->g.key1 = off;
        h->g.nkeys = off + 1;  // one key space; its last key holds removed particles
        for (auto& g : h->sgeom) g.nkeys = h->g.nkeys;
    }
    fill_solver_const(h);
    mlp_init_attributes();
    ws_init_attributes();
    int r = alloc_scene(h);
    if (!r && nscenes > 1) {
        // per-scene state: grids, then one block for the BatchDev arrays
        const size_t S = (size_t)nscenes;
        const size_t bytes = S * (sizeof(float) + 9 * sizeof(int) + 3 * sizeof(double)) + 256 + sizeof(int);
        if (cudaMalloc((void**)&h->d_geom, S * sizeof(GridGeom)) != cudaSuccess ||
            cudaMalloc(&h->d_batch, bytes) != cudaSuccess) {
            r = SPHGPU_ENOMEM;
        } else {
            copy_sync(h->d_geom, h->sgeom.data(), S * sizeof(GridGeom), cudaMemcpyHostToDevice);
            memset_sync(h->d_batch, 0, bytes);
            char* q = (char*)h->d_batch;
            BatchDev& b = h->d.b;
            b.err_density = (double*)q; q += S * sizeof(double);
            b.err_div = (double*)q; q += S * sizeof(double);
            b.vmax = (double*)q; q += S * sizeof(double);
            b.dt = (float*)q; q += S * sizeof(float);
            b.active = (int*)q; q += S * sizeof(int);
            b.it_density = (int*)q; q += S * sizeof(int);
            b.it_div = (int*)q; q += S * sizeof(int);
            b.total_it_density = (int*)q; q += S * sizeof(int);
            b.total_it_div = (int*)q; q += S * sizeof(int);
            b.n = (int*)q; q += S * sizeof(int);
            b.sticket = (unsigned*)q; q += S * sizeof(unsigned);
            b.chunk0 = (int*)q; q += (S + 1) * sizeof(int);
            b.status = (unsigned*)q;
            b.geom = h->d_geom;
            std::vector<float> dts(S, p->dt);
            copy_sync(b.dt, dts.data(), S * sizeof(float), cudaMemcpyHostToDevice);
        }
    }
    h->d.nscenes = nscenes;
    if (r) {
        free_scene(h);
        delete h;
        return r;
    }
    *out = h;
    return 0;
}

int sphgpu_create(const SphParams* p, int device, int max_fluid, sphgpu_t* out) {
    return create_impl(p, device, max_fluid, 1, nullptr, nullptr, out);
}

int sphgpu_destroy(sphgpu_t h) {
    if (!h) return SPHGPU_EINVAL;
    cudaSetDevice(h->device);
    cudaStreamSynchronize(h->stream);
    free_scene(h);
    cudaStreamSynchronize(h->stream3);
    cudaStreamSynchronize(h->stream4);
    cudaStreamDestroy(h->stream);
    cudaStreamDestroy(h->stream2);
    cudaStreamDestroy(h->stream3);
    cudaStreamDestroy(h->stream4);
    cudaEventDestroy(h->ev_out[0]);
    cudaEventDestroy(h->ev_out[1]);
    cudaEventDestroy(h->ev_in[0]);
    cudaEventDestroy(h->ev_in[1]);
    delete h;
    return 0;
}

int sphgpu_set_params(sphgpu_t h, const SphParams* p) {
    if (!h || !p) return SPHGPU_EINVAL;
    for (int i = 0; i < 3; ++i)
        if (p->spaceMin[i] != h->P.spaceMin[i] || p->spaceMax[i] != h->P.spaceMax[i]) {
            h->err = "the simulation domain is fixed at creation";
            return SPHGPU_EINVAL;
        }
    if (p->smoothRadius_h != h->P.smoothRadius_h || p->max_neighbours != h->P.max_neighbours) {
        h->err = "smoothRadius_h and max_neighbours are fixed at creation";
        return SPHGPU_EINVAL;
    }
    cudaSetDevice(h->device);
    h->P = *p;
    fill_solver_const(h);
    invalidate_graphs(h);
    float dt = p->dt;
    CK(cudaMemcpyAsync(h->d.dt, &dt, sizeof(float), cudaMemcpyHostToDevice, h->stream));
    if (h->nscenes > 1) {
        std::vector<float> dts(h->nscenes, dt);
        CK(copy_sync(h->d.b.dt, dts.data(), sizeof(float) * h->nscenes, cudaMemcpyHostToDevice));
    }
    CK(cudaStreamSynchronize(h->stream));
    return 0;
}

// Boundary particles of all scenes (scene == NULL: the single scene).
static int set_boundary_impl(sphgpu_t h, int n, const float* xyz, const int* solid_id, const int* scene, const float* volume) {
    if (!h || n < 0 || (n > 0 && !xyz)) return SPHGPU_EINVAL;
    cudaSetDevice(h->device);
    DevScene& d = h->d;
    if (scene)
        for (int i = 0; i < n; ++i)
            if (scene[i] < 0 || scene[i] >= h->nscenes) { h->err = "boundary scene index out of range"; return SPHGPU_EINVAL; }
    free_rigid(h);
    if (d.bpos) { cudaFree(d.bpos); cudaFree(d.bvel); cudaFree(d.bgid); cudaFree(d.bpv); d.bpos = nullptr; }
    for (void* q : {(void*)d.bsid, (void*)d.bnbr, (void*)d.bncount, (void*)d.bivs, (void*)d.bivo})
        if (q) cudaFree(q);
    d.bsid = d.bnbr = d.bncount = nullptr;
    d.bivs = d.bivo = nullptr;
    h->nb = n;
    d.nb = n;
    std::vector<float4> bp(n);
    for (int i = 0; i < n; ++i) bp[i] = make_float4(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], volume ? volume[i] : 0.f);
    if (dalloc(h, &d.bpos, n) || dalloc(h, &d.bvel, n) || dalloc(h, &d.bgid, n) || dalloc(h, &d.bpv, 2 * (size_t)n))
        return SPHGPU_ENOMEM;
    d.bpf = d.bpv;
    // cell keys on the device, each particle with its scene's grid
    std::vector<int> keys(n);
    {
        std::vector<int> ord(n);
        std::iota(ord.begin(), ord.end(), 0);
        if (scene) std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return scene[a] < scene[b]; });
        std::vector<float4> tmp(n);
        for (int i = 0; i < n; ++i) tmp[i] = bp[ord[i]];
        int* dkeys = nullptr;
        if (dalloc(h, &dkeys, n)) return SPHGPU_ENOMEM;
        CK(copy_sync(d.bpos, tmp.data(), sizeof(float4) * n, cudaMemcpyHostToDevice));
        for (int a = 0; a < n;) {
            int b = a;
            const int sc = scene ? scene[ord[a]] : 0;
            while (b < n && (scene ? scene[ord[b]] : 0) == sc) ++b;
            const GridGeom& G = h->nscenes > 1 ? h->sgeom[sc] : h->g;
            launch_boundary_keys(d.bpos + a, b - a, G, dkeys + a, h->stream);
            a = b;
        }
        CK(cudaStreamSynchronize(h->stream));
        std::vector<int> k2(n);
        CK(copy_sync(k2.data(), dkeys, sizeof(int) * n, cudaMemcpyDeviceToHost));
        cudaFree(dkeys);
        for (int i = 0; i < n; ++i) keys[ord[i]] = k2[i];
    }
    // reference insertion rank: solids in order, each in index order (the
    // caller's order, grouped by solid id; in a batch, by scene first)
    std::vector<int> rank(n);
    {
        std::vector<int> ord(n);
        std::iota(ord.begin(), ord.end(), 0);
        std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) {
            const int sa = scene ? scene[a] : 0, sb = scene ? scene[b] : 0;
            if (sa != sb) return sa < sb;
            return solid_id ? solid_id[a] < solid_id[b] : false;
        });
        for (int i = 0; i < n; ++i) rank[ord[i]] = i;
    }
    for (int i = 0; i < n; ++i)
        if (keys[i] < 0) {
            h->err = "boundary particle outside the grid";
            return SPHGPU_EINVAL;
        }
    std::vector<int> perm(n);
    std::iota(perm.begin(), perm.end(), 0);
    std::sort(perm.begin(), perm.end(), [&](int a, int b) {
        return keys[a] != keys[b] ? keys[a] < keys[b] : rank[a] > rank[b];
    });
    std::vector<float4> sp(n), sv(n, make_float4(0, 0, 0, 0));
    h->bgid_h.resize(n);
    h->bsolid_h.resize(n);
    std::vector<int> start(h->g.nkeys + 1, 0);
    for (int i = 0; i < n; ++i) {
        sp[i] = bp[perm[i]];
        h->bgid_h[i] = perm[i];
        h->bsolid_h[i] = solid_id ? solid_id[perm[i]] : 0;
        start[keys[perm[i]] + 1]++;
    }
    for (int k = 0; k < h->g.nkeys; ++k) start[k + 1] += start[k];
    h->iv_multi_solid = 0;
    for (int i = 1; i < n; ++i)
        if (h->bsolid_h[i] != h->bsolid_h[0]) h->iv_multi_solid = 1;
    fill_solver_const(h);
    CK(copy_sync(d.bpos, sp.data(), sizeof(float4) * n, cudaMemcpyHostToDevice));
    CK(copy_sync(d.bvel, sv.data(), sizeof(float4) * n, cudaMemcpyHostToDevice));
    CK(copy_sync(d.bgid, h->bgid_h.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    CK(copy_sync(d.bcell_start, start.data(), sizeof(int) * (h->g.nkeys + 1), cudaMemcpyHostToDevice));
    if (!volume) {
        // each scene's walls with its own grid: its sorted range is contiguous
        for (int sc = 0; sc < h->nscenes; ++sc) {
            const GridGeom& G = h->nscenes > 1 ? h->sgeom[sc] : h->g;
            launch_boundary_volume(d, G, h->P.particle_d, h->c.h2cut, h->ncap, start[G.key0], start[G.key1],
                                   h->stream);
        }
        CK(cudaStreamSynchronize(h->stream));
    }
    // packed {(x, y, z, volume), velocity} records for the sweeps
    if (n) {
        CK(copy2d_sync(d.bpv, 2 * sizeof(float4), d.bpos, sizeof(float4), sizeof(float4), n, cudaMemcpyDeviceToDevice));
        CK(copy2d_sync(d.bpv + 1, 2 * sizeof(float4), d.bvel, sizeof(float4), sizeof(float4), n,
                        cudaMemcpyDeviceToDevice));
    }
    invalidate_graphs(h);
    h->ns_valid = false;
    return 0;
}

int sphgpu_set_boundary(sphgpu_t h, int n, const float* xyz, const int* solid_id, const float* volume) {
    if (h && h->nscenes > 1) { h->err = "a batch takes its walls through sphgpu_batch_set_boundary"; return SPHGPU_EINVAL; }
    return set_boundary_impl(h, n, xyz, solid_id, nullptr, volume);
}

// Append fluid particles: a new phase of the single scene (scene == NULL),
// or, in a batch, particles of the given scenes (all in phase 0; the global
// index order is scene by scene, each scene in the caller's order).
static int add_fluid_impl(sphgpu_t h, int n, const float* xyz, const float* vel, float rho0, float visc_alpha,
                          const int* scene) {
    if (!h || n <= 0 || !xyz || !(rho0 > 0)) return SPHGPU_EINVAL;
    if (!scene && h->rho0_ph.size() >= 4) { h->err = "at most 4 fluid phases"; return SPHGPU_EINVAL; }
    if (scene && !h->rho0_ph.empty() && (h->rho0_ph[0] != rho0 || h->alpha_ph[0] != visc_alpha)) {
        h->err = "the scenes of a batch share one rest density and viscosity";
        return SPHGPU_EINVAL;
    }
    std::vector<int> sord;  // batch: particles grouped by scene, stable
    if (scene) {
        for (int i = 0; i < n; ++i)
            if (scene[i] < 0 || scene[i] >= h->nscenes) { h->err = "scene index out of range"; return SPHGPU_EINVAL; }
        sord.resize(n);
        std::iota(sord.begin(), sord.end(), 0);
        std::stable_sort(sord.begin(), sord.end(), [&](int a, int b) { return scene[a] < scene[b]; });
        if (scene[sord[0]] < h->last_scene) {
            h->err = "batch fluid must be added scene by scene in increasing order";
            return SPHGPU_EINVAL;
        }
    }
    cudaSetDevice(h->device);
    CK(cudaStreamSynchronize(h->stream));
    int cur = h->h_stats->n_active;
    if (cur + n > h->cap) { h->err = "fluid capacity exceeded"; return SPHGPU_EINVAL; }
    int phase = scene ? 0 : (int)h->rho0_ph.size();
    // bring the existing particles into staging in reference order
    std::vector<float4> P(cur + n), V(cur + n);
    std::vector<float4> carried[3];
    for (auto& c4 : carried) c4.assign(cur + n, make_float4(0.f, 0.f, 0.f, 0.f));
    if (cur > 0) {
        std::vector<int> gid;
        int m;
        if (download_gid(h, gid, m, h->in_staging)) return SPHGPU_ECUDA;
        std::vector<float4> tp(m), tv(m);
        CK(copy_sync(tp.data(), h->in_staging ? h->d.pos_s : h->d.pos, sizeof(float4) * m, cudaMemcpyDeviceToHost));
        CK(copy_sync(tv.data(), h->in_staging ? h->d.vel_s : h->d.vel, sizeof(float4) * m, cudaMemcpyDeviceToHost));
        std::vector<int> order;
        ref_order(gid, order);
        for (int k = 0; k < m; ++k) { P[k] = tp[order[k]]; V[k] = tv[order[k]]; }
        // carried PCISPH / IISPH_M state follows its particles
        const float4* srcs[3] = {h->in_staging ? h->d.cA_s : h->d.cA, h->in_staging ? h->d.cB_s : h->d.cB,
                                 h->in_staging ? h->d.cC_s : h->d.cC};
        for (int a = 0; a < 3; ++a) {
            std::vector<float4> t(m);
            CK(copy_sync(t.data(), srcs[a], sizeof(float4) * m, cudaMemcpyDeviceToHost));
            for (int k = 0; k < m; ++k) carried[a][k] = t[order[k]];
        }
    }
    for (int k = 0; k < n; ++k) {
        const int i = scene ? sord[k] : k;
        const int w = phase | (scene ? scene[i] << 4 : 0);
        P[cur + k] = make_float4(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], int_bits_as_float(w));
        V[cur + k] = vel ? make_float4(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2], 0.f) : make_float4(0, 0, 0, 0);
        // a new particle's density is its rest density (as the reference's
        // scene setup leaves it before the first step)
        carried[1][cur + k] = make_float4(0.f, 0.f, 0.f, rho0);
    }
    std::vector<int> G(cur + n);
    std::iota(G.begin(), G.end(), 0);
    CK(copy_sync(h->d.pos_s, P.data(), sizeof(float4) * (cur + n), cudaMemcpyHostToDevice));
    CK(copy_sync(h->d.vel_s, V.data(), sizeof(float4) * (cur + n), cudaMemcpyHostToDevice));
    CK(copy_sync(h->d.gid_s, G.data(), sizeof(int) * (cur + n), cudaMemcpyHostToDevice));
    CK(copy_sync(h->d.cA_s, carried[0].data(), sizeof(float4) * (cur + n), cudaMemcpyHostToDevice));
    CK(copy_sync(h->d.cB_s, carried[1].data(), sizeof(float4) * (cur + n), cudaMemcpyHostToDevice));
    CK(copy_sync(h->d.cC_s, carried[2].data(), sizeof(float4) * (cur + n), cudaMemcpyHostToDevice));
    h->h_stats->n_active = cur + n;
    CK(copy_sync(&h->d.st->n_active, &h->h_stats->n_active, sizeof(int), cudaMemcpyHostToDevice));
    if (!scene || h->rho0_ph.empty()) {
        h->rho0_ph.push_back(rho0);
        h->alpha_ph.push_back(visc_alpha);
        h->phase_n.push_back(n);
    } else {
        h->phase_n[0] += n;
    }
    if (scene) h->last_scene = scene[sord[n - 1]];
    h->n_total = cur + n;
    fill_solver_const(h);
    invalidate_graphs(h);
    h->in_staging = true;
    h->ns_valid = false;
    return phase;
}

int sphgpu_add_fluid(sphgpu_t h, int n, const float* xyz, const float* vel, float rho0, float visc_alpha) {
    if (h && h->nscenes > 1) { h->err = "a batch takes its fluid through sphgpu_batch_add_fluid"; return SPHGPU_EINVAL; }
    return add_fluid_impl(h, n, xyz, vel, rho0, visc_alpha, nullptr);
}

int sphgpu_num_fluid(sphgpu_t h) {
    if (!h) return SPHGPU_EINVAL;
    cudaStreamSynchronize(h->stream);
    return h->h_stats->n_active;
}

int sphgpu_step_async(sphgpu_t h, int solver, int nsteps) {
    if (!h || nsteps < 0) return SPHGPU_EINVAL;
    cudaSetDevice(h->device);
    h->err.clear();
    return enq_steps(h, solver, nsteps);
}

int sphgpu_synchronize(sphgpu_t h, SphStepStats* stats) {
    if (!h) return SPHGPU_EINVAL;
    cudaSetDevice(h->device);
    CK(cudaStreamSynchronize(h->stream));
    CK(cudaGetLastError());
    h->total_removed += h->h_stats->removed;
    fill_stats(h, stats, 0);
    int rc = status_to_rc(h->h_stats->status);
    if (rc == SPHGPU_ENAN) h->err = "non-finite particle state";
    else if (rc == SPHGPU_EMAXITER) h->err = "solver loop reached its iteration cap";
    else if (rc == SPHGPU_EOUT_OF_DOMAIN) h->err = "a dynamic solid left the grid";
    if (h->rigid_fail) {
        h->rigid_fail = 0;
        h->err = "the rigid-body callback failed";
        return SPHGPU_EINVAL;
    }
    return rc;
}

int sphgpu_step(sphgpu_t h, int solver, int nsteps, SphStepStats* stats) {
    int r = sphgpu_step_async(h, solver, nsteps);
    if (r) return r;
    r = sphgpu_synchronize(h, stats);
    if (stats) stats->steps = nsteps;
    return r;
}

// One step from and to host buffers.  When the device holds a sorted state
// with valid lists (a DFSPH step ended there, no particle was ever removed),
// the incoming state is compared with it on the device: velocities are
// copied in, and only if a position differs are the positions staged for a
// new neighbour search -- a caller that hands back the previous step's
// output (the usual loop) pays for the transfers, not for a search.  The
// transfers are stream-ordered, with one host synchronisation for the
// comparison and one at the end.
// The outputs of a host-buffer step after the step was enqueued: the
// velocities (and, unless they left during the step, the positions) in
// reference order.
static int finish_host_step(sphgpu_scene* h, float* vel_out, float* xyz_out, SphStepStats* stats) {
    int r = 0;
    const int n0 = h->out_n;
    float* tv = (float*)h->d.vadv;
    if (h->out_xyz_done) {
        launch_to_ref_order(h->d.vel, h->d.gid, n0, tv, h->stream);
        CK(cudaMemcpyAsync(vel_out, tv, sizeof(float) * 3 * (size_t)n0, cudaMemcpyDeviceToHost, h->stream));
    }
    r = sphgpu_synchronize(h, stats);
    if (stats) stats->steps = 1;
    if (r && r != SPHGPU_EMAXITER) return r;
    if (h->out_xyz_done && h->total_removed == 0) return r;
    int r2 = 0;
    if (h->total_removed == 0 && xyz_out && vel_out) {
        // both outputs reordered on the device, copied out back to back
        DevScene& d = h->d;
        const int n = h->h_stats->n_active;
        const bool stg = h->in_staging;
        float* tx = (float*)d.aux4;
        launch_to_ref_order(stg ? d.pos_s : d.pos, stg ? d.gid_s : d.gid, n, tx, h->stream);
        launch_to_ref_order(stg ? d.vel_s : d.vel, stg ? d.gid_s : d.gid, n, tv, h->stream);
        CK(cudaMemcpyAsync(xyz_out, tx, sizeof(float) * 3 * (size_t)n, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaMemcpyAsync(vel_out, tv, sizeof(float) * 3 * (size_t)n, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        return r;
    }
    if (xyz_out) r2 = sphgpu_get_fluid(h, "position", xyz_out) < 0 ? SPHGPU_ECUDA : 0;
    if (!r2 && vel_out) r2 = sphgpu_get_fluid(h, "velocity", vel_out) < 0 ? SPHGPU_ECUDA : 0;
    return r2 ? r2 : r;
}

int sphgpu_step_host(sphgpu_t h, int solver, const float* xyz, const float* vel, float* xyz_out, float* vel_out,
                     SphStepStats* stats) {
    if (!h) return SPHGPU_EINVAL;
    int r = 0;
    cudaSetDevice(h->device);
    CK(cudaStreamSynchronize(h->stream));
    const bool fast = xyz && vel && solver == SPHGPU_DFSPH && h->total_removed == 0 && !h->in_staging &&
                      h->ns_valid && h->nscenes == 1 && h->R.nd == 0;
    // Speculative form (the common loop: the host hands back the state the
    // last step returned): the step's first part (forces, density loop, the
    // integrated positions) runs on the device state while stream4 copies
    // the host inputs in and compares them with that state bit for bit; part
    // 1 writes no carried per-particle array (the warm start's history is
    // written in part 2, its kappa sum restarts from zero), so when the
    // inputs differ the step is run again from them.
    const bool spec = fast && h->spec && xyz_out && vel_out && h->use_graphs && !h->prof.on &&
                      h->P.enable_vortex == 0 && !h->record_ksum && (!h->mlp || h->ws_mode <= 1);
    const int n_in = h->h_stats->n_active;
    if (spec) {
        DevScene& d = h->d;
        const size_t b3 = sizeof(float) * 3 * (size_t)h->cap;
        if (!h->h_diff) {
            // all four or none: a partial allocation is released again
            if (cudaMalloc((void**)&h->in_xyz, b3) != cudaSuccess ||
                cudaMalloc((void**)&h->in_vel, b3) != cudaSuccess ||
                cudaMalloc((void**)&h->d_diff, sizeof(int)) != cudaSuccess ||
                cudaMallocHost((void**)&h->h_diff, sizeof(int)) != cudaSuccess) {
                for (void* q : {(void*)h->in_xyz, (void*)h->in_vel, (void*)h->d_diff})
                    if (q) cudaFree(q);
                h->in_xyz = h->in_vel = nullptr;
                h->d_diff = nullptr;
                h->h_diff = nullptr;
                cudaGetLastError();  // the failed allocation's error, reported here instead
                h->err = "out of device memory (host-step input buffers)";
                return SPHGPU_ENOMEM;
            }
        }
        cudaStream_t s4 = h->stream4;
        CK(cudaEventRecord(h->ev_in[0], h->stream));
        CK(cudaStreamWaitEvent(s4, h->ev_in[0], 0));
        CK(cudaMemsetAsync(h->d_diff, 0, sizeof(int), s4));
        CK(cudaMemcpyAsync(h->in_xyz, xyz, sizeof(float) * 3 * (size_t)n_in, cudaMemcpyHostToDevice, s4));
        CK(cudaMemcpyAsync(h->in_vel, vel, sizeof(float) * 3 * (size_t)n_in, cudaMemcpyHostToDevice, s4));
        launch_state_check(h->in_xyz, h->in_vel, d.gid, n_in, d.pos, d.vel, h->d_diff, s4);
        CK(cudaMemcpyAsync(h->h_diff, h->d_diff, sizeof(int), cudaMemcpyDeviceToHost, s4));
        CK(cudaEventRecord(h->ev_in[1], s4));
        h->spec_pending = true;
        h->spec_failed = false;
        h->out_xyz = xyz_out;
        h->out_n = n_in;
        h->out_xyz_done = false;
        r = sphgpu_step_async(h, solver, 1);
        h->out_xyz = nullptr;
        const bool checked = !h->spec_pending;
        h->spec_pending = false;
        if (!checked) CK(cudaStreamSynchronize(s4));  // the step did not take the two-graph path
        if (r) return r;
        if (h->spec_failed || (!checked && *h->h_diff)) {
            // the host state differs: back to the state the step started
            // from (part 1 changed no carried array; the kappa sum restarts)
            h->spec_failed = false;
            CK(cudaStreamSynchronize(h->stream));
            CK(cudaStreamSynchronize(h->stream3));
            if (!checked) {
                h->err = "host step: inputs differ after a step that was not speculative";
                return SPHGPU_ECUDA;
            }
            if (h->mlp && h->ws_mode == 1) CK(cudaMemsetAsync(d.ksum, 0, sizeof(float) * h->cap, h->stream));
        } else {
            return finish_host_step(h, vel_out, xyz_out, stats);
        }
    }
    if (fast) {
        DevScene& d = h->d;
        const int n = n_in;
        float* tx = (float*)d.aux4;
        float* tv = (float*)d.vadv;
        if (spec) {
            // the inputs are on the device already
            tx = h->in_xyz;
            tv = h->in_vel;
        } else {
            CK(cudaMemcpyAsync(tx, xyz, sizeof(float) * 3 * (size_t)n, cudaMemcpyHostToDevice, h->stream));
            CK(cudaMemcpyAsync(tv, vel, sizeof(float) * 3 * (size_t)n, cudaMemcpyHostToDevice, h->stream));
        }
        CK(cudaMemsetAsync(&d.st->cont, 0, sizeof(int), h->stream));
        launch_state_in(tx, tv, d.gid, n, d.pos, d.vel, d.prv, &d.st->cont, h->stream);
        CK(cudaMemcpyAsync(h->h_cont, &d.st->cont, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        if (*h->h_cont) {
            // a position changed: the sorted state is staged and searched again
            launch_from_ref_order(tx, d.gid, n, d.pos, h->stream);
            h->ns_valid = false;
            stage_from_sorted(h, n);
            h->in_staging = true;
        }
    } else {
        if (xyz && (r = sphgpu_set_fluid(h, "position", xyz)) < 0) return r;
        if (vel && (r = sphgpu_set_fluid(h, "velocity", vel)) < 0) return r;
    }
    // With both outputs wanted and nothing removed so far, a graph-run DFSPH
    // step copies the integrated positions out (in reference order) while
    // its neighbour search and divergence loop run, and the velocities are
    // reordered and queued behind the step before the host waits.
    const int n0 = h->h_stats->n_active;
    const bool overlap = fast && xyz_out && vel_out && !h->in_staging;
    h->out_xyz = overlap ? xyz_out : nullptr;
    h->out_n = n0;
    h->out_xyz_done = false;
    r = sphgpu_step_async(h, solver, 1);
    h->out_xyz = nullptr;
    if (r) return r;
    return finish_host_step(h, vel_out, xyz_out, stats);
}

int sphgpu_get_fluid(sphgpu_t h, const char* field, float* out) {
    if (!h || !field || !out) return SPHGPU_EINVAL;
    cudaSetDevice(h->device);
    std::string f(field);
    bool state = (f == "position" || f == "velocity");
    bool staging = state && h->in_staging;
    if (state && h->total_removed == 0) {
        // device-side reorder into reference order, one copy out
        CK(cudaStreamSynchronize(h->stream));
        int n = h->h_stats->n_active;
        const float4* src = f == "position" ? (staging ? h->d.pos_s : h->d.pos) : (staging ? h->d.vel_s : h->d.vel);
        float* tmp3 = (float*)h->d.aux4;
        launch_to_ref_order(src, staging ? h->d.gid_s : h->d.gid, n, tmp3, h->stream);
        CK(cudaMemcpyAsync(out, tmp3, sizeof(float) * 3 * (size_t)n, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        return n;
    }
    if (f == "phase" || f == "scene") {
        // fluid phase (or batch scene) index of each particle, as floats
        std::vector<int> gid;
        int n;
        if (download_gid(h, gid, n, h->in_staging)) return SPHGPU_ECUDA;
        std::vector<int> order;
        ref_order(gid, order);
        std::vector<float4> t(n);
        CK(copy_sync(t.data(), h->in_staging ? h->d.pos_s : h->d.pos, sizeof(float4) * n, cudaMemcpyDeviceToHost));
        for (int k = 0; k < n; ++k) {
            int w;
            memcpy(&w, &t[order[k]].w, sizeof w);
            out[k] = (float)(f == "phase" ? (w & 15) : (w >> 4));
        }
        return n;
    }
    std::vector<int> gid;
    int n;
    if (download_gid(h, gid, n, staging)) return SPHGPU_ECUDA;
    std::vector<int> order;
    ref_order(gid, order);
    // arrays written before the last sort are read through the order the
    // integration staged (gid_s): order[k] becomes the slot the k-th particle
    // held then
    const bool acc_group = f == "acce_adv" || f == "acceleration" || f == "advectionAcceleration" ||
                           (f == "acce_presure" && h->last_solver != SPHGPU_IISPH);
    const bool vort_group = f == "omega" || f == "deltaVorticity" || f == "dOmega" || f == "psi";
    const bool loop_group = f == "DFkappa" || f == "kappa_sum" || f == "kappa_warm" || f == "density_adv" ||
                            f == "ws_features" || f == "VF_kappa" || f == "VF_advectionVolume";
    const long ep = acc_group ? h->ep_acc : (loop_group ? h->ep_loop : (vort_group ? h->ep_vort : h->sorts));
    if (!staging && ep == h->sorts - 1) {
        const int ns = h->h_stats->pad0;
        std::vector<int> gs(ns);
        if (ns) CK(copy_sync(gs.data(), h->d.gid_s, sizeof(int) * ns, cudaMemcpyDeviceToHost));
        int mx = 0;
        for (int v : gs) mx = std::max(mx, v);
        for (int v : gid) mx = std::max(mx, v);
        std::vector<int> inv((size_t)mx + 1, -1);
        for (int i = 0; i < ns; ++i) inv[gs[i]] = i;
        for (int k = 0; k < n; ++k) {
            const int o = inv[gid[order[k]]];
            if (o < 0) { h->err = "field " + f + " has no value for a particle of the last sort"; return SPHGPU_EINVAL; }
            order[k] = o;
        }
    }
    int comps = 1;
    const void* src = nullptr;
    bool f4 = false;
    DevScene& d = h->d;
    if (f == "position") { src = staging ? d.pos_s : d.pos; f4 = true; comps = 3; }
    else if (f == "velocity") { src = staging ? d.vel_s : d.vel; f4 = true; comps = 3; }
    else if (f == "vel_adv") {
        CK(copy2d_sync(d.vadv, sizeof(float4), d.pv + 1, 2 * sizeof(float4), sizeof(float4), n,
                        cudaMemcpyDeviceToDevice));
        src = d.vadv;
        f4 = true;
        comps = 3;
    }
    else if (f == "acce_adv" || f == "acceleration" || (f == "acce_presure" && h->last_solver != SPHGPU_IISPH) ||
             f == "advectionAcceleration") {
        src = d.acc;
        f4 = true;
        comps = 3;
    }
    else if (f == "acce_presure") { src = d.ap; f4 = true; comps = 3; }
    // DFSPH vorticity options' vectors (see sph_vortex.cu)
    else if (f == "omega" || f == "deltaVorticity") { src = d.vA; f4 = true; comps = 3; }
    else if (f == "dOmega" || f == "psi") { src = d.vB; f4 = true; comps = 3; }
    else if (f == "angular_velocity" || f == "n0Vorticity") { src = d.cA; f4 = true; comps = 3; }
    else if (f == "advectionVelocity") {
        CK(copy2d_sync(d.vadv, sizeof(float4), d.pv + 1, 2 * sizeof(float4), sizeof(float4), n,
                        cudaMemcpyDeviceToDevice));
        src = d.vadv;
        f4 = true;
        comps = 3;
    }
    else if (f == "sphDensity" || f == "VF_gamma" || f == "VF_sphVolume" || f == "VF_alpha") {
        std::vector<float4> t(n);
        CK(copy_sync(t.data(), d.ivs, sizeof(float4) * n, cudaMemcpyDeviceToHost));
        for (int k = 0; k < n; ++k) {
            const float4& v = t[order[k]];
            out[k] = f == "VF_gamma" ? v.x : (f == "VF_sphVolume" ? v.y : (f == "VF_alpha" ? v.z : v.w));
        }
        return n;
    }
    else if (f == "VF_kappa") src = d.kappa;
    else if (f == "VF_kappaV") src = d.kappav;
    else if (f == "VF_advectionVolume") src = d.aux0;
    else if (f == "VF_divergenceDeviation") src = d.aux1;
    else if (f == "acce_pressure") { src = d.ap; f4 = true; comps = 3; }
    else if (f == "pos_prediction") { src = d.aux4; f4 = true; comps = 3; }
    else if (f == "dii") { src = d.cB; f4 = true; comps = 3; }
    else if (f == "sum_dijpj") { src = d.cC; f4 = true; comps = 3; }
    else if (f == "ii_vel_adv") { src = d.cA; f4 = true; comps = 3; }
    else if (f == "ws_features") {
        // normalised BF16 network inputs of the last warm-start step (n*16)
        if (!h->xn) { h->err = "no learned warm start attached"; return SPHGPU_EINVAL; }
        std::vector<__nv_bfloat16> t((size_t)n * MLP_IN);
        CK(copy_sync(t.data(), h->xn, sizeof(__nv_bfloat16) * t.size(), cudaMemcpyDeviceToHost));
        for (int k = 0; k < n; ++k)
            for (int i = 0; i < MLP_IN; ++i) out[(size_t)k * MLP_IN + i] = __bfloat162float(t[(size_t)order[k] * MLP_IN + i]);
        return n;
    }
    else if (f == "aii" || f == "p_l") {
        std::vector<float4> t(n);
        CK(copy_sync(t.data(), f == "aii" ? d.cC : d.cA, sizeof(float4) * n, cudaMemcpyDeviceToHost));
        for (int k = 0; k < n; ++k) out[k] = t[order[k]].w;
        return n;
    }
    else if (f == "rho_adv") src = d.aux1;
    else if (f == "density") src = d.rho;
    else if (f == "DFalpha") src = d.alpha;
    else if (f == "DFkappa") src = d.kappa;
    else if (f == "DFkappaV") src = d.kappav;
    else if (f == "kappa_sum") src = d.ksum;
    else if (f == "kappa_warm") src = d.kwarm;
    else if (f == "ws_hist") {
        CK(copy2d_sync(d.vadv, sizeof(float4), d.hist, sizeof(float4), sizeof(float4), n, cudaMemcpyDeviceToDevice));
        src = d.vadv;
        f4 = true;
        comps = 3;
    }
    else if (f == "density_adv") src = d.aux0;
    else if (f == "divergenceDeviation") src = d.aux1;
    else if (f == "presure") src = d.kr;
    else if (f == "neighbour_count") {
        std::vector<int> cnt(n);
        CK(copy_sync(cnt.data(), d.ncount, sizeof(int) * n, cudaMemcpyDeviceToHost));
        for (int k = 0; k < n; ++k) out[k] = (float)cnt[order[k]];
        return n;
    } else {
        h->err = "unknown field " + f;
        return SPHGPU_EINVAL;
    }
    if (f4) {
        std::vector<float4> t(n);
        CK(copy_sync(t.data(), src, sizeof(float4) * n, cudaMemcpyDeviceToHost));
        for (int k = 0; k < n; ++k) {
            const float4& v = t[order[k]];
            out[3 * k] = v.x; out[3 * k + 1] = v.y; out[3 * k + 2] = v.z;
        }
    } else {
        std::vector<float> t(n);
        CK(copy_sync(t.data(), src, sizeof(float) * n, cudaMemcpyDeviceToHost));
        for (int k = 0; k < n; ++k) out[k] = t[order[k]];
    }
    (void)comps;
    return n;
}

int sphgpu_set_fluid(sphgpu_t h, const char* field, const float* in) {
    if (!h || !field || !in) return SPHGPU_EINVAL;
    cudaSetDevice(h->device);
    std::string f(field);
    std::vector<int> gid;
    int n;
    bool staging = h->in_staging && (f == "position" || f == "velocity");
    const bool on_device = (f == "position" || f == "velocity") && h->total_removed == 0;
    if (on_device) {
        // reordered on the device: only the count is needed on the host
        CK(cudaStreamSynchronize(h->stream));
        n = h->h_stats->n_active;
    } else if (download_gid(h, gid, n, staging)) {
        return SPHGPU_ECUDA;
    }
    DevScene& d = h->d;
    if (on_device) {
        float4* dst = f == "position" ? (staging ? d.pos_s : d.pos) : (staging ? d.vel_s : d.vel);
        float* tmp3 = (float*)d.aux4;
        CK(cudaMemcpyAsync(tmp3, in, sizeof(float) * 3 * (size_t)n, cudaMemcpyHostToDevice, h->stream));
        launch_from_ref_order(tmp3, staging ? d.gid_s : d.gid, n, dst, h->stream);
        if (!staging) {
            // the sorted arrays are the state: stage them so the next search
            // rebuilds lists, rho/alpha and the packed sweep records
            h->ns_valid = false;
            stage_from_sorted(h, n);
            h->in_staging = true;
        }
        CK(cudaStreamSynchronize(h->stream));
        return n;
    }
    if (f == "position" || f == "velocity") {
        float4* dst = f == "position" ? (staging ? d.pos_s : d.pos) : (staging ? d.vel_s : d.vel);
        std::vector<float4> t(n);
        CK(copy_sync(t.data(), dst, sizeof(float4) * n, cudaMemcpyDeviceToHost));
        std::vector<int> order;
        ref_order(gid, order);
        for (int k = 0; k < n; ++k) {
            float4& v = t[order[k]];
            v.x = in[3 * k]; v.y = in[3 * k + 1]; v.z = in[3 * k + 2];
        }
        CK(copy_sync(dst, t.data(), sizeof(float4) * n, cudaMemcpyHostToDevice));
        if (!staging) {
            // positions changed: lists and rho/alpha must be rebuilt
            h->ns_valid = false;
            // the sorted arrays are the state; stage them for the next sort
            stage_from_sorted(h, n);
            CK(cudaStreamSynchronize(h->stream));
            h->in_staging = true;
        }
        return n;
    }
    if (f == "density") {
        // the density the PCISPH / IISPH_M non-pressure forces read is the
        // carried one (previous step): keep it in step with rho
        bool stg = h->in_staging;
        std::vector<int> g2;
        int n2;
        if (download_gid(h, g2, n2, stg)) return SPHGPU_ECUDA;
        std::vector<int> o2;
        ref_order(g2, o2);
        float4* cb = stg ? d.cB_s : d.cB;
        std::vector<float4> t(n2);
        CK(copy_sync(t.data(), cb, sizeof(float4) * n2, cudaMemcpyDeviceToHost));
        for (int k = 0; k < n2; ++k) t[o2[k]].w = in[k];
        CK(copy_sync(cb, t.data(), sizeof(float4) * n2, cudaMemcpyHostToDevice));
    }
    float* dst = nullptr;
    if (f == "density") dst = d.rho;
    else if (f == "DFalpha") dst = d.alpha;
    else if (f == "kappa_warm") dst = d.kwarm;
    else if (f == "kappa_sum") dst = d.ksum;
    else { h->err = "field not settable: " + f; return SPHGPU_EINVAL; }
    std::vector<int> order;
    ref_order(gid, order);
    std::vector<float> t(n);
    for (int k = 0; k < n; ++k) t[order[k]] = in[k];
    CK(copy_sync(dst, t.data(), sizeof(float) * n, cudaMemcpyHostToDevice));
    if (dst == d.rho && n)  // the force kernel's record carries rho too
        CK(copy2d_sync(reinterpret_cast<char*>(d.prv) + 3 * sizeof(float), 2 * sizeof(float4), d.rho, sizeof(float),
                        sizeof(float), n, cudaMemcpyDeviceToDevice));
    return n;
}

int sphgpu_get_boundary(sphgpu_t h, const char* field, float* out) {
    if (!h || !field || !out) return SPHGPU_EINVAL;
    cudaSetDevice(h->device);
    CK(cudaStreamSynchronize(h->stream));
    int n = h->nb;
    std::vector<float4> t(n);
    CK(copy_sync(t.data(), h->d.bpos, sizeof(float4) * n, cudaMemcpyDeviceToHost));
    std::string f(field);
    if (h->R.nd) {
        if (int r = sync_boundary_order(h)) return r;
        if (f == "velocity" || f == "force" || f == "kerSumFromSelf") {
            if (f == "velocity") {
                std::vector<float4> rec(2 * (size_t)n);
                CK(copy_sync(rec.data(), h->d.bpf, sizeof(float4) * 2 * n, cudaMemcpyDeviceToHost));
                for (int i = 0; i < n; ++i) t[i] = rec[2 * (size_t)i + 1];
            } else if (f == "force") {
                CK(copy_sync(t.data(), h->d.bforce, sizeof(float4) * n, cudaMemcpyDeviceToHost));
            } else {
                std::vector<float> ks(n);
                CK(copy_sync(ks.data(), h->d.bks, sizeof(float) * n, cudaMemcpyDeviceToHost));
                for (int i = 0; i < n; ++i) out[h->bgid_h[i]] = ks[i];
                return n;
            }
            for (int i = 0; i < n; ++i) {
                const int k = h->bgid_h[i];
                out[3 * k] = t[i].x;
                out[3 * k + 1] = t[i].y;
                out[3 * k + 2] = t[i].z;
            }
            return n;
        }
    }
    if (f != "position" && f != "volume") {
        // IISph boundary loop state
        static const char* names[8] = {"VF_gamma", "VF_sphVolume", "VF_alpha", nullptr,
                                       "VF_kappa", "VF_kappaV", "VF_advectionVolume", "VF_divergenceDeviation"};
        int which = -1;
        for (int i = 0; i < 8; ++i)
            if (names[i] && f == names[i]) which = i;
        if (which < 0) { h->err = "unknown boundary field"; return SPHGPU_EINVAL; }
        if (!h->d.bivs) { h->err = "no IISph boundary state (run an IISph step first)"; return SPHGPU_EINVAL; }
        CK(copy_sync(t.data(), which < 4 ? h->d.bivs : h->d.bivo, sizeof(float4) * n, cudaMemcpyDeviceToHost));
        for (int i = 0; i < n; ++i) {
            const float4& v = t[i];
            const int c = which & 3;
            out[h->bgid_h[i]] = c == 0 ? v.x : (c == 1 ? v.y : (c == 2 ? v.z : v.w));
        }
        return n;
    }
    for (int i = 0; i < n; ++i) {
        int k = h->bgid_h[i];
        if (f == "position") { out[3 * k] = t[i].x; out[3 * k + 1] = t[i].y; out[3 * k + 2] = t[i].z; }
        else out[k] = t[i].w;
    }
    return n;
}

int sphgpu_stage(sphgpu_t h, const char* name, SphStepStats* stats) {
    if (!h || !name) return SPHGPU_EINVAL;
    if (h->nscenes > 1) { h->err = "stages are for single scenes"; return SPHGPU_EINVAL; }
    cudaSetDevice(h->device);
    h->err.clear();
    std::string s(name);
    DevScene& d = h->d;
    cudaStream_t st = h->stream;
    int r = 0;
    launch_call_begin(d, st);
    launch_step_begin(d, st);
    if (s == "neighbourSearch" || s == "DF_constantDensitySolverFirst" || s == "wc_computePressure") {
        int mode = s == "wc_computePressure" ? 2 : 1;
        if (h->R.nd && mode != 1) { h->err = "dynamic solids are coupled in the DFSPH step"; return SPHGPU_ENOTIMPL; }
        enq_boundary_update(h, st);
        if (h->in_staging) {
            enq_ns(h, 0, mode, st, h->P.enable_vortex ? 3 : 1);
            ++h->sorts;
            h->in_staging = false;
        } else {
            if (h->R.nd) {
                launch_merge_starts(d, h->g, st);
                launch_rigid_volume(d, h->R, h->g, h->P.particle_d, h->c.h2cut, h->ncap, st);
            }
            launch_build(d, h->g, h->c, mode, h->cap, st);
        }
        h->ns_valid = mode == 1;
    } else if (s == "updateSolids") {
        CK(cudaStreamSynchronize(st));
        run_rigid_callback(h);
    } else if (s == "DF_forceExceptPressure") {
        if (h->in_staging) { h->err = "run neighbourSearch first"; return SPHGPU_EINVAL; }
        launch_df_forces(d, h->c, h->cap, 0, st);
        h->ep_acc = h->sorts;
    } else if (s == "DF_constantDensitySolverSecond") {
        if (h->in_staging) { h->err = "run neighbourSearch first"; return SPHGPU_EINVAL; }
        if (h->P.cfl) launch_cfl(d, h->cap, h->P.cfl_factor, h->P.particle_d, h->P.dt_max, h->P.dt_min, st);
        launch_df_forces(d, h->c, h->cap, 0, st);
        if (h->P.enable_vortex)
            launch_vortex_second(d, h->c, h->P.enable_vortex, h->P.vort_alpha, h->P.vort_zeta, h->P.vort_nu_t,
                                 h->P.spacing_r, h->cap, st);
        if (h->mlp && h->ws_mode == 1) {
            launch_ws_features(d, h->c, h->mlp->m, 1, h->P.dt_max, h->alpha_ref, nullptr, h->xn, h->cap, st);
            launch_ws_infer(d, h->c, h->mlp->m, h->xn, h->cap, h->sm_count, st);
            launch_df_warm_correction(d, h->c, h->cap, st);
        }
        const bool dyn = h->R.nd > 0;
        if (dyn && !(h->mlp && h->ws_mode == 1)) cudaMemsetAsync(d.ksum, 0, sizeof(float) * h->cap, st);
        const int rec = h->record_ksum;
        h->record_ksum = rec || dyn;
        r = enq_df_density_loop(h, false);
        h->record_ksum = rec;
        if (r) return r;
        enq_rigid_forces(h, st);
        if (dyn && h->mlp && h->ws_mode == 1) launch_ws_post(d, h->c, nullptr, h->cap, st);
        // integrate into staging (the reference updates positions in place)
        cudaMemsetAsync(d.cell_count, 0, sizeof(int) * ((size_t)h->g.nkeys + 1), st);
        launch_hash(d, h->g, h->P.enable_vortex ? 3 : 1, h->cap, st);
        h->ep_acc = h->ep_loop = h->sorts;
        if (h->P.enable_vortex == 1 || h->P.enable_vortex == 2) h->ep_vort = h->sorts;
        h->in_staging = true;
        h->ns_valid = false;
    } else if (s == "DF_divergenceFreeSolver") {
        if (h->in_staging) { h->err = "run neighbourSearch first"; return SPHGPU_EINVAL; }
        r = enq_df_div_loop(h, false);
        if (r) return r;
        if (h->P.enable_vortex == 3) {
            launch_vortex_after_div(d, h->c, h->P.spacing_r, h->cap, st);
            h->ep_vort = h->sorts;
        }
    } else if (s == "VF_prepareAttribute") {
        if ((r = ensure_iv_boundary(h))) return r;
        if (h->in_staging) ++h->sorts;
        enq_iv_prepare(h, h->in_staging, st);
        h->in_staging = false;
        h->ns_valid = false;
    } else if (s == "advectionStep" || s == "VF_divergenceFreeSolver" || s == "VF_constantVolumeSolver" ||
               s == "iv_updateFluids") {
        if (h->in_staging || (h->nb > 0 && !d.bivs)) { h->err = "run VF_prepareAttribute first"; return SPHGPU_EINVAL; }
        if (s == "advectionStep") launch_iv_forces(d, h->c, h->cap, h->tune.forces, st);
        else if (s == "iv_updateFluids") {
            launch_iv_integrate(d, h->cap, st);
            h->in_staging = true;
        } else if ((r = enq_iv_loops(h, false, s == "VF_divergenceFreeSolver"))) return r;
        h->ep_acc = h->ep_loop = h->sorts;
    } else if (s == "wc_computeForce") {
        if (h->in_staging) { h->err = "run neighbourSearch first"; return SPHGPU_EINVAL; }
        const bool surf = h->P.th_h != 0.f || h->P.th_r != 0.f || h->P.th_bt != 0.f;
        if (surf) launch_wc_normal(d, h->c, h->cap, st);
        launch_wc_force(d, h->c, h->cap, st, surf, h->c.lanes);
        h->ep_acc = h->sorts;
        h->in_staging = true;
        h->ns_valid = false;
    } else {
        h->err = "unknown stage " + s;
        return SPHGPU_EINVAL;
    }
    CK(cudaMemcpyAsync(h->h_stats, d.st, sizeof(DevStats), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    CK(cudaGetLastError());
    h->total_removed += h->h_stats->removed;
    fill_stats(h, stats, 0);
    return status_to_rc(h->h_stats->status);
}

int sphgpu_get_neighbours(sphgpu_t h, int* counts, int* t, int* idx) {
    if (!h || !counts || !t || !idx) return SPHGPU_EINVAL;
    cudaSetDevice(h->device);
    if (h->in_staging) { h->err = "no neighbour lists (run neighbourSearch)"; return SPHGPU_EINVAL; }
    if (int rs = sync_boundary_order(h)) return rs;
    std::vector<int> gid;
    int n;
    if (download_gid(h, gid, n, false)) return SPHGPU_ECUDA;
    std::vector<int> cnt(n), L((size_t)h->stride * ((h->ncap + 3) / 4) * 4);
    CK(copy_sync(cnt.data(), h->d.ncount, sizeof(int) * n, cudaMemcpyDeviceToHost));
    CK(copy_sync(L.data(), h->d.nbr, sizeof(int) * L.size(), cudaMemcpyDeviceToHost));
    std::vector<float4> pos(n);
    CK(copy_sync(pos.data(), h->d.pos, sizeof(float4) * n, cudaMemcpyDeviceToHost));
    // phase starts in global fluid index space
    std::vector<int> pstart(h->phase_n.size() + 1, 0);
    for (size_t k = 0; k < h->phase_n.size(); ++k) pstart[k + 1] = pstart[k] + h->phase_n[k];
    auto fluid_pidx = [&](int g, int& tt, int& ii) {
        int k = 0;
        while (k + 1 < (int)pstart.size() - 1 && g >= pstart[k + 1]) ++k;
        tt = -(k + 1);
        ii = g - pstart[k];
    };
    // boundary: solid ids and within-solid index
    int ns = 0;
    for (int v : h->bsolid_h) ns = std::max(ns, v + 1);
    std::vector<int> solid_of(h->nb), idx_in_solid(h->nb);
    {
        std::vector<int> sid(h->nb);
        for (int i = 0; i < h->nb; ++i) sid[h->bgid_h[i]] = h->bsolid_h[i];
        std::vector<int> cntS(std::max(ns, 1), 0);
        for (int g = 0; g < h->nb; ++g) { idx_in_solid[g] = cntS[sid[g]]++; solid_of[g] = sid[g]; }
    }
    std::vector<int> order;
    ref_order(gid, order);
    const int cap = h->ncap;
    for (int k = 0; k < n; ++k) {
        int p = order[k];
        counts[k] = cnt[p];
        for (int j = 0; j < cnt[p]; ++j) {
            unsigned e = (unsigned)L[((size_t)(j >> 2) * h->stride + p) * 4 + (j & 3)];
            int tt, ii;
            if (e & BND_FLAG) {
                int g = h->bgid_h[e & BND_MASK];
                tt = solid_of[g] + 1;
                ii = idx_in_solid[g];
            } else {
                fluid_pidx(gid[e], tt, ii);
            }
            t[(size_t)k * cap + j] = tt;
            idx[(size_t)k * cap + j] = ii;
        }
    }
    return cap;
}

int sphgpu_get_cells(sphgpu_t h, long long* cell) {
    if (h && h->nscenes > 1) { h->err = "reference cell indices are for single scenes"; return SPHGPU_EINVAL; }
    if (!h || !cell) return SPHGPU_EINVAL;
    cudaSetDevice(h->device);
    std::vector<float> p(3 * (size_t)std::max(1, h->h_stats->n_active));
    int n = sphgpu_get_fluid(h, "position", p.data());
    if (n < 0) return n;
    // gridOfPos (SphBase.h:700-701) on the host from the same float values;
    // the device computes keys with the identical round-to-nearest ops.
    const GridGeom& g = h->g;
    for (int i = 0; i < n; ++i) {
        int c[3];
        for (int a = 0; a < 3; ++a) {
            volatile float t = p[3 * i + a] - g.min[a];
            volatile float u = t * g.divisor;
            c[a] = (int)u;
        }
        cell[i] = (long long)c[0] + (long long)c[1] * g.num[0] + (long long)c[2] * g.num[0] * g.num[1];
    }
    return n;
}

void* sphgpu_stream(sphgpu_t h) { return h ? (void*)h->stream : nullptr; }

int sphgpu_profile(sphgpu_t h, int enable) {
    if (!h) return SPHGPU_EINVAL;
    h->prof.on = enable != 0;
    h->prof.acc.clear();
    return 0;
}

int sphgpu_profile_read(sphgpu_t h, char* names, int name_len, double* ms, int* launches, int cap) {
    if (!h) return SPHGPU_EINVAL;
    int i = 0;
    for (auto& kv : h->prof.acc) {
        if (i >= cap) break;
        if (names) {
            strncpy(names + (size_t)i * name_len, kv.first.c_str(), name_len - 1);
            names[(size_t)i * name_len + name_len - 1] = 0;
        }
        if (ms) ms[i] = kv.second.first;
        if (launches) launches[i] = kv.second.second;
        ++i;
    }
    return i;
}

int sphgpu_last_error(sphgpu_t h, char* buf, int len) {
    if (!h || !buf || len <= 0) return SPHGPU_EINVAL;
    strncpy(buf, h->err.c_str(), len - 1);
    buf[len - 1] = 0;
    return (int)h->err.size();
}

// ---------------- learned warm start ----------------

int sphgpu_mlp_create(int device, int dataset_cap, uint64_t seed, sphgpu_mlp_t* out) {
    if (!out || dataset_cap < 0) return SPHGPU_EINVAL;
    *out = nullptr;
    if (cudaSetDevice(device) != cudaSuccess) return SPHGPU_ECUDA;
    sphgpu_mlp* m = new sphgpu_mlp();
    m->device = device;
    cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking);
    MlpDev& d = m->m;
    bool ok = cudaMalloc(&d.master, sizeof(float) * MLP_NPARAM_PAD) == cudaSuccess &&
              cudaMalloc(&d.grad, sizeof(float) * MLP_NPARAM_PAD) == cudaSuccess &&
              cudaMalloc(&d.adam_m, sizeof(float) * MLP_NPARAM_PAD) == cudaSuccess &&
              cudaMalloc(&d.adam_v, sizeof(float) * MLP_NPARAM_PAD) == cudaSuccess &&
              cudaMalloc(&d.w_bf16, sizeof(__nv_bfloat16) * MLP_NPARAM_PAD) == cudaSuccess &&
              cudaMalloc(&d.loss, sizeof(float)) == cudaSuccess &&
              cudaMalloc(&d.norm, sizeof(float) * (2 * MLP_IN + 2)) == cudaSuccess &&
              cudaMalloc(&m->ds_count, sizeof(int)) == cudaSuccess &&
              cudaMalloc(&m->dsX, sizeof(float) * MLP_IN * ((size_t)dataset_cap + 1)) == cudaSuccess &&
              cudaMalloc(&m->dsy, sizeof(float) * ((size_t)dataset_cap + 1)) == cudaSuccess;
    if (!ok) {
        sphgpu_mlp_destroy(m);
        return SPHGPU_ENOMEM;
    }
    m->ds_cap = dataset_cap;
    // Xavier-uniform initial weights, zero biases (host RNG, seeded)
    std::vector<float> w(MLP_NPARAM_PAD, 0.f);
    uint64_t x = seed * 6364136223846793005ull + 1442695040888963407ull;
    auto uni = [&]() {
        x ^= x << 13; x ^= x >> 7; x ^= x << 17;
        return (double)(x >> 11) * (1.0 / 9007199254740992.0);
    };
    auto fill = [&](int off, int fan_in, int fan_out) {
        const double a = std::sqrt(6.0 / (fan_in + fan_out));
        for (int i = 0; i < fan_in * fan_out; ++i) w[off + i] = (float)((2 * uni() - 1) * a);
    };
    fill(MLP_OFF_W1, MLP_IN, MLP_H);
    fill(MLP_OFF_W2, MLP_H, MLP_H);
    fill(MLP_OFF_W3, MLP_H, 1);
    std::vector<float> norm(2 * MLP_IN + 2, 0.f);
    for (int i = 0; i < MLP_IN; ++i) norm[MLP_IN + i] = 1.f;
    norm[2 * MLP_IN + 1] = 1.f;
    copy_sync(d.master, w.data(), sizeof(float) * MLP_NPARAM_PAD, cudaMemcpyHostToDevice);
    memset_sync(d.grad, 0, sizeof(float) * MLP_NPARAM_PAD);
    memset_sync(d.adam_m, 0, sizeof(float) * MLP_NPARAM_PAD);
    memset_sync(d.adam_v, 0, sizeof(float) * MLP_NPARAM_PAD);
    copy_sync(d.norm, norm.data(), sizeof(float) * norm.size(), cudaMemcpyHostToDevice);
    memset_sync(m->ds_count, 0, sizeof(int));
    mlp_init_attributes();
    launch_mlp_sync_bf16(d, m->stream);
    if (cudaStreamSynchronize(m->stream) != cudaSuccess) {
        sphgpu_mlp_destroy(m);
        return SPHGPU_ECUDA;
    }
    *out = m;
    return 0;
}

int sphgpu_mlp_destroy(sphgpu_mlp_t m) {
    if (!m) return SPHGPU_EINVAL;
    cudaSetDevice(m->device);
    MlpDev& d = m->m;
    void* ptrs[] = {d.master, d.grad, d.adam_m, d.adam_v, d.w_bf16, d.loss, d.norm, d.gpart, m->ds_count, m->dsX,
                    m->dsy};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (m->stream) cudaStreamDestroy(m->stream);
    delete m;
    return 0;
}

int sphgpu_mlp_set_params(sphgpu_mlp_t m, const float* params) {
    if (!m || !params) return SPHGPU_EINVAL;
    cudaSetDevice(m->device);
    if (copy_sync(m->m.master, params, sizeof(float) * MLP_NPARAM, cudaMemcpyHostToDevice) != cudaSuccess)
        return SPHGPU_ECUDA;
    launch_mlp_sync_bf16(m->m, m->stream);
    return cudaStreamSynchronize(m->stream) == cudaSuccess ? 0 : SPHGPU_ECUDA;
}

int sphgpu_mlp_get_params(sphgpu_mlp_t m, float* params) {
    if (m) cudaDeviceSynchronize();  // written on the network's and on scenes' streams
    if (!m || !params) return SPHGPU_EINVAL;
    cudaSetDevice(m->device);
    return copy_sync(params, m->m.master, sizeof(float) * MLP_NPARAM, cudaMemcpyDeviceToHost) == cudaSuccess
               ? MLP_NPARAM : SPHGPU_ECUDA;
}

int sphgpu_mlp_set_norm(sphgpu_mlp_t m, const float* norm) {
    if (!m || !norm) return SPHGPU_EINVAL;
    cudaSetDevice(m->device);
    return copy_sync(m->m.norm, norm, sizeof(float) * (2 * MLP_IN + 2), cudaMemcpyHostToDevice) == cudaSuccess
               ? 0 : SPHGPU_ECUDA;
}

int sphgpu_mlp_get_norm(sphgpu_mlp_t m, float* norm) {
    if (m) cudaDeviceSynchronize();  // written on the network's and on scenes' streams
    if (!m || !norm) return SPHGPU_EINVAL;
    cudaSetDevice(m->device);
    return copy_sync(norm, m->m.norm, sizeof(float) * (2 * MLP_IN + 2), cudaMemcpyDeviceToHost) == cudaSuccess
               ? 0 : SPHGPU_ECUDA;
}

int sphgpu_mlp_dataset_size(sphgpu_mlp_t m) {
    if (m) cudaDeviceSynchronize();  // written on the network's and on scenes' streams
    if (!m) return SPHGPU_EINVAL;
    cudaSetDevice(m->device);
    int n = 0;
    if (copy_sync(&n, m->ds_count, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return SPHGPU_ECUDA;
    return std::min(n, m->ds_cap);
}

int sphgpu_mlp_dataset_set(sphgpu_mlp_t m, const float* X, const float* y, int n) {
    if (!m || n < 0 || n > m->ds_cap || (n && (!X || !y))) return SPHGPU_EINVAL;
    cudaSetDevice(m->device);
    if (n) {
        if (copy_sync(m->dsX, X, sizeof(float) * MLP_IN * (size_t)n, cudaMemcpyHostToDevice) != cudaSuccess ||
            copy_sync(m->dsy, y, sizeof(float) * n, cudaMemcpyHostToDevice) != cudaSuccess)
            return SPHGPU_ECUDA;
    }
    return copy_sync(m->ds_count, &n, sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess ? 0 : SPHGPU_ECUDA;
}

int sphgpu_mlp_dataset_get(sphgpu_mlp_t m, float* X, float* y, int max_n) {
    if (m) cudaDeviceSynchronize();  // written on the network's and on scenes' streams
    if (!m || max_n < 0) return SPHGPU_EINVAL;
    int n = std::min(sphgpu_mlp_dataset_size(m), max_n);
    if (n < 0) return n;
    if (n && X && copy_sync(X, m->dsX, sizeof(float) * MLP_IN * (size_t)n, cudaMemcpyDeviceToHost) != cudaSuccess)
        return SPHGPU_ECUDA;
    if (n && y && copy_sync(y, m->dsy, sizeof(float) * n, cudaMemcpyDeviceToHost) != cudaSuccess) return SPHGPU_ECUDA;
    return n;
}

// Train for `epochs` passes over the dataset in mini-batches of `batch` rows
// (dataset order; shuffle it first with sphgpu_mlp_dataset_shuffle), Adam at
// learning rate lr.  loss_per_epoch[e] = mean squared error (normalised
// labels) of epoch e.
// per-tile gradient slots for mini-batches of up to `rows` rows
static int mlp_ensure_gpart(sphgpu_mlp_t m, int rows) {
    const int blocks = mlp_train_blocks(rows);
    if (blocks <= m->gpart_blocks) return 0;
    if (m->m.gpart) cudaFree(m->m.gpart);
    m->m.gpart = nullptr;
    m->gpart_blocks = 0;
    if (cudaMalloc(&m->m.gpart, sizeof(float) * ((size_t)blocks * MLP_NPARAM_PAD + blocks)) != cudaSuccess) {
        m->m.gpart = nullptr;
        m->err = "cudaMalloc failed (training gradient slots)";
        return SPHGPU_ENOMEM;
    }
    m->gpart_blocks = blocks;
    return 0;
}

int sphgpu_mlp_train(sphgpu_mlp_t m, int epochs, int batch, float lr, float* loss_per_epoch) {
    if (!m || epochs < 0 || batch <= 0) return SPHGPU_EINVAL;
    cudaSetDevice(m->device);
    const int n = sphgpu_mlp_dataset_size(m);
    if (n <= 0) { m->err = "empty dataset"; return SPHGPU_EINVAL; }
    if (int r = mlp_ensure_gpart(m, std::min(batch, n))) return r;
    for (int e = 0; e < epochs; ++e) {
        cudaMemsetAsync(m->m.loss, 0, sizeof(float), m->stream);
        for (int b0 = 0; b0 < n; b0 += batch) {
            const int bsz = std::min(batch, n - b0);
            launch_mlp_train_batch(m->m, m->dsX, m->dsy, n, b0, bsz, 1.f / (float)bsz, m->stream);
            launch_mlp_adam(m->m, lr, ++m->adam_t, m->stream);
        }
        float l = 0;
        if (cudaMemcpyAsync(&l, m->m.loss, sizeof(float), cudaMemcpyDeviceToHost, m->stream) != cudaSuccess ||
            cudaStreamSynchronize(m->stream) != cudaSuccess)
            return SPHGPU_ECUDA;
        if (loss_per_epoch) loss_per_epoch[e] = l / (float)n;
    }
    return cudaGetLastError() == cudaSuccess ? 0 : SPHGPU_ECUDA;
}

// Shuffle the dataset rows (host permutation from a seeded RNG, device gather).
int sphgpu_mlp_dataset_shuffle(sphgpu_mlp_t m, uint64_t seed) {
    if (!m) return SPHGPU_EINVAL;
    const int n = sphgpu_mlp_dataset_size(m);
    if (n <= 1) return 0;
    std::vector<float> X((size_t)n * MLP_IN), y(n), X2((size_t)n * MLP_IN), y2(n);
    if (sphgpu_mlp_dataset_get(m, X.data(), y.data(), n) != n) return SPHGPU_ECUDA;
    std::vector<int> perm(n);
    std::iota(perm.begin(), perm.end(), 0);
    uint64_t x = seed * 0x9E3779B97F4A7C15ull + 7;
    for (int i = n - 1; i > 0; --i) {
        x ^= x << 13; x ^= x >> 7; x ^= x << 17;
        std::swap(perm[i], perm[(int)(x % (uint64_t)(i + 1))]);
    }
    for (int i = 0; i < n; ++i) {
        memcpy(&X2[(size_t)i * MLP_IN], &X[(size_t)perm[i] * MLP_IN], sizeof(float) * MLP_IN);
        y2[i] = y[perm[i]];
    }
    return sphgpu_mlp_dataset_set(m, X2.data(), y2.data(), n);
}

// Gradient of the mean squared error over (X, y) (host arrays, n rows, one
// mini-batch) w.r.t. the FP32 parameter vector; no update.  For checking the
// backward kernels against a CPU restatement.
int sphgpu_mlp_gradient(sphgpu_mlp_t m, const float* X, const float* y, int n, float* grad, float* loss) {
    if (!m || !X || !y || n <= 0 || !grad) return SPHGPU_EINVAL;
    cudaSetDevice(m->device);
    float *dX = nullptr, *dy = nullptr;
    if (cudaMalloc(&dX, sizeof(float) * MLP_IN * (size_t)n) != cudaSuccess ||
        cudaMalloc(&dy, sizeof(float) * n) != cudaSuccess) {
        cudaFree(dX);
        return SPHGPU_ENOMEM;
    }
    if (int r = mlp_ensure_gpart(m, n)) {
        cudaFree(dX);
        cudaFree(dy);
        return r;
    }
    copy_sync(dX, X, sizeof(float) * MLP_IN * (size_t)n, cudaMemcpyHostToDevice);
    copy_sync(dy, y, sizeof(float) * n, cudaMemcpyHostToDevice);
    cudaMemsetAsync(m->m.grad, 0, sizeof(float) * MLP_NPARAM_PAD, m->stream);
    cudaMemsetAsync(m->m.loss, 0, sizeof(float), m->stream);
    launch_mlp_train_batch(m->m, dX, dy, n, 0, n, 1.f / (float)n, m->stream);
    cudaMemcpyAsync(grad, m->m.grad, sizeof(float) * MLP_NPARAM, cudaMemcpyDeviceToHost, m->stream);
    float l = 0;
    cudaMemcpyAsync(&l, m->m.loss, sizeof(float), cudaMemcpyDeviceToHost, m->stream);
    cudaMemsetAsync(m->m.grad, 0, sizeof(float) * MLP_NPARAM_PAD, m->stream);
    cudaError_t e = cudaStreamSynchronize(m->stream);
    cudaFree(dX);
    cudaFree(dy);
    if (loss) *loss = l / (float)n;
    return e == cudaSuccess ? 0 : SPHGPU_ECUDA;
}

int sphgpu_mlp_predict(sphgpu_mlp_t m, const float* X, float* y, int n) {
    if (!m || !X || !y || n < 0) return SPHGPU_EINVAL;
    if (!n) return 0;
    cudaSetDevice(m->device);
    float *dX = nullptr, *dy = nullptr;
    if (cudaMalloc(&dX, sizeof(float) * MLP_IN * (size_t)n) != cudaSuccess ||
        cudaMalloc(&dy, sizeof(float) * n) != cudaSuccess) {
        cudaFree(dX);
        return SPHGPU_ENOMEM;
    }
    copy_sync(dX, X, sizeof(float) * MLP_IN * (size_t)n, cudaMemcpyHostToDevice);
    launch_mlp_predict(m->m, dX, dy, n, m->stream);
    cudaMemcpyAsync(y, dy, sizeof(float) * n, cudaMemcpyDeviceToHost, m->stream);
    cudaError_t e = cudaStreamSynchronize(m->stream);
    cudaFree(dX);
    cudaFree(dy);
    return e == cudaSuccess ? 0 : SPHGPU_ECUDA;
}

// Attach a network to a scene: mode 0 detaches, 1 applies the learned warm
// start every DFSPH step, 2 records (features, converged stiffness) of every
// `record_every`-th particle of every step into the network's dataset.
int sphgpu_attach_warm_start(sphgpu_t h, sphgpu_mlp_t m, int mode, int record_every) {
    if (!h || mode < 0 || mode > 3 || (mode && !m) || (mode == 2 && record_every <= 0)) return SPHGPU_EINVAL;
    cudaSetDevice(h->device);
    if (mode && m->device != h->device) { h->err = "network and scene on different devices"; return SPHGPU_EINVAL; }
    if (mode == 2 && !h->recX) {
        if (dalloc(h, &h->recX, (size_t)h->cap * MLP_IN) || dalloc(h, &h->recY, (size_t)h->cap)) return SPHGPU_ENOMEM;
    }
    if (mode == 1 && !h->xn) {
        if (dalloc(h, &h->xn, (size_t)h->cap * MLP_IN)) return SPHGPU_ENOMEM;
        cudaMemsetAsync(h->xn, 0, sizeof(__nv_bfloat16) * (size_t)h->cap * MLP_IN, h->stream);
    }
    h->mlp = mode ? m : nullptr;
    h->ws_mode = mode;
    h->ws_every = record_every > 0 ? record_every : 1;
    h->ws_offset = 0;
    cudaMemsetAsync(&h->d.st->pad2, 0, sizeof(int), h->stream);
    h->P.warm_start = mode == 1 || mode == 3;
    if (mode != 1 && mode != 3) cudaMemsetAsync(h->d.kwarm, 0, sizeof(float) * h->cap, h->stream);
    invalidate_graphs(h);
    return cudaStreamSynchronize(h->stream) == cudaSuccess ? 0 : SPHGPU_ECUDA;
}

// ---- autotuner ----
// Measures the DFSPH step kernels at 64, 128 and 256 threads per block on the
// handle's own scene (steps_per_candidate real steps each, timed per kernel
// with CUDA events) and keeps, per kernel class, the fastest block size.
// The scene advances by 3 * steps_per_candidate steps.  report (optional)
// receives a JSON summary.
int sphgpu_autotune(sphgpu_t h, int solver, int steps_per_candidate, char* report, int report_len) {
    if (!h || steps_per_candidate <= 0) return SPHGPU_EINVAL;
    if (solver != SPHGPU_DFSPH) { h->err = "the autotuner covers the DFSPH step"; return SPHGPU_ENOTIMPL; }
    cudaSetDevice(h->device);
    preload_sweep_kernels();
    preload_build_kernels();
    const int cands[3] = {64, 128, 256};
    const char* cls[4] = {"forces", "sweep_a", "sweep_b", "build"};
    double best_t[4] = {1e30, 1e30, 1e30, 1e30};
    int best_b[4] = {128, 128, 128, 128};
    std::string rep = "{\"candidates\": {";
    const bool was_on = h->prof.on;
    for (int ci = 0; ci < 3; ++ci) {
        const int b = cands[ci];
        h->tune.forces = h->tune.sweep_a = h->tune.sweep_b = h->tune.build = b;
        h->prof.on = true;
        h->prof.acc.clear();
        int r = sphgpu_step(h, solver, steps_per_candidate, nullptr);
        if (r < 0 && r != SPHGPU_EMAXITER) { h->prof.on = was_on; return r; }
        auto avg = [&](std::initializer_list<const char*> names) {
            double t = 0;
            int n = 0;
            for (const char* nm : names) {
                auto it = h->prof.acc.find(nm);
                if (it != h->prof.acc.end()) { t += it->second.first; n += it->second.second; }
            }
            return n ? t / n : 1e30;
        };
        const double t[4] = {avg({"df_forces"}), avg({"df_density_a", "df_div_a"}), avg({"df_density_b", "df_div_b"}),
                             avg({"build_first", "build_first_div"})};
        char buf[256];
        snprintf(buf, sizeof buf, "%s\"%d\": {\"forces\": %.2f, \"sweep_a\": %.2f, \"sweep_b\": %.2f, \"build\": %.2f}",
                 ci ? ", " : "", b, 1e3 * t[0], 1e3 * t[1], 1e3 * t[2], 1e3 * t[3]);
        rep += buf;
        for (int k = 0; k < 4; ++k)
            if (t[k] < best_t[k]) { best_t[k] = t[k]; best_b[k] = b; }
    }
    h->prof.on = was_on;
    h->prof.acc.clear();
    h->tune.forces = best_b[0];
    h->tune.sweep_a = best_b[1];
    h->tune.sweep_b = best_b[2];
    h->tune.build = best_b[3];
    invalidate_graphs(h);
    char buf[256];
    snprintf(buf, sizeof buf, "}, \"chosen\": {\"%s\": %d, \"%s\": %d, \"%s\": %d, \"%s\": %d}}", cls[0], best_b[0],
             cls[1], best_b[1], cls[2], best_b[2], cls[3], best_b[3]);
    rep += buf;
    if (report && report_len > 0) {
        strncpy(report, rep.c_str(), report_len - 1);
        report[report_len - 1] = 0;
    }
    return 0;
}

// ---- batch of independent scenes ----
int sphgpu_batch_create(const SphParams* p, int nscenes, const float* space_min, const float* space_max, int device,
                        int max_fluid, sphgpu_t* out) {
    if (nscenes < 1 || !space_min || !space_max) return SPHGPU_EINVAL;
    if (nscenes == 1) {
        SphParams q = *p;
        for (int i = 0; i < 3; ++i) { q.spaceMin[i] = space_min[i]; q.spaceMax[i] = space_max[i]; }
        return create_impl(&q, device, max_fluid, 1, nullptr, nullptr, out);
    }
    return create_impl(p, device, max_fluid, nscenes, space_min, space_max, out);
}

int sphgpu_batch_num_scenes(sphgpu_t h) { return h ? h->nscenes : SPHGPU_EINVAL; }

int sphgpu_batch_set_boundary(sphgpu_t h, int n, const float* xyz, const int* scene) {
    if (!h || (n > 0 && !scene)) return SPHGPU_EINVAL;
    return set_boundary_impl(h, n, xyz, nullptr, h->nscenes > 1 ? scene : nullptr, nullptr);
}

int sphgpu_batch_add_fluid(sphgpu_t h, int n, const float* xyz, const float* vel, const int* scene, float rho0,
                           float visc_alpha) {
    if (!h || (n > 0 && !scene)) return SPHGPU_EINVAL;
    return add_fluid_impl(h, n, xyz, vel, rho0, visc_alpha, h->nscenes > 1 ? scene : nullptr);
}

int sphgpu_batch_stats(sphgpu_t h, SphStepStats* out, int cap) {
    if (!h || !out || cap <= 0) return SPHGPU_EINVAL;
    cudaSetDevice(h->device);
    CK(cudaStreamSynchronize(h->stream));
    if (h->nscenes == 1) {
        fill_stats(h, out, 0);
        return 1;
    }
    const int S = h->nscenes;
    const BatchDev& b = h->d.b;
    std::vector<double> ed(S), ev(S);
    std::vector<float> dt(S);
    std::vector<int> itd(S), itv(S), ttd(S), ttv(S), nn(S);
    std::vector<unsigned> stt(S);
    CK(copy_sync(ed.data(), b.err_density, S * sizeof(double), cudaMemcpyDeviceToHost));
    CK(copy_sync(ev.data(), b.err_div, S * sizeof(double), cudaMemcpyDeviceToHost));
    CK(copy_sync(dt.data(), b.dt, S * sizeof(float), cudaMemcpyDeviceToHost));
    CK(copy_sync(itd.data(), b.it_density, S * sizeof(int), cudaMemcpyDeviceToHost));
    CK(copy_sync(itv.data(), b.it_div, S * sizeof(int), cudaMemcpyDeviceToHost));
    CK(copy_sync(ttd.data(), b.total_it_density, S * sizeof(int), cudaMemcpyDeviceToHost));
    CK(copy_sync(ttv.data(), b.total_it_div, S * sizeof(int), cudaMemcpyDeviceToHost));
    CK(copy_sync(nn.data(), b.n, S * sizeof(int), cudaMemcpyDeviceToHost));
    CK(copy_sync(stt.data(), b.status, S * sizeof(unsigned), cudaMemcpyDeviceToHost));
    const int m = std::min(cap, S);
    for (int i = 0; i < m; ++i) {
        SphStepStats& o = out[i];
        memset(&o, 0, sizeof(o));
        o.n_fluid = nn[i];
        o.iter_density = itd[i];
        o.iter_divergence = itv[i];
        o.err_density = ed[i];
        o.err_divergence = ev[i];
        o.dt = dt[i];
        o.status = stt[i];
        o.total_iter_density = ttd[i];
        o.total_iter_divergence = ttv[i];
    }
    return m;
}

int sphgpu_batch_scene_range(sphgpu_t h, int scene, int* first, int* count) {
    if (!h || scene < 0 || scene >= h->nscenes || !first || !count) return SPHGPU_EINVAL;
    cudaSetDevice(h->device);
    CK(cudaStreamSynchronize(h->stream));
    if (h->nscenes == 1) { *first = 0; *count = h->h_stats->n_active; return 0; }
    std::vector<int> nn(h->nscenes);
    if (h->in_staging && !h->ns_valid && h->frame == 0) {
        // before the first step: counts as added
        std::vector<float4> P(h->h_stats->n_active);
        CK(copy_sync(P.data(), h->d.pos_s, sizeof(float4) * P.size(), cudaMemcpyDeviceToHost));
        std::fill(nn.begin(), nn.end(), 0);
        for (auto& q : P) {
            int w;
            memcpy(&w, &q.w, sizeof w);
            nn[w >> 4]++;
        }
    } else {
        CK(copy_sync(nn.data(), h->d.b.n, sizeof(int) * h->nscenes, cudaMemcpyDeviceToHost));
    }
    int f = 0;
    for (int i = 0; i < scene; ++i) f += nn[i];
    *first = f;
    *count = nn[scene];
    return 0;
}

// Internal controls used by the Python host layer (not part of the
// reference-facing surface): record the summed density-loop stiffness per
// particle (training labels for the warm-start network), and switch CUDA
// graphs off (host-driven loops).

int sphgpu_set_solid_dynamic(sphgpu_t h, int solid_id, const float* inner_xyz, const SphRigidState* state) {
    if (!h || !inner_xyz || !state) return SPHGPU_EINVAL;
    if (h->nscenes > 1) { h->err = "dynamic solids are for single scenes"; return SPHGPU_EINVAL; }
    cudaSetDevice(h->device);
    CK(cudaStreamSynchronize(h->stream));
    if (int rs = sync_boundary_order(h)) return rs;
    // the solid's range in reference order (solids by id, each in insertion order)
    std::vector<int> sid_ref(h->nb);
    for (int q = 0; q < h->nb; ++q) sid_ref[h->bgid_h[q]] = h->bsolid_h[q];
    int r0 = -1, r1 = -1;
    for (int k = 0; k < h->nb; ++k)
        if (sid_ref[k] == solid_id) {
            if (r0 < 0) r0 = k;
            r1 = k + 1;
        }
    if (r0 < 0) { h->err = "no boundary particle has this solid id"; return SPHGPU_EINVAL; }
    int r = rigid_init(h);
    if (r) return r;
    int di = dyn_index(h, solid_id);
    if (di < 0) {
        if ((r = rigid_reserve(h, (int)h->dyn_ids.size() + 1))) return r;
        di = (int)h->dyn_ids.size();
        h->dyn_ids.push_back(solid_id);
        h->dyn_r0.push_back(r0);
        h->dyn_r1.push_back(r1);
    }
    RigidDev& R = h->R;
    R.nd = (int)h->dyn_ids.size();
    const int n = r1 - r0;
    // body-frame positions, keeping kerSumFromSelf in .w
    std::vector<float4> x0(n);
    CK(copy_sync(x0.data(), R.x0 + r0, sizeof(float4) * n, cudaMemcpyDeviceToHost));
    for (int i = 0; i < n; ++i) {
        x0[i].x = inner_xyz[3 * i];
        x0[i].y = inner_xyz[3 * i + 1];
        x0[i].z = inner_xyz[3 * i + 2];
    }
    CK(copy_sync(R.x0 + r0, x0.data(), sizeof(float4) * n, cudaMemcpyHostToDevice));
    std::vector<int> dv(n, di);
    CK(copy_sync(R.dyn + r0, dv.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    memcpy(h->h_rstate + 25 * di, state, sizeof(SphRigidState));
    // SphWithBullet::addSolid: updatePaticles, then prepareSolidPartWeight
    enq_boundary_update(h, h->stream);
    launch_rigid_prepare(h->d, R, h->g, h->P.particle_d, h->c.h2cut, h->ncap, h->stream);
    CK(cudaStreamSynchronize(h->stream));
    CK(cudaGetLastError());
    CK(copy_sync(h->bgid_h.data(), h->d.bgid, sizeof(int) * h->nb, cudaMemcpyDeviceToHost));
    CK(copy_sync(h->bsolid_h.data(), h->d.bsid, sizeof(int) * h->nb, cudaMemcpyDeviceToHost));
    // the fluid lists hold the old boundary order: the next step searches anew
    if (!h->in_staging) stage_from_sorted(h, h->h_stats->n_active);
    h->in_staging = true;
    h->ns_valid = false;
    invalidate_graphs(h);
    return 0;
}

int sphgpu_set_rigid_callback(sphgpu_t h, sphgpu_rigid_fn fn, void* user) {
    if (!h) return SPHGPU_EINVAL;
    h->rigid_fn = fn;
    h->rigid_user = user;
    return 0;
}

int sphgpu_set_solid_state(sphgpu_t h, int solid_id, const SphRigidState* state) {
    if (!h || !state) return SPHGPU_EINVAL;
    const int di = dyn_index(h, solid_id);
    if (di < 0) { h->err = "not a dynamic solid"; return SPHGPU_EINVAL; }
    cudaSetDevice(h->device);
    CK(cudaStreamSynchronize(h->stream));
    memcpy(h->h_rstate + 25 * di, state, sizeof(SphRigidState));
    return 0;
}

int sphgpu_get_solid_state(sphgpu_t h, int solid_id, SphRigidState* state) {
    if (!h || !state) return SPHGPU_EINVAL;
    const int di = dyn_index(h, solid_id);
    if (di < 0) { h->err = "not a dynamic solid"; return SPHGPU_EINVAL; }
    cudaSetDevice(h->device);
    CK(cudaStreamSynchronize(h->stream));
    memcpy(state, h->h_rstate + 25 * di, sizeof(SphRigidState));
    return 0;
}

int sphgpu_get_solid_force(sphgpu_t h, int solid_id, double force[3], double torque[3]) {
    if (!h || !force || !torque) return SPHGPU_EINVAL;
    const int di = dyn_index(h, solid_id);
    if (di < 0) { h->err = "not a dynamic solid"; return SPHGPU_EINVAL; }
    cudaSetDevice(h->device);
    CK(cudaStreamSynchronize(h->stream));
    for (int c = 0; c < 3; ++c) {
        force[c] = h->h_rout[6 * di + c];
        torque[c] = h->h_rout[6 * di + 3 + c];
    }
    return 0;
}

// Test and measurement switches (not part of the drop-in interface):
//   use_graphs             0: host-driven loops, each kernel its own launch
//   record_kappa_sum       sum the density loop's kappa per particle
//   reset_kappa_sum        clear that sum
//   carveout_sweeps/_build preferred L1/shared split of the sweeps / list build
//   l2_policy              L2 eviction priorities of the sweeps' list and record loads
//   fuse_div               DFSPH: the list build runs the divergence loop's first sweep A
//   fuse_ws                warm start: feature gather and network in one kernel
//   speculative_host_step  sphgpu_step_host runs part 1 while checking its inputs
//   wc_lanes               WCSPH threads per particle (0 by size, 1, 4)
int sphgpu_debug_set(sphgpu_t h, const char* key, int value) {
    if (!h || !key) return SPHGPU_EINVAL;
    std::string k(key);
    if (k == "record_kappa_sum") { h->record_ksum = value; invalidate_graphs(h); return 0; }
    if (k == "use_graphs") { h->use_graphs = value != 0; return 0; }
    if (k == "fuse_div") { h->fuse_div = value != 0; invalidate_graphs(h); return 0; }
    if (k == "fuse_ws") { h->fuse_ws = value != 0; invalidate_graphs(h); return 0; }
    if (k == "wc_lanes") {
        if (value != 0 && value != 1 && value != 4) return SPHGPU_EINVAL;
        h->wc_lanes = value;
        fill_solver_const(h);
        invalidate_graphs(h);
        return 0;
    }
    if (k == "speculative_host_step") { h->spec = value != 0; return 0; }
    if (k == "l2_policy") {
        // measurement knob: L2 eviction priorities of the sweeps' list and
        // record loads (SolverConst::l2pol)
        h->l2pol = value & 15;
        fill_solver_const(h);
        invalidate_graphs(h);
        return 0;
    }
    if (k == "carveout_sweeps" || k == "carveout_build") {
        // measurement knob: the kernels' preferred L1/shared split
        cudaSetDevice(h->device);
        if (k == "carveout_sweeps") set_sweep_carveout(value);
        else set_build_carveout(value);
        invalidate_graphs(h);
        return cudaPeekAtLastError() == cudaSuccess ? 0 : SPHGPU_ECUDA;
    }
    if (k == "reset_kappa_sum") {
        cudaMemsetAsync(h->d.ksum, 0, sizeof(float) * h->cap, h->stream);
        return cudaStreamSynchronize(h->stream) == cudaSuccess ? 0 : SPHGPU_ECUDA;
    }
    return SPHGPU_EINVAL;
}

}  // extern "C"

// ======================= output and restart =======================
namespace {

// a float4 field in reference order from the sorted or the staging copy
int ref_order_field(sphgpu_scene* h, const float4* sorted, const float4* staging, std::vector<float4>& out) {
    std::vector<int> gid;
    int n;
    if (download_gid(h, gid, n, h->in_staging)) return SPHGPU_ECUDA;
    std::vector<int> order;
    ref_order(gid, order);
    std::vector<float4> t(n);
    if (n) CK(copy_sync(t.data(), h->in_staging ? staging : sorted, sizeof(float4) * n, cudaMemcpyDeviceToHost));
    out.resize(n);
    for (int k = 0; k < n; ++k) out[k] = t[order[k]];
    return 0;
}

const char SNAP_MAGIC[8] = {'S', 'P', 'H', 'G', 'P', 'U', 'S', '1'};

template <class T>
bool put(FILE* f, const T* p, size_t n) { return n == 0 || fwrite(p, sizeof(T), n, f) == n; }
template <class T>
bool get(FILE* f, T* p, size_t n) { return n == 0 || fread(p, sizeof(T), n, f) == n; }

}  // namespace

extern "C" {

// .pos file of one fluid phase in the reference's format (write_fluid_particles,
// fUtility.h:254-303): four text lines, then per particle the chosen
// components in the reference's fixed order, as float32.
int sphgpu_write_pos(sphgpu_t h, const char* path, int phase, const char* components, const char* log_name) {
    if (!h || !path || phase < 0) return SPHGPU_EINVAL;
    cudaSetDevice(h->device);
    std::string comp = components ? components : "position";
    static const char* order[] = {"position", "velocity", "color", "density", "presure", "acceleration"};
    std::vector<std::string> use;
    for (const char* o : order)
        if (comp.find(o) != std::string::npos) use.push_back(o);
    if (use.empty()) { h->err = "no known component in '" + comp + "'"; return SPHGPU_EINVAL; }
    for (auto& u : use)
        if (u == "color") { h->err = "particle colours are not part of the GPU state"; return SPHGPU_EINVAL; }
    int n = sphgpu_num_fluid(h);
    if (n < 0) return n;
    std::vector<float> ph(n);
    int r = sphgpu_get_fluid(h, "phase", ph.data());
    if (r < 0) return r;
    std::vector<std::vector<float>> cols;
    std::vector<int> width;
    for (auto& u : use) {
        const int w = (u == "density" || u == "presure") ? 1 : 3;
        std::vector<float> v((size_t)n * w);
        const char* f = u.c_str();
        if (u == "density" && h->last_solver == SPHGPU_IISPH) f = "sphDensity";
        if (u == "acceleration") f = h->last_solver == SPHGPU_IISPH ? "acce_presure" : "acceleration";
        if ((r = sphgpu_get_fluid(h, f, v.data())) < 0) return r;
        cols.push_back(std::move(v));
        width.push_back(w);
    }
    std::vector<int> mine;
    for (int i = 0; i < n; ++i)
        if ((int)ph[i] == phase) mine.push_back(i);
    FILE* fo = fopen(path, "wb");
    if (!fo) { h->err = std::string("cannot open ") + path; return SPHGPU_EINVAL; }
    std::string mask = "<";
    for (auto& u : use) mask += " " + u + " ";
    mask += ">";
    fprintf(fo, "for parameters and scene info, please refer to \"%s\"\n", log_name ? log_name : "");
    fprintf(fo, "components writed: %s\n", mask.c_str());
    fprintf(fo, "%d (frame number), fluid index: %d\n", h->frame, phase);
    fprintf(fo, "%zu (num particles)\n", mine.size());
    bool ok = true;
    for (int i : mine)
        for (size_t c = 0; c < cols.size(); ++c) ok = ok && put(fo, &cols[c][(size_t)i * width[c]], width[c]);
    ok = (fclose(fo) == 0) && ok;
    if (!ok) { h->err = std::string("write failed: ") + path; return SPHGPU_EINVAL; }
    return (int)mine.size();
}

// read_fluid_particles (fUtility.h:486-510): the header's component mask and
// frame number, and the packed float32 records
long long sphgpu_read_pos(const char* path, float* out, long long max_floats, char* mask, int mask_len, int* frame) {
    if (!path) return SPHGPU_EINVAL;
    FILE* f = fopen(path, "rb");
    if (!f) return SPHGPU_EINVAL;
    char l1[512], l2[512], l3[512], l4[512];
    if (!fgets(l1, sizeof l1, f) || !fgets(l2, sizeof l2, f) || !fgets(l3, sizeof l3, f) || !fgets(l4, sizeof l4, f)) {
        fclose(f);
        return SPHGPU_EINVAL;
    }
    long long num = atoll(l4);
    std::string m(l2);
    const size_t colon = m.find(':');
    std::string msk = colon == std::string::npos ? m : m.substr(colon + 1);
    while (!msk.empty() && (msk.back() == '\n' || msk.back() == '\r')) msk.pop_back();
    while (!msk.empty() && msk.front() == ' ') msk.erase(msk.begin());
    int per = 0;  // floats per particle (get_part_size, fUtility.h:56-66)
    if (msk.find("position") != std::string::npos) per += 3;
    if (msk.find("velocity") != std::string::npos) per += 3;
    if (msk.find("color") != std::string::npos) per += 4;
    if (msk.find("density") != std::string::npos) per += 1;
    if (msk.find("presure") != std::string::npos) per += 1;
    if (msk.find("acceleration") != std::string::npos) per += 3;
    if (msk.find("dt") != std::string::npos) per += 1;
    if (mask && mask_len > 0) {
        strncpy(mask, msk.c_str(), (size_t)mask_len - 1);
        mask[mask_len - 1] = 0;
    }
    if (frame) *frame = atoi(l3);
    const long long total = num * per;
    if (out) {
        if (total > max_floats) { fclose(f); return SPHGPU_EINVAL; }
        if (!get(f, out, (size_t)total)) { fclose(f); return SPHGPU_EINVAL; }
    }
    fclose(f);
    return num;
}

// Snapshot for checkpoint / resume: parameters, walls, every fluid particle
// with the state the solvers carry between steps, the frame and the clock.
int sphgpu_save_snapshot(sphgpu_t h, const char* path) {
    if (!h || !path) return SPHGPU_EINVAL;
    if (h->nscenes > 1) { h->err = "snapshots are for single scenes"; return SPHGPU_EINVAL; }
    if (h->R.nd) { h->err = "snapshots hold static walls only"; return SPHGPU_EINVAL; }
    cudaSetDevice(h->device);
    CK(cudaStreamSynchronize(h->stream));
    DevScene& d = h->d;
    std::vector<float4> P, V, Hs, A, B, C;
    int r = ref_order_field(h, d.pos, d.pos_s, P);
    if (!r) r = ref_order_field(h, d.vel, d.vel_s, V);
    if (!r) r = ref_order_field(h, d.hist, d.hist_s, Hs);
    if (!r) r = ref_order_field(h, d.cA, d.cA_s, A);
    if (!r) r = ref_order_field(h, d.cB, d.cB_s, B);
    if (!r) r = ref_order_field(h, d.cC, d.cC_s, C);
    if (r) return r;
    const int nb = h->nb;
    std::vector<float4> bp(nb), bref(nb);
    std::vector<int> sid(nb);
    if (nb) CK(copy_sync(bp.data(), d.bpos, sizeof(float4) * nb, cudaMemcpyDeviceToHost));
    for (int i = 0; i < nb; ++i) {
        bref[h->bgid_h[i]] = bp[i];
        sid[h->bgid_h[i]] = h->bsolid_h[i];
    }
    float dt = 0.f;
    CK(copy_sync(&dt, d.dt, sizeof(float), cudaMemcpyDeviceToHost));
    FILE* f = fopen(path, "wb");
    if (!f) { h->err = std::string("cannot open ") + path; return SPHGPU_EINVAL; }
    const int hdr[8] = {SPHGPU_ABI_VERSION, (int)sizeof(SphParams), h->cap, nb, (int)P.size(),
                        (int)h->rho0_ph.size(), h->frame, h->last_solver};
    bool ok = put(f, SNAP_MAGIC, 8) && put(f, hdr, 8) && put(f, &h->P, 1) && put(f, &h->time, 1) && put(f, &dt, 1) &&
              put(f, h->rho0_ph.data(), h->rho0_ph.size()) && put(f, h->alpha_ph.data(), h->alpha_ph.size()) &&
              put(f, bref.data(), nb) && put(f, sid.data(), nb) && put(f, P.data(), P.size()) &&
              put(f, V.data(), V.size()) && put(f, Hs.data(), Hs.size()) && put(f, A.data(), A.size()) &&
              put(f, B.data(), B.size()) && put(f, C.data(), C.size());
    ok = (fclose(f) == 0) && ok;
    if (!ok) { h->err = std::string("write failed: ") + path; return SPHGPU_EINVAL; }
    return 0;
}

int sphgpu_load_snapshot(const char* path, int device, sphgpu_t* out) {
    if (!path || !out) return SPHGPU_EINVAL;
    *out = nullptr;
    FILE* f = fopen(path, "rb");
    if (!f) return SPHGPU_EINVAL;
    char magic[8];
    int hdr[8];
    SphParams P;
    double time = 0;
    float dt = 0;
    bool ok = get(f, magic, 8) && memcmp(magic, SNAP_MAGIC, 8) == 0 && get(f, hdr, 8) &&
              hdr[0] == SPHGPU_ABI_VERSION && hdr[1] == (int)sizeof(SphParams) && get(f, &P, 1) && get(f, &time, 1) &&
              get(f, &dt, 1);
    const int cap = ok ? hdr[2] : 0, nb = ok ? hdr[3] : 0, n = ok ? hdr[4] : 0, nph = ok ? hdr[5] : 0;
    ok = ok && cap > 0 && nb >= 0 && n >= 0 && n <= cap && nph >= 0 && nph <= 4;
    std::vector<float> rho0(nph), alpha(nph);
    std::vector<float4> bref(nb), Pp(n), V(n), Hs(n), A(n), B(n), C(n);
    std::vector<int> sid(nb);
    ok = ok && get(f, rho0.data(), nph) && get(f, alpha.data(), nph) && get(f, bref.data(), nb) &&
         get(f, sid.data(), nb) && get(f, Pp.data(), n) && get(f, V.data(), n) && get(f, Hs.data(), n) &&
         get(f, A.data(), n) && get(f, B.data(), n) && get(f, C.data(), n);
    fclose(f);
    if (!ok) return SPHGPU_EINVAL;
    sphgpu_t h = nullptr;
    int r = sphgpu_create(&P, device, cap, &h);
    if (r) return r;
    std::vector<float> xyz(3 * (size_t)nb), vol(nb);
    for (int i = 0; i < nb; ++i) {
        xyz[3 * i] = bref[i].x; xyz[3 * i + 1] = bref[i].y; xyz[3 * i + 2] = bref[i].z;
        vol[i] = bref[i].w;
    }
    if (nb && (r = sphgpu_set_boundary(h, nb, xyz.data(), sid.data(), vol.data())) < 0) { sphgpu_destroy(h); return r; }
    // phases in order (the reference order is phase-major)
    for (int ph = 0, a = 0; ph < nph; ++ph) {
        int b = a;
        int w;
        while (b < n && (memcpy(&w, &Pp[b].w, sizeof w), (w & 15) == ph)) ++b;
        std::vector<float> px(3 * (size_t)(b - a)), vx(3 * (size_t)(b - a));
        for (int i = a; i < b; ++i) {
            px[3 * (i - a)] = Pp[i].x; px[3 * (i - a) + 1] = Pp[i].y; px[3 * (i - a) + 2] = Pp[i].z;
            vx[3 * (i - a)] = V[i].x; vx[3 * (i - a) + 1] = V[i].y; vx[3 * (i - a) + 2] = V[i].z;
        }
        if (b > a) r = add_fluid_impl(h, b - a, px.data(), vx.data(), rho0[ph], alpha[ph], nullptr);
        else {
            // a phase that lost all its particles keeps its slot and constants
            h->rho0_ph.push_back(rho0[ph]);
            h->alpha_ph.push_back(alpha[ph]);
            h->phase_n.push_back(0);
            fill_solver_const(h);
            r = 0;
        }
        if (r < 0) { sphgpu_destroy(h); return r; }
        a = b;
    }
    // carried per-particle state into the staging arrays (gid = reference index)
    DevScene& d = h->d;
    cudaError_t e = cudaSuccess;
    if (n) {
        e = copy_sync(d.hist_s, Hs.data(), sizeof(float4) * n, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = copy_sync(d.cA_s, A.data(), sizeof(float4) * n, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = copy_sync(d.cB_s, B.data(), sizeof(float4) * n, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = copy_sync(d.cC_s, C.data(), sizeof(float4) * n, cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess) e = copy_sync(d.dt, &dt, sizeof(float), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) { sphgpu_destroy(h); return SPHGPU_ECUDA; }
    h->frame = hdr[6];
    h->last_solver = hdr[7];
    h->time = time;
    *out = h;
    return 0;
}

}  // extern "C"
