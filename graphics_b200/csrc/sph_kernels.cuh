// sph_kernels.cuh -- kernel declarations and the device-side state shared by
// the neighbour-search, DFSPH, WCSPH, PCISPH and IISPH kernels.
#pragma once
#include "sph_common.cuh"

// Device statistics of the current step (one instance per scene, in device
// memory; copied to pinned host memory at the end of each step).
struct DevStats {
    int n_active;          // fluid particles after the last neighbour search
    int it_density;        // iterations of the current/last density loop
    int it_div;            // iterations of the current/last divergence loop
    int removed;           // particles removed this step
    int overflow;          // pairs dropped by the neighbour cap
    int zero_dis;          // zero-distance pairs
    int max_nbrs;          // largest neighbour count
    int cont;              // loop-continue flag (host-driven loops)
    unsigned long long nbr_total;
    unsigned status;
    int total_it_density, total_it_div, steps, pad0;
    double err_density, err_div;
    double vmax;           // FP64 max |v| (CFL)
    float dt;              // current step length
    float pad1;
    unsigned ticket[4];    // last-block tickets of the reductions
    int pad2;              // warm-start recording: sampling offset
    int pad3;
    // PCISPH / IISPH_M loop state
    int pci_emax_bits;     // max relative density error of the iteration (float bits)
    int ii_iter;           // iterations of the current phase's pressure loop
    int ii_num;            // particles of the current phase
    int pad4;
    double ii_sum_cum;     // running sums of the reference's bookkeeping
    double ii_nb_cum;
};

// Per-scene state of a batch (many independent scenes in one set of
// arrays): each scene converges and picks its time step on its own.
struct BatchDev {
    const GridGeom* geom;  // [nscenes] grid of each scene (its key range)
    float* dt;             // [nscenes] step length
    int* active;           // [nscenes] 1 while the scene's current loop runs
    int* it_density;       // [nscenes] iterations of the last density / divergence loop
    int* it_div;
    int* total_it_density; // [nscenes] summed over the steps of the current call
    int* total_it_div;
    int* n;                // [nscenes] active particles
    unsigned* status;      // [nscenes] status bits
    double* err_density;   // [nscenes]
    double* err_div;
    double* vmax;
    // per-scene reductions in chunks of BATCH_CHUNK particles: chunk0[sc]
    // is the scene's first chunk (exclusive prefix, chunk0[nscenes] the
    // total), sticket[sc] counts the scene's finished chunks
    int* chunk0;           // [nscenes + 1]
    unsigned* sticket;     // [nscenes]
};
constexpr int BATCH_CHUNK = 4096;

// Per-scene device pointers passed to every kernel by value.
struct DevScene {
    // fluid, cell-sorted
    float4* pos;
    float4* vel;
    int* gid;
    float* rho;
    float* alpha;
    float4* vadv;       // scratch (reference-order transfers)
    float4* pv;         // 2 per particle: {position, loop velocity} -- the one
                        // 32-byte record the A sweeps gather per neighbour
    float4* pk;         // (x, y, z, kappa/rho) -- the record the B sweeps gather
    float4* prv;        // 2 per particle: {(x, y, z, rho), velocity} -- the record the
                        // DFSPH force kernel gathers (position and rho from the list
                        // build, velocity from the reorder / divergence sweep)
    float4* bpv;        // 2 per boundary particle: {(x,y,z,volume), velocity}
    float4* bpf;        // the record the DFSPH force kernel gathers for a boundary
                        // particle: {(x,y,z,volume), singleVelocity + velocity}
                        // (DFSPH.cpp:1349); the same array as bpv unless a solid
                        // is dynamic (bpv then keeps singleVelocity = 0, which is
                        // what the Jacobi loops read, DFSPH.cpp:615,822)
    float4* acc;        // a_adv (DFSPH) / acceleration (WCSPH) / pressure accel (PCISPH, IISPH)
    float* kr;          // kappa/rho (DFSPH), pressure (WCSPH/PCISPH/IISPH)
    float* kappa;       // DFkappa of the last density iteration
    float* kappav;      // DFkappaV of the last divergence iteration
    float* ksum;        // summed kappa over the density loop (warm-start label)
    float4* vA;         // DFSPH vorticity options: per-particle scratch vectors
    float4* vB;
    float* aux0;        // rho_adv (DFSPH density loop)
    float* aux1;        // divergence deviation (DFSPH), rho_adv (IISPH_M)
    float4* aux4;       // PCISPH predicted position; scratch for transfers
    float* kwarm;       // predicted initial kappa (learned warm start), 0 otherwise
    float4* hist;       // warm-start history: (khat, predicted error, divergence term) of the last step
    float2* wsbuf;      // this step's (predicted error, divergence term)
    // staging (unsorted) copies used by the reorder
    float4* pos_s;
    float4* vel_s;
    int* gid_s;
    float4* hist_s;
    // PCISPH / IISPH_M: carried per-particle state (sorted and staging) and
    // loop scratch
    float4* cA;         // IISPH_M: (v_adv, p_l)
    float4* cB;         // (d_ii, rho); PCISPH: w = rho of the previous step
    float4* cC;         // IISPH_M: (sum_j d_ij p_j, a_ii)
    float4* cA_s;
    float4* cB_s;
    float4* cC_s;
    float4* ap;         // PCISPH pressure acceleration; IISph acce_presure
    float* pl2;         // IISPH_M previous Jacobi iterate
    float4* ivs;        // IISph: (VF_gamma, VF_sphVolume, VF_alpha, sphDensity)
    int* key;
    int* slot;
    int* tmp;
    int* cell_count;    // nkeys + 1
    int* cell_start;    // nkeys + 1
    int2* cstart2;      // nkeys + 1: {fluid start, boundary start} per cell key
    // neighbour lists (ELL, column-major)
    int* nbr;
    int* ncount;
    // boundary, sorted once
    float4* bpos;       // (x, y, z, volume)
    float4* bvel;
    int* bcell_start;   // nkeys + 1
    int* bgid;          // boundary reference index (solid-major)
    int nb;
    // IISph boundary particles: their own per-step neighbour lists (fluid
    // entries, ELL4 with stride bstride) and loop state
    int* bsid;          // solid of each sorted boundary particle
    int* bnbr;
    int* bncount;
    float4* bivs;       // (VF_gamma, VF_sphVolume, VF_alpha, kappa/gamma of the current loop)
    float4* bivo;       // (VF_kappa, VF_kappaV, VF_advectionVolume, VF_divergenceDeviation)
    int bstride;
    // dynamic rigid solids: boundary force of the last DFSPH step and
    // kerSumFromSelf per sorted boundary particle
    float4* bforce;
    float* bks;
    int cap_fluid;      // fluid array capacity
    // reductions
    double* partial;    // >= number of blocks of a particle launch
    DevStats* st;
    float* dt;          // == &st->dt
    // batch of independent scenes (nscenes > 1); scene index in pos.w
    int nscenes;
    BatchDev b;
};

// Dynamic rigid solids (DFSPH): the boundary in reference order (solid by
// solid, each in insertion order), the per-solid rigid states, and the
// scratch of the per-step boundary re-sort and force reduction.
struct RigidDev {
    float4* x0;       // [nb] body-frame position (dynamic solid) or world position
                      // (static solid); w = kerSumFromSelf
    float* vol;       // [nb] current volume
    int* dyn;         // [nb] dense index of the particle's dynamic solid, -1 if static
    int* sid;         // [nb] solid id
    float* state;     // [nd * 25] transform[16] (OpenGL, column-major), com[3],
                      // linear velocity[3], angular velocity[3]
    float4* wpos;     // [nb] placed position (w = kerSumFromSelf)
    float4* wvel;     // [nb] rigid velocity of the placed particle
    int* key;         // [nb] cell key of each placed particle (reference order)
    int* slot;        // [nb] its arrival slot in the cell count
    int* tmp;         // [nb] sorted slot -> reference index, before the in-cell rank
    int* cnt;         // [nkeys + 1] particles per cell key
    int* binv;        // [nb] reference index -> sorted slot
    double* out;      // [nd * 6] joined force and torque of the last step
    double* partial;  // per-block partial sums, 6 per block
    unsigned* ticket; // [nd] last-block tickets
    int nb, nd;
};

// step length of the particle's scene
__device__ __forceinline__ float dt_of(const DevScene& s, float4 pa) {
    return s.nscenes > 1 ? s.b.dt[scene_of(pa)] : *s.dt;
}
// in a batch: is the particle's scene still iterating its current loop?
__device__ __forceinline__ bool scene_active(const DevScene& s, float4 pa) {
    return s.nscenes <= 1 || s.b.active[scene_of(pa)] != 0;
}

// last-block FP64 reduction of per-block partials; returns true in the
// thread that holds the total (thread 0 of the last block).  The partials
// are summed in block order, so the total is the same from run to run.
template <int BS>
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
    __shared__ double sh[BS / 32];
    double acc = 0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += BS) acc += ((volatile double*)partial)[i];
    double tot = block_sum_double<BS>(acc, sh);
    if (threadIdx.x == 0) {
        *total = tot;
        *ticket = 0u;
    }
    return threadIdx.x == 0;
}

// One pair's term of the DFSPH divergence sums, m_j gradW_ij . (v_i - v_j)
// (DFSPH.cpp:589-617, 795-825), accumulated into acc: neighbour j's record
// {pb = (x, y, z, volume or phase), vb = loop velocity}; boundary mass
// rho0 * volume.  The Jacobi sweeps and the list build's fused first
// divergence sweep share it, so both round the same way.
__device__ __forceinline__ float div_term(const SolverConst& c, float4 pa, float4 va, float4 pb, float4 vb, bool bnd,
                                          float acc) {
    const float m = bnd ? c.rho0 * pb.w : c.fm0;
    const float xx = pa.x - pb.x, xy = pa.y - pb.y, xz = pa.z - pb.z;
    const float f = grad_over_r(c.k, xx * xx + xy * xy + xz * xz);
    const float dot = xx * (va.x - vb.x) + xy * (va.y - vb.y) + xz * (va.z - vb.z);
    return fmaf(dot * f, m, acc);
}

// ---- neighbour search (sph_grid.cu) ----
// integrate: bit 0 the DFSPH position update, bit 1 carry cA, bit 2 the
// learned warm start's history from this step's sums (k_ws_post's job)
void launch_hash(const DevScene& s, const GridGeom& g, int integrate, int n_old, cudaStream_t st);
// carry: bit 0 hist, bit 1 cA, bit 2 cB, bit 3 cC (staging -> sorted)
void launch_scatter_reorder(const DevScene& s, const GridGeom& g, int n_old, int carry, cudaStream_t st);
void launch_count_active(const DevScene& s, const GridGeom& g, cudaStream_t st);
// mode 0: lists only; 1: lists + DFSPH rho/alpha; 2: lists + WCSPH rho/pressure;
// 3: lists + IISph VF_prepareAttribute / sphDensity (ivs); 4: mode 1 + the
// divergence loop's first sweep A (Drho/Dt, kappa_v, and for a single scene
// the FP64 error; a batch runs it with each scene's dt)
void launch_build(const DevScene& s, const GridGeom& g, const SolverConst& c, int mode, int n_max, cudaStream_t st,
                  int bs = 128);
void launch_to_ref_order(const float4* src, const int* gid, int n, float* dst3, cudaStream_t st);
void launch_integrated_to_ref(const DevScene& s, int n_max, float* out3, cudaStream_t st);
// host state (reference order) bit for bit against the sorted state: *differs |= 1
void launch_state_check(const float* xyz3, const float* vel3, const int* gid, int n, const float4* pos,
                        const float4* vel, int* differs, cudaStream_t st);
void set_sweep_carveout(int pct);
void set_build_carveout(int pct);
void preload_sweep_kernels();
void preload_build_kernels();
void launch_from_ref_order(const float* src3, const int* gid, int n, float4* dst, cudaStream_t st);
// host state (reference order) into a sorted state with valid lists:
// velocities copied in, *changed set when a position differs
void launch_state_in(const float* xyz3, const float* vel3, const int* gid, int n, const float4* pos, float4* vel,
                     float4* prv, int* changed, cudaStream_t st);
void launch_boundary_keys(const float4* bpos, int nb, const GridGeom& g, int* keys, cudaStream_t st);
// boundary particles [b0, b1) (one scene of a batch, or all)
void launch_boundary_volume(const DevScene& s, const GridGeom& g, float dpart, float h2cut, int cap, int b0, int b1,
                            cudaStream_t st);

// ---- DFSPH (sph_dfsph.cu) ----
// bs: threads per block (64, 128 or 256; the autotuner's choice)
void launch_df_forces(const DevScene& s, const SolverConst& c, int n_max, int warm, cudaStream_t st, int bs = 128);
void launch_df_dens_a(const DevScene& s, const SolverConst& c, int n_max, int record, cudaStream_t st, int bs = 128);
void launch_df_dens_b(const DevScene& s, const SolverConst& c, int n_max, double goal, int min_it, int max_it,
                      unsigned long long cond_handle, int use_handle, cudaStream_t st, int bs = 128);
void launch_df_div_a(const DevScene& s, const SolverConst& c, int n_max, cudaStream_t st, int bs = 128);
void launch_df_div_b(const DevScene& s, const SolverConst& c, int n_max, double goal_abs, double goal_rel,
                     int min_it, int max_it, unsigned long long cond_handle, int use_handle, cudaStream_t st,
                     int bs = 128);
void launch_df_warm_correction(const DevScene& s, const SolverConst& c, int n_max, cudaStream_t st, int bs = 128);
void launch_df_loop_reset(const DevScene& s, int which, cudaStream_t st);
void launch_cfl(const DevScene& s, int n_max, float cfl, float d, float dt_max, float dt_min, cudaStream_t st);
void launch_step_begin(const DevScene& s, cudaStream_t st);
void launch_call_begin(const DevScene& s, cudaStream_t st);

// ---- batch of scenes (sph_batch.cu) ----
void launch_batch_loop_reset(const DevScene& s, int nscenes, int which, cudaStream_t st);
// n_cap: particle capacity (bounds the number of chunks)
void launch_batch_decide(const DevScene& s, const SolverConst& c, int which, int nscenes, int n_cap, double goal_abs,
                         double goal_rel, int min_it, int max_it, unsigned long long cond_handle, int use_handle,
                         cudaStream_t st);
void launch_batch_cfl(const DevScene& s, int nscenes, int n_cap, float cfl, float d, float dt_max, float dt_min,
                      cudaStream_t st);
void launch_batch_call_begin(const DevScene& s, int nscenes, cudaStream_t st);
void launch_batch_count(const DevScene& s, int nscenes, cudaStream_t st);

// ---- WCSPH (sph_wcsph.cu) ----
// surf: with surface tension and adhesion (the normals of launch_wc_normal in vA)
// lanes: threads per particle (1, or 4 for small scenes)
void launch_wc_force(const DevScene& s, const SolverConst& c, int n_max, cudaStream_t st, bool surf = false,
                     int lanes = 1);
void launch_wc_normal(const DevScene& s, const SolverConst& c, int n_max, cudaStream_t st);

// ---- PCISPH / IISPH_M (sph_pci_ii.cu) ----
void launch_pci_force_except(const DevScene& s, const SolverConst& c, int n_max, cudaStream_t st);
void launch_pci_density(const DevScene& s, const SolverConst& c, float delta, int n_max, cudaStream_t st);
void launch_pci_pressure(const DevScene& s, const SolverConst& c, float eta, int min_it, int max_it,
                         unsigned long long cond_handle, int use_handle, int n_max, cudaStream_t st);
void launch_pci_finish(const DevScene& s, int n_max, cudaStream_t st);
void launch_ii_force_except(const DevScene& s, const SolverConst& c, int n_max, cudaStream_t st);
void launch_ii_phase_begin(const DevScene& s, cudaStream_t st);
void launch_ii_density(const DevScene& s, const SolverConst& c, int phase, int n_max, cudaStream_t st);
void launch_ii_aii(const DevScene& s, const SolverConst& c, int phase, int n_max, cudaStream_t st);
void launch_ii_sum(const DevScene& s, const SolverConst& c, int phase, int n_max, cudaStream_t st);
void launch_ii_press(const DevScene& s, const SolverConst& c, int phase, double omega, double eta_rel, int min_it,
                     int max_it, int compat, unsigned long long cond_handle, int use_handle, int n_max,
                     cudaStream_t st);
void launch_ii_force(const DevScene& s, const SolverConst& c, int compat, int n_max, cudaStream_t st);
// ---- IISph, volume form (sph_iisph.cu) ----
// boundary particles' neighbour lists and VF_prepareAttribute terms
void launch_iv_boundary_build(const DevScene& s, const GridGeom& g, const SolverConst& c, int bs, cudaStream_t st);
// advectionStep (gravity + viscosity); loop velocities start from the carried ones
void launch_iv_forces(const DevScene& s, const SolverConst& c, int n_max, int bs, cudaStream_t st);
void launch_iv_phase_begin(const DevScene& s, cudaStream_t st);
// loop velocity of phase `phase`: v (div) or v + a dt (constant volume); counts the phase
void launch_iv_loop_init(const DevScene& s, int phase, int div, int n_max, cudaStream_t st);
void launch_iv_boundary_sweep(const DevScene& s, const SolverConst& c, int div, int bs, cudaStream_t st);
void launch_iv_sweep_a(const DevScene& s, const SolverConst& c, int phase, int div, int n_max, int bs, cudaStream_t st);
void launch_iv_sweep_b(const DevScene& s, const SolverConst& c, int phase, int div, double goal, int min_it,
                       int max_it, unsigned long long cond_handle, int use_handle, int n_max, int bs, cudaStream_t st);
// acce_presure, v += acce_presure dt, x += v dt into the staging arrays (carried: v_adv)
void launch_iv_integrate(const DevScene& s, int n_max, cudaStream_t st);

// ---- DFSPH vorticity options (sph_vortex.cu) ----
// after the non-pressure forces: mode 1 TRRV, 2 micropolar (velocity and
// v_adv refined), 3 the vorticity at the start of the step (into cA)
void launch_vortex_second(const DevScene& s, const SolverConst& c, int mode, float alpha, float zeta, float nu_t,
                          float spacing, int n_max, cudaStream_t st);
// mode 3 after the divergence loop: stream-function correction of the velocity
void launch_vortex_after_div(const DevScene& s, const SolverConst& c, float spacing, int n_max, cudaStream_t st);

// ---- dynamic rigid solids (sph_rigid.cu) ----
// updatePaticles for every dynamic solid, then a counting sort of the whole
// boundary by cell key (within a cell: descending reference index) into the
// sorted arrays and the boundary cell table; scan_tmp / scan_bytes: CUB scan
// scratch for nkeys + 1 entries
void launch_rigid_place_sort(const DevScene& s, const RigidDev& R, const GridGeom& g, void* scan_tmp,
                             size_t scan_bytes, cudaStream_t st);
// prepareSolidPartWeight over the boundary alone: kerSumFromSelf and volume
void launch_rigid_prepare(const DevScene& s, const RigidDev& R, const GridGeom& g, float dpart, float h2cut, int cap,
                          cudaStream_t st);
// updateSolidPartWeight: volume = 1 / (kerSumFromSelf + other solids' terms)
void launch_rigid_volume(const DevScene& s, const RigidDev& R, const GridGeom& g, float dpart, float h2cut, int cap,
                         cudaStream_t st);
// boundary force of dynamic solid di (reference range [r0, r1)) and its
// joined force / torque (FP64)
void launch_rigid_force(const DevScene& s, const RigidDev& R, const SolverConst& c, const GridGeom& g, int r0, int r1,
                        int di, cudaStream_t st);
void launch_merge_starts(const DevScene& s, const GridGeom& g, cudaStream_t st);

// carried state of particles coming from another solver: cB = (0, rho), cA = cC = 0
// (staging: rho = the phase's rest density)
void launch_carry_init(const DevScene& s, const SolverConst& c, int staging, int n_max, cudaStream_t st);
