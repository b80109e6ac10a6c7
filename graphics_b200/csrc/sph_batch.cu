// sph_batch.cu -- many independent DFSPH scenes in one set of arrays.
//
// A batch packs every scene's particles into the same sorted arrays: each
// scene has its own grid (its own box), and the scenes' cell keys occupy
// disjoint ranges [key0, key1) of one key space, so one counting sort per
// step sorts all scenes at once, every scene's particles end up contiguous,
// and no neighbour list crosses scenes.  The sweep kernels are the
// single-scene ones (they read the scene index from pos.w for the scene's
// grid and time step); what is per scene lives here:
//   * the CFL step (FP64 max |v| over the scene's range),
//   * the loop decisions: the FP64 mean of rho_adv (density loop) or of
//     Drho/Dt (divergence loop) over the scene's range, the scene's own
//     iteration count and goal; a scene that has converged stops iterating
//     (its particles are skipped by the sweeps) while the others continue,
//     and the loop (a conditional graph node) runs while any scene is active.
// Each reduction runs over the scenes' contiguous ranges in chunks of
// BATCH_CHUNK particles, one block per chunk (a scene of 200k particles is
// 49 blocks, not one): the chunk's block sums (or maxima) go to partial[],
// the scene's last chunk to finish combines its chunks in chunk order and
// makes the scene's decision, and the last block of all makes the loop's.
// Sums are in a fixed order, so results are run-to-run deterministic.
#include "sph_kernels.cuh"

namespace {
constexpr int NT = 256;

__device__ __forceinline__ void scene_range(const DevScene& s, int sc, int& a, int& b) {
    const GridGeom& G = s.b.geom[sc];
    a = s.cell_start[G.key0];
    b = s.cell_start[G.key1];
}

__global__ void k_batch_call_begin(DevScene s, int nscenes) {
    const int sc = blockIdx.x * blockDim.x + threadIdx.x;
    if (sc >= nscenes) return;
    s.b.total_it_density[sc] = 0;
    s.b.total_it_div[sc] = 0;
    s.b.status[sc] = 0u;
}

// active particles per scene after a neighbour search, and the scenes'
// first chunks (one thread: a prefix over the scenes)
__global__ void k_batch_count(DevScene s, int nscenes) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    int c = 0;
    for (int sc = 0; sc < nscenes; ++sc) {
        int a, b;
        scene_range(s, sc, a, b);
        s.b.n[sc] = b - a;
        s.b.chunk0[sc] = c;
        c += (b - a + BATCH_CHUNK - 1) / BATCH_CHUNK;
    }
    s.b.chunk0[nscenes] = c;
}

// the scene of chunk `bid` (chunk0 ascending; empty scenes have no chunks)
__device__ __forceinline__ int chunk_scene(const DevScene& s, int nscenes, int bid) {
    int lo = 0, hi = nscenes - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (s.b.chunk0[mid] <= bid) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// start of a density (which 0) or divergence (which 1) loop
__global__ void k_batch_loop_reset(DevScene s, int nscenes, int which) {
    const int sc = blockIdx.x * blockDim.x + threadIdx.x;
    if (sc < nscenes) {
        s.b.active[sc] = s.b.n[sc] > 0 ? 1 : 0;
        if (which == 0) s.b.it_density[sc] = 0;
        else s.b.it_div[sc] = 0;
    }
    if (sc == 0) s.st->cont = 1;
}

// which 0: density loop (mean rho_adv, aux0); 1: divergence loop (mean
// Drho/Dt, aux1).  Same rules as the single-scene decisions in
// k_df_vupdate (DFSPH.cpp:566-700, 740-1024 with the FP64 mean and caps).
// One block per chunk of an active scene (grid: an upper bound on the chunks).
__global__ void __launch_bounds__(NT) k_batch_decide(DevScene s, SolverConst c, int which, int nscenes,
                                                     double goal_abs, double goal_rel, int min_it, int max_it,
                                                     cudaGraphConditionalHandle h, int use_handle) {
    const int bid = blockIdx.x;
    __shared__ double sh[NT / 32];
    __shared__ bool last;
    const int total = s.b.chunk0[nscenes];
    const int sc = bid < total ? chunk_scene(s, nscenes, bid) : -1;
    if (sc >= 0 && s.b.active[sc]) {  // uniform over the block
        int a, b;
        scene_range(s, sc, a, b);
        const int k = bid - s.b.chunk0[sc];
        const int c0 = a + k * BATCH_CHUNK, c1 = min(b, c0 + BATCH_CHUNK);
        const float* v = which == 0 ? s.aux0 : s.aux1;
        double acc = 0.0;
        for (int i = c0 + threadIdx.x; i < c1; i += NT) acc += (double)v[i];
        const double part = block_sum_double<NT>(acc, sh);
        if (threadIdx.x == 0) {
            s.partial[bid] = part;
            __threadfence();
            const int nch = s.b.chunk0[sc + 1] - s.b.chunk0[sc];
            last = atomicAdd(&s.b.sticket[sc], 1u) == (unsigned)(nch - 1);
        }
        __syncthreads();
        if (last && threadIdx.x == 0) {
            // the scene's last chunk: its chunks' sums in chunk order
            __threadfence();
            double tot = 0.0;
            for (int q = s.b.chunk0[sc]; q < s.b.chunk0[sc + 1]; ++q) tot += ((volatile double*)s.partial)[q];
            s.b.sticket[sc] = 0u;
            const double n = (double)(b - a);
            bool crit;
            int cont;
            if (which == 0) {
                const int it = ++s.b.it_density[sc];
                ++s.b.total_it_density[sc];
                const double err = (tot / n - (double)c.rho0) / (double)c.rho0;
                s.b.err_density[sc] = err;
                crit = err > goal_rel;
                cont = (crit || it < min_it) && it < max_it;
                if (!cont && crit) s.b.status[sc] |= 1u;
                if (!(err == err)) { cont = 0; s.b.status[sc] |= 4u; }
            } else {
                const int it = ++s.b.it_div[sc];
                ++s.b.total_it_div[sc];
                const double avg = tot / n;
                s.b.err_div[sc] = avg;
                const double dtd = (double)s.b.dt[sc];
                crit = goal_abs > 0 ? (avg > goal_abs) : (avg * dtd / (double)c.rho0 > goal_rel);
                cont = (crit || it < min_it) && it <= max_it;
                if (!cont && crit) s.b.status[sc] |= 2u;
                if (!(avg == avg)) { cont = 0; s.b.status[sc] |= 4u; }
            }
            if (!cont) s.b.active[sc] = 0;
        }
        __syncthreads();
    }
    // the last block to finish decides whether the loop runs again
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(&s.st->ticket[0], 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    int any = 0;
    unsigned st_or = 0u;
    for (int i = threadIdx.x; i < nscenes; i += NT) {
        any |= ((volatile int*)s.b.active)[i];
        st_or |= ((volatile unsigned*)s.b.status)[i];
    }
    any = __syncthreads_or(any);
    __shared__ unsigned sst;
    if (threadIdx.x == 0) sst = 0u;
    __syncthreads();
    if (st_or) atomicOr(&sst, st_or);
    __syncthreads();
    if (threadIdx.x == 0) {
        if (which == 0) ++s.st->it_density;
        else ++s.st->it_div;
        s.st->status |= sst;
        s.st->cont = any;
        s.st->ticket[0] = 0u;
        if (use_handle) cudaGraphSetConditional(h, any ? 1u : 0u);
    }
}

// per-scene CFL step: dt = clamp(cfl * d / max|v|, dt_min, dt_max), FP64
// max over the scene's chunks (the maximum is order-independent)
__global__ void __launch_bounds__(NT) k_batch_cfl(DevScene s, int nscenes, float cfl, float d, float dt_max,
                                                  float dt_min) {
    const int bid = blockIdx.x;
    const int total = s.b.chunk0[nscenes];
    if (bid == 0)  // scenes without particles (no chunks): dt_max
        for (int q = threadIdx.x; q < nscenes; q += NT)
            if (s.b.chunk0[q + 1] == s.b.chunk0[q]) {
                s.b.vmax[q] = 0.0;
                s.b.dt[q] = dt_max;
            }
    if (bid >= total) return;
    const int sc = chunk_scene(s, nscenes, bid);
    int a, b;
    scene_range(s, sc, a, b);
    const int k = bid - s.b.chunk0[sc];
    const int c0 = a + k * BATCH_CHUNK, c1 = min(b, c0 + BATCH_CHUNK);
    double m = 0.0;
    for (int i = c0 + threadIdx.x; i < c1; i += NT) {
        const float4 v = s.vel[i];
        const double x = v.x, y = v.y, z = v.z;
        m = fmax(m, sqrt(x * x + y * y + z * z));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    __shared__ double sh[NT / 32];
    __shared__ bool last;
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double bm = 0.0;
        for (int i = 0; i < NT / 32; ++i) bm = fmax(bm, sh[i]);
        s.partial[bid] = bm;
        __threadfence();
        const int nch = s.b.chunk0[sc + 1] - s.b.chunk0[sc];
        last = atomicAdd(&s.b.sticket[sc], 1u) == (unsigned)(nch - 1);
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        double vmax = 0.0;
        for (int q = s.b.chunk0[sc]; q < s.b.chunk0[sc + 1]; ++q) vmax = fmax(vmax, ((volatile double*)s.partial)[q]);
        s.b.sticket[sc] = 0u;
        double dt = vmax > 0 ? (double)cfl * (double)d / vmax : (double)dt_max;
        if (dt > dt_max) dt = dt_max;
        if (dt < dt_min) dt = dt_min;
        s.b.vmax[sc] = vmax;
        s.b.dt[sc] = (float)dt;
    }
}
}  // namespace

static inline int blocks_for(int n, int nt) { return (n + nt - 1) / nt; }

void launch_batch_call_begin(const DevScene& s, int nscenes, cudaStream_t st) {
    k_batch_call_begin<<<blocks_for(nscenes, 128), 128, 0, st>>>(s, nscenes);
}
void launch_batch_count(const DevScene& s, int nscenes, cudaStream_t st) {
    k_batch_count<<<1, 32, 0, st>>>(s, nscenes);
}
// an upper bound on the chunks of all scenes: sum ceil(n_s / C) <= n / C + scenes
static inline int max_chunks(int n_cap, int nscenes) { return n_cap / BATCH_CHUNK + nscenes + 1; }
void launch_batch_loop_reset(const DevScene& s, int nscenes, int which, cudaStream_t st) {
    k_batch_loop_reset<<<blocks_for(nscenes, 128), 128, 0, st>>>(s, nscenes, which);
}
void launch_batch_decide(const DevScene& s, const SolverConst& c, int which, int nscenes, int n_cap, double goal_abs,
                         double goal_rel, int min_it, int max_it, unsigned long long cond_handle, int use_handle,
                         cudaStream_t st) {
    k_batch_decide<<<max_chunks(n_cap, nscenes), NT, 0, st>>>(s, c, which, nscenes, goal_abs, goal_rel, min_it, max_it,
                                                             (cudaGraphConditionalHandle)cond_handle, use_handle);
}
void launch_batch_cfl(const DevScene& s, int nscenes, int n_cap, float cfl, float d, float dt_max, float dt_min,
                      cudaStream_t st) {
    k_batch_cfl<<<max_chunks(n_cap, nscenes), NT, 0, st>>>(s, nscenes, cfl, d, dt_max, dt_min);
}
