// sph_grid.cu -- uniform-grid neighbour search on the GPU.
//
// Replaces SphBase::gridSetup + SphBase::neighbourSearch
// (SphBase.cpp:849-1089).  The reference inserts every particle at the head
// of a per-cell linked list (solids first, then fluids, each in index order)
// and walks the 27 surrounding cells (x fastest, then y, then z;
// SphBase.cpp:980-986) and each list in list order, keeping a neighbour j when
// its float squared distance is < (d_i + d_j)^2 and stopping at 48 entries.
// The list order is therefore: per cell, fluids in descending (phase, index),
// then solids in descending (solid, index).
//
// Here: one counting sort per step by cell key (atomic histogram, exclusive
// scan, scatter), then a within-cell rank step that orders each cell's
// particles by descending global index -- exactly the reference's list order
// -- while reordering the particle state into the new layout.  Boundary
// particles are sorted once into their own cell table.  The neighbour-list
// kernel then walks the 27 cells in the reference's offset order, the fluid
// range of a cell before its boundary range, so the stored lists (and which
// entries a 48-cap truncates) are the reference's.  The cut test uses
// round-to-nearest float ops in the reference's evaluation order, so the
// neighbour sets are bit-identical.
#include "sph_kernels.cuh"

namespace {
constexpr int NT = 256;

__global__ void __launch_bounds__(NT) k_hash(DevScene s, GridGeom g, int integrate) {
    const int n = s.st->n_active;
    if (blockIdx.x == 0 && threadIdx.x == 0) s.st->pad0 = n;  // staged count
    int i = blockIdx.x * NT + threadIdx.x;
    int removed = 0, nan = 0;
    if (i < n) {
        float4 p, v;
        if (integrate) {
            // Second loop 2.4: velocity = vel_adv; position += velocity*dt
            // (DFSPH.cpp:705-715), in round-to-nearest float ops.
            p = s.pos[i];
            const float dt = dt_of(s, p);
            v = s.pv[2 * i + 1];  // v_adv of the density loop
            p.x = __fadd_rn(p.x, __fmul_rn(v.x, dt));
            p.y = __fadd_rn(p.y, __fmul_rn(v.y, dt));
            p.z = __fadd_rn(p.z, __fmul_rn(v.z, dt));
            v.w = 0.f;
            s.pos_s[i] = p;
            s.vel_s[i] = v;
            s.gid_s[i] = s.gid[i];
            if (integrate & 4) {
                // the learned warm start's history of this step (as k_ws_post):
                // the step's kappa sum with the applied prediction, and the
                // step's (predicted error, divergence term); the sum restarts
                const float2 w = s.wsbuf[i];
                s.hist_s[i] = make_float4(s.ksum[i] + s.kwarm[i], w.x, w.y, 0.f);
                s.ksum[i] = 0.f;
            } else {
                s.hist_s[i] = s.hist[i];
            }
            if (integrate & 2) s.cA_s[i] = s.cA[i];  // DFSPH vorticity state carried through the sort
        } else {
            p = s.pos_s[i];
        }
        // the particle's scene grid (the only grid unless this is a batch)
        const GridGeom G = s.nscenes > 1 ? s.b.geom[scene_of(p)] : g;
        // SphFluid::removeOutsideParts test (SphBase.cpp:34-44, Vec23.h:193-194)
        bool in = G.smin[0] <= p.x && G.smin[1] <= p.y && G.smin[2] <= p.z && p.x <= G.smax[0] &&
                  p.y <= G.smax[1] && p.z <= G.smax[2];
        int key = g.nkeys - 1;
        if (in) {
            int cx = cell_coord(p.x, G.min[0], G.divisor);
            int cy = cell_coord(p.y, G.min[1], G.divisor);
            int cz = cell_coord(p.z, G.min[2], G.divisor);
            if (cell_inside(G, cx, cy, cz)) key = cell_key(G, cx, cy, cz);
            else removed = 1;
        } else {
            removed = 1;
            if (!(isfinite(p.x) && isfinite(p.y) && isfinite(p.z))) nan = 1;
        }
        s.key[i] = key;
        s.slot[i] = atomicAdd(&s.cell_count[key], 1);
    }
    if (__syncthreads_or(removed)) {
        if (removed) atomicOr(&s.st->status, 16u | (nan ? 4u : 0u));
    }
}

__global__ void __launch_bounds__(NT) k_scatter(DevScene s) {
    const int n = s.st->pad0;
    int i = blockIdx.x * NT + threadIdx.x;
    if (i < n) s.tmp[s.cell_start[s.key[i]] + s.slot[i]] = i;
}

// For sorted slot q: its particle i, its cell range [a, b); its final place is
// a + #{particles of the cell with larger global index}.
__global__ void __launch_bounds__(NT) k_rank_reorder(DevScene s, int dead_key, int carry) {
    const int n = s.st->pad0;
    int q = blockIdx.x * NT + threadIdx.x;
    if (q >= n) return;
    int i = s.tmp[q];
    int key = s.key[i];
    if (key == dead_key) return;
    int a = s.cell_start[key], b = s.cell_start[key + 1];
    int my = s.gid_s[i], cnt = 0;
    for (int r = a; r < b; ++r) cnt += s.gid_s[s.tmp[r]] > my;
    int p = a + cnt;
    const float4 x = s.pos_s[i], v = s.vel_s[i];
    s.pos[p] = x;
    s.vel[p] = v;
    s.pv[2 * p] = x;
    s.pv[2 * p + 1] = v;
    s.prv[2 * p + 1] = v;
    s.pk[p] = make_float4(x.x, x.y, x.z, 0.f);
    s.gid[p] = my;
    if (carry & 1) s.hist[p] = s.hist_s[i];
    if (carry & 2) s.cA[p] = s.cA_s[i];
    if (carry & 4) s.cB[p] = s.cB_s[i];
    if (carry & 8) s.cC[p] = s.cC_s[i];
}

__global__ void k_count_active(DevScene s, int dead_key) {
    int staged = s.st->pad0;
    int act = s.cell_start[dead_key];
    s.st->removed += staged - act;
    s.st->n_active = act;
}

// interleaved {fluid start, boundary start} per cell key: one 8-byte load
// per cell bound in the neighbour-list kernel
__global__ void k_merge_starts(DevScene s, int nk) {
    const int k = blockIdx.x * NT + threadIdx.x;
    if (k <= nk) s.cstart2[k] = make_int2(s.cell_start[k], s.bcell_start[k]);
}

// Ints per thread of the shared-memory list staging (>= the cap of 48, a
// multiple of 4 so that every row starts on a 16-byte boundary; 52 also
// spreads the rows of 8 consecutive threads over distinct bank quads).
constexpr int LROW = 52;

// mode 0: neighbour lists only; 1: + DFSPH rho and alpha
// (DF_constantDensitySolverFirst, DFSPH.cpp:84-193); 2: + WCSPH rho and Tait
// pressure (WcSph::wc_computePressure, WcSph.cpp:99-153); 3: + IISph
// sphDensity, gamma, sphVolume and alpha (IISph.cpp:100-402); 4: mode 1 and,
// over the same list in the same pass, the first sweep A of the divergence
// loop that follows the neighbour search (DFSPH.cpp:795-835: Drho/Dt, its
// clamp, kappa_v, the FP64 error sum) -- every neighbour's 32-byte
// {position, velocity} record is gathered once for both, and the loop then
// starts with its velocity update (the per-pair term is div_term, the one the
// separate sweep uses, so the results are the same bit for bit); 5: mode 4 in
// a batch (each scene's own dt; the loop decisions reduce per scene).
//
// STAGED (cap <= 48): a kept neighbour is one predicated shared-memory store
// into the thread's row -- no divergent branch around a global store in the
// candidate loop -- and the finished list leaves in 16-byte groups (a warp
// writes whole sectors); the rho/alpha pass reads the list back from shared
// memory.  Otherwise entries go straight to the global ELL list.
// With staging, shared memory limits an SM to 1024 / BS blocks (26.6 KB
// each at 128 threads); saying so lets the compiler use the registers that
// occupancy leaves (60 instead of 48 with spills: 529 -> 520 us at 1 M).
template <int MODE, int BS, bool STAGED>
__global__ void __launch_bounds__(BS, STAGED ? 1024 / BS : 1) k_build(DevScene s, GridGeom g, SolverConst c) {
    constexpr bool DIV = MODE == 4 || MODE == 5;  // the fused first divergence sweep
    extern __shared__ int4 list_smem[];
    int* const row = reinterpret_cast<int*>(list_smem) + (STAGED ? threadIdx.x * LROW : 0);
    const int n = s.st->n_active;
    const int p = blockIdx.x * BS + threadIdx.x;
    int cnt = 0, over = 0;
    double ddiv = 0.0;  // MODE 4: this particle's Drho/Dt for the FP64 error
    const bool act = p < n;
    if (act) {
        const float4 pa = s.pos[p];
        const int ph = phase_of(pa);
        const float fm0 = c.fm_ph[ph], rho0 = c.rho0_ph[ph];
        const float4* __restrict__ P = s.pos;
        const float4* __restrict__ BP = s.bpos;
        const GridGeom G = s.nscenes > 1 ? s.b.geom[scene_of(pa)] : g;
        const int cx = cell_coord(pa.x, G.min[0], G.divisor);
        const int cy = cell_coord(pa.y, G.min[1], G.divisor);
        const int cz = cell_coord(pa.z, G.min[2], G.divisor);
        int* out = s.nbr;
        const size_t stride = (size_t)c.stride;
        const int cap = c.cap;
        // phase 1: candidate scan in the reference's order, append indices.
        // Every one of the 27 cells is scanned: skipping cells beyond the cut
        // per particle saves fewer tests than the per-cell test and the
        // divergence it causes among the lanes of one cell cost (measured).
        for (int dz = -1; dz <= 1; ++dz) {
            for (int dy = -1; dy <= 1; ++dy) {
                for (int dx = -1; dx <= 1; ++dx) {
                    const int x = cx + dx, y = cy + dy, z = cz + dz;
                    if (!cell_inside(G, x, y, z)) continue;
                    const int key = cell_key(G, x, y, z);
                    const int2 s0 = __ldg(s.cstart2 + key), s1 = __ldg(s.cstart2 + key + 1);
                    for (int q = s0.x; q < s1.x; ++q) {
                        const float4 pb = __ldg(P + q);
                        const float len2 = dis_square_rn(pa.x, pa.y, pa.z, pb.x, pb.y, pb.z);
                        const bool hit = len2 < c.h2cut && q != p;
                        if (STAGED) {
                            // cnt counts every hit; the first `cap` are kept
                            if (hit && cnt < cap) row[cnt] = q;
                            cnt += hit;
                        } else if (hit) {
                            if (cnt < cap) out[ell_index(stride, p, cnt++)] = q;
                            else ++over;
                        }
                    }
                    for (int q = s0.y; q < s1.y; ++q) {
                        const float4 pb = __ldg(BP + q);
                        const float len2 = dis_square_rn(pa.x, pa.y, pa.z, pb.x, pb.y, pb.z);
                        const bool hit = len2 < c.h2cut;
                        if (STAGED) {
                            if (hit && cnt < cap) row[cnt] = q | (int)BND_FLAG;
                            cnt += hit;
                        } else if (hit) {
                            if (cnt < cap) out[ell_index(stride, p, cnt++)] = q | (int)BND_FLAG;
                            else ++over;
                        }
                    }
                }
            }
        }
        if (STAGED) {
            over = cnt > cap ? cnt - cap : 0;
            cnt -= over;
            // the list in 16-byte groups (entries past the count are never
            // read: every sweep masks them)
            const int4* r4 = reinterpret_cast<const int4*>(row);
            int4* o4 = reinterpret_cast<int4*>(out);
            for (int gi = 0; gi < ((cnt + 3) >> 2); ++gi) o4[(size_t)gi * stride + p] = r4[gi];
        }
        s.ncount[p] = cnt;
        if (MODE == 3) {
            // IISph: sphDensity (DF_prepareAttribute, IISph.cpp:127-170) and
            // VF_prepareAttribute (IISph.cpp:309-402) over the stored list,
            // per-pair h = (d_a + d_b)/2 = d (one diameter for all particles)
            const float Va = c.iv_V, ma = c.iv_m[ph], rda = rho0;
            const float w0 = c.kd.theta;  // W(0, d)
            float density = w0 * ma;
            float gamma = Va * w0;
            float sphv = (float)((double)w0 * (double)Va * (double)Va);
            float a1x = 0.f, a1y = 0.f, a1z = 0.f, a2 = 0.f;
            for (int k = 0; k < cnt; ++k) {
                const unsigned e = STAGED ? (unsigned)row[k] : (unsigned)out[ell_index(stride, p, k)];
                const bool bnd = (e & BND_FLAG) != 0u;
                const float4 pb = __ldg((bnd ? BP : P) + (e & BND_MASK));
                const float xx = pa.x - pb.x, xy = pa.y - pb.y, xz = pa.z - pb.z;
                const float len2 = dis_square_rn(pa.x, pa.y, pa.z, pb.x, pb.y, pb.z);
                float w, f;
                kernel_pair_rn(c.kd, len2, w, f);
                const float Vb = bnd ? pb.w : Va;
                density = fmaf(bnd ? rda * Vb : c.iv_m[phase_of(pb)], w, density);
                gamma = fmaf(Vb, w, gamma);
                sphv = fmaf(Va * Vb, w, sphv);
                const float fv = f * Vb;
                a1x = fmaf(xx, fv, a1x);
                a1y = fmaf(xy, fv, a1y);
                a1z = fmaf(xz, fv, a1z);
                // V_b^2 |gradW|^2 / m_b: fluid neighbours only (boundary terms
                // belong to dynamic solids, IISph.cpp:386-393)
                if (!bnd) a2 = fmaf(fv * fv, len2 / c.iv_m[phase_of(pb)], a2);
            }
            float al = ((a1x * a1x + a1y * a1y + a1z * a1z) / ma + a2) / gamma;
            if (al < 1.0e-10f) al = 1.0e-10f;
            s.ivs[p] = make_float4(gamma, sphv, 1.f / al, density);
        } else if (MODE != 0) {
            // phase 2: rho and alpha over the stored list (all lanes busy)
            float density = ker_W(c.k, 0.f) * fm0;
            float a1x = 0.f, a1y = 0.f, a1z = 0.f, a2 = 0.f;
            float dacc = 0.f;  // MODE 4: the divergence sum
            const float4 va = DIV ? s.pv[2 * p + 1] : make_float4(0.f, 0.f, 0.f, 0.f);
            for (int k = 0; k < cnt; ++k) {
                const unsigned e = STAGED ? (unsigned)row[k] : (unsigned)out[ell_index(stride, p, k)];
                const bool bnd = (e & BND_FLAG) != 0u;
                float4 pb, vb;
                // pv / bpv hold {the position (boundary: with its volume) of
                // pos / bpos, the velocity}
                if (DIV) ld_record32((bnd ? s.bpv : s.pv) + 2 * (size_t)(e & BND_MASK), pb, vb);
                else pb = __ldg((bnd ? BP : P) + (e & BND_MASK));
                if (DIV) dacc = div_term(c, pa, va, pb, vb, bnd, dacc);
                const float xx = pa.x - pb.x, xy = pa.y - pb.y, xz = pa.z - pb.z;
                const float len2 = dis_square_rn(pa.x, pa.y, pa.z, pb.x, pb.y, pb.z);
                float w, f;
                kernel_pair(c.k, len2, w, f);
                const float m = bnd ? rho0 * pb.w : fm0;
                density = fmaf(m, w, density);
                if (MODE == 1 || DIV) {
                    const float fm = f * m;
                    a1x = fmaf(xx, fm, a1x);
                    a1y = fmaf(xy, fm, a1y);
                    a1z = fmaf(xz, fm, a1z);
                    const float t = bnd ? 0.f : fm * sqrtf(len2);  // |gradW| m, fluid only (DFSPH.cpp:161)
                    a2 = fmaf(t, t, a2);
                }
            }
            if (MODE == 1 || DIV) {
                s.rho[p] = density;
                s.prv[2 * p] = make_float4(pa.x, pa.y, pa.z, density);
                float al = a1x * a1x + a1y * a1y + a1z * a1z + a2;
                if (al < 1.0e-6f) al = 1.0e-6f;
                const float alpha = density / al;
                s.alpha[p] = alpha;
                if (DIV) {
                    // the divergence loop's first sweep A, as k_df_div_a
                    const float dt = MODE == 5 ? s.b.dt[scene_of(pa)] : *s.dt;
                    float dd = dacc;
                    if (dd < 0.f || (density + dd * dt) < c.rho0) dd = 0.f;  // DFSPH.cpp:829-832
                    const float kv = dd * alpha / dt;                         // DFSPH.cpp:835
                    s.pk[p] = make_float4(pa.x, pa.y, pa.z, kv / density);
                    s.kappav[p] = kv;
                    s.aux1[p] = dd;
                    ddiv = (double)dd;
                }
            } else {
                s.rho[p] = density;
                // Tait, WcSph.cpp:142-146 (NEGLECT_NEGATIVE_PRESSURE)
                float pr = c.wc_B * (powf(density / rho0, c.wc_gamma) - 1.f);
                if (pr < 0.f) pr = 0.f;
                s.kr[p] = pr;
            }
        }
    }
    __shared__ int sh[BS / 32];
    int tot = block_sum_int<BS>(act ? cnt : 0, sh);
    int ov = block_sum_int<BS>(over, sh);
    int mx = block_max_int<BS>(act ? cnt : 0, sh);
    if (threadIdx.x == 0) {
        if (tot) atomicAdd(&s.st->nbr_total, (unsigned long long)tot);
        if (ov) { atomicAdd(&s.st->overflow, ov); atomicOr(&s.st->status, 8u); }
        if (mx) atomicMax(&s.st->max_nbrs, mx);
    }
    if (MODE == 4) {
        // mean Drho/Dt of the iteration (k_df_div_a's FP64 error; a batch,
        // mode 5, reduces per scene in k_batch_decide)
        __shared__ double shd[BS / 32];
        const double bsum = block_sum_double<BS>(ddiv, shd);
        double t;
        if (finish_sum<BS>(s.partial, &s.st->ticket[1], bsum, &t)) s.st->err_div = n > 0 ? t / (double)n : 0.0;
    }
}

// WCSPH list build + density + Tait pressure (mode 2) with L threads per
// particle, for small scenes (one thread per particle leaves too few warps
// per SM to hide the candidate loads' latency).  Lane l scans a contiguous
// range of the 27 cells in the reference's order into its own staged row;
// the lanes' counts give each lane's offset in the particle's list, so the
// list (and its cap) is the one-thread kernel's exactly.  Density: each
// lane sums its kept entries, the partial sums are added in a fixed shuffle
// order (deterministic; the one-thread kernel's sum is in list order).
template <int L>
__global__ void __launch_bounds__(128) k_build_wc_lanes(DevScene s, GridGeom g, SolverConst c) {
    constexpr int BS = 128;
    extern __shared__ int4 list_smem[];
    int* const row = reinterpret_cast<int*>(list_smem) + threadIdx.x * LROW;
    const int n = s.st->n_active;
    const int t = blockIdx.x * BS + threadIdx.x;
    const int p = t / L, l = t % L;
    const bool act = p < n;
    // lane l scans cells [c0, c1) of the 27
    constexpr int PER = (27 + L - 1) / L;
    const int c0 = l * PER, c1 = min(27, c0 + PER);
    int cnt = 0;
    float4 pa = make_float4(0.f, 0.f, 0.f, 0.f);
    if (act) {
        pa = s.pos[p];
        const GridGeom G = s.nscenes > 1 ? s.b.geom[scene_of(pa)] : g;
        const int cx = cell_coord(pa.x, G.min[0], G.divisor);
        const int cy = cell_coord(pa.y, G.min[1], G.divisor);
        const int cz = cell_coord(pa.z, G.min[2], G.divisor);
        const int cap = c.cap;
        for (int ci = c0; ci < c1; ++ci) {
            const int x = cx + ci % 3 - 1, y = cy + (ci / 3) % 3 - 1, z = cz + ci / 9 - 1;
            if (!cell_inside(G, x, y, z)) continue;
            const int key = cell_key(G, x, y, z);
            const int2 s0 = __ldg(s.cstart2 + key), s1 = __ldg(s.cstart2 + key + 1);
            for (int q = s0.x; q < s1.x; ++q) {
                const float4 pb = __ldg(s.pos + q);
                const float len2 = dis_square_rn(pa.x, pa.y, pa.z, pb.x, pb.y, pb.z);
                const bool hit = len2 < c.h2cut && q != p;
                if (hit && cnt < cap) row[cnt] = q;
                cnt += hit;
            }
            for (int q = s0.y; q < s1.y; ++q) {
                const float4 pb = __ldg(s.bpos + q);
                const float len2 = dis_square_rn(pa.x, pa.y, pa.z, pb.x, pb.y, pb.z);
                const bool hit = len2 < c.h2cut;
                if (hit && cnt < cap) row[cnt] = q | (int)BND_FLAG;
                cnt += hit;
            }
        }
    }
    // exclusive prefix of the lanes' counts within the particle's group
    int pre = cnt;
#pragma unroll
    for (int off = 1; off < L; off <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, pre, off, L);
        if (l >= off) pre += v;
    }
    const int total = __shfl_sync(0xffffffffu, pre, L - 1, L);
    pre -= cnt;
    const int cap = c.cap;
    const int kept = min(total, cap);
    float density = 0.f;
    if (act) {
        const size_t stride = (size_t)c.stride;
        const int ph = phase_of(pa);
        const float fm0 = c.fm_ph[ph], rho0 = c.rho0_ph[ph];
        const int mine = max(0, min(cnt, cap - pre));
        for (int i = 0; i < mine; ++i) {
            const unsigned e = (unsigned)row[i];
            s.nbr[ell_index(stride, p, pre + i)] = (int)e;
            const bool bnd = (e & BND_FLAG) != 0u;
            const float4 pb = __ldg((bnd ? s.bpos : s.pos) + (e & BND_MASK));
            const float len2 = dis_square_rn(pa.x, pa.y, pa.z, pb.x, pb.y, pb.z);
            float w, f;
            kernel_pair(c.k, len2, w, f);
            density = fmaf(bnd ? rho0 * pb.w : fm0, w, density);
        }
        if (l == 0) density = fmaf(ker_W(c.k, 0.f), fm0, density);
    }
#pragma unroll
    for (int off = 1; off < L; off <<= 1) density += __shfl_xor_sync(0xffffffffu, density, off);
    if (act && l == 0) {
        const float rho0 = c.rho0_ph[phase_of(pa)];
        s.ncount[p] = kept;
        s.rho[p] = density;
        // Tait, WcSph.cpp:142-146 (NEGLECT_NEGATIVE_PRESSURE)
        float pr = c.wc_B * (powf(density / rho0, c.wc_gamma) - 1.f);
        if (pr < 0.f) pr = 0.f;
        s.kr[p] = pr;
    }
    __shared__ int sh[BS / 32];
    const bool lead = act && l == 0;
    int tot = block_sum_int<BS>(lead ? kept : 0, sh);
    int ov = block_sum_int<BS>(lead ? total - kept : 0, sh);
    int mx = block_max_int<BS>(lead ? kept : 0, sh);
    if (threadIdx.x == 0) {
        if (tot) atomicAdd(&s.st->nbr_total, (unsigned long long)tot);
        if (ov) { atomicAdd(&s.st->overflow, ov); atomicOr(&s.st->status, 8u); }
        if (mx) atomicMax(&s.st->max_nbrs, mx);
    }
}

__global__ void k_boundary_keys(const float4* bpos, int nb, GridGeom g, int* keys) {
    int i = blockIdx.x * NT + threadIdx.x;
    if (i >= nb) return;
    float4 p = bpos[i];
    int cx = cell_coord(p.x, g.min[0], g.divisor);
    int cy = cell_coord(p.y, g.min[1], g.divisor);
    int cz = cell_coord(p.z, g.min[2], g.divisor);
    keys[i] = cell_inside(g, cx, cy, cz) ? cell_key(g, cx, cy, cz) : -1;
}

// Boundary volume of a static rigid wall, SphBase::prepareSolidPartWeight
// (SphBase.cpp:766-813) with only boundary particles in the grid:
// V_b = 1 / (W(0, d) + sum over the (capped) boundary neighbour list of
// W(dis, (d_a + d_b)/2)).
__global__ void __launch_bounds__(128) k_boundary_volume(DevScene s, GridGeom g, float dpart, float h2cut, int cap,
                                                         int b0, int b1) {
    int p = b0 + blockIdx.x * 128 + threadIdx.x;
    if (p >= b1) return;
    float4 pa = s.bpos[p];
    int cx = cell_coord(pa.x, g.min[0], g.divisor);
    int cy = cell_coord(pa.y, g.min[1], g.divisor);
    int cz = cell_coord(pa.z, g.min[2], g.divisor);
    float h = dpart;
    float sum = ker_W_h(0.f, h);
    int cnt = 0;
    float hp = (dpart + dpart) / 2;
    for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) {
                int x = cx + dx, y = cy + dy, z = cz + dz;
                if (!cell_inside(g, x, y, z)) continue;
                int key = cell_key(g, x, y, z);
                int a = s.bcell_start[key], b = s.bcell_start[key + 1];
                for (int q = a; q < b; ++q) {
                    if (q == p) continue;
                    float4 pb = s.bpos[q];
                    float len2 = dis_square_rn(pa.x, pa.y, pa.z, pb.x, pb.y, pb.z);
                    if (len2 < h2cut && cnt < cap) {
                        ++cnt;
                        sum += ker_W_h(sqrtf(len2), hp);
                    }
                }
            }
    s.bpos[p].w = 1.f / sum;
}

// Reference-order transfers: gid is a permutation of [0, n) while no
// particle has been removed.
__global__ void k_to_ref_order(const float4* src, const int* gid, int n, float* dst3) {
    int p = blockIdx.x * NT + threadIdx.x;
    if (p >= n) return;
    float4 v = src[p];
    size_t g = (size_t)gid[p] * 3;
    dst3[g] = v.x;
    dst3[g + 1] = v.y;
    dst3[g + 2] = v.z;
}
// A host step's incoming state (reference order) against the sorted state
// whose lists are still valid: velocities go straight into the sorted
// arrays (vel and the velocity half of the force kernel's record); a
// position that differs from the device's sets *changed, and the caller
// then stages the positions and searches again.
__global__ void k_state_in(const float* xyz3, const float* vel3, const int* gid, int n, const float4* pos,
                           float4* vel, float4* prv, int* changed) {
    const int p = blockIdx.x * NT + threadIdx.x;
    int diff = 0;
    if (p < n) {
        const size_t g = (size_t)gid[p] * 3;
        const float4 x = pos[p];
        diff = x.x != xyz3[g] || x.y != xyz3[g + 1] || x.z != xyz3[g + 2];
        const float4 v = make_float4(vel3[g], vel3[g + 1], vel3[g + 2], 0.f);
        vel[p] = v;
        prv[2 * p + 1] = v;
    }
    if (__syncthreads_or(diff) && threadIdx.x == 0) atomicOr(changed, 1);
}

// Host state (reference order) against the sorted device state, bit for bit
// (positions and velocities): *differs set if any particle differs.  Reads
// only, so it can run while a step that has not yet re-sorted reads the same
// arrays.
__global__ void k_state_check(const float* xyz3, const float* vel3, const int* gid, int n, const float4* pos,
                              const float4* vel, int* differs) {
    const int p = blockIdx.x * NT + threadIdx.x;
    int diff = 0;
    if (p < n) {
        const size_t g = (size_t)gid[p] * 3;
        const float4 x = pos[p], v = vel[p];
        diff = (__float_as_int(x.x) != __float_as_int(xyz3[g])) | (__float_as_int(x.y) != __float_as_int(xyz3[g + 1])) |
               (__float_as_int(x.z) != __float_as_int(xyz3[g + 2])) | (__float_as_int(v.x) != __float_as_int(vel3[g])) |
               (__float_as_int(v.y) != __float_as_int(vel3[g + 1])) | (__float_as_int(v.z) != __float_as_int(vel3[g + 2]));
    }
    if (__syncthreads_or(diff) && threadIdx.x == 0) atomicOr(differs, 1);
}

// The positions the integration (k_hash, integrate mode) will write, in
// the same round-to-nearest operations, scattered into reference order:
// a host-buffer step copies them out while the rest of the step runs (the
// divergence loop changes velocities only).
__global__ void k_integrated_to_ref(DevScene s, float* out3) {
    const int n = s.st->n_active;
    const int i = blockIdx.x * NT + threadIdx.x;
    if (i >= n) return;
    float4 p = s.pos[i];
    const float dt = dt_of(s, p);
    const float4 v = s.pv[2 * i + 1];
    const size_t g = (size_t)s.gid[i] * 3;
    out3[g] = __fadd_rn(p.x, __fmul_rn(v.x, dt));
    out3[g + 1] = __fadd_rn(p.y, __fmul_rn(v.y, dt));
    out3[g + 2] = __fadd_rn(p.z, __fmul_rn(v.z, dt));
}

__global__ void k_from_ref_order(const float* src3, const int* gid, int n, float4* dst) {
    int p = blockIdx.x * NT + threadIdx.x;
    if (p >= n) return;
    size_t g = (size_t)gid[p] * 3;
    float4 v = dst[p];
    v.x = src3[g];
    v.y = src3[g + 1];
    v.z = src3[g + 2];
    dst[p] = v;
}
}  // namespace

static inline int nblk(int n, int nt) { return (n + nt - 1) / nt; }

void launch_to_ref_order(const float4* src, const int* gid, int n, float* dst3, cudaStream_t st) {
    if (n > 0) k_to_ref_order<<<nblk(n, NT), NT, 0, st>>>(src, gid, n, dst3);
}
void launch_state_in(const float* xyz3, const float* vel3, const int* gid, int n, const float4* pos, float4* vel,
                     float4* prv, int* changed, cudaStream_t st) {
    if (n > 0) k_state_in<<<nblk(n, NT), NT, 0, st>>>(xyz3, vel3, gid, n, pos, vel, prv, changed);
}
void launch_state_check(const float* xyz3, const float* vel3, const int* gid, int n, const float4* pos,
                        const float4* vel, int* differs, cudaStream_t st) {
    if (n > 0) k_state_check<<<nblk(n, NT), NT, 0, st>>>(xyz3, vel3, gid, n, pos, vel, differs);
}
void launch_integrated_to_ref(const DevScene& s, int n_max, float* out3, cudaStream_t st) {
    if (n_max > 0) k_integrated_to_ref<<<nblk(n_max, NT), NT, 0, st>>>(s, out3);
}
void launch_from_ref_order(const float* src3, const int* gid, int n, float4* dst, cudaStream_t st) {
    if (n > 0) k_from_ref_order<<<nblk(n, NT), NT, 0, st>>>(src3, gid, n, dst);
}


void launch_hash(const DevScene& s, const GridGeom& g, int integrate, int n_old, cudaStream_t st) {
    k_hash<<<nblk(n_old > 0 ? n_old : 1, NT), NT, 0, st>>>(s, g, integrate);
}

void launch_scatter_reorder(const DevScene& s, const GridGeom& g, int n_old, int carry, cudaStream_t st) {
    int nb = nblk(n_old > 0 ? n_old : 1, NT);
    k_scatter<<<nb, NT, 0, st>>>(s);
    k_rank_reorder<<<nb, NT, 0, st>>>(s, g.nkeys - 1, carry);
}

void launch_count_active(const DevScene& s, const GridGeom& g, cudaStream_t st) {
    k_count_active<<<1, 1, 0, st>>>(s, g.nkeys - 1);
    k_merge_starts<<<nblk(g.nkeys + 1, NT), NT, 0, st>>>(s, g.nkeys);
}

void launch_merge_starts(const DevScene& s, const GridGeom& g, cudaStream_t st) {
    k_merge_starts<<<nblk(g.nkeys + 1, NT), NT, 0, st>>>(s, g.nkeys);
}

template <int BS, bool STAGED>
static void launch_build_st(const DevScene& s, const GridGeom& g, const SolverConst& c, int mode, int nb,
                            cudaStream_t st) {
    const size_t sm = STAGED ? sizeof(int) * LROW * BS : 0;
    if (mode == 0) k_build<0, BS, STAGED><<<nb, BS, sm, st>>>(s, g, c);
    else if (mode == 1) k_build<1, BS, STAGED><<<nb, BS, sm, st>>>(s, g, c);
    else if (mode == 2) k_build<2, BS, STAGED><<<nb, BS, sm, st>>>(s, g, c);
    else if (mode == 4 && s.nscenes > 1) k_build<5, BS, STAGED><<<nb, BS, sm, st>>>(s, g, c);
    else if (mode == 4) k_build<4, BS, STAGED><<<nb, BS, sm, st>>>(s, g, c);
    else k_build<3, BS, STAGED><<<nb, BS, sm, st>>>(s, g, c);
}

template <int BS>
static void launch_build_bs(const DevScene& s, const GridGeom& g, const SolverConst& c, int mode, int n_max,
                            cudaStream_t st) {
    const int nb = nblk(n_max > 0 ? n_max : 1, BS);
    // staging needs the cap to fit a row and the rows to fit the default
    // 48 KB of dynamic shared memory (64 and 128 threads per block)
    if (c.cap <= LROW - 4 && BS * LROW * sizeof(int) <= 48 * 1024) launch_build_st<BS, true>(s, g, c, mode, nb, st);
    else launch_build_st<BS, false>(s, g, c, mode, nb, st);
}

// every block-size instantiation of the DFSPH list build (modes 1 and 4)
template <int BS, class F>
static void each_build_kernel_bs(F f) {
    f((const void*)k_build<1, BS, true>);
    f((const void*)k_build<1, BS, false>);
    f((const void*)k_build<4, BS, true>);
    f((const void*)k_build<4, BS, false>);
    f((const void*)k_build<5, BS, true>);
    f((const void*)k_build<5, BS, false>);
}
template <class F>
static void each_build_kernel(F f) {
    each_build_kernel_bs<64>(f);
    each_build_kernel_bs<128>(f);
    each_build_kernel_bs<256>(f);
}
// preferred shared-memory carveout of the DFSPH list build (percent; -1 =
// the driver's choice): the staged rows take shared memory from the L1 that
// caches the candidates' records
void set_build_carveout(int pct) {
    each_build_kernel([&](const void* k) { cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, pct); });
}
// loads every instantiation now (see preload_sweep_kernels)
void preload_build_kernels() {
    each_build_kernel([](const void* k) {
        cudaFuncAttributes a;
        cudaFuncGetAttributes(&a, k);
    });
}

void launch_build(const DevScene& s, const GridGeom& g, const SolverConst& c, int mode, int n_max, cudaStream_t st,
                  int bs) {
    if (mode == 2 && c.lanes == 4 && c.cap <= LROW - 4) {
        // small scenes: 4 threads per particle (sizes measured: 27 k particles,
        // 54 -> 35 us; 8 threads per particle 40 us)
        const int nb = (int)(((long long)(n_max > 0 ? n_max : 1) * 4 + 127) / 128);
        k_build_wc_lanes<4><<<nb, 128, sizeof(int) * LROW * 128, st>>>(s, g, c);
        return;
    }
    if (bs == 64) launch_build_bs<64>(s, g, c, mode, n_max, st);
    else if (bs == 256) launch_build_bs<256>(s, g, c, mode, n_max, st);
    else launch_build_bs<128>(s, g, c, mode, n_max, st);
}

void launch_boundary_keys(const float4* bpos, int nb, const GridGeom& g, int* keys, cudaStream_t st) {
    if (nb > 0) k_boundary_keys<<<nblk(nb, NT), NT, 0, st>>>(bpos, nb, g, keys);
}

void launch_boundary_volume(const DevScene& s, const GridGeom& g, float dpart, float h2cut, int cap, int b0, int b1,
                            cudaStream_t st) {
    if (b1 > b0) k_boundary_volume<<<nblk(b1 - b0, 128), 128, 0, st>>>(s, g, dpart, h2cut, cap, b0, b1);
}
