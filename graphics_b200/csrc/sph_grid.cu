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
// kernel (k_build_win, sph_dfsph.cu) then walks the 27 cells in the
// reference's offset order, the fluid range of a cell before its boundary
// range, so the stored lists (and which entries a 48-cap truncates) are the
// reference's.  The cut test uses round-to-nearest float ops in the
// reference's evaluation order, so the neighbour sets are bit-identical.
#include "sph_kernels.cuh"

namespace {
constexpr int NT = 256;

__global__ void __launch_bounds__(NT) k_hash(DevScene s, GridGeom g, float3 smin, float3 smax, int integrate) {
    const int n = s.st->n_active;
    if (blockIdx.x == 0 && threadIdx.x == 0) s.st->pad0 = n;  // staged count
    int i = blockIdx.x * NT + threadIdx.x;
    int removed = 0, nan = 0;
    if (i < n) {
        float4 p, v;
        if (integrate) {
            // Second loop 2.4: velocity = vel_adv; position += velocity*dt
            // (DFSPH.cpp:705-715), in round-to-nearest float ops.
            float dt = *s.dt;
            p = s.pos[i];
            v = s.vadv[i];
            p.x = __fadd_rn(p.x, __fmul_rn(v.x, dt));
            p.y = __fadd_rn(p.y, __fmul_rn(v.y, dt));
            p.z = __fadd_rn(p.z, __fmul_rn(v.z, dt));
            v.w = 0.f;
            s.pos_s[i] = p;
            s.vel_s[i] = v;
            s.gid_s[i] = s.gid[i];
            if (s.kwarm_s) s.kwarm_s[i] = s.kwarm[i];
        } else {
            p = s.pos_s[i];
        }
        // SphFluid::removeOutsideParts test (SphBase.cpp:34-44, Vec23.h:193-194)
        bool in = smin.x <= p.x && smin.y <= p.y && smin.z <= p.z && p.x <= smax.x && p.y <= smax.y &&
                  p.z <= smax.z;
        int key = g.nkeys - 1;
        if (in) {
            int cx = cell_coord(p.x, g.min[0], g.divisor);
            int cy = cell_coord(p.y, g.min[1], g.divisor);
            int cz = cell_coord(p.z, g.min[2], g.divisor);
            if (cell_inside(g, cx, cy, cz)) key = cell_key(g, cx, cy, cz);
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
__global__ void __launch_bounds__(NT) k_rank_reorder(DevScene s, int dead_key, int carry_kwarm) {
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
    s.pos[p] = s.pos_s[i];
    s.vel[p] = s.vel_s[i];
    s.gid[p] = my;
    if (carry_kwarm) s.kwarm[p] = s.kwarm_s[i];
}

__global__ void k_count_active(DevScene s, int dead_key) {
    int staged = s.st->pad0;
    int act = s.cell_start[dead_key];
    s.st->removed += staged - act;
    s.st->n_active = act;
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
__global__ void __launch_bounds__(128) k_boundary_volume(DevScene s, GridGeom g, float dpart, float h2cut, int cap) {
    int p = blockIdx.x * 128 + threadIdx.x;
    if (p >= s.nb) return;
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
void launch_from_ref_order(const float* src3, const int* gid, int n, float4* dst, cudaStream_t st) {
    if (n > 0) k_from_ref_order<<<nblk(n, NT), NT, 0, st>>>(src3, gid, n, dst);
}


void launch_hash(const DevScene& s, const GridGeom& g, const float* smin, const float* smax, int integrate,
                 int n_old, cudaStream_t st) {
    k_hash<<<nblk(n_old > 0 ? n_old : 1, NT), NT, 0, st>>>(s, g, make_float3(smin[0], smin[1], smin[2]),
                                                          make_float3(smax[0], smax[1], smax[2]), integrate);
}

void launch_scatter_reorder(const DevScene& s, const GridGeom& g, int n_old, int carry_kwarm, cudaStream_t st) {
    int nb = nblk(n_old > 0 ? n_old : 1, NT);
    k_scatter<<<nb, NT, 0, st>>>(s);
    k_rank_reorder<<<nb, NT, 0, st>>>(s, g.nkeys - 1, carry_kwarm);
}

void launch_count_active(const DevScene& s, const GridGeom& g, cudaStream_t st) {
    k_count_active<<<1, 1, 0, st>>>(s, g.nkeys - 1);
}

void launch_boundary_keys(const float4* bpos, int nb, const GridGeom& g, int* keys, cudaStream_t st) {
    if (nb > 0) k_boundary_keys<<<nblk(nb, NT), NT, 0, st>>>(bpos, nb, g, keys);
}

void launch_boundary_volume(const DevScene& s, const GridGeom& g, float dpart, float h2cut, int cap,
                            cudaStream_t st) {
    if (s.nb > 0) k_boundary_volume<<<nblk(s.nb, 128), 128, 0, st>>>(s, g, dpart, h2cut, cap);
}
