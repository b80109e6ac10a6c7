// sph_rigid.cu -- dynamic rigid solids coupled to the DFSPH step.
//
// The reference couples rigid bodies through Bullet (SphWithBullet.cpp:
// 180-224, called from DFSPH::sphStep, DFSPH.cpp:54): the DFSPH step
// accumulates a force on every boundary particle -- the reaction of the
// boundary viscosity term (`rb.force -= tmp`, DFSPH.cpp:1334-1359) and of
// every constant-density iteration's pressure term (`p_b.force += acc_p`,
// DFSPH.cpp:681-691), scaled by the particle mass of phase 0 at the end
// (DFSPH.cpp:723-737) -- then joins them per solid into a force and a torque
// about the centre of mass (SphSolid::rigidForceJoin, SphBase.cpp:131-143),
// hands them to Bullet, and moves the boundary particles with the body's new
// transform (SphSolid::updatePaticles, SphBase.cpp:95-128) before the
// neighbour search, which recomputes the boundary volumes
// (updateSolidPartWeight, SphBase.cpp:817-841).
//
// Here the rigid-body world stays on the host and exchanges only force,
// torque and state per solid and step; everything per particle runs on the
// device:
//   k_rigid_force     per boundary particle of a dynamic solid: gathers its
//                     fluid neighbours (the fluid particles whose capped list
//                     holds it), sums both reactions, and joins force and
//                     torque per solid in FP64 (block partials summed in a
//                     fixed order by the last block).  The pressure reaction
//                     uses the loop's summed stiffness (kappa summed over the
//                     iterations by the density sweep, plus the warm start's
//                     applied stiffness): the positions and densities are
//                     fixed during the loop, so the sum over iterations of
//                     gradW m kappa_i / rho factors exactly.
//   k_rigid_place     updatePaticles for every particle of a dynamic solid
//                     (transform in round-to-nearest float ops in the
//                     reference's evaluation order) and the cell keys of the
//                     whole boundary
//   radix sort        stable sort of the keys, fed in reversed reference
//                     order, so each cell lists its particles in descending
//                     reference index -- the reference's linked-list order
//   k_rigid_gather    sorted boundary arrays, inverse permutation
//   k_bcell_bounds    boundary cell table (lower bound per key)
//   k_rigid_volume    updateSolidPartWeight after the fluid sort: the
//                     boundary particle's capped list in the reference's
//                     order (fluid candidates count toward the cap; same-solid
//                     particles are skipped, SphBase.cpp:922)
//   k_rigid_prepare   prepareSolidPartWeight over the boundary alone
//                     (kerSumFromSelf and volume), when a solid turns dynamic
#include <cub/device/device_radix_sort.cuh>

#include "sph_kernels.cuh"

namespace {
constexpr int NT = 128;

__device__ __forceinline__ float dot3_rn(float a, float x, float b, float y, float c, float z, float d) {
    // a*x + b*y + c*z + d, left to right, no contraction
    return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(a, x), __fmul_rn(b, y)), __fmul_rn(c, z)), d);
}

__global__ void __launch_bounds__(NT) k_rigid_place(DevScene s, RigidDev R, GridGeom g) {
    const int r = blockIdx.x * NT + threadIdx.x;
    if (r >= R.nb) return;
    const float4 x0 = R.x0[r];
    const int di = R.dyn[r];
    float px = x0.x, py = x0.y, pz = x0.z, vx = 0.f, vy = 0.f, vz = 0.f;
    if (di >= 0) {
        const float* t = R.state + 25 * di;
        // SphBase.cpp:106-112: tranform[0-3] is the first column
        px = dot3_rn(t[0], x0.x, t[4], x0.y, t[8], x0.z, t[12]);
        py = dot3_rn(t[1], x0.x, t[5], x0.y, t[9], x0.z, t[13]);
        pz = dot3_rn(t[2], x0.x, t[6], x0.y, t[10], x0.z, t[14]);
        const float al = dot3_rn(t[3], x0.x, t[7], x0.y, t[11], x0.z, t[15]);
        px = __fdiv_rn(px, al);
        py = __fdiv_rn(py, al);
        pz = __fdiv_rn(pz, al);
        // velocity = v + w x (x - com), vec3::cross (Vec23.h:142-143)
        const float rx = __fsub_rn(px, t[16]), ry = __fsub_rn(py, t[17]), rz = __fsub_rn(pz, t[18]);
        const float ax = t[22], ay = t[23], az = t[24];
        vx = __fadd_rn(t[19], __fsub_rn(__fmul_rn(ay, rz), __fmul_rn(az, ry)));
        vy = __fadd_rn(t[20], __fsub_rn(__fmul_rn(az, rx), __fmul_rn(ax, rz)));
        vz = __fadd_rn(t[21], __fsub_rn(__fmul_rn(ax, ry), __fmul_rn(ay, rx)));
    }
    R.wpos[r] = make_float4(px, py, pz, x0.w);
    R.wvel[r] = make_float4(vx, vy, vz, 0.f);
    int key = g.nkeys - 1;  // the dead key: no cell scan reaches it
    const bool fin = isfinite(px) && isfinite(py) && isfinite(pz);
    if (fin) {
        const int cx = cell_coord(px, g.min[0], g.divisor);
        const int cy = cell_coord(py, g.min[1], g.divisor);
        const int cz = cell_coord(pz, g.min[2], g.divisor);
        if (cell_inside(g, cx, cy, cz)) key = cell_key(g, cx, cy, cz);
    }
    if (key == g.nkeys - 1) atomicOr(&s.st->status, 64u);
    R.key_in[R.nb - 1 - r] = key;
    R.val_in[R.nb - 1 - r] = r;
}

__global__ void __launch_bounds__(NT) k_rigid_gather(DevScene s, RigidDev R) {
    const int q = blockIdx.x * NT + threadIdx.x;
    if (q >= R.nb) return;
    const int r = R.val_out[q];
    const float4 p = R.wpos[r], v = R.wvel[r];
    const float vol = R.vol[r];
    const float4 pv = make_float4(p.x, p.y, p.z, vol);
    s.bpos[q] = pv;
    s.bks[q] = p.w;
    s.bpv[2 * q] = pv;
    s.bpv[2 * q + 1] = make_float4(0.f, 0.f, 0.f, 0.f);  // singleVelocity
    s.bpf[2 * q] = pv;
    s.bpf[2 * q + 1] = v;
    s.bgid[q] = r;
    s.bsid[q] = R.sid[r];
    R.binv[r] = q;
}

__global__ void __launch_bounds__(256) k_bcell_bounds(DevScene s, RigidDev R, int nkeys) {
    const int k = blockIdx.x * 256 + threadIdx.x;
    if (k > nkeys) return;
    int lo = 0, hi = R.nb;  // first sorted slot with key >= k
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (R.key_out[mid] < k) lo = mid + 1;
        else hi = mid;
    }
    s.bcell_start[k] = lo;
}

__device__ __forceinline__ void set_volume(DevScene& s, const RigidDev& R, int q, float vol) {
    s.bpos[q].w = vol;
    s.bpv[2 * q].w = vol;
    s.bpf[2 * q].w = vol;
    R.vol[s.bgid[q]] = vol;
}

// SphBase::prepareSolidPartWeight (SphBase.cpp:766-813), rigid branch, with
// only boundary particles in the grid: kerSumFromSelf = W(0) + same-solid
// terms, volume = 1 / (W(0) + all boundary terms) over the capped list.
__global__ void __launch_bounds__(NT) k_rigid_prepare(DevScene s, RigidDev R, GridGeom g, float dpart, float h2cut,
                                                      int cap) {
    const int q = blockIdx.x * NT + threadIdx.x;
    if (q >= R.nb) return;
    const float4 pa = s.bpos[q];
    const int sid = s.bsid[q];
    const int cx = cell_coord(pa.x, g.min[0], g.divisor);
    const int cy = cell_coord(pa.y, g.min[1], g.divisor);
    const int cz = cell_coord(pa.z, g.min[2], g.divisor);
    const float hp = (dpart + dpart) / 2;
    const float w0 = ker_W_h(0.f, dpart);
    float ks = w0, sum2 = w0;
    int cnt = 0;
    for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) {
                const int x = cx + dx, y = cy + dy, z = cz + dz;
                if (!cell_inside(g, x, y, z)) continue;
                const int key = cell_key(g, x, y, z);
                for (int b = s.bcell_start[key], e = s.bcell_start[key + 1]; b < e; ++b) {
                    if (b == q) continue;
                    const float4 pb = s.bpos[b];
                    const float len2 = dis_square_rn(pa.x, pa.y, pa.z, pb.x, pb.y, pb.z);
                    if (!(len2 < h2cut) || cnt >= cap) continue;
                    ++cnt;
                    const float w = ker_W_h(sqrtf(len2), hp);
                    if (s.bsid[b] == sid) ks += w;
                    sum2 += w;
                }
            }
    s.bks[q] = ks;
    R.x0[s.bgid[q]].w = ks;
    set_volume(s, R, q, 1.f / sum2);
}

// SphBase::updateSolidPartWeight (SphBase.cpp:817-841) over the boundary
// particle's per-step list (SphBase.cpp:911-935: the 27 cells in the
// reference's order, per cell its fluid particles, then the boundary
// particles of other solids; cap entries): volume = 1 / (kerSumFromSelf +
// sum of W(dis, (d_a + d_b)/2) over the listed boundary particles).
__global__ void __launch_bounds__(NT) k_rigid_volume(DevScene s, RigidDev R, GridGeom g, float dpart, float h2cut,
                                                     int cap) {
    const int q = blockIdx.x * NT + threadIdx.x;
    if (q >= R.nb) return;
    const float4 pa = s.bpos[q];
    const int sid = s.bsid[q];
    const int cx = cell_coord(pa.x, g.min[0], g.divisor);
    const int cy = cell_coord(pa.y, g.min[1], g.divisor);
    const int cz = cell_coord(pa.z, g.min[2], g.divisor);
    const float hp = (dpart + dpart) / 2;
    float sum = s.bks[q];
    int cnt = 0;
    for (int dz = -1; dz <= 1 && cnt < cap; ++dz)
        for (int dy = -1; dy <= 1 && cnt < cap; ++dy)
            for (int dx = -1; dx <= 1 && cnt < cap; ++dx) {
                const int x = cx + dx, y = cy + dy, z = cz + dz;
                if (!cell_inside(g, x, y, z)) continue;
                const int key = cell_key(g, x, y, z);
                const int2 s0 = s.cstart2[key], s1 = s.cstart2[key + 1];
                for (int a = s0.x; a < s1.x && cnt < cap; ++a) {
                    const float4 pb = s.pos[a];
                    cnt += dis_square_rn(pa.x, pa.y, pa.z, pb.x, pb.y, pb.z) < h2cut;
                }
                for (int b = s0.y; b < s1.y && cnt < cap; ++b) {
                    if (b == q || s.bsid[b] == sid) continue;
                    const float4 pb = s.bpos[b];
                    const float len2 = dis_square_rn(pa.x, pa.y, pa.z, pb.x, pb.y, pb.z);
                    if (!(len2 < h2cut)) continue;
                    ++cnt;
                    sum += ker_W_h(sqrtf(len2), hp);
                }
            }
    set_volume(s, R, q, 1.f / sum);
}

// Boundary force of the particles of dynamic solid di (reference indices
// [r0, r1)) after the density loop, and the solid's joined force and torque.
// Fluid particle a contributes when boundary particle q is in its list:
// within the cut (the same float test as the list build) and, if a's list
// is full, found among its entries.  Per pair, with the kernel gradient
// factor f = -W'(r)/r and x = x_a - x_q:
//   viscosity (DFSPH.cpp:1349-1357): if (v_a - v_q).x < 0,
//     tmp = x f (v_a - v_q).x / (r^2 + 0.01 h^2) (rho0 V_q / rho_a) 10 nu,
//     force -= tmp
//   pressure (DFSPH.cpp:687-689), summed over the iterations:
//     force += x f rho0 V_q (sum_it kappa_a) / rho_a
// and force *= rho0 * spacing_r^3 (DFSPH.cpp:723-737).
template <int BS>
__global__ void __launch_bounds__(BS) k_rigid_force(DevScene s, RigidDev R, SolverConst c, GridGeom g, int r0, int r1,
                                                    int di) {
    const int r = r0 + blockIdx.x * BS + threadIdx.x;
    double acc[6] = {0, 0, 0, 0, 0, 0};
    if (r < r1) {
        const int q = R.binv[r];
        const float4 pb = s.bpf[2 * q], vb = s.bpf[2 * q + 1];
        const float Vb = pb.w;
        const int cx = cell_coord(pb.x, g.min[0], g.divisor);
        const int cy = cell_coord(pb.y, g.min[1], g.divisor);
        const int cz = cell_coord(pb.z, g.min[2], g.divisor);
        const float den0 = 0.01f * c.hs * c.hs;
        const float visc = 10.f * c.nu;
        const size_t stride = (size_t)c.stride;
        const int me = (int)((unsigned)q | BND_FLAG);
        float px = 0.f, py = 0.f, pz = 0.f, vx = 0.f, vy = 0.f, vz = 0.f;
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    const int x = cx + dx, y = cy + dy, z = cz + dz;
                    if (!cell_inside(g, x, y, z)) continue;
                    const int key = cell_key(g, x, y, z);
                    const int a0 = s.cstart2[key].x, a1 = s.cstart2[key + 1].x;
                    for (int a = a0; a < a1; ++a) {
                        const float4 pa = s.pos[a];
                        const float len2 = dis_square_rn(pa.x, pa.y, pa.z, pb.x, pb.y, pb.z);
                        if (!(len2 < c.h2cut)) continue;
                        const int cnt = s.ncount[a];
                        if (cnt >= c.cap) {
                            bool listed = false;
                            for (int k = 0; k < cnt && !listed; ++k) listed = ell_get(s.nbr, stride, a, k) == me;
                            if (!listed) continue;
                        }
                        if (len2 == 0.f) continue;  // the reference skips zero distances (DFSPH.cpp:1338-1342)
                        const float xx = pa.x - pb.x, xy = pa.y - pb.y, xz = pa.z - pb.z;
                        const float f = grad_over_r(c.k, len2);
                        const float rhoa = s.rho[a];
                        const float kap = (s.ksum[a] + s.kwarm[a]) / rhoa;
                        const float tp = f * (c.rho0 * kap) * Vb;
                        px = fmaf(xx, tp, px);
                        py = fmaf(xy, tp, py);
                        pz = fmaf(xz, tp, pz);
                        const float4 va = s.vel[a];
                        const float pro = (va.x - vb.x) * xx + (va.y - vb.y) * xy + (va.z - vb.z) * xz;
                        if (pro < 0.f) {
                            const float m = c.rho0 * Vb / rhoa;
                            const float tv = f * pro / (len2 + den0) * m * visc;
                            vx = fmaf(xx, tv, vx);
                            vy = fmaf(xy, tv, vy);
                            vz = fmaf(xz, tv, vz);
                        }
                    }
                }
        const float fx = c.fm0 * (px - vx), fy = c.fm0 * (py - vy), fz = c.fm0 * (pz - vz);
        s.bforce[q] = make_float4(fx, fy, fz, 0.f);
        const float* st = R.state + 25 * di;
        const double rx = (double)pb.x - st[16], ry = (double)pb.y - st[17], rz = (double)pb.z - st[18];
        acc[0] = fx;
        acc[1] = fy;
        acc[2] = fz;
        acc[3] = ry * fz - rz * fy;
        acc[4] = rz * fx - rx * fz;
        acc[5] = rx * fy - ry * fx;
    }
    __shared__ double sh[BS / 32];
    double bs[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) bs[i] = block_sum_double<BS>(acc[i], sh);
    __shared__ bool last;
    if (threadIdx.x == 0) {
        for (int i = 0; i < 6; ++i) R.partial[6 * (size_t)blockIdx.x + i] = bs[i];
        __threadfence();
        last = atomicAdd(&R.ticket[di], 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    double tot[6] = {0, 0, 0, 0, 0, 0};
    for (int b = 0; b < (int)gridDim.x; ++b)
        for (int i = 0; i < 6; ++i) tot[i] += ((volatile double*)R.partial)[6 * (size_t)b + i];
    for (int i = 0; i < 6; ++i) R.out[6 * di + i] = tot[i];
    R.ticket[di] = 0u;
}
}  // namespace

static inline int nblk(int n, int bs) { return (n > 0 ? n + bs - 1 : bs) / bs; }

size_t rigid_sort_bytes(int nb, int end_bit) {
    size_t bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, bytes, (const int*)nullptr, (int*)nullptr, (const int*)nullptr,
                                    (int*)nullptr, nb, 0, end_bit);
    return bytes;
}

void launch_rigid_place_sort(const DevScene& s, const RigidDev& R, const GridGeom& g, void* sort_tmp,
                             size_t sort_bytes, int end_bit, cudaStream_t st) {
    if (R.nb <= 0) return;
    k_rigid_place<<<nblk(R.nb, NT), NT, 0, st>>>(s, R, g);
    size_t b = sort_bytes;
    cub::DeviceRadixSort::SortPairs(sort_tmp, b, (const int*)R.key_in, R.key_out, (const int*)R.val_in, R.val_out,
                                    R.nb, 0, end_bit, st);
    k_rigid_gather<<<nblk(R.nb, NT), NT, 0, st>>>(s, R);
    k_bcell_bounds<<<nblk(g.nkeys + 1, 256), 256, 0, st>>>(s, R, g.nkeys);
}

void launch_rigid_prepare(const DevScene& s, const RigidDev& R, const GridGeom& g, float dpart, float h2cut, int cap,
                          cudaStream_t st) {
    if (R.nb > 0) k_rigid_prepare<<<nblk(R.nb, NT), NT, 0, st>>>(s, R, g, dpart, h2cut, cap);
}

void launch_rigid_volume(const DevScene& s, const RigidDev& R, const GridGeom& g, float dpart, float h2cut, int cap,
                         cudaStream_t st) {
    if (R.nb > 0) k_rigid_volume<<<nblk(R.nb, NT), NT, 0, st>>>(s, R, g, dpart, h2cut, cap);
}

void launch_rigid_force(const DevScene& s, const RigidDev& R, const SolverConst& c, const GridGeom& g, int r0, int r1,
                        int di, cudaStream_t st) {
    if (r1 > r0) k_rigid_force<NT><<<nblk(r1 - r0, NT), NT, 0, st>>>(s, R, c, g, r0, r1, di);
}
