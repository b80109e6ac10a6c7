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
//   k_rigid_force     per boundary particle of a dynamic solid (one warp,
//                     a lane per neighbour cell): gathers its fluid
//                     neighbours (the fluid particles whose capped list
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
//   counting sort     per-cell counts (k_rigid_place), exclusive scan into
//                     the boundary cell table, scatter, then the in-cell rank
//                     by descending reference index -- the reference's
//                     linked-list order -- with the gather into the sorted
//                     arrays and the inverse permutation (k_rigid_rank)
//   k_rigid_volume    updateSolidPartWeight after the fluid sort: the
//                     boundary particle's capped list in the reference's
//                     order (fluid candidates count toward the cap; same-solid
//                     particles are skipped, SphBase.cpp:922)
//   k_rigid_prepare   prepareSolidPartWeight over the boundary alone
//                     (kerSumFromSelf and volume), when a solid turns dynamic
#include <cub/device/device_scan.cuh>

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
    R.key[r] = key;
    R.slot[r] = atomicAdd(&R.cnt[key], 1);
}

__global__ void __launch_bounds__(NT) k_rigid_scatter(DevScene s, RigidDev R) {
    const int r = blockIdx.x * NT + threadIdx.x;
    if (r < R.nb) R.tmp[s.bcell_start[R.key[r]] + R.slot[r]] = r;
}

// sorted slot q holds reference particle tmp[q] of cell [a, b); its final
// slot is a + #{particles of the cell with a larger reference index}
__global__ void __launch_bounds__(NT) k_rigid_rank(DevScene s, RigidDev R) {
    const int q0 = blockIdx.x * NT + threadIdx.x;
    if (q0 >= R.nb) return;
    const int r = R.tmp[q0];
    const int key = R.key[r];
    const int a = s.bcell_start[key], b = s.bcell_start[key + 1];
    int rank = 0;
    for (int j = a; j < b; ++j) rank += R.tmp[j] > r;
    const int q = a + rank;
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
    // no particle of another solid within the cut: the list adds nothing
    bool other = false;
    for (int dz = -1; dz <= 1 && !other; ++dz)
        for (int dy = -1; dy <= 1 && !other; ++dy)
            for (int dx = -1; dx <= 1 && !other; ++dx) {
                const int x = cx + dx, y = cy + dy, z = cz + dz;
                if (!cell_inside(g, x, y, z)) continue;
                const int key = cell_key(g, x, y, z);
                for (int b = s.bcell_start[key], e = s.bcell_start[key + 1]; b < e && !other; ++b) {
                    if (s.bsid[b] == sid) continue;
                    const float4 pb = s.bpos[b];
                    other = dis_square_rn(pa.x, pa.y, pa.z, pb.x, pb.y, pb.z) < h2cut;
                }
            }
    if (!other) {
        set_volume(s, R, q, 1.f / sum);
        return;
    }
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
// One warp per boundary particle, lane l < 27 scanning cell l of the 27 (x
// fastest); the lanes' sums meet in a fixed shuffle tree, the particles'
// FP64 force and torque in fixed-order block and grid sums.
template <int BS>
__global__ void __launch_bounds__(BS) k_rigid_force(DevScene s, RigidDev R, SolverConst c, GridGeom g, int r0, int r1,
                                                    int di) {
    constexpr int WPB = BS / 32;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int r = r0 + blockIdx.x * WPB + wid;
    __shared__ double wsum[WPB][6];
    if (r < r1) {
        const int q = R.binv[r];
        const float4 pb = s.bpf[2 * q], vb = s.bpf[2 * q + 1];
        const float Vb = pb.w;
        float px = 0.f, py = 0.f, pz = 0.f, vx = 0.f, vy = 0.f, vz = 0.f;
        if (lane < 27) {
            const int x = cell_coord(pb.x, g.min[0], g.divisor) + lane % 3 - 1;
            const int y = cell_coord(pb.y, g.min[1], g.divisor) + (lane / 3) % 3 - 1;
            const int z = cell_coord(pb.z, g.min[2], g.divisor) + lane / 9 - 1;
            if (cell_inside(g, x, y, z)) {
                const int key = cell_key(g, x, y, z);
                const int a0 = s.cstart2[key].x, a1 = s.cstart2[key + 1].x;
                const float den0 = 0.01f * c.hs * c.hs;
                const float visc = 10.f * c.nu;
                const size_t stride = (size_t)c.stride;
                const int me = (int)((unsigned)q | BND_FLAG);
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
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            px += __shfl_down_sync(0xffffffffu, px, o);
            py += __shfl_down_sync(0xffffffffu, py, o);
            pz += __shfl_down_sync(0xffffffffu, pz, o);
            vx += __shfl_down_sync(0xffffffffu, vx, o);
            vy += __shfl_down_sync(0xffffffffu, vy, o);
            vz += __shfl_down_sync(0xffffffffu, vz, o);
        }
        if (lane == 0) {
            const float fx = c.fm0 * (px - vx), fy = c.fm0 * (py - vy), fz = c.fm0 * (pz - vz);
            s.bforce[q] = make_float4(fx, fy, fz, 0.f);
            const float* st = R.state + 25 * di;
            const double rx = (double)pb.x - st[16], ry = (double)pb.y - st[17], rz = (double)pb.z - st[18];
            wsum[wid][0] = fx;
            wsum[wid][1] = fy;
            wsum[wid][2] = fz;
            wsum[wid][3] = ry * fz - rz * fy;
            wsum[wid][4] = rz * fx - rx * fz;
            wsum[wid][5] = rx * fy - ry * fx;
        }
    } else if (lane == 0) {
        for (int i = 0; i < 6; ++i) wsum[wid][i] = 0.0;
    }
    __syncthreads();
    __shared__ bool last;
    if (threadIdx.x == 0) {
        for (int i = 0; i < 6; ++i) {
            double b = 0.0;
            for (int w = 0; w < WPB; ++w) b += wsum[w][i];
            R.partial[6 * (size_t)blockIdx.x + i] = b;
        }
        __threadfence();
        last = atomicAdd(&R.ticket[di], 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    // the last block: thread t sums blocks t, t + BS, ... in order, then a
    // fixed tree over the threads
    __shared__ double sh[BS / 32];
    for (int i = 0; i < 6; ++i) {
        double v = 0.0;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += BS) v += ((volatile double*)R.partial)[6 * (size_t)b + i];
        const double tot = block_sum_double<BS>(v, sh);
        if (threadIdx.x == 0) R.out[6 * di + i] = tot;
    }
    if (threadIdx.x == 0) R.ticket[di] = 0u;
}
}  // namespace

static inline int nblk(int n, int bs) { return (n > 0 ? n + bs - 1 : bs) / bs; }

void launch_rigid_place_sort(const DevScene& s, const RigidDev& R, const GridGeom& g, void* scan_tmp,
                             size_t scan_bytes, cudaStream_t st) {
    if (R.nb <= 0) return;
    cudaMemsetAsync(R.cnt, 0, sizeof(int) * ((size_t)g.nkeys + 1), st);
    k_rigid_place<<<nblk(R.nb, NT), NT, 0, st>>>(s, R, g);
    size_t b = scan_bytes;
    cub::DeviceScan::ExclusiveSum(scan_tmp, b, R.cnt, s.bcell_start, g.nkeys + 1, st);
    k_rigid_scatter<<<nblk(R.nb, NT), NT, 0, st>>>(s, R);
    k_rigid_rank<<<nblk(R.nb, NT), NT, 0, st>>>(s, R);
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
    if (r1 > r0) k_rigid_force<NT><<<nblk(r1 - r0, NT / 32), NT, 0, st>>>(s, R, c, g, r0, r1, di);
}
