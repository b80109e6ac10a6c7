// sph_surface.cu -- surface reconstruction of a particle fluid on the GPU:
// the scalar field of surface_field (isotropic splat, surface_field.cpp:
// 43-75; anisotropic kernels after Yu & Turk 2010, surface_field.cpp:83-176)
// and marchingCubes (marching_cubes.cpp:45-120), behind the C ABI of
// include/sphgpu.h (sphgpu_surface_*).
//
// Field pipeline (one handle holds the grid of surface_setup,
// surface_field.cpp:8-41):
//   k_sf_key / counting sort   particles into the neighbour grid (cells of
//                              h_field = 2 r_h, surface_field.cpp:23-27),
//                              within a cell by ascending index
//   k_sf_kernel                per particle: the weighted mean of its
//                              neighbours within h_field (weights
//                              1 - (r/h_field)^3, Equation 11) and, with at
//                              least N_e = 25 neighbours, the weighted
//                              covariance about it, its eigen-decomposition
//                              (cyclic Jacobi, FP64), the clamped and scaled
//                              singular values (k_r, k_s) and
//                              G = V diag(1/s) V^T; otherwise the isotropic
//                              G = k_n (3 - 2 n / N_e) I.  Out: centre, G,
//                              det G and the node box the reference loops
//                              over (its cell +- int(h_cell_num s_max), +1 on
//                              the upper side, clamped to the grid)
//   tile binning               the grid in 8x16x16-node tiles; every particle
//                              is listed under each tile its box touches
//                              (count, scan, emit, stable radix sort by tile:
//                              within a tile in ascending particle order)
//   k_sf_field                 one CTA per tile: its particles staged in
//                              shared memory in chunks, each thread sums the
//                              8 nodes of its x-row, det G W(|G (x - c)|),
//                              over them in particle order (no atomics:
//                              deterministic); along a row |G (x - c)|^2 is
//                              a quadratic in the node index, so only the
//                              nodes in its root interval are evaluated
// The isotropic field is the same with G = I and the box +- h_cell_num.
//
// Marching cubes: k_mc_count (each thread 4 consecutive x-cubes: their case
// bytes, and the triangles per block from the case table), exclusive scan
// over the blocks, k_mc_emit (the block's case bytes again, an in-block
// scan; cubes with triangles gather their corners; cut-edge vertices
// interpolated as
// VertexInterp does, marching_cubes.cpp:39-40, in round-to-nearest float
// ops; triangles in cube order z, y, x, each cube's in table order).  The
// case table is built at start-up by mc_build_table() from first principles
// (face walks, see there); it cuts the same polygons out of every cube as the
// reference's table and may split them along other diagonals.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/sphgpu.h"
#include "sph_sync.cuh"

namespace {

// field tiles: 8 (x) x 16 (y) x 16 (z) nodes, one thread per x-row of 8
constexpr int TX = 8, TY = 16, TZ = 16;
constexpr int FT = TY * TZ;          // threads of the field kernel
constexpr int MCB = 256;             // threads per marching-cubes block
constexpr int MCX = 4;               // consecutive x-cubes per marching-cubes thread

// ---------------- marching-cubes case table ----------------
// Cube numbering of marching_cubes.cpp:9-31: vertex v at (x, y, z) bits
// below, edge e joins kEdge[e][0] -> kEdge[e][1] (the interpolation runs
// from the first vertex, as VertexInterp's arguments do, :79-102).
constexpr int kVert[8][3] = {{0, 0, 0}, {0, 0, 1}, {0, 1, 1}, {0, 1, 0}, {1, 0, 0}, {1, 0, 1}, {1, 1, 1}, {1, 1, 0}};
constexpr int kEdge[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6}, {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};

__constant__ signed char c_tri[256][16];
__constant__ unsigned char c_ntri[256];
__constant__ int c_vert[8][3];
__constant__ int c_edge[12][2];

// The table: on every face, walk its corners counter-clockwise seen from
// outside; each maximal run of "in" corners (value < iso) becomes one
// segment from the edge where the walk enters the run to the edge where it
// leaves it -- two diagonal "in" corners of a face are cut off separately,
// the same choice on both cubes sharing the face, so the mesh is closed.
// Each cut edge ends one segment and starts the next: the segments chain
// into closed loops, each loop of k edges fanned into k - 2 triangles
// (loop[0], loop[j + 1], loop[j]), the facing of the reference's output.
void mc_build_table(signed char tri[256][16], unsigned char ntri[256]) {
    // faces as corner cycles, counter-clockwise seen from outside
    int faces[6][4];
    for (int axis = 0, f = 0; axis < 3; ++axis)
        for (int side = 0; side < 2; ++side, ++f) {
            int cs[4], m = 0;
            for (int v = 0; v < 8; ++v)
                if (kVert[v][axis] == side) cs[m++] = v;
            const int a = (axis + 1) % 3, b = (axis + 2) % 3;
            const double sgn = side ? 1.0 : -1.0;  // outward normal along axis
            double ang[4];
            for (int i = 0; i < 4; ++i) {
                // in-plane coordinates about the face centre, in the frame
                // (e_a, n x e_a) that is right-handed with the normal n
                const double u = kVert[cs[i]][a] - 0.5, w = kVert[cs[i]][b] - 0.5;
                ang[i] = std::atan2(sgn * w, u);
            }
            int ord[4] = {0, 1, 2, 3};
            std::sort(ord, ord + 4, [&](int p, int q) { return ang[p] < ang[q]; });
            for (int i = 0; i < 4; ++i) faces[f][i] = cs[ord[i]];
        }
    auto edge_of = [](int p, int q) {
        for (int e = 0; e < 12; ++e)
            if ((kEdge[e][0] == p && kEdge[e][1] == q) || (kEdge[e][0] == q && kEdge[e][1] == p)) return e;
        return -1;
    };
    for (int c = 0; c < 256; ++c) {
        int nxt[12];
        for (int e = 0; e < 12; ++e) nxt[e] = -1;
        auto in = [&](int v) { return (c >> v) & 1; };
        for (int f = 0; f < 6; ++f) {
            const int* fc = faces[f];
            for (int i = 0; i < 4; ++i) {
                const int p = fc[i], q = fc[(i + 1) % 4];
                if (!in(p) && in(q)) {
                    int j = (i + 1) % 4;
                    while (in(fc[(j + 1) % 4])) j = (j + 1) % 4;
                    nxt[edge_of(p, q)] = edge_of(fc[j], fc[(j + 1) % 4]);
                }
            }
        }
        int n = 0;
        bool seen[12] = {false};
        for (int e = 0; e < 12; ++e) {
            if (nxt[e] < 0 || seen[e]) continue;
            int loop[12], k = 0, x = e;
            do {
                loop[k++] = x;
                seen[x] = true;
                x = nxt[x];
            } while (x != e && k < 12);
            for (int j = 1; j + 1 < k; ++j) {
                tri[c][3 * n] = (signed char)loop[0];
                tri[c][3 * n + 1] = (signed char)loop[j + 1];
                tri[c][3 * n + 2] = (signed char)loop[j];
                ++n;
            }
        }
        for (int i = 3 * n; i < 16; ++i) tri[c][i] = -1;
        ntri[c] = (unsigned char)n;
    }
}

// ---------------- field kernels ----------------
struct SfParams {
    float gmin[3];     // field grid min (surface_field.cpp:16)
    int gnum[3];       // field grid nodes per axis
    float cell;
    double gmin_d[3], gdiv_d;  // FP64 copies for the box (the reference's double math)
    float pmin[3];     // neighbour grid (cells of h_field)
    int pnum[3];
    float pdiv;
    float h_field, h_field2, inv_hf3;
    float r_h, r_h2;
    float p1, p2, p3, p4;  // ker_spline constants (times the particle volume)
    float k_r, k_s, k_n;
    int n_e;
    int h_cell_num;
    int tiles[3];
};

__device__ __forceinline__ int pcell(const SfParams& P, float4 p, int& cx, int& cy, int& cz) {
    cx = (int)((p.x - P.pmin[0]) * P.pdiv);
    cy = (int)((p.y - P.pmin[1]) * P.pdiv);
    cz = (int)((p.z - P.pmin[2]) * P.pdiv);
    if (cx < 0 || cy < 0 || cz < 0 || cx >= P.pnum[0] || cy >= P.pnum[1] || cz >= P.pnum[2]) return -1;
    return (cz * P.pnum[1] + cy) * P.pnum[0] + cx;
}

__global__ void k_sf_key(SfParams P, const float4* pos, int n, int* key, int* slot, int* cnt, int* bad) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int cx, cy, cz;
    int k = pcell(P, pos[i], cx, cy, cz);
    if (k < 0) {
        atomicAdd(bad, 1);
        k = P.pnum[0] * P.pnum[1] * P.pnum[2];  // outside: a cell no scan reaches
    }
    key[i] = k;
    slot[i] = atomicAdd(&cnt[k], 1);
}

__global__ void k_sf_scatter(const int* key, const int* slot, const int* start, int n, int* tmp) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) tmp[start[key[i]] + slot[i]] = i;
}

// within a cell by ascending particle index
__global__ void k_sf_rank(const int* key, const int* start, const int* tmp, int n, int* sorted) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const int i = tmp[q], k = key[i];
    const int a = start[k], b = start[k + 1];
    int r = 0;
    for (int j = a; j < b; ++j) r += tmp[j] < i;
    sorted[a + r] = i;
}

// symmetric 3x3 eigen-decomposition by cyclic Jacobi rotations (FP64):
// m is destroyed; eigenvalues on its diagonal, eigenvectors the columns of v
__device__ void jacobi3(double m[3][3], double v[3][3]) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) v[i][j] = i == j ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 32; ++sweep) {
        const double off = fabs(m[0][1]) + fabs(m[0][2]) + fabs(m[1][2]);
        const double dia = fabs(m[0][0]) + fabs(m[1][1]) + fabs(m[2][2]);
        if (off == 0.0 || off <= dia * 1e-300) break;
        for (int p = 0; p < 2; ++p)
            for (int q = p + 1; q < 3; ++q) {
                if (m[p][q] == 0.0) continue;
                const double th = (m[q][q] - m[p][p]) / (2.0 * m[p][q]);
                const double t = (th >= 0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < 3; ++k) {
                    const double a = m[k][p], b = m[k][q];
                    m[k][p] = c * a - s * b;
                    m[k][q] = s * a + c * b;
                }
                for (int k = 0; k < 3; ++k) {
                    const double a = m[p][k], b = m[q][k];
                    m[p][k] = c * a - s * b;
                    m[q][k] = s * a + c * b;
                }
                for (int k = 0; k < 3; ++k) {
                    const double a = v[k][p], b = v[k][q];
                    v[k][p] = c * a - s * b;
                    v[k][q] = s * a + c * b;
                }
            }
    }
}

// Per particle: centre, G (symmetric, 6 values), det G, node box.
// rec0 = (cx, cy, cz, det), rec1 = (gxx, gxy, gxz, gyy), rec2 = (gyz, gzz, -, -),
// box_lo / box_hi = inclusive node ranges.
__global__ void __launch_bounds__(128) k_sf_kernel(SfParams P, const float4* pos, int n, const int* sorted,
                                                   const int* start, int aniso, float4* rec0, float4* rec1,
                                                   float4* rec2, int4* box_lo, int4* box_hi) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 pi = pos[i];
    float cxr = pi.x, cyr = pi.y, czr = pi.z;  // centre
    float g[6] = {1.f, 0.f, 0.f, 1.f, 0.f, 1.f};
    float det = 1.f;
    double smax = 1.0;
    double ext[3] = {-1.0, -1.0, -1.0};  // the ellipsoid's half-extents per axis (aniso only)
    if (aniso) {
        int cx, cy, cz;
        const int home = pcell(P, pi, cx, cy, cz);
        float sw = 0.f, sx = 0.f, sy = 0.f, sz = 0.f;
        int nn = 0;
        if (home >= 0) {
            for (int dz = -1; dz <= 1; ++dz)
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dx = -1; dx <= 1; ++dx) {
                        const int x = cx + dx, y = cy + dy, z = cz + dz;
                        if (x < 0 || y < 0 || z < 0 || x >= P.pnum[0] || y >= P.pnum[1] || z >= P.pnum[2]) continue;
                        const int k = (z * P.pnum[1] + y) * P.pnum[0] + x;
                        for (int q = start[k]; q < start[k + 1]; ++q) {
                            const int j = sorted[q];
                            if (j == i) continue;
                            const float4 pj = pos[j];
                            const float ex = pj.x - pi.x, ey = pj.y - pi.y, ez = pj.z - pi.z;
                            const float l2 = ex * ex + ey * ey + ez * ez;
                            if (!(l2 <= P.h_field2)) continue;
                            const float r = sqrtf(l2);
                            const float w = 1.f - r * r * r * P.inv_hf3;  // Equation (11)
                            sw += w;
                            sx = fmaf(w, ex, sx);
                            sy = fmaf(w, ey, sy);
                            sz = fmaf(w, ez, sz);
                            ++nn;
                        }
                    }
        }
        if (nn >= P.n_e) {
            // weighted mean (Equation 10), relative to the particle; lambda = 1 (Equation 6)
            const float mx = sx / sw, my = sy / sw, mz = sz / sw;
            double C[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
            for (int dz = -1; dz <= 1; ++dz)
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dx = -1; dx <= 1; ++dx) {
                        const int x = cx + dx, y = cy + dy, z = cz + dz;
                        if (x < 0 || y < 0 || z < 0 || x >= P.pnum[0] || y >= P.pnum[1] || z >= P.pnum[2]) continue;
                        const int k = (z * P.pnum[1] + y) * P.pnum[0] + x;
                        for (int q = start[k]; q < start[k + 1]; ++q) {
                            const int j = sorted[q];
                            if (j == i) continue;
                            const float4 pj = pos[j];
                            const float ex = pj.x - pi.x, ey = pj.y - pi.y, ez = pj.z - pi.z;
                            const float l2 = ex * ex + ey * ey + ez * ez;
                            if (!(l2 <= P.h_field2)) continue;
                            const float r = sqrtf(l2);
                            const double w = 1.f - r * r * r * P.inv_hf3;
                            const double ax = (double)ex - mx, ay = (double)ey - my, az = (double)ez - mz;
                            C[0][0] += w * ax * ax;
                            C[0][1] += w * ax * ay;
                            C[0][2] += w * ax * az;
                            C[1][1] += w * ay * ay;
                            C[1][2] += w * ay * az;
                            C[2][2] += w * az * az;
                        }
                    }
            C[1][0] = C[0][1];
            C[2][0] = C[0][2];
            C[2][1] = C[1][2];
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) C[a][b] /= (double)sw;  // Equation (9)
            double V[3][3];
            jacobi3(C, V);
            double ev[3] = {fabs(C[0][0]), fabs(C[1][1]), fabs(C[2][2])};
            int o[3] = {0, 1, 2};
            for (int a = 0; a < 3; ++a)
                for (int b = a + 1; b < 3; ++b)
                    if (ev[o[b]] > ev[o[a]]) { const int t = o[a]; o[a] = o[b]; o[b] = t; }
            double s[3] = {ev[o[0]], ev[o[1]], ev[o[2]]};
            s[1] = fmax(s[1], s[0] / P.k_r);  // Equation (15)
            s[2] = fmax(s[2], s[0] / P.k_r);
            for (int a = 0; a < 3; ++a) s[a] = fmax(s[a] * P.k_s, 1e-30);
            double G[3][3];
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) {
                    double t = 0;
                    for (int k = 0; k < 3; ++k) t += V[a][o[k]] * V[b][o[k]] / s[k];
                    G[a][b] = t;
                }
            g[0] = (float)G[0][0];
            g[1] = (float)G[0][1];
            g[2] = (float)G[0][2];
            g[3] = (float)G[1][1];
            g[4] = (float)G[1][2];
            g[5] = (float)G[2][2];
            det = (float)(1.0 / (s[0] * s[1] * s[2]));
            smax = s[0];
            // {x : |G (x - c)| <= r_h} = {c + V diag(s) V^T u : |u| <= r_h}:
            // along axis a it reaches r_h |row a of V diag(s)|
            for (int a = 0; a < 3; ++a) {
                double e2 = 0.0;
                for (int k = 0; k < 3; ++k) e2 += V[a][o[k]] * s[k] * V[a][o[k]] * s[k];
                ext[a] = (double)P.r_h * sqrt(e2);
            }
            cxr = pi.x + mx;
            cyr = pi.y + my;
            czr = pi.z + mz;
        } else {
            const float k = P.k_n * (3.f - 2.f * (float)nn / (float)P.n_e);
            g[0] = g[3] = g[5] = k;
            det = k * k * k;
            smax = 1.0 / P.k_n;
        }
    }
    rec0[i] = make_float4(cxr, cyr, czr, det);
    rec1[i] = make_float4(g[0], g[1], g[2], g[3]);
    rec2[i] = make_float4(g[4], g[5], 0.f, 0.f);
    // the node box of surface_field.cpp:140-145 (66-70 isotropic)
    const int hw = aniso ? (int)(P.h_cell_num * smax) : P.h_cell_num;
    const double cc[3] = {cxr, cyr, czr};
    int lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
        const int c = (int)((cc[a] - P.gmin_d[a]) * P.gdiv_d);
        lo[a] = max(c - hw, 0);
        hi[a] = min(c + hw + 1, P.gnum[a] - 1);
        // The reference's box bounds the ellipsoid's circumscribed sphere;
        // nodes outside the ellipsoid add nothing (W = 0 beyond r_h), so the
        // box is cut to the ellipsoid's axis-aligned extent, one node of
        // margin each side (the field's own r <= r_h test decides within).
        if (ext[a] >= 0.0) {
            const double u = (cc[a] - P.gmin_d[a]) * P.gdiv_d, e = ext[a] * P.gdiv_d;
            lo[a] = max(lo[a], (int)floor(u - e) - 1);
            hi[a] = min(hi[a], (int)ceil(u + e) + 1);
        }
    }
    box_lo[i] = make_int4(lo[0], lo[1], lo[2], 0);
    box_hi[i] = make_int4(hi[0], hi[1], hi[2], 0);
}

// tiles a particle's box touches
__device__ __forceinline__ int tile_span(int4 lo, int4 hi, int a) {
    const int l = (&lo.x)[a], h = (&hi.x)[a];
    const int t = a == 0 ? TX : (a == 1 ? TY : TZ);
    return h < l ? 0 : h / t - l / t + 1;
}

__global__ void k_sf_tile_count(const int4* box_lo, const int4* box_hi, int n, int* npair) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int4 lo = box_lo[i], hi = box_hi[i];
    npair[i] = tile_span(lo, hi, 0) * tile_span(lo, hi, 1) * tile_span(lo, hi, 2);
}

__global__ void k_sf_tile_emit(SfParams P, const int4* box_lo, const int4* box_hi, int n, const int* off, int* ptile,
                               int* ppart) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int4 lo = box_lo[i], hi = box_hi[i];
    if (hi.x < lo.x || hi.y < lo.y || hi.z < lo.z) return;
    int o = off[i];
    for (int tz = lo.z / TZ; tz <= hi.z / TZ; ++tz)
        for (int ty = lo.y / TY; ty <= hi.y / TY; ++ty)
            for (int tx = lo.x / TX; tx <= hi.x / TX; ++tx) {
                ptile[o] = (tz * P.tiles[1] + ty) * P.tiles[0] + tx;
                ppart[o] = i;
                ++o;
            }
}

__global__ void k_sf_tile_bounds(const int* tile_sorted, long long npairs, int ntiles, int* tstart) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t > ntiles) return;
    long long lo = 0, hi = npairs;
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        if (tile_sorted[mid] < t) lo = mid + 1;
        else hi = mid;
    }
    tstart[t] = (int)lo;
}

// PTX sqrt.approx (relative error within a few ulp; sqrt(0) = 0), for the
// splat's distances, which only feed the spline
__device__ __forceinline__ float sqrt_approx(float x) {
    float y;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// ker_spline (surface_field.cpp:235-249), times the particle volume
__device__ __forceinline__ float sf_spline(const SfParams& P, float r) {
    const float hr = P.r_h - r;
    return r < 0.5f * P.r_h ? fmaf(P.p3 * r, r * r, fmaf(P.p2, r * r, P.p1)) : P.p4 * hr * hr * hr;
}

// One CTA per tile, one thread per x-row of 8 nodes.  Along a row the
// transformed offset u = G (x - c) is linear in the node index k, so
// r^2(k) = |u0|^2 + 2 (u0.du) k + |du|^2 k^2 (du = G e_x cell, staged with the
// particle) and r^2 <= r_h^2 holds on the interval between the quadratic's
// roots (widened by one node each side); the nodes in it are tested directly
// with r^2 from the polynomial in k.
__global__ void __launch_bounds__(FT) k_sf_field(SfParams P, const int* tstart, const int* ppart, const float4* rec0,
                                                 const float4* rec1, const float4* rec2, const int4* box_lo,
                                                 const int4* box_hi, float* field) {
    const int t = blockIdx.x;
    const int tx = t % P.tiles[0], ty = (t / P.tiles[0]) % P.tiles[1], tz = t / (P.tiles[0] * P.tiles[1]);
    __shared__ float4 s0[FT], s1[FT], s3[FT];
    __shared__ float4 s2[FT];
    __shared__ int4 slo[FT], shi[FT];
    const int y = ty * TY + (int)(threadIdx.x % TY), z = tz * TZ + (int)(threadIdx.x / TY);
    const int x0 = tx * TX;
    const bool row = y < P.gnum[1] && z < P.gnum[2];
    const int xlast = min(TX - 1, P.gnum[0] - 1 - x0);
    const float px0 = P.gmin[0] + (float)x0 * P.cell;
    const float py = P.gmin[1] + (float)y * P.cell, pz = P.gmin[2] + (float)z * P.cell;
    const float rh = P.r_h, rh2 = P.r_h2, hh = 0.5f * P.r_h;
    float acc[TX];
#pragma unroll
    for (int k = 0; k < TX; ++k) acc[k] = 0.f;
    const int a0 = tstart[t], a1 = tstart[t + 1];
    for (int base = a0; base < a1; base += FT) {
        const int m = min(FT, a1 - base);
        __syncthreads();
        if ((int)threadIdx.x < m) {
            const int i = ppart[base + threadIdx.x];
            const float4 g = rec1[i], g2 = rec2[i];
            s0[threadIdx.x] = rec0[i];
            s1[threadIdx.x] = g;
            const float dx = g.x * P.cell, dy = g.y * P.cell, dz = g.z * P.cell;
            const float A = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            s2[threadIdx.x] = make_float4(g2.x, g2.y, 1.f / A, 0.f);
            s3[threadIdx.x] = make_float4(dx, dy, dz, A);
            slo[threadIdx.x] = box_lo[i];
            shi[threadIdx.x] = box_hi[i];
        }
        __syncthreads();
        if (!row) continue;
        for (int j = 0; j < m; ++j) {
            const int4 lo = slo[j], hi = shi[j];
            if (y < lo.y || y > hi.y || z < lo.z || z > hi.z) continue;
            const int xa = max(lo.x - x0, 0), xb = min(hi.x - x0, xlast);
            if (xa > xb) continue;
            const float4 c = s0[j], g = s1[j], g2 = s2[j], du = s3[j];
            const float vx = px0 - c.x, vy = py - c.y, vz = pz - c.z;
            // G = [[gxx gxy gxz] [gxy gyy gyz] [gxz gyz gzz]]; u0 = G v
            const float ux = fmaf(g.x, vx, fmaf(g.y, vy, g.z * vz));
            const float uy = fmaf(g.y, vx, fmaf(g.w, vy, g2.x * vz));
            const float uz = fmaf(g.z, vx, fmaf(g2.x, vy, g2.y * vz));
            const float B = fmaf(ux, du.x, fmaf(uy, du.y, uz * du.z));
            const float C0 = fmaf(ux, ux, fmaf(uy, uy, uz * uz));
            const float disc = fmaf(B, B, -du.w * (C0 - rh2));
            // min_k r^2 = r_h^2 - disc / |du|^2: the row misses the ellipsoid
            // (kept when within rounding of touching it)
            if (disc < -1e-5f * rh2 * du.w) continue;
            const float sq = disc > 0.f ? disc * rsqrtf(disc) : 0.f;
            const int ka = max(xa, (int)floorf((-B - sq) * g2.z) - 1);
            const int kb = min(xb, (int)ceilf((-B + sq) * g2.z) + 1);
            const float B2 = 2.f * B;
            // the row's two halves, each evaluated only when the interval
            // reaches it (adjacent rows of a warp mostly agree)
#pragma unroll
            for (int half = 0; half < 2; ++half) {
                if (half == 0 ? ka >= TX / 2 : kb < TX / 2) continue;
#pragma unroll
                for (int k = half * (TX / 2); k < (half + 1) * (TX / 2); ++k) {
                    if (k < ka || k > kb) continue;
                    const float fk = (float)k;
                    const float r2 = fmaf(fmaf(du.w, fk, B2), fk, C0);
                    if (!(r2 <= rh2)) continue;
                    // ker_spline (surface_field.cpp:235-249), times the particle
                    // volume: p1 + r^2 (p2 + p3 r) inside h/2, p4 (h - r)^3 beyond
                    const float r = sqrt_approx(r2);
                    const float hr = rh - r;
                    const float w = r < hh ? fmaf(fmaf(P.p3, r, P.p2), r2, P.p1) : (P.p4 * hr) * (hr * hr);
                    acc[k] = fmaf(c.w, w, acc[k]);
                }
            }
        }
    }
    if (row) {
        const size_t base = ((size_t)z * P.gnum[1] + y) * P.gnum[0] + x0;
#pragma unroll
        for (int k = 0; k < TX; ++k)
            if (k <= xlast) field[base + k] = acc[k];
    }
}

// ---------------- marching cubes ----------------
struct McParams {
    int res[3];          // nodes per axis
    int ref_rows;        // 1: the reference's row pairing (see sphgpu.h)
    float iso;
    const float* cx_lo;  // per cube index: its x, y, z extents
    const float* cx_hi;
    const float* cy_lo;
    const float* cy_hi;
    const float* cz_lo;
    const float* cz_hi;
};

__device__ __forceinline__ void mc_corners(const McParams& M, const float* f, long long c, int& x, int& y, int& z,
                                           float v[8]) {
    const int nx = M.res[0] - 1, ny = M.res[1] - 1;
    x = (int)(c % nx);
    y = (int)((c / nx) % ny);
    z = (int)(c / ((long long)nx * ny));
    // y rows of the cube's low and high side: y, y + 1; with ref_rows the
    // reference's caches give rows max(y - 1, 0) and y (marching_cubes.cpp:56-65)
    const int ylo = M.ref_rows ? max(y - 1, 0) : y, yhi = M.ref_rows ? y : y + 1;
    const long long plane = (long long)M.res[0] * M.res[1];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int xx = x + c_vert[k][0], yy = c_vert[k][1] ? yhi : ylo, zz = z + c_vert[k][2];
        v[k] = f[zz * plane + (long long)yy * M.res[0] + xx];
    }
}

__device__ __forceinline__ int mc_case(const McParams& M, const float v[8]) {
    int cs = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) cs |= (v[k] < M.iso) << k;
    return cs;
}

// A thread takes MCX consecutive cubes of one x-row (a group); groups are
// numbered row by row, so group order is cube order.
__device__ __forceinline__ void mc_group(const McParams& M, long long g, int gpr, int& x0, int& xe, int& y, int& z) {
    const int ncx = M.res[0] - 1, ncy = M.res[1] - 1;
    const long long r = g / gpr;
    x0 = (int)(g % gpr) * MCX;
    xe = min(x0 + MCX, ncx);
    y = (int)(r % ncy);
    z = (int)(r / ncy);
}

// pass 1: the case of every cube (one byte) and the triangles per block of
// MCB groups; a group reads its 4 node rows once (MCX + 1 nodes each)
__global__ void __launch_bounds__(MCB) k_mc_count(McParams M, const float* f, long long ngroups, int gpr,
                                                  unsigned char* cases, int* bcount) {
    const long long g = (long long)blockIdx.x * MCB + threadIdx.x;
    int n = 0;
    if (g < ngroups) {
        int x0, xe, y, z;
        mc_group(M, g, gpr, x0, xe, y, z);
        const int ylo = M.ref_rows ? max(y - 1, 0) : y, yhi = M.ref_rows ? y : y + 1;
        const long long plane = (long long)M.res[0] * M.res[1];
        // rows of vertices 0, 1, 2, 3 (x low side; 4..7 are the same rows at x + 1)
        const float* r0 = f + z * plane + (long long)ylo * M.res[0];
        const float* r1 = f + (z + 1) * plane + (long long)ylo * M.res[0];
        const float* r2 = f + (z + 1) * plane + (long long)yhi * M.res[0];
        const float* r3 = f + z * plane + (long long)yhi * M.res[0];
        int lo = (r0[x0] < M.iso) | ((r1[x0] < M.iso) << 1) | ((r2[x0] < M.iso) << 2) | ((r3[x0] < M.iso) << 3);
        const long long c0 = ((long long)z * (M.res[1] - 1) + y) * (M.res[0] - 1);
        for (int x = x0; x < xe; ++x) {
            const int hi =
                (r0[x + 1] < M.iso) | ((r1[x + 1] < M.iso) << 1) | ((r2[x + 1] < M.iso) << 2) | ((r3[x + 1] < M.iso) << 3);
            const int cs = lo | (hi << 4);
            cases[c0 + x] = (unsigned char)cs;
            n += c_ntri[cs];
            lo = hi;
        }
    }
    __shared__ int sh[MCB / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) n += __shfl_down_sync(0xffffffffu, n, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = n;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int w = 0; w < MCB / 32; ++w) t += sh[w];
        bcount[blockIdx.x] = t;
    }
}

// pass 2: the cases again, offsets by an in-block scan after the block's
// offset; only cubes with triangles gather their corners
__global__ void __launch_bounds__(MCB) k_mc_emit(McParams M, const float* f, long long ngroups, int gpr,
                                                 const unsigned char* cases, const int* bcount, const int* boff,
                                                 float* out) {
    // most blocks of cubes hold no surface: the whole block leaves at once
    if (bcount[blockIdx.x] == 0) return;
    const long long g = (long long)blockIdx.x * MCB + threadIdx.x;
    int x0 = 0, xe = 0, y = 0, z = 0, n = 0;
    long long c0 = 0;
    if (g < ngroups) {
        mc_group(M, g, gpr, x0, xe, y, z);
        c0 = ((long long)z * (M.res[1] - 1) + y) * (M.res[0] - 1);
        for (int x = x0; x < xe; ++x) n += c_ntri[cases[c0 + x]];
    }
    __shared__ int wsum[MCB / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int inc = n;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) wsum[wid] = inc;
    __syncthreads();
    int before = 0;
    for (int w = 0; w < wid; ++w) before += wsum[w];
    if (n == 0) return;
    long long first = (long long)boff[blockIdx.x] + before + inc - n;
    for (int x = x0; x < xe; ++x) {
        const int cs = cases[c0 + x];
        const int nc = c_ntri[cs];
        if (!nc) continue;
        int cx, cy, cz;
        float v[8];
        mc_corners(M, f, c0 + x, cx, cy, cz, v);
        const float lo[3] = {M.cx_lo[cx], M.cy_lo[cy], M.cz_lo[cz]};
        const float hi[3] = {M.cx_hi[cx], M.cy_hi[cy], M.cz_hi[cz]};
        float* o = out + 9 * first;
        for (int t = 0; t < 3 * nc; ++t) {
            const int e = c_tri[cs][t];
            const int a = c_edge[e][0], b = c_edge[e][1];
            const float va = v[a], vb = v[b];
            // VertexInterp (marching_cubes.cpp:39-40)
            const float mu = __fdiv_rn(__fsub_rn(M.iso, va), __fsub_rn(vb, va));
#pragma unroll
            for (int ax = 0; ax < 3; ++ax) {
                const float pa = c_vert[a][ax] ? hi[ax] : lo[ax];
                const float pb = c_vert[b][ax] ? hi[ax] : lo[ax];
                o[3 * t + ax] = __fadd_rn(pa, __fmul_rn(mu, __fsub_rn(pb, pa)));
            }
        }
        first += nc;
    }
}

inline int nblk(long long n, int bs) { return (int)((n + bs - 1) / bs); }

}  // namespace

// ======================= handle =======================
struct sphgpu_surface {
    int device = 0;
    cudaStream_t stream = nullptr;
    SfParams P{};
    double gmin[3] = {0, 0, 0}, cell = 0;
    int gnum[3] = {0, 0, 0};
    long long nnodes = 0;
    int ntiles = 0;
    long long npairs = 0;    // (tile, particle) pairs of the last field
    long long kernels = 0;   // this file's kernel launches, cumulative
    float* field = nullptr;
    // particles
    int pcap = 0;
    float* xyz = nullptr;  // host positions staged on the device
    float4 *pos = nullptr, *rec0 = nullptr, *rec1 = nullptr, *rec2 = nullptr;
    int4 *blo = nullptr, *bhi = nullptr;
    int *key = nullptr, *slot = nullptr, *tmp = nullptr, *sorted = nullptr, *npair = nullptr, *poff = nullptr;
    int* pcnt = nullptr;    // neighbour-grid cells + 2
    int* pstart = nullptr;
    int* bad = nullptr;
    // tile pairs
    long long paircap = 0;
    int *ptile = nullptr, *ppart = nullptr, *ptile_s = nullptr, *ppart_s = nullptr;
    int* tstart = nullptr;
    // marching cubes
    long long cubecap = 0, tricap = 0, ntris = 0;
    int* ntri = nullptr;  // triangles per block of MCB cube groups
    int* toff = nullptr;  // and the blocks' offsets
    unsigned char* cases = nullptr;  // case byte per cube
    long long casecap = 0;
    float* tris = nullptr;
    float* coords = nullptr;  // 6 coordinate tables
    void* tmpbuf = nullptr;
    size_t tmpbytes = 0;
    std::string err;
};

namespace {
#define SCK(x)                                                                                      \
    do {                                                                                            \
        cudaError_t e_ = (x);                                                                       \
        if (e_ != cudaSuccess) {                                                                    \
            s->err = std::string(#x) + ": " + cudaGetErrorString(e_);                               \
            return SPHGPU_ECUDA;                                                                    \
        }                                                                                           \
    } while (0)

// the case table lives in each device's constant memory
unsigned long long g_table_ready = 0;  // bit d: device d has it

int ensure_table(sphgpu_surface* s) {
    if (s->device < 64 && ((g_table_ready >> s->device) & 1ull)) return 0;
    signed char tri[256][16];
    unsigned char nt[256];
    mc_build_table(tri, nt);
    SCK(cudaMemcpyToSymbol(c_tri, tri, sizeof tri));
    SCK(cudaMemcpyToSymbol(c_ntri, nt, sizeof nt));
    SCK(cudaMemcpyToSymbol(c_vert, kVert, sizeof kVert));
    SCK(cudaMemcpyToSymbol(c_edge, kEdge, sizeof kEdge));
    if (s->device < 64) g_table_ready |= 1ull << s->device;
    return 0;
}

template <class T>
int salloc(sphgpu_surface* s, T** p, size_t n) {
    if (*p) cudaFree(*p);
    *p = nullptr;
    cudaError_t e = cudaMalloc((void**)p, std::max<size_t>(n, 1) * sizeof(T));
    if (e != cudaSuccess) {
        s->err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
        return SPHGPU_ENOMEM;
    }
    return 0;
}

int ensure_tmp(sphgpu_surface* s, size_t bytes) {
    if (bytes <= s->tmpbytes) return 0;
    if (s->tmpbuf) cudaFree(s->tmpbuf);
    s->tmpbuf = nullptr;
    if (cudaMalloc(&s->tmpbuf, bytes + 256) != cudaSuccess) {
        s->err = "cudaMalloc (scratch) failed";
        return SPHGPU_ENOMEM;
    }
    s->tmpbytes = bytes;
    return 0;
}

int ensure_particles(sphgpu_surface* s, int n) {
    if (n <= s->pcap) return 0;
    const int cap = std::max(n, 2 * s->pcap);
    int r = salloc(s, &s->pos, cap) | salloc(s, &s->rec0, cap) | salloc(s, &s->rec1, cap) | salloc(s, &s->rec2, cap) |
            salloc(s, &s->blo, cap) | salloc(s, &s->bhi, cap) | salloc(s, &s->key, cap) | salloc(s, &s->slot, cap) |
            salloc(s, &s->tmp, cap) | salloc(s, &s->sorted, cap) | salloc(s, &s->npair, (size_t)cap + 1) |
            salloc(s, &s->poff, (size_t)cap + 1) | salloc(s, &s->xyz, 3 * (size_t)cap);
    if (r) return SPHGPU_ENOMEM;
    s->pcap = cap;
    return 0;
}

__global__ void k_pack_xyz(const float* xyz, int n, float4* pos) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) pos[i] = make_float4(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], 0.f);
}

// the field of the n particles in s->pos
int run_field(sphgpu_surface* s, int n, int aniso) {
    cudaStream_t st = s->stream;
    const SfParams& P = s->P;
    const int pcells = P.pnum[0] * P.pnum[1] * P.pnum[2];
    // neighbour grid (anisotropic kernels only)
    if (aniso && n > 0) {
        SCK(cudaMemsetAsync(s->pcnt, 0, sizeof(int) * ((size_t)pcells + 2), st));
        SCK(cudaMemsetAsync(s->bad, 0, sizeof(int), st));
        s->kernels += 3;
        k_sf_key<<<nblk(n, 256), 256, 0, st>>>(P, s->pos, n, s->key, s->slot, s->pcnt, s->bad);
        size_t b = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, b, s->pcnt, s->pstart, pcells + 2, st);
        if (int r = ensure_tmp(s, b)) return r;
        cub::DeviceScan::ExclusiveSum(s->tmpbuf, b, s->pcnt, s->pstart, pcells + 2, st);
        k_sf_scatter<<<nblk(n, 256), 256, 0, st>>>(s->key, s->slot, s->pstart, n, s->tmp);
        k_sf_rank<<<nblk(n, 256), 256, 0, st>>>(s->key, s->pstart, s->tmp, n, s->sorted);
    }
    s->kernels += n > 0;
    if (n > 0)
        k_sf_kernel<<<nblk(n, 128), 128, 0, st>>>(P, s->pos, n, s->sorted, s->pstart, aniso, s->rec0, s->rec1, s->rec2,
                                                    s->blo, s->bhi);
    // tile pairs
    long long npairs = 0;
    if (n > 0) {
        ++s->kernels;
        k_sf_tile_count<<<nblk(n, 256), 256, 0, st>>>(s->blo, s->bhi, n, s->npair);
        SCK(cudaMemsetAsync(s->npair + n, 0, sizeof(int), st));
        size_t b = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, b, s->npair, s->poff, n + 1, st);
        if (int r = ensure_tmp(s, b)) return r;
        cub::DeviceScan::ExclusiveSum(s->tmpbuf, b, s->npair, s->poff, n + 1, st);
        int tot = 0;
        SCK(cudaMemcpyAsync(&tot, s->poff + n, sizeof(int), cudaMemcpyDeviceToHost, st));
        SCK(cudaStreamSynchronize(st));
        npairs = tot;
    }
    if (npairs > s->paircap) {
        const long long cap = std::max(npairs, 2 * s->paircap);
        if (salloc(s, &s->ptile, cap) | salloc(s, &s->ppart, cap) | salloc(s, &s->ptile_s, cap) |
            salloc(s, &s->ppart_s, cap))
            return SPHGPU_ENOMEM;
        s->paircap = cap;
    }
    if (npairs > 0) {
        ++s->kernels;
        k_sf_tile_emit<<<nblk(n, 256), 256, 0, st>>>(P, s->blo, s->bhi, n, s->poff, s->ptile, s->ppart);
        int bits = 1;
        while (bits < 31 && (1ll << bits) <= (long long)s->ntiles) ++bits;
        size_t b = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, b, s->ptile, s->ptile_s, s->ppart, s->ppart_s, (int)npairs, 0, bits,
                                        st);
        if (int r = ensure_tmp(s, b)) return r;
        cub::DeviceRadixSort::SortPairs(s->tmpbuf, b, s->ptile, s->ptile_s, s->ppart, s->ppart_s, (int)npairs, 0, bits,
                                        st);
    }
    s->npairs = npairs;
    s->kernels += 2;
    k_sf_tile_bounds<<<nblk((long long)s->ntiles + 1, 256), 256, 0, st>>>(s->ptile_s, npairs, s->ntiles, s->tstart);
    k_sf_field<<<s->ntiles, FT, 0, st>>>(P, s->tstart, s->ppart_s, s->rec0, s->rec1, s->rec2, s->blo, s->bhi,
                                          s->field);
    SCK(cudaGetLastError());
    SCK(cudaStreamSynchronize(st));
    return 0;
}
}  // namespace

// ======================= C ABI =======================
extern "C" {

int sphgpu_mc_table(int* ntri, signed char* tri) {
    if (!ntri || !tri) return SPHGPU_EINVAL;
    signed char t[256][16];
    unsigned char n[256];
    mc_build_table(t, n);
    for (int c = 0; c < 256; ++c) {
        ntri[c] = n[c];
        for (int k = 0; k < 16; ++k) tri[16 * c + k] = t[c][k];
    }
    return 0;
}

int sphgpu_surface_create(const double* mn, const double* mx, double r_p, double r_h, double cell_size, int device,
                          sphgpu_surface_t* out) {
    if (!mn || !mx || !out || !(r_p > 0) || !(r_h > 0) || !(cell_size > 0)) return SPHGPU_EINVAL;
    *out = nullptr;
    if (cudaSetDevice(device) != cudaSuccess) return SPHGPU_ECUDA;
    sphgpu_surface* s = new sphgpu_surface();
    s->device = device;
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete s;
        return SPHGPU_ECUDA;
    }
    // surface_setup (surface_field.cpp:8-41), in double as the reference
    SfParams& P = s->P;
    const double vol = r_p * r_p * r_p;
    s->cell = cell_size;
    for (int a = 0; a < 3; ++a) {
        s->gmin[a] = mn[a] - r_h * 0.75;
        s->gnum[a] = (int)((mx[a] - mn[a] + r_h * 1.5) / cell_size) + 1;
        P.gmin[a] = (float)s->gmin[a];
        P.gmin_d[a] = s->gmin[a];
        P.gnum[a] = s->gnum[a];
        P.tiles[a] = (s->gnum[a] + (a == 0 ? TX : (a == 1 ? TY : TZ)) - 1) / (a == 0 ? TX : (a == 1 ? TY : TZ));
    }
    P.gdiv_d = 1.0 / cell_size;
    P.cell = (float)cell_size;
    const double hf = 2 * r_h;
    for (int a = 0; a < 3; ++a) {
        P.pmin[a] = (float)(mn[a] - hf * 1.25);
        P.pnum[a] = (int)((mx[a] - mn[a] + hf * 2.5) / hf) + 1;
    }
    P.pdiv = (float)(1.0 / hf);
    P.h_field = (float)hf;
    P.h_field2 = (float)(hf * hf);
    P.inv_hf3 = (float)(1.0 / (hf * hf * hf));
    P.r_h = (float)r_h;
    P.r_h2 = (float)(r_h * r_h);
    P.p1 = (float)(8.0 / (M_PI * std::pow(r_h, 3.0)) * vol);
    P.p2 = (float)(-48.0 / (M_PI * std::pow(r_h, 5.0)) * vol);
    P.p3 = (float)(48.0 / (M_PI * std::pow(r_h, 6.0)) * vol);
    P.p4 = (float)(16.0 / (M_PI * std::pow(r_h, 6.0)) * vol);
    P.k_r = 4.f;                                         // Equation (15)
    P.k_s = (float)(1.0 / (0.16 * hf * hf) * 1.6);
    P.k_n = 0.95f;
    P.n_e = 25;
    P.h_cell_num = (int)(r_h / cell_size);
    s->nnodes = (long long)s->gnum[0] * s->gnum[1] * s->gnum[2];
    s->ntiles = P.tiles[0] * P.tiles[1] * P.tiles[2];
    const long long pcells = (long long)P.pnum[0] * P.pnum[1] * P.pnum[2];
    if (s->nnodes <= 0 || s->nnodes > (1ll << 40) || pcells > (1ll << 31) - 4) {
        s->err = "grid too large";
        sphgpu_surface_destroy(s);
        return SPHGPU_EINVAL;
    }
    if (salloc(s, &s->field, (size_t)s->nnodes) || salloc(s, &s->tstart, (size_t)s->ntiles + 1) ||
        salloc(s, &s->pcnt, (size_t)pcells + 2) || salloc(s, &s->pstart, (size_t)pcells + 2) ||
        salloc(s, &s->bad, 1) || salloc(s, &s->coords, 6 * (size_t)std::max({s->gnum[0], s->gnum[1], s->gnum[2]}))) {
        sphgpu_surface_destroy(s);
        return SPHGPU_ENOMEM;
    }
    memset_sync(s->field, 0, sizeof(float) * (size_t)s->nnodes);
    if (ensure_table(s)) {
        sphgpu_surface_destroy(s);
        return SPHGPU_ECUDA;
    }
    *out = s;
    return 0;
}

int sphgpu_surface_destroy(sphgpu_surface_t s) {
    if (!s) return SPHGPU_EINVAL;
    cudaSetDevice(s->device);
    void* ptrs[] = {s->field, s->xyz, s->pos, s->rec0, s->rec1, s->rec2, s->blo, s->bhi, s->key, s->slot, s->tmp, s->sorted,
                    s->npair, s->poff, s->pcnt, s->pstart, s->bad, s->ptile, s->ppart, s->ptile_s, s->ppart_s,
                    s->tstart, s->ntri, s->toff, s->cases, s->tris, s->coords, s->tmpbuf};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return 0;
}

int sphgpu_surface_grid(sphgpu_surface_t s, double* mn, int* num, double* cell) {
    if (!s) return SPHGPU_EINVAL;
    for (int a = 0; a < 3; ++a) {
        if (mn) mn[a] = s->gmin[a];
        if (num) num[a] = s->gnum[a];
    }
    if (cell) *cell = s->cell;
    return 0;
}

int sphgpu_surface_field(sphgpu_surface_t s, int aniso, const float* xyz, int n, int on_device) {
    if (!s || n < 0 || (n > 0 && !xyz)) return SPHGPU_EINVAL;
    cudaSetDevice(s->device);
    s->err.clear();
    if (int r = ensure_particles(s, n)) return r;
    if (n > 0) {
        float* d = nullptr;
        if (on_device) {
            d = const_cast<float*>(xyz);
        } else {
            d = s->xyz;
            SCK(cudaMemcpyAsync(d, xyz, sizeof(float) * 3 * (size_t)n, cudaMemcpyHostToDevice, s->stream));
        }
        ++s->kernels;
        k_pack_xyz<<<nblk(n, 256), 256, 0, s->stream>>>(d, n, s->pos);
    }
    int r = run_field(s, n, aniso);
    if (r) return r;
    int bad = 0;
    if (aniso && n > 0) {
        SCK(copy_sync(&bad, s->bad, sizeof(int), cudaMemcpyDeviceToHost));
        if (bad) {
            s->err = std::to_string(bad) + " particles outside the reconstruction box";
            return SPHGPU_EOUT_OF_DOMAIN;
        }
    }
    return 0;
}

int sphgpu_surface_get_field(sphgpu_surface_t s, float* out) {
    if (!s || !out) return SPHGPU_EINVAL;
    cudaSetDevice(s->device);
    SCK(copy_sync(out, s->field, sizeof(float) * (size_t)s->nnodes, cudaMemcpyDeviceToHost));
    return 0;
}

int sphgpu_surface_set_field(sphgpu_surface_t s, const float* in) {
    if (!s || !in) return SPHGPU_EINVAL;
    cudaSetDevice(s->device);
    SCK(copy_sync(s->field, in, sizeof(float) * (size_t)s->nnodes, cudaMemcpyHostToDevice));
    return 0;
}

long long sphgpu_surface_mesh(sphgpu_surface_t s, float iso, int ref_rows, float* out, long long max_tris) {
    if (!s || max_tris < 0) return SPHGPU_EINVAL;
    cudaSetDevice(s->device);
    s->err.clear();
    cudaStream_t st = s->stream;
    const int* g = s->gnum;
    if (g[0] < 2 || g[1] < 2 || g[2] < 2) return 0;
    const long long ncubes = (long long)(g[0] - 1) * (g[1] - 1) * (g[2] - 1);
    if (ncubes > 0x7fffffffll) {
        s->err = "more than 2^31 - 1 cubes";
        return SPHGPU_EINVAL;
    }
    const int gpr = (g[0] - 1 + MCX - 1) / MCX;  // groups per x-row
    const long long ngroups = (long long)gpr * (g[1] - 1) * (g[2] - 1);
    const long long nblocks = (ngroups + MCB - 1) / MCB;
    if (nblocks > s->cubecap) {
        if (salloc(s, &s->ntri, (size_t)nblocks) || salloc(s, &s->toff, (size_t)nblocks)) return SPHGPU_ENOMEM;
        s->cubecap = nblocks;
    }
    if (ncubes > s->casecap) {
        if (salloc(s, &s->cases, (size_t)ncubes)) return SPHGPU_ENOMEM;
        s->casecap = ncubes;
    }
    // cube extents per index: nodes at min + i * cell; with ref_rows the
    // reference's running float sums (marching_cubes.cpp:53-66)
    const int m = std::max({g[0], g[1], g[2]});
    std::vector<float> tab(6 * (size_t)m, 0.f);
    const float mnf[3] = {(float)s->gmin[0], (float)s->gmin[1], (float)s->gmin[2]};
    const float cf = (float)s->cell;
    for (int a = 0; a < 3; ++a) {
        float* lo = &tab[(size_t)(2 * a) * m];
        float* hi = &tab[(size_t)(2 * a + 1) * m];
        if (ref_rows) {
            float l = mnf[a], h = mnf[a] + cf;
            for (int i = 0; i + 1 < g[a]; ++i) {
                lo[i] = l;
                hi[i] = a == 0 ? l + cf : h;  // x: xmax = xmin + cell per cube; y, z: running sums
                l += cf;
                h += cf;
            }
        } else {
            // node i at min + i * cell from the float min and cell that
            // marchingCubes receives, evaluated in double
            for (int i = 0; i + 1 < g[a]; ++i) {
                lo[i] = (float)((double)mnf[a] + (double)i * (double)cf);
                hi[i] = (float)((double)mnf[a] + (double)(i + 1) * (double)cf);
            }
        }
    }
    SCK(cudaMemcpyAsync(s->coords, tab.data(), sizeof(float) * tab.size(), cudaMemcpyHostToDevice, st));
    McParams M;
    for (int a = 0; a < 3; ++a) M.res[a] = g[a];
    M.ref_rows = ref_rows;
    M.iso = iso;
    M.cx_lo = s->coords;
    M.cx_hi = s->coords + m;
    M.cy_lo = s->coords + 2 * (size_t)m;
    M.cy_hi = s->coords + 3 * (size_t)m;
    M.cz_lo = s->coords + 4 * (size_t)m;
    M.cz_hi = s->coords + 5 * (size_t)m;
    ++s->kernels;
    k_mc_count<<<(int)nblocks, MCB, 0, st>>>(M, s->field, ngroups, gpr, s->cases, s->ntri);
    size_t b = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, b, s->ntri, s->toff, (int)nblocks, st);
    if (int r = ensure_tmp(s, b)) return r;
    cub::DeviceScan::ExclusiveSum(s->tmpbuf, b, s->ntri, s->toff, (int)nblocks, st);
    int last_off = 0;
    int last_n = 0;
    SCK(cudaMemcpyAsync(&last_off, s->toff + nblocks - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    SCK(cudaMemcpyAsync(&last_n, s->ntri + nblocks - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    SCK(cudaStreamSynchronize(st));
    const long long total = (long long)last_off + last_n;  // < 2^31: 5 triangles per cube at most
    if (total > s->tricap) {
        if (salloc(s, &s->tris, 9 * (size_t)total)) return SPHGPU_ENOMEM;
        s->tricap = total;
    }
    s->kernels += total > 0;
    if (total > 0)
        k_mc_emit<<<(int)nblocks, MCB, 0, st>>>(M, s->field, ngroups, gpr, s->cases, s->ntri, s->toff, s->tris);
    SCK(cudaGetLastError());
    SCK(cudaStreamSynchronize(st));
    s->ntris = total;
    if (out && total > 0)
        SCK(copy_sync(out, s->tris, sizeof(float) * 9 * (size_t)std::min(total, max_tris), cudaMemcpyDeviceToHost));
    return total;
}

void* sphgpu_surface_stream(sphgpu_surface_t s) { return s ? (void*)s->stream : nullptr; }

int sphgpu_surface_stats(sphgpu_surface_t s, long long* n_pairs, int* n_tiles, long long* kernels) {
    if (!s) return SPHGPU_EINVAL;
    if (n_pairs) *n_pairs = s->npairs;
    if (n_tiles) *n_tiles = s->ntiles;
    if (kernels) *kernels = s->kernels;
    return 0;
}

int sphgpu_surface_last_error(sphgpu_surface_t s, char* buf, int len) {
    if (!s || !buf || len <= 0) return SPHGPU_EINVAL;
    snprintf(buf, len, "%s", s->err.c_str());
    return 0;
}

}  // extern "C"
