// sph_window.cuh -- brick windows in shared memory.
//
// Particles are sorted by cell key, with cells enumerated 4x4x4 brick by
// brick (sph_common.cuh), so the particles of one brick are one contiguous
// range.  A thread block works on one brick: it stages the particles of the
// brick's 6x6x6-cell window (the brick plus a one-cell halo, which contains
// every neighbour of every particle of the brick, since cell = support) into
// shared memory, then sweeps the neighbour lists of the brick's own particles
// out of shared memory.
//
// Window slots: the fluid particles of the 216 window cells in window-cell
// order (w = (wz*6 + wy)*6 + wx), then the boundary particles in the same
// cell order.  Neighbour lists store these slots as 16-bit entries, column
// major (entry k of particle p at nbr16[k * stride + p]).  A window larger
// than WIN_MAX slots is "wide": its particles keep 32-bit global lists
// (fluid j, or boundary b | BND_FLAG) in `nbr` and are swept from global
// memory.
#pragma once
#include "sph_kernels.cuh"

#define WIN_CELLS 216
#define WIN_MAX 3072
#define WIN_NT 256

struct WinHead {
    int fstart[WIN_CELLS + 1];   // fluid slot prefix per window cell
    int bstart[WIN_CELLS + 1];   // boundary slot prefix per window cell
    int fglob[WIN_CELLS];        // global start of each cell's fluid range
    int bglob[WIN_CELLS];        // global start of each cell's boundary range
    int nf, nbnd;                // window fluid / boundary counts
    int own_a, own_b;            // the brick's own particle range [own_a, own_b)
    int wide;                    // window exceeds WIN_MAX
    int bx, by, bz;              // brick coordinates
};

__device__ __forceinline__ int win_cell_key(const GridGeom& g, int bx, int by, int bz, int w, bool& inside) {
    int wx = w % 6, wy = (w / 6) % 6, wz = w / 36;
    int cx = bx * 4 - 1 + wx, cy = by * 4 - 1 + wy, cz = bz * 4 - 1 + wz;
    inside = cell_inside(g, cx, cy, cz);
    return inside ? cell_key(g, cx, cy, cz) : 0;
}

// Block-wide set-up of the window head (counts, prefix sums).  All threads
// call it; returns with __syncthreads() done.
__device__ __forceinline__ void win_setup(const DevScene& s, const GridGeom& g, int brick, WinHead& H) {
    const int nbx = g.nb[0], nby = g.nb[1];
    if (threadIdx.x == 0) {
        H.bx = brick % nbx;
        H.by = (brick / nbx) % nby;
        H.bz = brick / (nbx * nby);
        H.own_a = s.cell_start[brick * 64];
        H.own_b = s.cell_start[brick * 64 + 64];
    }
    __syncthreads();
    if (H.own_b <= H.own_a) return;  // empty brick (uniform across the block)
    for (int w = threadIdx.x; w < WIN_CELLS; w += blockDim.x) {
        bool in;
        int key = win_cell_key(g, H.bx, H.by, H.bz, w, in);
        int fa = 0, fb = 0, ba = 0, bb = 0;
        if (in) {
            fa = s.cell_start[key];
            fb = s.cell_start[key + 1];
            ba = s.bcell_start[key];
            bb = s.bcell_start[key + 1];
        }
        H.fglob[w] = fa;
        H.bglob[w] = ba;
        H.fstart[w + 1] = fb - fa;  // counts, prefixed below
        H.bstart[w + 1] = bb - ba;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        // warp prefix over 216 entries (7 per lane)
        const int lane = threadIdx.x;
        int fl[7], bl[7], fs = 0, bs = 0;
#pragma unroll
        for (int i = 0; i < 7; ++i) {
            int w = lane * 7 + i;
            fl[i] = w < WIN_CELLS ? H.fstart[w + 1] : 0;
            bl[i] = w < WIN_CELLS ? H.bstart[w + 1] : 0;
            fs += fl[i];
            bs += bl[i];
        }
        int fx = fs, bxs = bs;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int a = __shfl_up_sync(0xffffffffu, fx, o), b = __shfl_up_sync(0xffffffffu, bxs, o);
            if (lane >= o) { fx += a; bxs += b; }
        }
        int f0 = fx - fs, b0 = bxs - bs;
#pragma unroll
        for (int i = 0; i < 7; ++i) {
            int w = lane * 7 + i;
            if (w < WIN_CELLS) {
                H.fstart[w] = f0;
                H.bstart[w] = b0;
                f0 += fl[i];
                b0 += bl[i];
            }
        }
        if (lane == 31) {
            H.fstart[WIN_CELLS] = fx;
            H.bstart[WIN_CELLS] = bxs;
            H.nf = fx;
            H.nbnd = bxs;
            H.wide = (fx + bxs) > WIN_MAX;
        }
    }
    __syncthreads();
}

// window cell of a window slot (binary search over the prefix)
__device__ __forceinline__ int win_cell_of(const int* start, int slot) {
    int lo = 0, hi = WIN_CELLS;  // start[lo] <= slot < start[hi]
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (start[mid] <= slot) lo = mid;
        else hi = mid;
    }
    return lo;
}

// global index of window slot q (fluid j, or boundary b | BND_FLAG)
__device__ __forceinline__ unsigned win_global(const WinHead& H, int q) {
    if (q < H.nf) {
        int c = win_cell_of(H.fstart, q);
        return (unsigned)(H.fglob[c] + (q - H.fstart[c]));
    }
    int t = q - H.nf;
    int c = win_cell_of(H.bstart, t);
    return (unsigned)(H.bglob[c] + (t - H.bstart[c])) | BND_FLAG;
}

// Stage a float4 field of the window (fluid from F, boundary from B) into S.
__device__ __forceinline__ void win_stage4(const WinHead& H, const float4* F, const float4* B, float4* S) {
    const int tot = H.nf + H.nbnd;
    for (int q = threadIdx.x; q < tot; q += blockDim.x) {
        unsigned gq = win_global(H, q);
        S[q] = (gq & BND_FLAG) ? B[gq & BND_MASK] : F[gq];
    }
}
