"""Marching-cubes case table built from first principles (TEST
INFRASTRUCTURE: the checker for the library's table and its GPU marching
cubes).

Cube numbering of the reference's marching_cubes.cpp:9-31,36-37 (vertex
v: (x, y, z) bits; edge e joins two vertices):
  v0 (0,0,0) v1 (0,0,1) v2 (0,1,1) v3 (0,1,0) v4 (1,0,0) v5 (1,0,1) v6 (1,1,1) v7 (1,1,0)
  e0 0-1  e1 1-2  e2 2-3  e3 3-0  e4 4-5  e5 5-6  e6 6-7  e7 7-4  e8 0-4  e9 1-5  e10 2-6  e11 3-7
A vertex is "in" when its value is below the iso value (cubeindex bit set,
marching_cubes.cpp:62-72).

Construction (this repository's own, not a copy of a published table): on
every face, walk its corners counter-clockwise seen from outside the cube;
each maximal run of "in" corners gives one segment from the edge where the
walk enters the run to the edge where it leaves it -- so on a face with two
diagonal "in" corners the two are cut off separately, the same choice on
both cubes that share the face, which keeps the mesh closed.  Every cut edge
ends one segment and starts another, so the segments chain into closed
loops; each loop of k edges becomes k - 2 triangles fanned from its first
edge.  Triangles are listed (loop[0], loop[k + 1], loop[k]), the facing
of the reference's emitted triangles (its output order t0, t2, t1 of each
table row, marching_cubes.cpp:109-112).
"""
import numpy as np

VERT = [(0, 0, 0), (0, 0, 1), (0, 1, 1), (0, 1, 0), (1, 0, 0), (1, 0, 1), (1, 1, 1), (1, 1, 0)]
EDGES = [(0, 1), (1, 2), (2, 3), (3, 0), (4, 5), (5, 6), (6, 7), (7, 4), (0, 4), (1, 5), (2, 6), (3, 7)]


def _faces():
    """The six faces as corner lists, counter-clockwise seen from outside."""
    out = []
    for axis in range(3):
        for side in (0, 1):
            corners = [v for v in range(8) if VERT[v][axis] == side]
            n = np.zeros(3)
            n[axis] = 1.0 if side else -1.0
            c = np.mean([VERT[v] for v in corners], axis=0)
            a = np.zeros(3)
            a[(axis + 1) % 3] = 1.0
            b = np.cross(n, a)
            ang = [np.arctan2(np.dot(np.subtract(VERT[v], c), b), np.dot(np.subtract(VERT[v], c), a)) for v in corners]
            out.append([corners[i] for i in np.argsort(ang)])
    return out


FACES = _faces()
EDGE_OF = {frozenset(e): k for k, e in enumerate(EDGES)}


def case_loops(case):
    """Closed loops (lists of edge ids) of the cube case."""
    inside = [(case >> v) & 1 for v in range(8)]
    nxt = {}
    for f in FACES:
        m = len(f)
        if all(inside[v] for v in f) or not any(inside[v] for v in f):
            continue
        for i in range(m):
            a, b = f[i], f[(i + 1) % m]
            if not inside[a] and inside[b]:  # the walk enters a run of "in" corners
                j = (i + 1) % m
                while inside[f[(j + 1) % m]]:
                    j = (j + 1) % m
                e_in = EDGE_OF[frozenset((a, b))]
                e_out = EDGE_OF[frozenset((f[j], f[(j + 1) % m]))]
                nxt[e_in] = e_out
    loops, seen = [], set()
    for e in sorted(nxt):
        if e in seen:
            continue
        loop = [e]
        seen.add(e)
        k = nxt[e]
        while k != e:
            loop.append(k)
            seen.add(k)
            k = nxt[k]
        loops.append(loop)
    return loops


def tri_table():
    """tri[case] = list of (e_a, e_b, e_c) triangles."""
    tab = []
    for case in range(256):
        tris = []
        for loop in case_loops(case):
            for k in range(1, len(loop) - 1):
                tris.append((loop[0], loop[k + 1], loop[k]))
        tab.append(tris)
    return tab


def edge_mask(case):
    inside = [(case >> v) & 1 for v in range(8)]
    return sum(1 << k for k, (a, b) in enumerate(EDGES) if inside[a] != inside[b])


def cube_extents(res, mn, cell, ref_rows):
    """Per axis, the low and high coordinate of cube i (float32): nodes at
    mn + i * cell (float32 mn and cell, evaluated in double), or with
    ref_rows the running float
    sums of the reference's loops (marching_cubes.cpp:53-66: x_max = x_min +
    cell per cube; y and z minima and maxima each summed)."""
    ext = []
    f32 = np.float32
    for a in range(3):
        n = res[a] - 1
        lo = np.zeros(n, np.float32)
        hi = np.zeros(n, np.float32)
        if ref_rows:
            l, h = f32(mn[a]), f32(f32(mn[a]) + f32(cell))
            for i in range(n):
                lo[i] = l
                hi[i] = f32(l + f32(cell)) if a == 0 else h
                l = f32(l + f32(cell))
                h = f32(h + f32(cell))
        else:
            for i in range(n):
                lo[i] = f32(float(f32(mn[a])) + i * float(f32(cell)))
                hi[i] = f32(float(f32(mn[a])) + (i + 1) * float(f32(cell)))
        ext.append((lo, hi))
    return ext


def marching_cubes(field, res, mn, cell, iso, ref_rows=False, table=None, per_cube=False):
    """CPU marching cubes over field[z][y][x] (res = (nx, ny, nz)) with the
    table above: cubes in z, y, x order (x fastest), each cube's triangles in
    table order, vertices interpolated on the cut edges as the reference's
    VertexInterp does (marching_cubes.cpp:39-40) in float32.  ref_rows: cube
    y spans node rows max(y - 1, 0) and y, as the reference's row caches
    give them (marching_cubes.cpp:56-65), with its running coordinates.
    Returns (T, 3, 3) float32 (and the per-cube triangle counts of the cubes
    that have any, as (cube index, count), with per_cube)."""
    tab = table or tri_table()
    nx, ny, nz = res
    f = np.asarray(field, np.float32).reshape(nz, ny, nx)
    iso = np.float32(iso)
    ext = cube_extents(res, mn, cell, ref_rows)
    out, counts = [], []
    for z in range(nz - 1):
        for y in range(ny - 1):
            ylo, yhi = (max(y - 1, 0), y) if ref_rows else (y, y + 1)
            for x in range(nx - 1):
                val = [f[z + VERT[v][2], yhi if VERT[v][1] else ylo, x + VERT[v][0]] for v in range(8)]
                case = sum(1 << v for v in range(8) if val[v] < iso)
                if not tab[case]:
                    continue
                lo = (ext[0][0][x], ext[1][0][y], ext[2][0][z])
                hi = (ext[0][1][x], ext[1][1][y], ext[2][1][z])
                pts = {}
                for e in set(k for t in tab[case] for k in t):
                    a, b = EDGES[e]
                    va, vb = val[a], val[b]
                    mu = np.float32(np.float32(iso - va) / np.float32(vb - va))
                    p = []
                    for ax in range(3):
                        pa = hi[ax] if VERT[a][ax] else lo[ax]
                        pb = hi[ax] if VERT[b][ax] else lo[ax]
                        p.append(np.float32(pa + np.float32(mu * np.float32(pb - pa))))
                    pts[e] = p
                for t in tab[case]:
                    out.append([pts[t[0]], pts[t[1]], pts[t[2]]])
                counts.append(((z * (ny - 1) + y) * (nx - 1) + x, len(tab[case])))
    tris = np.array(out, np.float32).reshape(-1, 3, 3)
    return (tris, counts) if per_cube else tris
