"""Shared set-up for the parity tests: one seeded scene loaded both into the
GPU path (through the C ABI) and into the CPU oracle (restatement)."""
import numpy as np

from graphics_b200.scene import small_dam_break
from graphics_b200.sph import GpuScene, params_for_scene
from oracle import make_scene_oracle

COMMON = dict(dt=1e-3, nu=1e-3, soundSpeed_cs=100.0, df_density_goal=1e-4, df_density_min_iter=2,
              df_density_max_iter=100, df_div_goal_abs=2.5, df_div_goal_rel=1e-3, df_div_min_iter=1,
              df_div_max_iter=30, cfl=0, cfl_factor=0.4, dt_max=5e-3, dt_min=1e-6, wc_gamma=7.0)
GPU_ONLY = ("max_neighbours", "boundary_visc", "warm_start")


def make_pair(scene=None, visc_alpha=0.0, boundary_visc=0.0, cap=48, **kw):
    if scene is None:
        scene = small_dam_break((12, 12, 12), r=0.025, seed=7)
    p = dict(COMMON)
    p.update(kw)
    gp = params_for_scene(scene, max_neighbours=cap, boundary_visc=boundary_visc,
                          **{k: v for k, v in p.items() if k not in ("float_err",)})
    g = GpuScene(gp, scene.n_fluid)
    g.set_boundary(scene.boundary_pos, scene.meta.get("solid_id"))
    if scene.phase is None:
        g.add_fluid(scene.fluid_pos, scene.fluid_vel, rho0=scene.rho0, visc_alpha=visc_alpha)
    else:
        for ph, rho in enumerate(scene.rho0_phases):
            m = scene.phase == ph
            g.add_fluid(scene.fluid_pos[m], scene.fluid_vel[m], rho0=rho, visc_alpha=visc_alpha)
    o = make_scene_oracle(scene, visc_alpha=visc_alpha, solid_visc=boundary_visc, cap=cap,
                          **{k: v for k, v in p.items() if k not in GPU_ONLY})
    return scene, g, o


def rel_err(a, b, scale=None):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    if scale is None:
        scale = np.max(np.abs(b)) if b.size else 1.0
    return float(np.max(np.abs(a - b)) / max(scale, 1e-30)) if a.size else 0.0


def elem_rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-30))) if a.size else 0.0


def closed_and_oriented(tris, tol):
    """A triangle mesh (T, 3, 3) is closed and consistently oriented: after
    welding vertices closer than tol (a cut edge's vertex is interpolated
    from either end by the cubes that share the edge, so copies can differ by
    an ulp), every directed side appears once and its reverse once."""
    from scipy.spatial import cKDTree
    pts = np.asarray(tris, np.float64).reshape(-1, 3)
    parent = np.arange(len(pts))

    def find(i):
        while parent[i] != i:
            parent[i] = parent[parent[i]]
            i = parent[i]
        return i

    for i, j in cKDTree(pts).query_pairs(tol):
        a, b = find(i), find(j)
        if a != b:
            parent[max(a, b)] = min(a, b)
    lab = np.array([find(i) for i in range(len(pts))]).reshape(-1, 3)
    sides = {}
    for t in lab:
        if len(set(t)) < 3:
            continue  # a degenerate sliver (vertex on a node)
        for k in range(3):
            s = (t[k], t[(k + 1) % 3])
            sides[s] = sides.get(s, 0) + 1
    return all(v == 1 for v in sides.values()) and all((b, a) in sides for (a, b) in sides)


def build_surface_dropin(out_dir):
    """Compile tests/cpp/surface_dropin_main.cpp against include/ and the
    library; returns the executable's path."""
    import os
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = os.path.join(str(out_dir), "surface_dropin")
    lib = os.path.join(root, "graphics_b200")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I" + os.path.join(root, "include"),
                    os.path.join(root, "tests", "cpp", "surface_dropin_main.cpp"), "-L" + lib, "-lsphgpu",
                    "-Wl,-rpath," + lib, "-o", exe], check=True, capture_output=True)
    return exe
