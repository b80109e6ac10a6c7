#!/usr/bin/env python3
"""Benchmark: DFSPH particle-steps/s on the 1M-particle dam break.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one "step" = one DFSPH solver step, DFSPH::sphStep): 100x100x100
fluid particles (r = 0.01 m, seeded +-0.1 r jitter) in a 4 x 2 x 2 m box with
2-layer static walls; cubic spline support 4r; density loop to 0.01 % mean
density error (FP64), divergence loop to 0.1 % (mean Drho/Dt * dt / rho0, FP64),
capped at 1000 / 100 iterations; CFL dt = min(0.4 d / max|v|, 2e-3 s).  The
timed window starts after --settle (300) untimed steps.

ours      : the sm_100a kernels through libsphgpu.so (C ABI).  `value` is timed
            with CUDA events on the scene's stream over K steps with all
            inputs resident in HBM (each step one CUDA graph); `e2e` drives the
            same steps through sphgpu_step_host with pinned host buffers
            (positions and velocities copied in and out every step).
reference : the reference's own DFSPH CPU code (oracle/_ref, OpenMP, all host
            cores), same scene and goals, on a time-bounded sample of steps.

Multi-GPU (torchrun, one rank per GPU): the single-scene workload does not
shard, so every rank runs an independent replica ("replicas only"); value is
the sum over ranks of particle-steps divided by the max-over-ranks time.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "DFSPH particle-steps/s @1M, plain vs learned warm-start at 0.01% rho error"
UNIT = "particle-steps/s"
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM = 6650.0

# Algorithmic bytes per fluid particle of each kernel class, as the hot-path
# byte model defines them (compulsory traffic: own-particle state in and out
# and the 4-byte neighbour index list; gathers of neighbour state are cache
# traffic and not counted; nb = mean stored neighbours):
#   hash + cell id 24, integrate 64, counting sort 32, reindex 80, cell
#   ranges 4, list build 20 + 4 nb, density + alpha 24 + 4 nb, forces + v_adv
#   48 + 4 nb, Jacobi sweep A (rho_adv / Drho/Dt + kappa) 40 + 4 nb, Jacobi
#   sweep B (v_adv update) 56 + 4 nb.
# Fused kernels count the bytes of every stage they perform (the hash kernel
# also integrates; the list build also sums rho and alpha).
ALG_BYTES = {
    "df_density_a": lambda nb: 16 + 16 + 4 + 4 * nb + 4,
    "df_density_b": lambda nb: 16 + 4 + 4 + 32 + 4 * nb,
    "df_div_a": lambda nb: 16 + 16 + 4 + 4 * nb + 4,
    "df_div_b": lambda nb: 16 + 4 + 4 + 32 + 4 * nb,
    "df_forces": lambda nb: 32 + 4 * nb + 16,
    "build_first": lambda nb: (16 + 4 + 4 * nb) + (16 + 4 * nb + 8),
    # the list build with rho/alpha and the divergence loop's first sweep A
    "build_first_div": lambda nb: (16 + 4 + 4 * nb) + (16 + 4 * nb + 8) + (16 + 16 + 4 + 4 * nb + 4),
    "hash": lambda nb: 24 + 64,
    "reorder": lambda nb: 32 + 80,
    # IISph (volume form) loop sweeps (not in the byte model; own compulsory
    # sets): A reads pv (pos, v_adv), ivs (gamma, sphVolume, alpha), count,
    # list and writes kappa, V_adv / div, pk.w; B reads pk, pos (phase),
    # v_adv, count, list and writes v_adv (+ vel in the divergence loop)
    "iv_cv_a": lambda nb: 16 + 16 + 16 + 4 + 4 * nb + 4 + 4 + 4,
    "iv_cv_b": lambda nb: 16 + 16 + 16 + 4 + 4 * nb + 16,
    "iv_div_a": lambda nb: 16 + 16 + 16 + 4 + 4 * nb + 4 + 4 + 4,
    "iv_div_b": lambda nb: 16 + 16 + 16 + 4 + 4 * nb + 16 + 16,
}
# cell ranges: 4 B per particle plus 8 B per cell key (count, start)
SCAN_BYTES_PER_PARTICLE = 4
SCAN_BYTES_PER_KEY = 8


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--profile-steps", type=int, default=3)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--cpu-budget", type=float, default=60.0, help="seconds of reference CPU work per sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--scale", type=int, default=100, help="fluid block edge (100 -> 1M particles)")
    ap.add_argument("--max-iter", type=int, default=1000, help="density-loop iteration cap")
    ap.add_argument("--settle", type=int, default=300,
                    help="untimed steps before warm-up, so the timed window is in the collapsing flow "
                         "(t ~ 0.5 s) rather than the first steps from rest")
    ap.add_argument("--no-warm-start", action="store_true", help="skip the learned warm-start arm")
    ap.add_argument("--no-iisph", action="store_true",
                    help="skip the IISph (volume form) arm timed on the same settled state")
    ap.add_argument("--no-subarms", action="store_true",
                    help="skip the short GPU runs of the other configurations (2M warm start, 27k WCSPH, "
                         "500k two-phase IISPH_M / PCISPH)")
    ap.add_argument("--train-seeds", default="1,2", help="jitter seeds of the training runs")
    ap.add_argument("--train-steps", type=int, default=350, help="recorded plain steps per training seed")
    ap.add_argument("--train-every", type=int, default=175, help="record every n-th particle per step")
    ap.add_argument("--workload", default="dam_break_1m",
                    choices=["dam_break_1m", "batched_64", "floating_box_1m", "surface_1m"],
                    help="dam_break_1m: the headline 1M-particle DFSPH dam break; batched_64: 64 independent "
                         "dam breaks of 10k-200k particles in one batch")
    ap.add_argument("--no-graphs", action="store_true",
                    help="host-driven solver loops instead of CUDA graphs (for ncu: kernels inside graphs "
                         "with conditional nodes cannot be profiled)")
    return ap.parse_args()


def workload_seed(scale, seed):
    from graphics_b200.scene import dam_break
    return dam_break((scale, scale, scale), 0.01, (4.0, 2.0, 2.0), seed=seed)


def workload(scale):
    """The 1M-particle dam break (scale=100); smaller blocks in the same box
    for quick checks."""
    from graphics_b200.scene import dam_break
    return dam_break((scale, scale, scale), 0.01, (4.0, 2.0, 2.0), seed=0)


# dt_max: 2e-3 s.  The reference's DFSPH (as restated by the CPU oracle, and
# on the GPU) is unstable on this scene at 5e-3 s (velocities blow up by
# t = 0.05 s for nu up to 1e-2, CFL factor down to 0.2 and 20% headroom);
# 2e-3 s is the largest stable cap measured.
SOLVER_KW = dict(cfl=1, cfl_factor=0.4, dt_max=2e-3, dt_min=1e-6, dt=2e-3, nu=1e-3,
                 df_density_goal=1e-4, df_density_min_iter=2, df_density_max_iter=1000,
                 df_div_goal_abs=0.0, df_div_goal_rel=1e-3, df_div_min_iter=1, df_div_max_iter=100)


SETTLE = [0]


def config_dict(sc, world=1):
    """The workload as both arms describe it (the reference arm prints the
    same dictionary, so the two lines are for the same configuration)."""
    return {"workload": "dfsph_dam_break_%dk" % (sc.n_fluid // 1000), "n_fluid": sc.n_fluid,
            "n_boundary": sc.n_boundary, "r": sc.r, "box": list(sc.meta["box"]), "cfl": 0.4,
            "dt_max": SOLVER_KW["dt_max"], "settle_steps": SETTLE[0],
            "density_goal": 1e-4, "divergence_goal": 1e-3, "max_iter": SOLVER_KW["df_density_max_iter"],
            "div_max_iter": SOLVER_KW["df_div_max_iter"], "neighbour_cap": 48,
            "window": "the steps after settle_steps + warmup DFSPH steps from the seeded lattice",
            "l2": "inputs larger than L2 (neighbour lists %.0f MB + state)" % (sc.n_fluid * 48 * 4 / 1e6),
            "parallelism": "replicas x%d" % world if world > 1 else "single"}


def peaks():
    try:
        j = json.load(open(PEAKS))
        return float(j["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM, "fallback"


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


class ClockSampler:
    """nvidia-smi samples (every 50 ms) of SM clock, power and throttle
    reasons between start() and stop()."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.p = None
        self.path = os.path.join(os.environ.get("SPH_BENCH_OUT", os.path.join(ROOT, "_bench_out")),
                                 "clocks_%d.csv" % gpu_index)

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + self.QUERY,
                                       "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        return self

    def wait_first(self, timeout=5.0):
        """Block until nvidia-smi has written its first sample (its start-up
        takes a fraction of a second), so that the timed region is covered."""
        t0 = time.perf_counter()
        while self.p and time.perf_counter() - t0 < timeout:
            try:
                if os.path.getsize(self.path) > 0:
                    return self
            except OSError:
                pass
            time.sleep(0.02)
        return self

    def stop(self):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(5)
            except Exception:
                self.p.kill()
            self.f.close()

    def __enter__(self):
        return self.start().wait_first()

    def __exit__(self, *a):
        self.stop()

    def summary(self, covers="the timed region"):
        if not self.p:
            return None
        sm, mx, reasons = [], 0.0, set()
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm),
                "covers": covers}


def window_dt(vel, d):
    """The CFL step the GPU computes at the start of a step from these
    velocities: clamp(0.4 d / max|v|, dt_min, dt_max) with an FP64 max."""
    vmax = float(np.sqrt((np.asarray(vel, np.float64) ** 2).sum(1)).max()) if len(vel) else 0.0
    dt = SOLVER_KW["cfl_factor"] * d / vmax if vmax > 0 else SOLVER_KW["dt_max"]
    return float(np.float32(min(max(dt, SOLVER_KW["dt_min"]), SOLVER_KW["dt_max"])))


def cpu_reference_window(sc, pos, vel, dts, budget, max_steps, start_note):
    """The reference's own DFSPH (oracle/_ref/libref_dfsph_capped.so: float,
    OpenMP on every host core; DFSPH.cpp with only its loop bookkeeping
    changed to an FP64 density mean and 100-iteration caps) from the GPU
    window's start state, step k at the GPU window's k-th CFL step dts[k]
    (the reference has no CFL rule; its m_TH.dt is set before each step).
    The frame-0 neighbour search and rho/alpha run untimed (the GPU did them
    at the end of the previous step); then whole steps until `budget`
    seconds or `max_steps`."""
    import dataclasses
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import make_scene_oracle
    dt = dts[0]
    t0 = time.perf_counter()
    sc2 = dataclasses.replace(sc, fluid_pos=np.ascontiguousarray(pos, np.float32),
                              fluid_vel=np.ascontiguousarray(vel, np.float32))
    o = make_scene_oracle(sc2, kind="reference", solver="dfsph_capped", nu=SOLVER_KW["nu"], dt=dt)
    for name in ("neighbourSearch", "updateSolidPartWeight", "DF_constantDensitySolverFirst"):
        o.stage(name)
    o.set_frame(1)
    o.df_iters()
    setup = time.perf_counter() - t0
    steps, t_run = 0, 0.0
    while True:
        o.set_dt(dts[steps % len(dts)])
        t1 = time.perf_counter()
        o.stage("runOneStep")
        t_run += time.perf_counter() - t1
        steps += 1
        if t_run >= budget or steps >= max_steps:
            break
    it_d, it_v = o.df_iters()
    cores = o.threads()
    rho = np.asarray(o.get("density"), np.float64)
    o.close()
    used = [dts[k % len(dts)] for k in range(steps)]
    return {"value": sc.n_fluid * steps / t_run, "unit": UNIT, "cores": cores, "cpu_model": cpu_model(),
            "kind": "reference", "dt_first": used[0], "dt_mean": float(np.mean(used)),
            "iterations_per_step": {"density": it_d / steps, "divergence": it_v / steps},
            "sample": "%d DFSPH step(s) of the %d-particle dam break from %s, each at the GPU window's CFL step "
                      "of the same index (%.3e..%.3e s); reference DFSPH.cpp via oracle/_ref (float, density "
                      "mean FP64 and loops capped at 100), %d OpenMP threads; setup %.1f s untimed"
                      % (steps, sc.n_fluid, start_note, min(used), max(used), cores, setup),
            "seconds": round(t_run, 2), "mean_density_error": float(np.mean(rho) / sc.rho0 - 1.0)}


def settle_on_gpu(sc, steps, device, window):
    """The window's start state -- `steps` DFSPH steps of the GPU path from
    the seeded lattice -- and the CFL steps of the `window` steps that follow
    (input preparation only; nothing here is timed)."""
    from graphics_b200.sph import scene_to_gpu
    g = scene_to_gpu(sc, device=device, **SOLVER_KW)
    g.step("dfsph", steps)
    pos, vel = g.get("position"), g.get("velocity")
    dts = [g.step("dfsph", 1)["dt"] for _ in range(window)]
    g.close()
    return pos, vel, dts


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    sc = workload(args.scale)
    try:
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("no CUDA device for the window's start state")
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        pos, vel, dts = settle_on_gpu(sc, SETTLE[0] + max(args.warmup, 1), int(os.environ.get("LOCAL_RANK", "0")),
                                      args.steps)
        note = ("the state after %d + %d DFSPH steps (settle + warm-up, the GPU arm's window start, "
                "prepared untimed on the GPU)" % (SETTLE[0], max(args.warmup, 1)))
    except Exception as e:
        pos, vel = sc.fluid_pos, sc.fluid_vel
        dts = [window_dt(vel, sc.d)]
        note = "rest (the window's start state could not be prepared: %s)" % e
    try:
        cb = cpu_reference_window(sc, pos, vel, dts, budget=max(30.0, args.cpu_budget * 2), max_steps=args.steps,
                                  start_note=note)
    except Exception as e:  # the reference build is missing
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU build not loadable: %s" % e}))
        return
    v = cb["value"]
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sc.n_fluid / v,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded dam break)", "config": config_dict(sc, world),
            "cpu_baseline": cb, "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def init_dist(torch):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return world, rank, local, dist


def timed_window(g, solver, steps, stream, torch, dist, nvtx=None):
    """K steps of `solver` on `g`, bracketed by CUDA events on the scene's
    stream (inputs resident); returns (max-over-ranks ms, stats)."""
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    if nvtx:
        torch.cuda.nvtx.range_push(nvtx)
    e0.record(stream)
    g.step_async(solver, steps)
    e1.record(stream)
    st = g.synchronize()
    if nvtx:
        torch.cuda.nvtx.range_pop()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    return ms, st


def run_ours(args):
    import torch
    world, rank, local, dist = init_dist(torch)
    from graphics_b200.sph import scene_to_gpu

    sc = workload(args.scale)
    g = scene_to_gpu(sc, device=local, **SOLVER_KW)
    if args.no_graphs:
        g.debug_set("use_graphs", 0)
    stream = torch.cuda.ExternalStream(g.lib.sphgpu_stream(g.h), device=torch.device("cuda", local))

    # learned warm start: train on plain runs of other jitter seeds (untimed)
    net, train_info = None, None
    if not args.no_warm_start:
        from graphics_b200.warmstart import train_for_scenes
        t0 = time.perf_counter()
        seeds = [int(x) for x in args.train_seeds.split(",") if x]
        net, losses = train_for_scenes(lambda sd: workload_seed(args.scale, sd), seeds, settle=0,
                                       record_steps=args.train_steps, every=args.train_every, epochs=20, lr=1e-3,
                                       batch=8192, device=local, dataset_cap=4_200_000, **SOLVER_KW)
        train_info = {"seeds": seeds, "samples": net.dataset_size(), "epochs": 20, "lr": 1e-3,
                      "loss_first": round(float(losses[0]), 4), "loss_last": round(float(losses[-1]), 4),
                      "seconds": round(time.perf_counter() - t0, 1)}

    # settle into the flow, then warm up (also builds the step graph)
    if args.settle > 0:
        g.step("dfsph", args.settle)
    settle_pos, settle_vel = g.get("position"), g.get("velocity")
    # clock samples from the warm-up on (nvidia-smi's first sample arrives
    # before the timed region starts)
    clk = ClockSampler(local).start()
    g.step("dfsph", max(args.warmup, 1))

    # snapshot of the state the timed region starts from; the end-to-end run,
    # the FP64 check and the CPU baseline all start from it
    n0 = g.n_fluid
    snap_pos = torch.empty((n0, 3), dtype=torch.float32, pin_memory=True).numpy()
    snap_vel = torch.empty((n0, 3), dtype=torch.float32, pin_memory=True).numpy()
    snap_pos[:] = g.get("position")
    snap_vel[:] = g.get("velocity")
    g.set("position", snap_pos)  # same restaging the host-buffer path performs
    g.step("dfsph", 0)
    clk.wait_first()
    ms_max, st = timed_window(g, "dfsph", args.steps, stream, torch, dist, nvtx="timed_plain")
    end_pos = g.get("position")
    st_plain = st
    n_active = st["n_fluid"]
    value = n_active * args.steps * world / (ms_max / 1e3)
    it_rho = st["total_iter_density"] / args.steps
    it_div = st["total_iter_divergence"] / args.steps
    launches = args.steps * 13 + 2 * (st["total_iter_density"] + st["total_iter_divergence"])

    # per-kernel durations: the same kernels as individual launches bracketed
    # by CUDA events (host-driven loops), on the steps right after the timed
    # window (same flow state, same iteration counts)
    hbm, peak_kind = peaks()
    kern, roof = {}, None
    if args.profile_steps > 0:
        roof, kern = profile_kernels(g, args, hbm, peak_kind, sc)

    # learned warm start on the same window: restore the settled state, warm
    # up with the network attached (builds the per-particle history), time K
    warm = None
    if net is not None:
        from graphics_b200.warmstart import attach
        g.set("position", settle_pos)
        g.set("velocity", settle_vel)
        attach(g, net, 1)
        g.step("dfsph", max(args.warmup, 1))
        wms, stw = timed_window(g, "dfsph", args.steps, stream, torch, dist, nvtx="timed_warm")
        wval = stw["n_fluid"] * args.steps * world / (wms / 1e3)
        warm = {"value": wval, "ms_per_step": round(wms / args.steps, 4),
                "speedup_vs_plain": round(wval / value, 3),
                "iterations_per_step": {"density": stw["total_iter_density"] / args.steps,
                                        "divergence": stw["total_iter_divergence"] / args.steps},
                "err_density_last": stw["err_density"], "status": stw["status"], "training": train_info,
                "network": "16-64-64-1 GELU, BF16 weights/activations (mma.sync), FP32 accumulate"}
        if args.profile_steps > 0:
            g.profile(True)
            g.step("dfsph", args.profile_steps)
            prof = g.profile_read()
            g.profile(False)
            g.synchronize()
            warm["kernels_us_per_step"] = {k: round(1e3 * t / args.profile_steps, 1) for k, (t, c) in prof.items()}
        attach(g, None, 0)
        g.set("position", end_pos)  # continue from the plain run's state

    e2e = run_e2e(args, g, snap_pos, snap_vel, end_pos, world, dist, torch)
    clk.stop()

    iisph = None
    if not args.no_iisph:
        def barrier():
            if dist:
                dist.barrier()
            torch.cuda.synchronize()

        iisph = run_iisph_arm(args, g, sc, settle_pos, settle_vel, st_plain["dt"], barrier, stream, dist,
                              world, torch)

    fp64 = cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        dts = [window_dt(snap_vel, sc.d)]
        try:
            fp64, dts = fp64_window_check(sc, g, snap_pos, snap_vel, args.steps)
        except Exception as e:
            fp64 = {"unavailable": str(e)}
        try:
            cpu = cpu_reference_window(sc, snap_pos, snap_vel, dts, budget=args.cpu_budget, max_steps=args.steps,
                                       start_note="the GPU window's start state (after %d + %d GPU steps)"
                                                  % (args.settle, max(args.warmup, 1)))
            cpu["gpu_window"] = {"dt_mean": float(np.mean(dts)),
                                 "iterations_per_step": {"density": it_rho, "divergence": it_div}}
        except Exception as e:
            cpu = {"unavailable": str(e)}
    g.close()

    subarms = {}
    if not args.no_subarms and world == 1:
        subarms = run_subarms(args, net, local, stream, torch)
    if net is not None:
        net.close()

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded dam break)",
                "config": config_dict(sc, world),
                "iterations_per_step": {"density": it_rho, "divergence": it_div},
                "last_step": {"err_density": st["err_density"], "err_divergence": st["err_divergence"],
                              "dt": st["dt"], "status": st["status"], "neighbour_overflow": st["neighbour_overflow"]},
                "kernels": kern, "iisph": iisph, "roofline": roof, "fp64_check": fp64, "cpu_baseline": cpu,
                "e2e": e2e, "gpu_launches": launches, "subarms": subarms, "warm_start": warm,
                "clocks": clk.summary("the warm-up, the plain and warm-start timed windows, the kernel profiles "
                                      "and the e2e replay")}
        print(json.dumps(line))
    if dist:
        dist.destroy_process_group()


def run_e2e(args, g, snap_pos, snap_vel, end_pos, world, dist, torch):
    """End to end through the C ABI with pinned host buffers: the same K
    steps, replayed from the snapshot taken before the timed region."""
    if args.e2e_steps <= 0:
        return None
    n = snap_pos.shape[0]
    pos, vel = snap_pos.copy(), snap_vel.copy()
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    pos, vel = pin(pos), pin(vel)
    po = torch.empty((n, 3), dtype=torch.float32, pin_memory=True).numpy()
    vo = torch.empty((n, 3), dtype=torch.float32, pin_memory=True).numpy()
    g.step_host("dfsph", pos, vel, po, vo)  # untimed: builds the step graphs (the inputs stay the snapshot)
    # back to the snapshot (sorted and searched as the device window had it),
    # so the timed loop is the steady state: each step's inputs are the
    # previous step's outputs
    g.set("position", snap_pos)
    g.set("velocity", snap_vel)
    g.step("dfsph", 0)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        g.step_host("dfsph", pos, vel, po, vo)
        pos, po = po, pos
        vel, vo = vo, vel
    sec = time.perf_counter() - t0
    if dist:
        t = torch.tensor([sec], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        sec = float(t.item())
    return {"value": n * args.steps * world / sec, "unit": UNIT, "h2d_bytes_per_step": int(n * 24),
            "d2h_bytes_per_step": int(n * 24), "steps": args.steps,
            "same_trajectory_as_timed": bool(np.array_equal(pos, end_pos)),
            "note": "sphgpu_step_host: pinned positions+velocities in, step, positions+velocities out"}


def fp64_window_check(sc, g, pos, vel, window):
    """The window's first step on the GPU against the FP64 build of the CPU
    restatement (oracle/liboracle_f64.so) from the same state: the error of
    the timed result against an FP64 oracle.  Also returns the CFL steps of
    the window (the GPU replays it step by step from the same state)."""
    import dataclasses
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import make_scene_oracle
    g.set("position", pos)
    g.set("velocity", vel)
    st = g.step("dfsph", 1)
    rg = g.get("density").astype(np.float64)
    vg = g.get("velocity").astype(np.float64)
    xg = g.get("position").astype(np.float64)
    dts = [st["dt"]] + [g.step("dfsph", 1)["dt"] for _ in range(window - 1)]
    t0 = time.perf_counter()
    sc2 = dataclasses.replace(sc, fluid_pos=np.ascontiguousarray(pos), fluid_vel=np.ascontiguousarray(vel))
    o = make_scene_oracle(sc2, f64=True, **SOLVER_KW)
    o.stage("df_step")
    it, err, dt, _ = o.stats()
    ro, vo, xo = o.get("density"), o.get("velocity"), o.get("position")
    o.close()
    vs = max(float(np.abs(vo).max()), 1e-30)
    return {"oracle": "oracle/liboracle_f64.so (CPU restatement, FP64), same start state and CFL rule",
            "max_rel_density": float(np.max(np.abs(rg - ro) / ro)),
            "max_rel_velocity": float(np.max(np.abs(vg - vo)) / vs),
            "max_abs_position_m": float(np.max(np.abs(xg - xo))),
            "mean_density_error": {"gpu": float(np.mean(rg) / sc.rho0 - 1), "oracle_f64": float(np.mean(ro) / sc.rho0 - 1)},
            "iterations": {"gpu": [st["iter_density"], st["iter_divergence"]], "oracle_f64": [it[0], it[1]]},
            "dt": {"gpu": st["dt"], "oracle_f64": dt}, "oracle_seconds": round(time.perf_counter() - t0, 1)}, dts


def run_iisph_arm(args, g, sc, settle_pos, settle_vel, dt, barrier, stream, dist, world, torch):
    """The reference's IISph class (volume form: divergence-free and
    constant-volume loops, boundary particles with their own loop state) on
    the settled state of the same scene: fixed dt = the plain run's last CFL
    step (IISph has no CFL rule), the particles' kinematic viscosity = nu.
    (The reference's default 0.1 m^2/s belongs to its demo's 0.3 m
    particles; explicit viscosity at d = 0.02 m needs 10 nu dt / h^2 << 1.)"""
    from graphics_b200.sph import params_for_scene
    nu = SOLVER_KW["nu"]
    g.set_params(params_for_scene(sc, **{**SOLVER_KW, "cfl": 0, "dt": dt, "iv_kvisc": nu, "iv_kvisc_b": nu}))
    g.set("position", settle_pos)
    g.set("velocity", settle_vel)
    g.step("iisph", max(args.warmup, 1))
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.nvtx.range_push("timed_iisph")
    e0.record(stream)
    g.step_async("iisph", args.steps)
    e1.record(stream)
    st = g.synchronize()
    torch.cuda.nvtx.range_pop()
    barrier()
    ms = e0.elapsed_time(e1)
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    out = {"solver": "IISph (IISph.cpp, volume form)", "value": st["n_fluid"] * args.steps * world / (ms / 1e3),
           "unit": UNIT, "ms_per_step": ms / args.steps, "dt": dt, "kinematic_viscosity": nu,
           "iterations_per_step": {"constant_volume": st["total_iter_density"] / args.steps,
                                   "divergence_free": st["total_iter_divergence"] / args.steps},
           "last_step": {"err_volume": st["err_density"], "err_divergence": st["err_divergence"],
                         "status": st["status"]}}
    if args.profile_steps > 0:
        g.profile(True)
        g.step("iisph", args.profile_steps)
        prof = g.profile_read()
        g.profile(False)
        st_p = g.synchronize()
        nb = st_p["mean_neighbours"]
        kern = {}
        for k, (tot_ms, cnt) in prof.items():
            ent = {"n": cnt, "us": round(1e3 * tot_ms / max(cnt, 1), 1)}
            if k in ALG_BYTES:
                ent["gbs"] = round(ALG_BYTES[k](nb) * st_p["n_fluid"] / (tot_ms / cnt / 1e3) / 1e9, 1)
            kern[k] = ent
        out["kernels"] = kern
    g.set_params(params_for_scene(sc, **SOLVER_KW))
    return out


def profile_kernels(g, args, hbm, peak_kind, sc):
    g.profile(True)
    g.step("dfsph", args.profile_steps)
    prof = g.profile_read()
    g.profile(False)
    st_p = g.synchronize()
    nb = st_p["mean_neighbours"]
    n = st_p["n_fluid"]
    nkeys = cell_keys(sc)
    kern, full = {}, {}
    for k, (tot_ms, cnt) in prof.items():
        avg = tot_ms / max(cnt, 1)
        ent = {"n": cnt, "us": round(1e3 * avg, 1)}
        b = None
        if k in ALG_BYTES:
            b = ALG_BYTES[k](nb) * n
        elif k == "scan":
            b = SCAN_BYTES_PER_PARTICLE * n + SCAN_BYTES_PER_KEY * nkeys
        if b is not None:
            ent["gbs"] = round(b / (avg / 1e3) / 1e9, 1)
        kern[k] = ent
        full[k] = (avg, b, tot_ms)
    # the dominant kernel: the largest share of the step among the kernels
    # with an algorithmic byte count
    dom = max((k for k in full if k in ALG_BYTES), key=lambda k: full[k][2])
    traffic = None
    tf = os.path.join(ROOT, "profiles", "dram_traffic_1m.json")
    if os.path.exists(tf):
        try:
            traffic = json.load(open(tf)).get(dom)
        except Exception:
            traffic = None
    ach = full[dom][1] / (full[dom][0] / 1e3) / 1e9
    roof = {"bound": "hbm", "kernel": dom, "achieved": round(ach, 1), "peak": hbm, "unit": "GB/s",
            "frac": round(ach / hbm, 4), "traffic": traffic,
            "traffic_source": "ncu capture of this kernel (dram__bytes_read.sum + dram__bytes_write.sum), read "
                              "from profiles/dram_traffic_1m.json, not measured in this run",
            "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback",
            "alg_bytes_per_particle": round(ALG_BYTES[dom](nb), 1), "mean_neighbours": round(nb, 2)}
    # neighbour + density kernels (hash with integration, cell ranges,
    # counting sort + reindex, list build with rho/alpha)
    ns_keys = [k for k in ("hash", "scan", "reorder", "build_first", "build_first_div") if k in full]
    ns_s = sum(full[k][0] for k in ns_keys) / 1e3
    ns_bytes = sum(full[k][1] for k in ns_keys)
    roof["neighbour_density_group"] = {"kernels": ns_keys, "us_per_step": round(ns_s * 1e6, 1),
                                       "gbs": round(ns_bytes / ns_s / 1e9, 1),
                                       "frac": round(ns_bytes / ns_s / 1e9 / hbm, 4)}
    return roof, kern


# ---- the other configurations, as short GPU runs inside the default bench ----

# two-phase column (rest densities 1000 below, 3000 above): Monaghan
# viscosity 0.02 in the fluid and 0.01 at the walls, fixed dt = 1e-3 s
MULTI_KW = dict(dt=1e-3, nu=1e-3, soundSpeed_cs=20.0, cfl=0)
MULTI_VISC = dict(visc_alpha=0.02, boundary_visc=0.01)
IISPH_M_KW = dict(ii_omega=0.5, ii_eta_rel=5e-4, ii_min_iter=2, ii_max_iter=100, ii_compat=0)
PCISPH_KW = dict(densityErro_eta=5e-3, pci_min_iter=3, pci_max_iter=50)
# WCSPH dam break: Tait B = 50,000 Pa (c_s = sqrt(B gamma / rho0)), gamma 7,
# Monaghan viscosity 0.01, fixed dt = 2.5e-4 s
WCSPH_KW = dict(dt=2.5e-4, soundSpeed_cs=18.708287, wc_gamma=7.0, cfl=0)
WCSPH_VISC = dict(visc_alpha=0.01, boundary_visc=0.01)


def gpu_scene(sc, device, visc_alpha=0.0, boundary_visc=0.0, **kw):
    from graphics_b200.sph import GpuScene, params_for_scene
    g = GpuScene(params_for_scene(sc, boundary_visc=boundary_visc, **kw), sc.n_fluid, device=device)
    g.set_boundary(sc.boundary_pos, sc.meta.get("solid_id"))
    if sc.phase is None:
        g.add_fluid(sc.fluid_pos, sc.fluid_vel, rho0=sc.rho0, visc_alpha=visc_alpha)
    else:
        for ph, rho in enumerate(sc.rho0_phases):
            m = sc.phase == ph
            g.add_fluid(sc.fluid_pos[m], sc.fluid_vel[m], rho0=rho, visc_alpha=visc_alpha)
    return g


def _stream(g, torch, device):
    return torch.cuda.ExternalStream(g.lib.sphgpu_stream(g.h), device=torch.device("cuda", device))


def subarm_warm_2m(args, net, device, torch):
    """The learned warm start at 2,000,000 particles (200 x 100 x 100 block,
    r = 0.008 m, the 1M dam break's box and goals): the same window (after
    settle + warm-up steps) timed plain, with a network trained the way the
    1M arm's is -- on recorded plain runs of this configuration with other
    jitter seeds (every 350th particle of 350 steps per seed, 20 epochs) --
    and with the 1M-trained network (features are dimensionless, so it
    transfers; how well is the second figure)."""
    from graphics_b200.scene import config_dfsph_2m
    from graphics_b200.warmstart import attach, train_for_scenes
    from graphics_b200.sph import scene_to_gpu
    sc = config_dfsph_2m()
    g = scene_to_gpu(sc, device=device, **SOLVER_KW)
    s = _stream(g, torch, device)
    g.step("dfsph", SETTLE[0])
    pos, vel = g.get("position"), g.get("velocity")
    g.step("dfsph", max(args.warmup, 1))
    ms, st = timed_window(g, "dfsph", args.steps, s, torch, None)
    out = {"config": "DFSPH dam break 2M (200x100x100, r=0.008), settle %d" % SETTLE[0],
           "plain": {"value": st["n_fluid"] * args.steps / (ms / 1e3), "ms_per_step": round(ms / args.steps, 3),
                     "iterations_per_step": st["total_iter_density"] / args.steps}}

    def warm_window(network):
        g.set("position", pos)
        g.set("velocity", vel)
        attach(g, network, 1)
        g.step("dfsph", max(args.warmup, 1))
        wms, sw = timed_window(g, "dfsph", args.steps, s, torch, None)
        attach(g, None, 0)
        return {"value": sw["n_fluid"] * args.steps / (wms / 1e3), "ms_per_step": round(wms / args.steps, 3),
                "iterations_per_step": sw["total_iter_density"] / args.steps, "err_density_last": sw["err_density"]}

    if not args.no_warm_start:
        t0 = time.perf_counter()
        seeds = [int(x) for x in args.train_seeds.split(",") if x]
        own, losses = train_for_scenes(config_dfsph_2m, seeds, settle=0, record_steps=args.train_steps,
                                       every=2 * args.train_every, epochs=20, lr=1e-3, batch=8192, device=device,
                                       dataset_cap=4_200_000, **SOLVER_KW)
        out["warm"] = warm_window(own)
        out["speedup_vs_plain"] = round(out["warm"]["value"] / out["plain"]["value"], 3)
        out["training"] = {"seeds": seeds, "samples": own.dataset_size(), "epochs": 20,
                           "loss_first": round(float(losses[0]), 4), "loss_last": round(float(losses[-1]), 4),
                           "seconds": round(time.perf_counter() - t0, 1)}
        own.close()
        out["network"] = "trained on 2M runs of seeds %s (untimed)" % ",".join(map(str, seeds))
    if net is not None:
        w1 = warm_window(net)
        out["warm_1m_network"] = dict(w1, speedup_vs_plain=round(w1["value"] / out["plain"]["value"], 3))
    g.close()
    return out


def subarm_wcsph_27k(args, device, torch):
    """The 27,000-particle WCSPH dam break (r = 0.025 m): 1,000 steps of
    2.5e-4 s from the seeded lattice, all timed."""
    from graphics_b200.scene import config_wcsph_27k
    sc = config_wcsph_27k()
    g = gpu_scene(sc, device, **WCSPH_VISC, **WCSPH_KW)
    s = _stream(g, torch, device)
    g.step("wcsph", 0)
    ms, st = timed_window(g, "wcsph", 1000, s, torch, None)
    rho = g.get("density").astype(np.float64)
    g.close()
    return {"config": "WCSPH dam break 27k (30^3, r=0.025), fixed dt 2.5e-4 s, 1000 steps from the lattice",
            "value": st["n_fluid"] * 1000 / (ms / 1e3), "ms_per_step": round(ms / 1000, 4),
            "mean_density_error_last": float(rho.mean() / sc.rho0 - 1.0), "status": st["status"]}


def settled_column_500k(device, steps=300):
    """The 500k column settled under gravity: the reference's iterative
    multiphase solvers do not hold a 126-layer column started from the
    lattice at rest (PCISPH and IISPH_M reach their iteration caps in the
    first steps, compress it past the neighbour cap and blow it apart, in
    the CPU restatement as on the GPU), so, as the reference's own settled
    column fixture is made, the column first settles as one fluid under
    DFSPH (fixed dt 1e-3 s, `steps` steps); then the particles above the
    perturbed interface become the heavy phase."""
    import dataclasses
    from graphics_b200.scene import config_multiphase_500k
    sc = config_multiphase_500k()
    one = dataclasses.replace(sc, phase=None, rho0_phases=(sc.rho0,))
    g = gpu_scene(one, device, **MULTI_VISC, **{**SOLVER_KW, "cfl": 0, "dt": 1e-3})
    g.step("dfsph", steps)
    pos, vel = g.get("position"), g.get("velocity")
    g.close()
    x, y, z = (pos[:, k].astype(np.float64) for k in range(3))
    box = sc.meta["box"]
    iface = box[1] / 2 + 0.02 * np.sin(2 * np.pi * x) * np.sin(2 * np.pi * z)
    return dataclasses.replace(sc, fluid_pos=np.ascontiguousarray(pos), fluid_vel=np.ascontiguousarray(vel),
                               phase=(y > iface).astype(np.int32))


def subarm_multiphase_500k(args, device, torch):
    """The 500k two-phase Rayleigh-Taylor column (settled first, see
    settled_column_500k): IISPH_M (relaxed Jacobi, omega 0.5, 0.05 %) and
    PCISPH (0.5 %, at most 50 iterations), fixed dt = 1e-3 s; each timed
    over K steps after W warm-up steps."""
    sc = settled_column_500k(device)
    out = {"config": "two-phase column 500,094 (63x126x63, rho0 1000/3000), fixed dt 1e-3 s, from the column "
                     "settled as one fluid (300 DFSPH steps)"}
    for name, solver, kw in (("iisph_m", "iisph_m", IISPH_M_KW), ("pcisph", "pcisph", PCISPH_KW)):
        g = gpu_scene(sc, device, **MULTI_VISC, **MULTI_KW, **kw)
        s = _stream(g, torch, device)
        g.step(solver, max(args.warmup, 1))
        ms, st = timed_window(g, solver, args.steps, s, torch, None)
        out[name] = {"value": st["n_fluid"] * args.steps / (ms / 1e3), "ms_per_step": round(ms / args.steps, 3),
                     "iterations_per_step": st["total_iter_density"] / args.steps, "status": st["status"],
                     "n_fluid": st["n_fluid"]}
        g.close()
    return out


def run_subarms(args, net, device, stream, torch):
    out = {}
    for name, fn in (("config5_warm_start_2m", lambda: subarm_warm_2m(args, net, device, torch)),
                     ("config1_wcsph_27k", lambda: subarm_wcsph_27k(args, device, torch)),
                     ("config3_multiphase_500k", lambda: subarm_multiphase_500k(args, device, torch)),
                     ("config4_batched_64", lambda: subarm_batched_64(args, device, torch))):
        try:
            out[name] = fn()
        except Exception as e:
            out[name] = {"error": str(e)[:300]}
    return out


def lpt_shards(sizes, world):
    """Longest-processing-time-first assignment of scenes to ranks."""
    load = [0] * world
    parts = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda i: -sizes[i]):
        r = min(range(world), key=lambda r: load[r])
        parts[r].append(i)
        load[r] += sizes[i]
    return [sorted(p) for p in parts]


def batched_window(scenes, args, device, torch, dist, unbatched):
    """One batch of independent dam breaks on this GPU: settle (at most 100
    steps), the block-size autotuner, W warm-up steps, then K steps timed
    with CUDA events (max over ranks).  Also: the per-kernel event times of
    a few host-driven steps, whose sum against the graph-timed step gives
    the launch overhead per step; with `unbatched`, the same scenes from the
    same states stepped one single-scene handle after another."""
    from graphics_b200.sph import batch_to_gpu, scene_to_gpu
    b = batch_to_gpu(scenes, device=device, **SOLVER_KW)
    stream = torch.cuda.ExternalStream(b.lib.sphgpu_stream(b.h), device=torch.device("cuda", device))
    settle = min(args.settle, 100)
    if settle:
        b.step("dfsph", settle)
    tune = b.autotune("dfsph", 2)
    b.step("dfsph", max(args.warmup, 1))
    n0 = b.n_fluid
    snap = [(b.get_scene("position", k), b.get_scene("velocity", k)) for k in range(len(scenes))]
    ms, st = timed_window(b, "dfsph", args.steps, stream, torch, dist)
    per = b.scene_stats()
    its = [p_["total_iter_density"] / args.steps for p_ in per]
    # kernel time per step (individual launches with events) on the next steps
    b.profile(True)
    nprof = 3
    b.step("dfsph", nprof)
    prof = b.profile_read()
    b.profile(False)
    post = b.scene_stats()
    kern_ms = sum(t for t, c in prof.values()) / nprof
    launches = sum(c for t, c in prof.values()) / nprof
    b.close()
    unb = None
    if unbatched:
        t_seq = 0.0
        for k, sc in enumerate(scenes):
            g = scene_to_gpu(sc, device=device, **SOLVER_KW)
            g.set("position", snap[k][0])
            g.set("velocity", snap[k][1])
            s2 = torch.cuda.ExternalStream(g.lib.sphgpu_stream(g.h), device=torch.device("cuda", device))
            g.step("dfsph", 1)
            g.set("position", snap[k][0])
            g.set("velocity", snap[k][1])
            g.step("dfsph", 0)
            f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            f0.record(s2)
            g.step_async("dfsph", args.steps)
            f1.record(s2)
            g.synchronize()
            torch.cuda.synchronize()
            t_seq += f0.elapsed_time(f1)
            g.close()
        unb = {"value": n0 * args.steps / (t_seq / 1e3), "unit": UNIT, "ms_per_step": t_seq / args.steps,
               "note": "the same scenes from the same states, one single-scene handle after another"}
    # a loop runs while any scene is active: its trips are the most any scene
    # took (the per-scene totals count the last step call)
    it_prof = sum(max(q[k] for q in post) for k in ("total_iter_density", "total_iter_divergence")) / nprof
    return {"ms": ms, "st": st, "n0": n0, "settle": settle, "tune": tune, "unbatched": unb,
            "iterations_per_step": {"density_min": min(its), "density_max": max(its),
                                    "density_mean": sum(its) / len(its)},
            "launch_overhead": {"kernel_ms_per_step": round(kern_ms, 4),
                                "launches_per_step": round(launches, 1),
                                "loop_iterations_per_step": round(it_prof, 2),
                                "note": "sum of the event-timed kernels of host-driven steps; against the graph-timed "
                                        "ms_per_step (different steps, same flow) the difference is the launch and "
                                        "dependency overhead of the graph's kernel nodes"}}


def run_batched(args):
    """64 independent dam breaks (10k-200k particles, log-uniform) in one
    batch per GPU: one neighbour search and one launch per sweep for all of
    them, per-scene CFL step and loop convergence.  Multi-GPU: scenes sharded
    over ranks (longest first), no data-path collective; value = all ranks'
    particle-steps / max-over-ranks time."""
    import torch
    world, rank, local, dist = init_dist(torch)
    from graphics_b200.scene import config_batched_dfsph
    scenes_all = config_batched_dfsph(64, seed=0)
    mine = lpt_shards([s.n_fluid for s in scenes_all], world)[rank]
    scenes = [scenes_all[i] for i in mine]
    with ClockSampler(local) as clk:
        r = batched_window(scenes, args, local, torch, dist, unbatched=(world == 1))
    ms_max, st = r["ms"], r["st"]
    if dist:
        tot = torch.tensor([float(st["n_fluid"])], device="cuda")
        dist.all_reduce(tot)
        n_all = tot.item()
    else:
        n_all = st["n_fluid"]
    value = n_all * args.steps / (ms_max / 1e3)
    unb = r["unbatched"]
    if rank == 0:
        line = {"metric": "batched DFSPH particle-steps/s (64 independent scenes, 10k-200k particles each)",
                "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak" if world == 1 else
                "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded dam breaks)",
                "config": {"workload": "batched_dfsph_64", "n_scenes": len(scenes_all),
                           "n_fluid_total": int(sum(s.n_fluid for s in scenes_all)),
                           "n_boundary_total": int(sum(s.n_boundary for s in scenes_all)),
                           "scenes_on_rank0": len(scenes), "r": 0.01, "settle_steps": r["settle"],
                           "parallelism": "scene shards x%d (LPT)" % world if world > 1 else "single",
                           "l2": "inputs larger than L2"},
                "iterations_per_step": r["iterations_per_step"], "launch_overhead": r["launch_overhead"],
                "autotune": r["tune"], "unbatched": unb,
                "speedup_vs_unbatched": (value / unb["value"]) if unb else None,
                "gpu_launches": int(round(r["launch_overhead"]["launches_per_step"] * args.steps)),
                "clocks": clk.summary()}
        print(json.dumps(line))
    if dist:
        dist.destroy_process_group()


def subarm_batched_64(args, device, torch):
    """The batched configuration (64 independent dam breaks of 10k-200k
    particles in one batch), compactly: value, the autotuner's choice, the
    launch overhead per step and the speed-up over the same scenes stepped
    one handle after another."""
    from graphics_b200.scene import config_batched_dfsph
    scenes = config_batched_dfsph(64, seed=0)
    r = batched_window(scenes, args, device, torch, None, unbatched=True)
    value = r["st"]["n_fluid"] * args.steps / (r["ms"] / 1e3)
    unb = r["unbatched"]
    return {"config": "64 dam breaks, %d fluid particles in all, settle %d" % (r["n0"], r["settle"]),
            "value": value, "ms_per_step": round(r["ms"] / args.steps, 3),
            "iterations_per_step": r["iterations_per_step"], "launch_overhead": r["launch_overhead"],
            "autotune": r["tune"].get("chosen", r["tune"]),
            "unbatched_value": unb["value"], "speedup_vs_unbatched": round(value / unb["value"], 3)}


# Dynamic rigid body: the DFSPH step with a 0.4 m box of density 500
# floating half submerged in a 1 m deep pool filling the 4 x 2 x 2 m tank
# (200 x 50 x 100 fluid lattice, r = 0.01 m, ~995k fluid particles after the
# box's volume is cleared; 2,402 body and ~180k wall particles), the host
# rigid-body world (graphics_b200.rigid) in the loop every step.
RIGID_BODY = dict(half=(0.2, 0.2, 0.2), center=(2.0, 1.0, 1.0), density=500.0,
                  q=(float(np.cos(0.05)), 0.0, 0.0, float(np.sin(0.05))))
# Algorithmic bytes per boundary particle (every wall and body particle) of
# the per-step boundary kernels, and per body particle of the force kernel:
#   rigid_place  : place (x0, dyn -> wpos, wvel, key, slot, count = 64 B),
#                  scatter (key, slot, cell start -> tmp = 16 B), in-cell
#                  rank and gather (tmp, key, cell range, wpos, wvel, vol,
#                  sid -> bpos, bks, bpv, bpf, bgid, bsid, binv = 156 B);
#                  plus 12 B per cell key (count clear, scan read + write)
#   rigid_volume : bpos, bsid, bks, bgid in; volume into bpos, bpv, bpf and
#                  the reference-order copy (44 B)
#   rigid_force  : binv, bpf record in, force out (52 B)
RIGID_ALG = {"rigid_place": 236, "rigid_volume": 44, "rigid_force": 52}
RIGID_ALG_PER_KEY = {"rigid_place": 12}


def cell_keys(sc):
    """Cell keys of the scene's grid (4x4x4 bricks of smoothRadius_h cells
    over [spaceMin - 2h, spaceMax + 2h], as the library enumerates them)."""
    h = np.float32(sc.smooth_radius)
    lo, hi = np.float32(sc.space_min), np.float32(sc.space_max)
    num = ((hi - lo + h * np.float32(2)) * (np.float32(1) / h)).astype(np.int64) + 2
    return int(np.prod((num + 3) // 4) * 64 + 1)


def rigid_workload(seed=0):
    from graphics_b200.scene import floating_box
    b = RIGID_BODY
    return floating_box((200, 50, 100), 0.01, (4.0, 2.0, 2.0), b["half"], b["center"], seed=seed)


def rigid_world(sc):
    from graphics_b200.rigid import RigidBody, RigidWorld
    b, m = RIGID_BODY, sc.meta["bodies"][0]
    w = RigidWorld()
    w.add(m["solid_id"], RigidBody.box(b["density"], b["half"], b["center"], q=b["q"]))
    return w


def cpu_rigid_sample(sc, budget, dt):
    """The reference's DFSPH with the rigid stand-in of the oracle harness
    (rigidForceJoin, the same host world, updatePaticles) on all host cores,
    steps from rest until `budget` seconds."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import make_scene_oracle
    t0 = time.perf_counter()
    o = make_scene_oracle(sc, kind="reference", solver="dfsph_capped", nu=SOLVER_KW["nu"], dt=dt)
    w = rigid_world(sc)
    m = sc.meta["bodies"][0]
    o.set_solid_dynamic(m["solid_id"], m["inner"], w.state(m["solid_id"]))
    o.set_rigid_world(w)
    setup = time.perf_counter() - t0
    steps, t_run = 0, 0.0
    while True:
        t1 = time.perf_counter()
        o.stage("runOneStep")
        t_run += time.perf_counter() - t1
        steps += 1
        if t_run >= budget or steps >= 50:
            break
    cores = o.threads()
    o.close()
    return {"value": sc.n_fluid * steps / t_run, "unit": UNIT, "cores": cores, "kind": "reference",
            "sample": "%d DFSPH step(s) of the %d-particle floating-box scene from rest at fixed dt=%.1e s with "
                      "the dynamic box coupled every step (reference DFSPH.cpp + SphBase.cpp rigidForceJoin / "
                      "updatePaticles via oracle/_ref, float, all threads; density loop FP64-summed and capped "
                      "at 100), setup %.1f s untimed" % (steps, sc.n_fluid, dt, setup),
            "seconds": t_run}


def run_rigid(args):
    """DFSPH with a dynamic rigid body (one GPU; the scene does not shard)."""
    import torch
    from graphics_b200.sph import scene_to_gpu
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    world_n = int(os.environ.get("WORLD_SIZE", "1"))
    torch.cuda.set_device(local)
    sc = rigid_workload()
    m = sc.meta["bodies"][0]
    g = scene_to_gpu(sc, device=local, **SOLVER_KW)
    if args.no_graphs:
        g.debug_set("use_graphs", 0)
    w = rigid_world(sc)
    g.set_solid_dynamic(m["solid_id"], m["inner"], w.state(m["solid_id"]))
    g.set_rigid_world(w)
    stream = torch.cuda.ExternalStream(g.lib.sphgpu_stream(g.h), device=torch.device("cuda", local))
    settle = min(args.settle, 150)
    if settle:
        g.step("dfsph", settle)
    g.step("dfsph", max(args.warmup, 1))
    import copy
    snap_pos, snap_vel = g.get("position"), g.get("velocity")
    body0 = copy.deepcopy(w.bodies[m["solid_id"]])
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.nvtx.range_push("timed_rigid")  # lets an ncu launch list select the timed steps
        e0.record(stream)
        st = g.step("dfsph", args.steps)
        e1.record(stream)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
    ms = e0.elapsed_time(e1)
    n = st["n_fluid"]
    value = n * args.steps / (ms / 1e3)
    log = w.log[-args.steps:]
    hbm, peak_kind = peaks()
    # per-kernel durations (individual launches, CUDA events), next steps
    g.profile(True)
    g.step("dfsph", args.profile_steps)
    prof = g.profile_read()
    g.profile(False)
    st_p = g.synchronize()
    nbp = sc.n_boundary
    nbody = len(m["inner"])
    kern = {}
    for k, (tot_ms, cnt) in prof.items():
        ent = {"launches": cnt, "avg_us": round(1e3 * tot_ms / max(cnt, 1), 2),
               "us_per_step": round(1e3 * tot_ms / args.profile_steps, 1)}
        if k in RIGID_ALG:
            units = nbody if k == "rigid_force" else nbp
            b = RIGID_ALG[k] * units + RIGID_ALG_PER_KEY.get(k, 0) * cell_keys(sc)
            ent["alg_bytes"] = b
            ent["gbs"] = round(b / (tot_ms / cnt / 1e3) / 1e9, 1)
        kern[k] = ent
    dom = max((k for k in kern if k in RIGID_ALG), key=lambda k: kern[k]["us_per_step"])
    roof = {"bound": "hbm", "kernel": dom, "achieved": kern[dom]["gbs"], "peak": hbm, "unit": "GB/s",
            "frac": round(kern[dom]["gbs"] / hbm, 4), "traffic": None,
            "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback",
            "alg_bytes_per_boundary_particle": RIGID_ALG[dom] if dom != "rigid_force" else None,
            "rigid_us_per_step": round(sum(kern[k]["us_per_step"] for k in kern if k in RIGID_ALG), 1)}
    # the same state with the body held static (one more static solid)
    bpos = g.get_boundary("position")
    g.close()
    from graphics_b200.sph import params_for_scene, GpuScene
    g2 = GpuScene(params_for_scene(sc, **SOLVER_KW), sc.n_fluid, device=local)
    g2.set_boundary(bpos, sc.meta["solid_id"])
    g2.add_fluid(snap_pos, snap_vel, rho0=sc.rho0)
    g2.step("dfsph", max(args.warmup, 1))
    g2.set("position", snap_pos)
    g2.set("velocity", snap_vel)
    g2.step("dfsph", 0)
    s2 = torch.cuda.ExternalStream(g2.lib.sphgpu_stream(g2.h), device=torch.device("cuda", local))
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(s2)
    st2 = g2.step("dfsph", args.steps)
    f1.record(s2)
    torch.cuda.synchronize()
    ms2 = f0.elapsed_time(f1)
    g2.close()
    # end to end: host positions/velocities in and out every step, the world
    # in the loop, from the snapshot of the timed region's start
    e2e = None
    if args.e2e_steps > 0:
        g3 = scene_to_gpu(sc, device=local, **SOLVER_KW)
        w3 = rigid_world(sc)
        w3.bodies[m["solid_id"]] = copy.deepcopy(body0)
        g3.set_solid_dynamic(m["solid_id"], m["inner"], w3.state(m["solid_id"]))
        g3.set_rigid_world(w3)
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
        pos, vel = pin(snap_pos), pin(snap_vel)
        po, vo = pin(np.empty_like(snap_pos)), pin(np.empty_like(snap_vel))
        g3.step_host("dfsph", pos, vel, po, vo)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            g3.step_host("dfsph", pos, vel, po, vo)
            pos, po = po, pos
            vel, vo = vo, vel
        sec = time.perf_counter() - t0
        e2e = {"value": n * args.steps / sec, "unit": UNIT, "h2d_bytes_per_step": int(n * 24),
               "d2h_bytes_per_step": int(n * 24), "steps": args.steps,
               "note": "sphgpu_step_host with the rigid world in the loop: pinned positions+velocities in, "
                       "step, positions+velocities out"}
        g3.close()
    cpu = None
    if rank == 0 and world_n == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_rigid_sample(sc, budget=args.cpu_budget, dt=st["dt"])
        except Exception as e:
            cpu = {"unavailable": str(e)}
    if rank == 0:
        F = np.array([f for _, f, _, _ in log])[:, 0]
        line = {"metric": "DFSPH particle-steps/s with a dynamic rigid body coupled every step", "value": value,
                "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded pool with a floating box)",
                "config": {"workload": "dfsph_floating_box_%dk" % (sc.n_fluid // 1000), "n_fluid": sc.n_fluid,
                           "n_boundary": nbp, "n_body_particles": nbody, "body": RIGID_BODY, "r": sc.r,
                           "box": list(sc.meta["box"]), "settle_steps": settle, "cfl": 0.4,
                           "dt_max": SOLVER_KW["dt_max"], "density_goal": 1e-4, "divergence_goal": 1e-3,
                           "parallelism": "single", "l2": "inputs larger than L2"},
                "iterations_per_step": {"density": st["total_iter_density"] / args.steps,
                                        "divergence": st["total_iter_divergence"] / args.steps},
                "static_body": {"ms_per_step": ms2 / args.steps,
                                "iterations_per_step": {"density": st2["total_iter_density"] / args.steps,
                                                        "divergence": st2["total_iter_divergence"] / args.steps},
                                "note": "the same state with the box as a static solid"},
                "body_force_last": F[-1].tolist(), "body_state_last": w.state(m["solid_id"])[16:22].tolist(),
                "roofline": roof, "kernels": kern, "cpu_baseline": cpu, "e2e": e2e,
                "gpu_launches": int(round(sum(kern[k]["launches"] for k in kern) * args.steps
                                          / max(args.profile_steps, 1))),
                "clocks": clk.summary()}
        print(json.dumps(line))


# Surface reconstruction: the reference's reconstruction driver (re.c:29,
# 107, 112) on the 1M-particle dam-break block (100^3 jittered lattice,
# r_p = 0.01 m): surface_setup(bbox, r_p, r_h = 2 r_p, cell = r_p / 4),
# surface_aniso, marchingCubes at iso 0.5.  One "step" = field + mesh.
SURF = dict(r_p=0.01, r_h=0.02, cell=0.0025, iso=0.5)
# algorithmic bytes of the field kernel per launch: every node written once
# (4 B), every (tile, particle) pair's record read once (centre + det, G,
# box = 64 B) with its particle index (4 B)
SURF_ALG_NODE, SURF_ALG_PAIR = 4, 68


def cpu_surface_sample(pos, budget):
    """The reference's surface_aniso + marchingCubes (oracle/_ref, one
    thread: surface_aniso has no OpenMP) on a sub-block of the workload,
    grown until it takes about `budget` seconds."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import RefSurface
    lo = pos.min(0)
    side, t_run, n = 10, 0.0, 0
    while True:
        m = np.all(pos < lo + side * 2 * SURF["r_p"], axis=1)
        sub = pos[m].astype(np.float64)
        rs = RefSurface(sub.min(0), sub.max(0), SURF["r_p"], SURF["r_h"], SURF["cell"])
        t0 = time.perf_counter()
        f = rs.field(sub, aniso=True)
        tris = RefSurface.marching_cubes(SURF["iso"], f, rs.grid_min.astype(np.float32), rs.grid_num,
                                         np.float32(rs.cell))
        t_run = time.perf_counter() - t0
        n = len(sub)
        rs.close()
        if t_run >= budget / 4 or side >= 100:
            break
        side = int(side * 1.6)
    return {"value": n / t_run, "unit": "particles/s", "cores": 1, "kind": "reference",
            "sample": "%d particles (a %d^3 corner of the block): surface_aniso + marchingCubes of the reference "
                      "(oracle/_ref, float field, FP64 kernels; single-threaded as written), %d triangles"
                      % (n, side, len(tris)),
            "seconds": t_run}


def run_surface(args):
    """Surface reconstruction of the 1M-particle block (one GPU; a single
    field does not shard)."""
    import torch
    from graphics_b200.scene import lattice_block
    from graphics_b200.surface import surface_field
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    pos = lattice_block((args.scale,) * 3, SURF["r_p"], jitter=0.1, seed=0)
    n = len(pos)
    sf = surface_field(device=local)
    sf.surface_setup(pos.min(0).astype(np.float64), pos.max(0).astype(np.float64), SURF["r_p"], SURF["r_h"],
                     SURF["cell"])
    dpos = torch.from_numpy(pos).to("cuda")
    stream = torch.cuda.ExternalStream(sf.lib.sphgpu_surface_stream(sf.h), device=torch.device("cuda", local))
    lib = sf.lib

    def step():
        rc = lib.sphgpu_surface_field(sf.h, 1, dpos.data_ptr(), n, 1)
        assert rc == 0, rc
        return lib.sphgpu_surface_mesh(sf.h, SURF["iso"], 0, None, 0)

    for _ in range(max(args.warmup, 1)):
        ntri = step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    k0 = sf.stats()[2]
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            ntri = step()
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    npairs, ntiles, k1 = sf.stats()
    value = n * args.steps / (ms / 1e3)
    # per-kernel durations: the field and mesh calls bracketed by events
    f0, f1, f2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    tf = tm = 0.0
    reps = max(args.profile_steps, 1)
    for _ in range(reps):
        f0.record(stream)
        lib.sphgpu_surface_field(sf.h, 1, dpos.data_ptr(), n, 1)
        f1.record(stream)
        lib.sphgpu_surface_mesh(sf.h, SURF["iso"], 0, None, 0)
        f2.record(stream)
        torch.cuda.synchronize()
        tf += f0.elapsed_time(f1)
        tm += f1.elapsed_time(f2)
    nodes = int(np.prod(sf.get_grid_num()))
    # end to end: host positions in, host triangles out
    e2e = None
    if args.e2e_steps > 0:
        pin = torch.from_numpy(pos).pin_memory().numpy()
        out = torch.empty((ntri, 3, 3), dtype=torch.float32, pin_memory=True).numpy()
        import ctypes as C
        t0 = time.perf_counter()
        for _ in range(args.steps):
            lib.sphgpu_surface_field(sf.h, 1, pin.ctypes.data, n, 0)
            m = lib.sphgpu_surface_mesh(sf.h, SURF["iso"], 0, out.ctypes.data_as(C.POINTER(C.c_float)), ntri)
        sec = time.perf_counter() - t0
        e2e = {"value": n * args.steps / sec, "unit": "particles/s", "h2d_bytes_per_step": int(n * 12),
               "d2h_bytes_per_step": int(m * 36), "steps": args.steps,
               "note": "sphgpu_surface_field from host positions, sphgpu_surface_mesh into host memory"}
    hbm, peak_kind = peaks()
    # the field kernel (the largest share of the step): its algorithmic bytes
    # over its event-timed duration; bound by instruction issue in practice
    # (every row of a tile tests every particle listed under the tile), so
    # the HBM fraction is low by construction
    field_bytes = nodes * SURF_ALG_NODE + npairs * SURF_ALG_PAIR
    roof = {"kernel": "k_sf_field (+ per-particle kernels and tile binning of sphgpu_surface_field)",
            "bound": "hbm", "achieved": field_bytes / (tf / reps * 1e-3) / 1e9, "peak": hbm, "unit": "GB/s",
            "traffic": None, "alg_bytes": int(field_bytes), "tile_pairs": int(npairs), "tiles": int(ntiles),
            "peak_source": peak_kind}
    roof["frac"] = roof["achieved"] / hbm
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        try:
            cpu = cpu_surface_sample(pos, args.cpu_budget)
        except Exception as e:
            cpu = {"unavailable": str(e)}
    if rank == 0:
        line = {"metric": "surface reconstruction particles/s (anisotropic field + marching cubes)", "value": value,
                "unit": "particles/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic (seeded jittered lattice block)",
                "config": {"workload": "surface_aniso_block_%dk" % (n // 1000), "n_particles": n, **SURF,
                           "grid_nodes": nodes, "grid": sf.get_grid_num().tolist(), "triangles": int(ntri),
                           "parallelism": "single", "l2": "field %.1f GB > L2" % (nodes * 4 / 1e9)},
                "kernels": {"field_ms": tf / reps, "mesh_ms": tm / reps},
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(k1 - k0),
                "clocks": clk.summary()}
        print(json.dumps(line))
    sf.close()


def main():
    args = parse()
    SOLVER_KW["df_density_max_iter"] = args.max_iter
    SETTLE[0] = args.settle
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batched_64":
        run_batched(args)
    elif args.workload == "floating_box_1m":
        run_rigid(args)
    elif args.workload == "surface_1m":
        run_surface(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
