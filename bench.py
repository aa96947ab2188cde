#!/usr/bin/env python
"""Benchmark of the B200 SPH step engine on the IISPH dam break with
4,194,304 fluid particles (256 x 128 x 128 lattice, spacing 0.005, jitter
+-0.05 h, 2 x 1 x 1 box with one layer of Akinci wall particles, Wendland C2,
rest density 1000, viscosity 0.01, relaxed Jacobi omega = 0.5 to 0.1 % average
density error, adaptive dt from the reference's CFL controller with
lambda = 0.4).

A step is one iteration of the reference main loop (main.cu:60-78): dt
controller (CFL max-velocity reduction), uniform-grid build + reorder of the
state, IISPH step, hard bounds; the bounds and the max-velocity reduction run
inside the step's integrating kernel. Inputs are resident in HBM for `value`; `e2e`
repeats the step through the C ABI with the state uploaded from and downloaded
to pinned host memory inside the timed region.

By default the FP32 solver and the two mixed-precision solvers (neighbour
velocities, densities and pressure accelerations FP16; in mixed_pos16 also
16-bit neighbour positions; FP32 arithmetic, FP64 convergence reduction) are
timed on the same scene; the fastest is the headline ("headline_precision"),
the others are reported beside it, with "mixed_over_fp32".

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]
                       [--precision all|mixed|mixed_pos16|fp32]
Under torchrun (N > 1) every rank advances its own independently seeded scene
(weak scaling, no data-path collective); rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import ctypes
import datetime
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s, 4M IISPH, mixed vs FP32 at ≤0.1% ρ err; % of HBM peak"
UNIT = "particle-steps/s"
WORKLOAD = "iisph_dam_break_4M"

# Algorithmic (compulsory) bytes per fluid particle of each kernel: every
# array the kernel's reference counterpart reads or writes, once, FP32;
# neighbour data assumed cache-resident. Boundary samples add 16 B each to the
# density pass, the only pass that visits them.
ALG_BYTES = {
    "k_density": 12 + 4 + 4,          # x, m -> rho
    "k_nonpressure": 12 + 12 + 4 + 4 + 12 + 12,  # x, v, m, rho -> a, v*
    "k_iisph_diag": 12 + 12 + 4 + 4 + 4 + 4 + 4,  # x, v*, m, rho -> a_ii, s_i; p warm start
    "k_iisph_pacc": 12 + 4 + 4 + 12,  # x, m, p -> a
    "k_iisph_jacobi": 12 + 4 + 12 + 8 + 4 + 4,  # x, m, a, p r/w, a_ii, s_i
    "k_iisph_final": 12 + 4 + 4 + 12 + 12 + 12 + 12,  # x, m, p, v* -> a, x, v
    # the same passes over 16-byte neighbour records (mixed_pos16): the same
    # compulsory arrays of their reference counterparts
    "k_np_rec": 12 + 12 + 4 + 4 + 12 + 12,
    "k_diag_pacc_rec": 12 + 12 + 4 + 4 + 4 + 4 + 4 + 12,
    "k_diag_rec": 12 + 12 + 4 + 4 + 4 + 4 + 4,
    "k_pacc_rec": 12 + 4 + 4 + 12,
    "k_jacobi_rec": 12 + 4 + 12 + 8 + 4 + 4,
    "k_final_rec": 12 + 4 + 4 + 12 + 12 + 12 + 12,
    "k_keys_count": 12 + 4,           # x -> key (+ histogram)
    "k_scatter": 4 + 4 + 4,           # key, prefix -> slot
    "k_canonical": 4 + 4 + 4 + 4,     # slot, key, prefix -> sorted
    "k_gather": 4 + 28 + 28 + 32,     # perm, 7 arrays in/out, packed copies
    "k_vmax": 12,
    "k_bounds_enforce": 24 + 12,
    "k_unpack_acc": 16 + 12,
}


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--scale", type=int, default=1,
                    help="divide the lattice by this factor per axis (testing only)")
    ap.add_argument("--precision", choices=["all", "mixed", "mixed_pos16", "fp32"],
                    default="all",
                    help="all: time FP32 and mixed_pos16, then report the mixed path beside them")
    ap.add_argument("--order", choices=["xyz", "zorder"], default="xyz",
                    help="cell order of the grid the state is sorted by")
    ap.add_argument("--workload", choices=["iisph_4m", "batched_pcisph", "batched_iisph",
                                           "column_16m", "mesh_lbvh"],
                    default="iisph_4m",
                    help="batched_pcisph: 256 independent PCISPH scenes; batched_iisph: "
                         "about 4M particles of independent IISPH scenes in FP32 and the "
                         "mixed modes; column_16m: the "
                         "16.7M-particle column collapse onto a sphere; mesh_lbvh: LBVH "
                         "closest-point queries and boundary sampling of a 327,680-face mesh "
                         "(none is the headline)")
    ap.add_argument("--scenes", type=int, default=0,
                    help="batched workloads: scene count (0: 256 for PCISPH, 96 for IISPH)")
    ap.add_argument("--no-sequential", action="store_true",
                    help="batched_pcisph: skip the scene-by-scene comparison run")
    ap.add_argument("--no-autotune", action="store_true",
                    help="skip the block-size / cell-ratio autotuner (128 threads, cell r/2)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--reorder-every", type=int, default=1,
                    help="column_16m: reorder the state every K steps, the steps between on "
                         "grids built without reorder")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-precision-check", action="store_true",
                    help="iisph_4m: skip the error of every precision mode against the "
                         "FP64 checker on the benchmark scene")
    ap.add_argument("--develop-steps", type=int, default=2500,
                    help="iisph_4m: untimed FP32 steps that develop the flow before the "
                         "'developed' leg times every precision from the same state "
                         "(0: no developed leg)")
    return ap.parse_args()


NU = 0.01
LAMBDA = 0.4
DT0 = 5e-4
# the steps both arms time with the reference's own constants: the reference
# arm on the reference's CUDA, the engine arm on the engine
REF_CUDA_STEPS = 5
REF_CUDA_DT = 2e-4


def workload_config(n: int, nb: int, h: float, rho0: float, world: int) -> dict:
    """The workload as both arms state it (the same keys and values): scene,
    kernel, solver constants and dt rule. Engine settings (precision, block
    size, cell size, reorder interval) are reported under "engine"."""
    return {"workload": WORKLOAD, "particles_per_gpu": n, "boundary_particles": nb,
            "kernel": "C2", "h": h, "rho0": rho0, "nu": NU, "omega": 0.5,
            "convergence": "avg density error <= 0.1% (FP64 reduction)",
            "dt": f"min(simple_dt_controller(lambda={LAMBDA}, target 10 iters, "
                  f"0.1%/step) from {DT0}, 0.08 h^2/nu = {viscous_dt_limit(h, NU):.2e})",
            "parallelism": f"replicas{world}",
            "l2": "inputs larger than L2 (state 4M x 28 B + grid 70 MB per step)"}


def scene_spec(rank: int, scale: int) -> dict:
    return dict(counts=(256 // scale, 128 // scale, 128 // scale), h=0.005 * scale,
                box=(2.0, 1.0, 1.0), rho0=1000.0, jitter=0.05, seed=3 + rank,
                mass_kernel="C2", gap=1.5)


def scene_for(rank: int, scale: int):
    """The workload built on the host (for the CPU arms)."""
    from reyn_b200 import scenes
    return scenes.dam_break(name=WORKLOAD, **scene_spec(rank, scale))


class DeviceScene:
    """The workload generated on the GPU: the same arrays as scene_for."""

    def __init__(self, rank: int, scale: int):
        from reyn_b200 import scenes
        spec = scene_spec(rank, scale)
        self.st, self.walls, self.box_min, self.box_max = scenes.dam_break_on_device(**spec)
        self.h, self.rho0 = spec["h"], spec["rho0"]
        self.n = self.st.n
        self.nb = int(self.walls[0].numel())


def viscous_dt_limit(h: float, nu: float) -> float:
    """Explicit-viscosity stability bound of the artificial viscosity term
    (solver.cuh:62-63): dt <= 0.08 h^2 / nu (2e-4 s at h = 0.005, nu = 0.01)."""
    return 0.08 * h * h / nu


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_field(kernel: str, precision: str, key: str):
    """A numeric field of the committed ncu summary of `kernel` on this
    workload (profiles/<kernel>_iisph_4m[_mixed].txt, line '<key>: value')."""
    suffix = "" if precision == "fp32" else "_" + precision
    path = os.path.join(ROOT, "profiles", f"{kernel}_iisph_4m{suffix}.txt")
    try:
        for line in open(path):
            if line.startswith(key + ":"):
                return float(line.split(":", 1)[1].split()[0])
    except (OSError, ValueError):
        pass
    return None


def profile_traffic(kernel: str, precision: str):
    """DRAM bytes per launch of `kernel` on this workload, from its committed
    ncu summary (line 'traffic_bytes_per_launch:')."""
    return profile_field(kernel, precision, "traffic_bytes_per_launch")


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.p = None
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200",
                                       "-i", gpu_id], stdout=subprocess.PIPE,
                                      stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.p.terminate()
        out, _ = self.p.communicate(timeout=10)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                    device_id=torch.device("cuda", local))
        else:  # host-only ranks (the reference arm's CPU leg, CPU tests)
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(world, v: float) -> float:
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---- engine arm ---------------------------------------------------------------

class EngineRun:
    """The workload on the engine: one scene, its grid, boundary and solver,
    and the main-loop step (main.cu:64-75)."""

    def __init__(self, rank: int, scale: int, dev, precision: str, order: str = "xyz",
                 ratio: float = 0.5, block: int = 0, reorder_every: int = 1):
        import reyn_b200 as rb

        self.rb = rb
        self.precision = precision
        self.sc = sc = DeviceScene(rank, scale)
        self.n = sc.n
        self.st = sc.st
        self.bd = rb.Boundary(*sc.walls, None, h=sc.h, rho0=sc.rho0, mass_iters=5)
        self.grid = rb.Grid(sc.box_min, sc.box_max, 2 * sc.h, ratio,
                            rb.ORDER_ZORDER if order == "zorder" else rb.ORDER_XYZ)
        prm = self.params(rb, sc, precision)
        prm.block_size = block
        self.sv = rb.Solver(rb.IISPH, prm, sc.n)
        self.dt, self.iters = DT0, 0
        # the state is reordered every `reorder_every` steps; the steps
        # between run on grids built without reorder (Resort::no)
        self.reorder_every, self.k = reorder_every, 0
        self.dt_visc = viscous_dt_limit(sc.h, NU)
        self.log = []
        self.limit_hits = 0

    @staticmethod
    def params(rb, sc, precision):
        prm = rb.reference_params(rb.IISPH, rb.C2, sc.h, sc.rho0, NU)
        prm.convergence = rb.CONV_AVERAGE
        prm.eta = 0.001
        prm.max_iter = 1000
        prm.precision = {"mixed": rb.PRECISION_MIXED, "mixed_pos16": rb.PRECISION_MIXED_POS16,
                         "fp32": rb.PRECISION_FP32}[precision]
        return prm

    def step(self, S, ready=None):
        """One main-loop step on stream S. ready = (positions, everything):
        callables that make S wait for the host uploads of the positions and
        of the whole state; the grid is then built while the velocities and
        masses still arrive and the state reordered after them."""
        rb, sc = self.rb, self.sc
        dt_next = lambda: min(self.sv.next_dt(self.st, self.iters, self.dt, LAMBDA, sc.h,
                                              (0.0, -9.81, 0.0), 10, 0.001, stream=S),
                              self.dt_visc)
        # simple_dt_controller (cfl.cu:39-52) at lambda 0.4, capped by the
        # explicit-viscosity bound; its max |v| comes from the previous
        # step's integrating kernel, which also applied the hard bounds
        # (scene.cu:466-491)
        if ready is not None and self.k % self.reorder_every == 0:
            ready[0]()
            self.grid.construct_state(self.st, stream=S)
            ready[1]()
            self.dt = dt_next()
            self.grid.reorder(self.st, stream=S)
        else:
            if ready is not None:
                ready[1]()
            self.dt = dt_next()
            if self.k % self.reorder_every == 0:
                self.grid.construct_and_reorder(self.st, stream=S)
            else:
                self.grid.construct_state(self.st, stream=S)
        self.k += 1
        try:
            it = self.sv.step(self.st, self.grid, self.bd, self.dt, stream=S,
                              bounds=(sc.box_min, sc.box_max))
        except rb.ReynError as e:
            if e.code != rb.ERR_ITER_LIMIT:
                raise
            it = self.sv.stats().iters
            self.limit_hits += 1
        self.iters = it
        self.log.append((it, self.sv.stats().avg_density_error, self.dt))

    def checkpoint(self):
        return (self.st.download(), self.sv.pressure(), self.dt, self.iters, self.k)

    def restore(self, ck):
        state, p, dt, iters, k = ck
        self.st.upload(state)
        self.sv.set_pressure(self.st, p)
        self.dt, self.iters, self.k = dt, iters, k

    def close(self):
        for o in (self.sv, self.grid, self.bd, self.st):
            o.close()


def timed_steps(run, a, world, stream, dev):
    """W warm-up steps, checkpoint, then K steps timed with CUDA events
    (max over ranks), with per-kernel launch counts and device time and the
    SM clocks sampled during the timed region."""
    import torch

    rb = run.rb
    S = stream.cuda_stream
    for _ in range(a.warmup):
        run.step(S)
    torch.cuda.synchronize()
    ck = run.checkpoint()  # the timed region starts here (replayed for e2e)
    run.log.clear()
    gpu_uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    clocks = ClockSampler(gpu_uuid)
    time.sleep(0.3)
    rb.profile_reset()
    rb.profile_enable(True)
    barrier(world)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(a.steps):
        run.step(S)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    rb.profile_enable(False)
    prof = rb.profile_read()
    ck_clocks = clocks.stop()
    ms = e0.elapsed_time(e1)
    ms_max = max_over_ranks(world, ms)
    return ck, ms, ms_max, prof, ck_clocks, list(run.log)


def leg_summary(run, a, world, ms_max, log):
    return {"value": round(world * run.n * a.steps / (ms_max / 1e3), 1), "unit": UNIT,
            "ms_per_step": round(ms_max / a.steps, 3),
            "iters_per_step": [x[0] for x in log],
            "avg_density_error_per_step": [round(x[1], 7) for x in log],
            "iter_limit_hits": run.limit_hits}


def developed_leg(a, world, rank, dev, stream, names, config):
    """The flow developed by a.develop_steps untimed FP32 main-loop steps
    (the dam break's column collapsing), checkpointed; every precision then
    runs W warm-up and K timed steps from that same state. The sweeps per
    step there exceed the 3 of the first steps from rest."""
    import torch

    S = stream.cuda_stream
    base = EngineRun(rank, a.scale, dev, "fp32", a.order, *config["fp32"][:2]
                     if "fp32" in config else (0.5, 0))
    for _ in range(a.develop_steps):
        base.step(S)
    torch.cuda.synchronize()
    ck = base.checkpoint()
    t_sim = float(sum(x[2] for x in base.log))
    base_iters = [x[0] for x in base.log[-10:]]
    base.close()
    out = {"develop_steps": a.develop_steps, "simulated_seconds": round(t_sim, 5),
           "iters_last_develop_steps": base_iters}
    for name in names:
        ratio, block, _, every = config[name]
        r = EngineRun(rank, a.scale, dev, name, a.order, ratio, block, every)
        r.restore(ck)
        _, _, ms_max, prof, clk, log = timed_steps(r, a, world, stream, dev)
        leg = leg_summary(r, a, world, ms_max, log)
        leg["dt_per_step"] = [float(f"{x[2]:.4e}") for x in log]
        leg["clocks"] = clk
        leg["kernels_ms_per_step"] = {
            k: round(v[1] / a.steps, 3)
            for k, v in sorted(prof.items(), key=lambda kv: -kv[1][1])[:8]}
        out[name] = leg
        r.close()
    mixed = [k for k in ("mixed", "mixed_pos16") if k in out]
    if "fp32" in out and mixed:
        out["mixed_over_fp32_by_mode"] = {k: round(out[k]["value"] / out["fp32"]["value"], 3)
                                          for k in mixed}
    return out


PREC_STEPS, PREC_SWEEPS, PREC_DT = 2, 4, 2e-4
PREC_FIELDS = ("x", "y", "z", "vx", "vy", "vz", "rho", "p", "aii", "sii")


def precision_vs_fp64(rank: int, scale: int, names, stream=None):
    """Error of each precision mode against the FP64 restatement of the IISPH
    step (oracle/fp64.py, the checker: torch float64 on this GPU, pairs by
    cube bucketing) on the benchmark scene itself: PREC_STEPS main-loop steps
    of exactly PREC_SWEEPS Jacobi sweeps at dt PREC_DT from rest, the same
    initial state and boundary masses for every run. Per quantity the largest
    error relative to the field's largest magnitude, and the mean
    |rho - rho_FP64| / rho0."""
    import torch

    import reyn_b200 as rb
    from oracle import fp64

    S = None if stream is None else stream.cuda_stream
    sc = DeviceScene(rank, scale)
    bd = rb.Boundary(*sc.walls, None, h=sc.h, rho0=sc.rho0, mass_iters=5)
    fluid = sc.st.download()
    (px, py, pz, pm), nb = bd.arrays()
    bdy = {"x": rb.device_to_numpy(px, nb), "y": rb.device_to_numpy(py, nb),
           "z": rb.device_to_numpy(pz, nb), "m": rb.device_to_numpy(pm, nb)}
    grav = (0.0, -9.81, 0.0)
    t0 = time.perf_counter()
    want = fp64.iisph_run(rb.C2, fluid, bdy, sc.box_min, sc.box_max, sc.h, sc.rho0, NU, grav,
                          PREC_DT, PREC_STEPS, PREC_SWEEPS, 0.5, True, device="cuda")
    t_fp64 = time.perf_counter() - t0
    out = {"what": "error against the FP64 restatement (checker) on the benchmark scene, "
                   f"{PREC_STEPS} steps of {PREC_SWEEPS} Jacobi sweeps at dt {PREC_DT} from "
                   "rest; per field max |err| / max |field|, and mean |rho - rho_FP64| / rho0",
           "particles": sc.n, "fp64_seconds": round(t_fp64, 1)}
    dev = torch.device("cuda")
    ids0 = torch.arange(sc.n, dtype=torch.float32, device=dev)
    for name in names:
        sc.st.upload(fluid)
        ids = ids0.clone()
        prm = rb.reference_params(rb.IISPH, rb.C2, sc.h, sc.rho0, NU)
        prm.min_iter = prm.max_iter = PREC_SWEEPS
        prm.eta = 1.0  # met after every sweep: exactly PREC_SWEEPS sweeps
        prm.precision = {"mixed": rb.PRECISION_MIXED, "mixed_pos16": rb.PRECISION_MIXED_POS16,
                         "fp32": rb.PRECISION_FP32}[name]
        sv = rb.Solver(rb.IISPH, prm, sc.n)
        grid = rb.Grid(sc.box_min, sc.box_max, 2 * sc.h)
        for _ in range(PREC_STEPS):
            grid.construct_and_reorder(sc.st, [ids], stream=S)
            sv.step(sc.st, grid, bd, PREC_DT, stream=S, bounds=(sc.box_min, sc.box_max))
        torch.cuda.synchronize()
        got = sc.st.download()
        buf = sv.buffers()
        for k in ("rho", "p", "aii", "sii"):
            got[k] = rb.device_to_numpy(getattr(buf, k), sc.n)
        order = np.argsort(ids.cpu().numpy().astype(np.int64))
        err = {}
        for k in PREC_FIELDS:
            g = np.asarray(got[k], np.float64)[order]
            w = np.asarray(want[k], np.float64)
            err[k] = float(f"{np.abs(g - w).max() / max(np.abs(w).max(), 1e-30):.3g}")
        drho = np.abs(np.asarray(got["rho"], np.float64)[order] - want["rho"])
        err["mean_abs_rho_rel"] = float(f"{np.mean(drho) / sc.rho0:.3g}")
        out[name] = err
        sv.close()
        grid.close()
    bd.close()
    sc.st.close()
    return out


def reference_constants_leg(a, rank, dev, stream, names):
    """The engine on the steps the reference arm's "reference_cuda" leg times:
    the scene at rest, REF_CUDA_STEPS main-loop steps at the fixed dt
    REF_CUDA_DT with the reference's hard-coded IISPH constants
    (reyn_params_reference: any particle above 0.5 % error, min 3 sweeps,
    omega 0.5, warm start), after one untimed run of the same steps; FP32
    and each mixed mode."""
    import torch

    import reyn_b200 as rb

    S = stream.cuda_stream
    out = {"what": "the engine on the steps of the reference arm's reference_cuda leg "
                   "(reference constants, fixed dt, from rest)",
           "steps": REF_CUDA_STEPS, "dt": REF_CUDA_DT}
    for name in names:
        sc = DeviceScene(rank, a.scale)
        bd = rb.Boundary(*sc.walls, None, h=sc.h, rho0=sc.rho0, mass_iters=5)
        grid = rb.Grid(sc.box_min, sc.box_max, 2 * sc.h)
        prm = rb.reference_params(rb.IISPH, rb.C2, sc.h, sc.rho0, NU)
        prm.precision = {"mixed": rb.PRECISION_MIXED, "mixed_pos16": rb.PRECISION_MIXED_POS16,
                         "fp32": rb.PRECISION_FP32}[name]
        sv = rb.Solver(rb.IISPH, prm, sc.n)
        init = sc.st.download()

        def steps():
            it = []
            for _ in range(REF_CUDA_STEPS):
                grid.construct_and_reorder(sc.st, stream=S)
                it.append(sv.step(sc.st, grid, bd, REF_CUDA_DT, stream=S,
                                  bounds=(sc.box_min, sc.box_max)))
            return it

        steps()
        sc.st.upload(init)
        sv.set_pressure(sc.st, np.zeros(sc.n, np.float32))
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        it = steps()
        e1.record(stream)
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / REF_CUDA_STEPS
        out[name] = {"ms_per_step": round(t, 3), "value": round(sc.n / (t / 1e3), 1),
                     "unit": UNIT, "iters_per_step": it}
        for o in (sv, grid, bd, sc.st):
            o.close()
    return out


def run_engine(a, world, rank, local):
    import torch

    import reyn_b200 as rb

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)
    S = stream.cuda_stream

    names = ["fp32", "mixed", "mixed_pos16"] if a.precision == "all" else [a.precision]
    # the autotuner (block size of the neighbour passes, cell size) for every
    # precision, from the scene's initial state
    config = {name: (0.5, 0, None, 1) for name in names}
    if not a.no_autotune:
        sc = DeviceScene(rank, a.scale)
        bd = rb.Boundary(*sc.walls, None, h=sc.h, rho0=sc.rho0, mass_iters=5)
        for name in names:
            prm = EngineRun.params(rb, sc, name)
            best, pts = rb.autotune(rb.IISPH, prm, sc.st, bd, viscous_dt_limit(sc.h, NU),
                                    steps=3, bounds=(sc.box_min, sc.box_max), stream=S)
            # then the reorder interval at that block size and cell ratio
            prm.block_size = best.block_size
            every = (1, 2, 5, 10)
            k_best, k_ms = rb.autotune_reorder(rb.IISPH, prm, sc.st, bd,
                                               viscous_dt_limit(sc.h, NU),
                                               (sc.box_min, sc.box_max), best.cell_ratio,
                                               every, steps=10, stream=S)
            config[name] = (best.cell_ratio, best.block_size,
                            [{"block_size": p.block_size, "cell_ratio": p.cell_ratio,
                              "ms_per_step": round(p.ms_per_step, 3)} for p in pts]
                            + [{"reorder_every": e, "ms_per_step": round(m, 3)}
                               for e, m in zip(every, k_ms)], k_best)
        bd.close()
        sc.st.close()
        torch.cuda.synchronize()

    # every precision on the same scene; the fastest is the headline (the
    # others are reported beside it), then timed end to end
    results = {}
    for name in names:
        ratio, block, _, every = config[name]
        run = EngineRun(rank, a.scale, dev, name, a.order, ratio, block, every)
        results[name] = (run, timed_steps(run, a, world, stream, dev))
    headline = min(names, key=lambda k: results[k][1][2])  # ms_max: the same on every rank
    legs = {}
    for name in names:
        if name == headline:
            continue
        r, (_, _, msl, _, clk, logl) = results[name]
        legs[name] = leg_summary(r, a, world, msl, logl)
        legs[name]["clocks"] = clk
        legs[name]["cell_ratio"], legs[name]["block_size"] = config[name][0], config[name][1]
        legs[name]["reorder_every"] = config[name][3]
        r.close()
    torch.cuda.synchronize()
    run, (ck, ms, ms_max, prof, ck_clocks, log) = results[headline]
    n = run.n
    value = world * n * a.steps / (ms_max / 1e3)

    # dominant kernel and its roofline (CUDA events around its launches)
    launches = sum(v[0] for v in prof.values())
    dom_name, (dom_launches, dom_ms) = max(prof.items(), key=lambda kv: kv[1][1])
    per_launch_s = dom_ms / 1e3 / max(dom_launches, 1)
    alg = ALG_BYTES.get(dom_name, 0) * n + (16 * run.sc.nb if dom_name == "k_density" else 0)
    peak, peak_kind = peaks()
    achieved = alg / per_launch_s / 1e9 if per_launch_s > 0 else 0.0
    roofline = {"bound": "hbm", "kernel": dom_name, "achieved": round(achieved, 1),
                "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
                "traffic": profile_traffic(dom_name, headline), "peak_source": peak_kind,
                # what bounds these passes instead (ncu, committed summary):
                # instruction issue, and the L1 that serves their gathers
                "issue_active_pct": profile_field(dom_name, headline, "issue_active_pct"),
                "l1tex_throughput_pct": profile_field(dom_name, headline,
                                                      "l1tex_throughput_pct"),
                "dram_traffic_over_alg": (round(profile_traffic(dom_name, headline) / alg, 2)
                                          if alg and profile_traffic(dom_name, headline)
                                          else None),
                "alg_bytes_per_launch": alg, "ms_per_launch": round(per_launch_s * 1e3, 4),
                "share_of_step": round(dom_ms / ms, 4)}
    kernels = {k: {"launches": v[0], "ms": round(v[1], 3)} for k, v in
               sorted(prof.items(), key=lambda kv: -kv[1][1])}

    # e2e: the same K steps again from the checkpoint, through the C ABI
    # with the state uploaded from / downloaded to pinned host memory
    e2e = None
    if not a.no_e2e:
        run.restore(ck)
        host = {k: torch.empty(n, dtype=torch.float32, pin_memory=True).numpy()
                for k in ("x", "y", "z", "vx", "vy", "vz", "m")}
        for k in host:
            host[k][:] = ck[0][k]
        L = rb.lib()
        hp = [host[k].ctypes.data for k in ("x", "y", "z", "vx", "vy", "vz", "m")]
        run.log.clear()
        # the copies run field by field on two copy streams: the upload of
        # a field for step k + 1 waits only for that field's download of step
        # k, so the two directions of the link overlap, and the grid is built
        # as soon as the positions are in
        up, down = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
        su, sd = up.cuda_stream, down.cuda_stream
        ev_down = [torch.cuda.Event() for _ in range(6)]
        ev_up, ev_step, ev_xyz = torch.cuda.Event(), torch.cuda.Event(), torch.cuda.Event()

        def one(f):
            ptrs = [None] * 7
            ptrs[f] = hp[f]
            return ptrs

        barrier(world)
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        up.wait_stream(stream)
        for k in range(a.steps):
            if k:
                up.wait_event(ev_step)  # the state's arrays are free again
            for f in (0, 1, 2, 6, 3, 4, 5):  # positions first, then the masses
                if k and f < 6:
                    up.wait_event(ev_down[f])
                rb.check(L.reyn_particles_upload(run.st.h, *one(f), su))
                if f == 2:
                    ev_xyz.record(up)
            ev_up.record(up)
            run.step(S, ready=(lambda: stream.wait_event(ev_xyz),
                               lambda: stream.wait_event(ev_up)))
            ev_step.record(stream)
            down.wait_event(ev_step)
            for f in range(6):
                rb.check(L.reyn_particles_download_async(run.st.h, *one(f), sd))
                ev_down[f].record(down)
        stream.wait_stream(down)
        t1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        ems = max_over_ranks(world, t0.elapsed_time(t1))
        e2e = {"value": round(world * n * a.steps / (ems / 1e3), 1), "unit": UNIT,
               "h2d_bytes_per_step": 28 * n, "d2h_bytes_per_step": 24 * n,
               "copies": "one field per call, uploads and downloads on two streams",
               "ms_per_step": round(ems / a.steps, 3),
               "iters_per_step": [x[0] for x in run.log]}

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cpu = cpu_baseline_from(ck, run)
    run.close()

    developed = None
    if a.develop_steps > 0:
        developed = developed_leg(a, world, rank, dev, stream, names, config)
    ref_constants = None
    if world == 1 and a.scale == 1:
        ref_constants = reference_constants_leg(a, rank, dev, stream, names)
    precision_error = None
    if rank == 0 and world == 1 and not a.no_precision_check:
        precision_error = precision_vs_fp64(rank, a.scale, names, stream)

    precision = {
        "fp32": "fp32 storage and math",
        "mixed": "mixed: neighbour velocities, densities and pressure accelerations FP16; "
                 "positions, own data and all arithmetic FP32; Kahan density and divergence "
                 "sums; FP64 convergence reduction",
        "mixed_pos16": "mixed_pos16: every neighbour pass reads one 16-byte record per "
                       "neighbour (positions 16-bit fixed point at 1/16384 cell, masses, "
                       "velocities and m a FP16, m p FP32); own data and all arithmetic "
                       "FP32; Kahan density and divergence sums; FP64 convergence "
                       "reduction"}[headline]
    out = {
        "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(ms_max / a.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded lattice + jitter dam break; Akinci box walls)",
        "config": workload_config(n, run.sc.nb, run.sc.h, run.sc.rho0, world),
        "engine": {"precision": precision, "cell_order": a.order,
                   "block_size": config[headline][1] or 128, "cell_ratio": config[headline][0],
                   "reorder_every": config[headline][3]},
        "clocks": ck_clocks, "e2e": e2e, "gpu_launches": launches, "roofline": roofline,
        "cpu_baseline": cpu, "autotune": config[headline][2],
        "iters_per_step": [x[0] for x in log],
        "avg_density_error_per_step": [round(x[1], 7) for x in log],
        "dt_per_step": [float(f"{x[2]:.4e}") for x in log],
        "iter_limit_hits": run.limit_hits, "kernels": kernels,
        "developed": developed, "reference_constants": ref_constants,
        "precision_error": precision_error,
    }
    out["headline_precision"] = headline
    out.update(legs)
    vals = dict({k: v["value"] for k, v in legs.items()}, **{headline: value})
    mixed = [k for k in ("mixed", "mixed_pos16") if k in vals]
    if "fp32" in vals and mixed:
        best = max(mixed, key=lambda k: vals[k])
        out["mixed_over_fp32"] = round(vals[best] / vals["fp32"], 3)
        out["mixed_over_fp32_by_mode"] = {k: round(vals[k] / vals["fp32"], 3) for k in mixed}
    if rank == 0:
        print(json.dumps(out), flush=True)


def oracle_params(h: float, rho0: float):
    import oracle
    op = oracle.reference_params(2, 0, h, rho0, NU)
    op.iisph_avg = 1
    op.eta = 0.001
    op.max_iter = 1000
    return op


def cpu_baseline_from(ck, run):
    """One IISPH step of the oracle (C++/OpenMP, all host threads) from the
    checkpoint the GPU's timed region started from."""
    import oracle
    import reyn_b200 as rb

    state, p, dt_prev, iters = ck[:4]
    sc = run.sc
    fl = {k: v.copy() for k, v in state.items()}
    fl["id"] = np.arange(sc.n, dtype=np.float32)
    (px, py, pz, pm), nb = run.bd.arrays()
    bdy = {"x": rb.device_to_numpy(px, nb), "y": rb.device_to_numpy(py, nb),
           "z": rb.device_to_numpy(pz, nb), "m": rb.device_to_numpy(pm, nb)}
    g = oracle.f32([0.0, -9.81, 0.0])
    t0 = time.perf_counter()
    dt = min(float(oracle.lib().orc_dt_controller(iters, dt_prev, LAMBDA, sc.h, sc.n,
                                                  fl["vx"], fl["vy"], fl["vz"], g, 10, 0.001)),
             viscous_dt_limit(sc.h, NU))
    r = oracle.run(oracle_params(sc.h, sc.rho0), fl, bdy, sc.box_min, sc.box_max, dt, 1, p0=p)
    secs = time.perf_counter() - t0
    return {"value": round(sc.n / secs, 1), "unit": UNIT, "cores": oracle.threads(),
            "kind": "port",
            "sample": f"1 step of the same workload from the state the GPU timing started "
                      f"from ({sc.n} particles, {int(r.iters[0])} Jacobi sweeps) on the "
                      f"C++/OpenMP oracle: {secs:.2f} s"}


# ---- reference arm -------------------------------------------------------------

def run_reference(a, world, rank):
    """The reference's path timed on the host cores. The reference has no CPU
    implementation of its step; its algorithm as restated in the C++/OpenMP
    oracle (every host thread) runs the same scene, parameters and dt rule
    as the engine arm: W warm-up steps, then K timed steps."""
    if rank != 0:
        return
    import oracle

    sc = scene_for(0, a.scale)
    t0 = time.perf_counter()
    bm = oracle.boundary_masses(sc.bdy["x"], sc.bdy["y"], sc.bdy["z"], sc.h, sc.rho0, 5)
    setup = time.perf_counter() - t0
    bdy = dict(sc.bdy, m=bm)
    op = oracle_params(sc.h, sc.rho0)
    fl = {k: v.copy() for k, v in sc.fluid.items()}
    p = np.zeros(sc.n, np.float32)
    dt, iters = DT0, 0
    g = oracle.f32([0.0, -9.81, 0.0])
    dt_visc = viscous_dt_limit(sc.h, NU)
    log = []

    def one():
        nonlocal dt, iters, p, fl
        dt = min(float(oracle.lib().orc_dt_controller(iters, dt, LAMBDA, sc.h, sc.n, fl["vx"],
                                                      fl["vy"], fl["vz"], g, 10, 0.001)),
                 dt_visc)
        r = oracle.run(op, fl, bdy, sc.box_min, sc.box_max, dt, 1, p0=p)
        fl = dict(r.state)
        p = r.p
        iters = int(r.iters[0])
        log.append(iters)

    for _ in range(a.warmup):
        one()
    log.clear()
    t0 = time.perf_counter()
    for _ in range(a.steps):
        one()
    secs = time.perf_counter() - t0
    v = sc.n * a.steps / secs
    out = {"impl": "reference", "metric": METRIC, "value": round(v, 1), "unit": UNIT,
           "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
           "ms_per_step": round(secs / a.steps * 1e3, 3), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
           "config": workload_config(sc.n, int(sc.bdy["x"].size), sc.h, sc.rho0, world),
           "reference_run": {"threads": oracle.threads(), "setup_s": round(setup, 1),
                             "iters_per_step": log},
           "cpu_baseline": {"value": round(v, 1), "unit": UNIT, "cores": oracle.threads(),
                            "kind": "port",
                            "sample": f"{a.steps} timed steps of the full workload after "
                                      f"{a.warmup} warm-up steps, C++/OpenMP restatement "
                                      f"of the reference's algorithm"},
           "e2e": {"value": round(v, 1), "unit": UNIT, "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    out["reference_cuda"] = reference_cuda_leg(sc, bm)
    print(json.dumps(out), flush=True)


def reference_cuda_leg(sc, bm):
    """The reference's own CUDA step (its src/ compiled unmodified for sm_100a
    into oracle/_ref/ by oracle/ref/Makefile) on the same scene and boundary
    masses: REF_CUDA_STEPS main-loop steps (construct_and_reorder, IISPH step
    with the reference's hard-coded constants, hard bounds) at the fixed dt
    REF_CUDA_DT from rest, device-timed, after one untimed run of the same
    steps (kernel loading, allocation). The engine arm's "reference_constants"
    leg runs the same steps with the same constants."""
    import ctypes

    import oracle
    try:
        L = oracle.ref_cuda()
    except (OSError, FileNotFoundError) as e:
        return {"unavailable": f"reference CUDA library not built: {e}"}
    try:
        import torch
        if not torch.cuda.is_available():
            return {"unavailable": "no GPU"}
    except ImportError:
        return {"unavailable": "no torch"}
    P = lambda x: x.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    F32 = lambda x: np.ascontiguousarray(x, np.float32)  # noqa: E731
    keys = ("x", "y", "z", "vx", "vy", "vz", "m", "id")
    bx, by, bz, bmf = F32(sc.bdy["x"]), F32(sc.bdy["y"]), F32(sc.bdy["z"]), F32(bm)
    lo, hi = F32(sc.box_min), F32(sc.box_max)
    iters = np.zeros(REF_CUDA_STEPS, np.uint32)
    ms = np.zeros(1, np.float32)
    for _ in range(2):  # the second run, from the same state, is the one reported
        st = {k: F32(sc.fluid[k]).copy() for k in keys}
        rc = L.ref_run_timed(2, 0, ctypes.c_uint(sc.n), *(P(st[k]) for k in keys),
                             ctypes.c_uint(int(bx.size)), P(bx), P(by), P(bz), P(bmf), P(lo),
                             P(hi), ctypes.c_float(sc.h), ctypes.c_float(sc.rho0),
                             ctypes.c_float(NU), ctypes.c_float(REF_CUDA_DT),
                             ctypes.c_uint(REF_CUDA_STEPS), P(iters), P(ms))
        if rc:
            return {"unavailable": "reference CUDA run failed: "
                    + L.ref_last_error().decode()}
    t = float(ms[0])
    return {"what": "the reference's own CUDA IISPH main-loop step on this GPU (reference "
                    "constants: any particle above 0.5 % error, min 3 sweeps; fixed dt)",
            "steps": REF_CUDA_STEPS, "dt": REF_CUDA_DT, "ms_per_step": round(t, 3),
            "value": round(sc.n / (t / 1e3), 1), "unit": UNIT,
            "iters_per_step": iters.tolist()}


# ---- batched workload ----------------------------------------------------------

BATCH_DT = 2e-4


def run_batched(a, world, rank, local):
    """256 independent PCISPH dam breaks (cube particle counts log-uniform in
    [2000, 200000], spacing 0.01, cubic B-spline, 1 % density tolerance,
    fixed dt 2e-4) stepped as one batch: one grid, boundary and solver over
    all scenes, one launch per phase. For comparison the same scenes are
    then stepped one after another, each with its own grid, boundary and
    solver (the same engine without batching)."""
    import torch

    import reyn_b200 as rb
    from reyn_b200 import scenes
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)
    S = stream.cuda_stream
    b = scenes.batched_pcisph(n_scenes=a.scenes or 256, seed=4 + rank)
    n = int(b.first[-1])

    def params():
        prm = rb.reference_params(rb.PCISPH, rb.B3, b.h, b.rho0, NU)
        prm.eta = 0.01  # 1 % average density error
        prm.max_iter = 100
        return prm

    st = rb.Particles(n, b.rho0)
    st.upload(b.fluid)
    bd = rb.Boundary(*(torch.tensor(b.bdy[k], device=dev) for k in ("x", "y", "z")), None,
                     h=b.h, rho0=b.rho0, scene_first=b.bfirst)
    tuned, ratio, block = None, 0.5, 0
    if not a.no_autotune:
        best, pts = rb.autotune(rb.PCISPH, params(), st, bd, BATCH_DT, steps=2,
                                scene_first=b.first, scene_min=b.box_min, scene_max=b.box_max,
                                stream=S)
        ratio, block = best.cell_ratio, best.block_size
        tuned = [{"block_size": p.block_size, "cell_ratio": p.cell_ratio,
                  "ms_per_step": round(p.ms_per_step, 3)} for p in pts]
    grid = rb.Grid(b.frame_min, b.frame_max, 2 * b.h, ratio, 0, scene_first=b.first,
                   scene_min=b.box_min, scene_max=b.box_max)
    prm = params()
    prm.block_size = block
    sv = rb.Solver(rb.PCISPH, prm, n)
    its = []

    def step():
        grid.construct_and_reorder(st, stream=S)
        its.append(sv.step_batched(st, grid, bd, BATCH_DT, stream=S))

    for _ in range(a.warmup):
        step()
    its.clear()
    torch.cuda.synchronize()
    start = st.download()  # the graph leg starts from the same state
    gpu_uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    clocks = ClockSampler(gpu_uuid)
    time.sleep(0.3)
    rb.profile_reset()
    rb.profile_enable(True)
    barrier(world)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(a.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    rb.profile_enable(False)
    prof = rb.profile_read()
    ck_clocks = clocks.stop()
    ms = max_over_ranks(world, e0.elapsed_time(e1))
    value = world * n * a.steps / (ms / 1e3)
    it = np.array(its)

    # the same steps from the same state as CUDA-graph replays: one launch per
    # step, the pressure loop in a device-side while node, no host round trip
    st.upload(start)
    torch.cuda.synchronize()
    graph = rb.StepGraph(sv, st, grid, bd, BATCH_DT, bounds=((0, 0, 0), (0, 0, 0)))
    for _ in range(a.warmup):
        graph.launch(stream=S)
    graph.stats(stream=S)
    st.upload(start)
    torch.cuda.synchronize()
    barrier(world)
    e0.record(stream)
    for _ in range(a.steps):
        graph.launch(stream=S)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    gms = max_over_ranks(world, e0.elapsed_time(e1))
    g_last = graph.stats(stream=S)
    g_step_k, g_sweep_k = graph.info()
    graph_leg = {"value": round(world * n * a.steps / (gms / 1e3), 1), "unit": UNIT,
                 "ms_per_step": round(gms / a.steps, 3),
                 "kernels_per_step": g_step_k, "kernels_per_sweep": g_sweep_k,
                 "last_step_sweeps": g_last.iters,
                 "note": "same scenes, state and dt; graph launches back to back"}
    graph.close()
    for o in (sv, grid, bd, st):
        o.close()

    seq = None
    if not a.no_sequential:
        # the same scenes, each with its own grid, boundary and solver,
        # stepped one after another
        runs = []
        for s in range(b.n_scenes):
            lo, hi = int(b.first[s]), int(b.first[s + 1])
            blo, bhi = int(b.bfirst[s]), int(b.bfirst[s + 1])
            pst = rb.Particles(hi - lo, b.rho0)
            pst.upload({k: v[lo:hi] for k, v in b.fluid.items()})
            pbd = rb.Boundary(*(torch.tensor(b.bdy[k][blo:bhi], device=dev)
                                for k in ("x", "y", "z")), None, h=b.h, rho0=b.rho0)
            pg = rb.Grid(b.box_min[s], b.box_max[s], 2 * b.h, ratio)
            psv = rb.Solver(rb.PCISPH, prm, hi - lo)
            runs.append((pst, pbd, pg, psv, (b.box_min[s], b.box_max[s])))

        def seq_step():
            for pst, pbd, pg, psv, box in runs:
                pg.construct_and_reorder(pst, stream=S)
                psv.step(pst, pg, pbd, BATCH_DT, stream=S, bounds=box)

        for _ in range(a.warmup):
            seq_step()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(a.steps):
            seq_step()
        e1.record(stream)
        torch.cuda.synchronize()
        sms = max_over_ranks(world, e0.elapsed_time(e1))
        seq = {"value": round(world * n * a.steps / (sms / 1e3), 1), "unit": UNIT,
               "ms_per_step": round(sms / a.steps, 3),
               "launches_per_step": "one set of phase launches per scene"}
        for r in runs:
            for o in r[:4]:
                o.close()

    launches = sum(v[0] for v in prof.values())
    out = {
        "metric": "particle-steps/s, batched PCISPH, 256 scenes", "value": round(value, 1),
        "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": round(ms / a.steps, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded log-uniform cube sizes, lattice + jitter, Akinci box walls)",
        "config": {"workload": "batched_pcisph", "scenes": b.n_scenes, "particles": n,
                   "boundary_particles": int(b.bfirst[-1]), "kernel": "B3", "h": b.h,
                   "tolerance": "1 % average density error", "dt": BATCH_DT,
                   "precision": "fp32 (the mixed modes are IISPH only)",
                   "block_size": block or 128, "cell_ratio": ratio,
                   "parallelism": f"replicas{world}"},
        "autotune": tuned,
        "clocks": ck_clocks, "gpu_launches": launches,
        "iters_per_step_max": it.max(1).tolist(), "iters_per_step_mean":
            [round(float(x), 2) for x in it.mean(1)],
        "kernels": {k: {"launches": v[0], "ms": round(v[1], 3)} for k, v in
                    sorted(prof.items(), key=lambda kv: -kv[1][1])},
        "sequential": seq,
        "graph": graph_leg,
        "graph_over_plain": round(graph_leg["value"] / value, 3),
    }
    if seq:
        out["batched_over_sequential"] = round(value / seq["value"], 3)
    if rank == 0:
        print(json.dumps(out), flush=True)


def run_batched_iisph(a, world, rank, local):
    """Batched IISPH: independent dam breaks (96 cubes of log-uniform particle
    counts in [2000, 200000] at spacing 0.01, about 4M particles, Wendland C2
    masses), 0.1 % average density error, fixed dt 2e-4. The same batch from
    the same start is stepped in FP32, MIXED and MIXED_POS16 (one launch per
    phase for all scenes); the fastest is the headline, and a CUDA-graph leg
    replays its step."""
    import torch

    import reyn_b200 as rb
    from reyn_b200 import scenes
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)
    S = stream.cuda_stream
    ns = a.scenes or 96
    counts = scenes.batch_counts(ns, 2000, 200000, 4 + rank)
    b = scenes.batched_dam_breaks(counts, 0.01, seed=4 + rank, mass_kernel="C2")
    n = int(b.first[-1])
    st = rb.Particles(n, b.rho0)
    st.upload(b.fluid)
    bd = rb.Boundary(*(torch.tensor(b.bdy[k], device=dev) for k in ("x", "y", "z")), None,
                     h=b.h, rho0=b.rho0, scene_first=b.bfirst)
    grid = rb.Grid(b.frame_min, b.frame_max, 2 * b.h, 0.5, 0, scene_first=b.first,
                   scene_min=b.box_min, scene_max=b.box_max)

    def params(precision):
        prm = rb.reference_params(rb.IISPH, rb.C2, b.h, b.rho0, NU)
        prm.convergence = rb.CONV_AVERAGE
        prm.eta = 0.001
        prm.max_iter = 1000
        prm.precision = precision
        return prm

    modes = (("fp32", rb.PRECISION_FP32), ("mixed", rb.PRECISION_MIXED),
             ("mixed_pos16", rb.PRECISION_MIXED_POS16))
    legs = {}
    gpu_uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    for name, prec in modes:
        st.upload(b.fluid)
        sv = rb.Solver(rb.IISPH, params(prec), n)
        its = []

        def step():
            grid.construct_and_reorder(st, stream=S)
            its.append(sv.step_batched(st, grid, bd, BATCH_DT, stream=S))

        for _ in range(a.warmup):
            step()
        its.clear()
        torch.cuda.synchronize()
        clocks = ClockSampler(gpu_uuid)
        time.sleep(0.3)
        rb.profile_reset()
        rb.profile_enable(True)
        barrier(world)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(a.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        rb.profile_enable(False)
        prof = rb.profile_read()
        ck = clocks.stop()
        ms = max_over_ranks(world, e0.elapsed_time(e1))
        it = np.array(its)
        legs[name] = {"value": round(world * n * a.steps / (ms / 1e3), 1), "unit": UNIT,
                      "ms_per_step": round(ms / a.steps, 3), "clocks": ck,
                      "gpu_launches": sum(v[0] for v in prof.values()),
                      "iters_per_step_max": it.max(1).tolist(),
                      "iters_per_step_mean": [round(float(x), 2) for x in it.mean(1)],
                      "kernels": {k: {"launches": v[0], "ms": round(v[1], 3)} for k, v in
                                  sorted(prof.items(), key=lambda kv: -kv[1][1])}}
        sv.close()
    head = max(legs, key=lambda k: legs[k]["value"])
    # the headline mode's step as CUDA-graph replays, from the same start
    st.upload(b.fluid)
    sv = rb.Solver(rb.IISPH, params(dict(modes)[head]), n)
    graph = rb.StepGraph(sv, st, grid, bd, BATCH_DT, bounds=((0, 0, 0), (0, 0, 0)))
    for _ in range(a.warmup):
        graph.launch(stream=S)
    graph.stats(stream=S)
    torch.cuda.synchronize()
    barrier(world)
    e0.record(stream)
    for _ in range(a.steps):
        graph.launch(stream=S)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    gms = max_over_ranks(world, e0.elapsed_time(e1))
    graph.close()
    sv.close()
    for o in (grid, bd, st):
        o.close()
    top = legs[head]
    out = {
        "metric": f"particle-steps/s, batched IISPH, {ns} scenes",
        "value": top["value"], "unit": UNIT, "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": top["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded log-uniform cube sizes, lattice + jitter, Akinci box walls)",
        "config": {"workload": "batched_iisph", "scenes": ns, "particles": n,
                   "boundary_particles": int(b.bfirst[-1]), "kernel": "C2", "h": b.h,
                   "tolerance": "0.1 % average density error", "dt": BATCH_DT,
                   "headline_precision": head, "parallelism": f"replicas{world}"},
        "clocks": top["clocks"], "gpu_launches": top["gpu_launches"],
        "legs": legs,
        "mixed_over_fp32": round(legs["mixed"]["value"] / legs["fp32"]["value"], 3),
        "mixed_pos16_over_fp32": round(legs["mixed_pos16"]["value"] / legs["fp32"]["value"], 3),
        "graph": {"precision": head, "ms_per_step": round(gms / a.steps, 3),
                  "value": round(world * n * a.steps / (gms / 1e3), 1)},
    }
    if rank == 0:
        print(json.dumps(out), flush=True)


# ---- large column collapse ----------------------------------------------------

def run_column(a, world, rank, local):
    """IISPH column collapse onto an obstacle: a 256^3 lattice (16,777,216
    particles, spacing 0.004, seeded jitter +-0.05 h) in a 3 x 1.5 x 1.5 box
    with one layer of wall samples, a sphere of radius 0.2 at the floor's
    centre sampled on the Fibonacci spiral at the same spacing, Wendland C6
    (masses calibrated to its lattice density), viscosity 0.005, 0.1 %
    average density error, dt = min(0.4 CFL controller, 0.08 h^2 / nu),
    MIXED_POS16 unless --precision names another mode, the grid in XYZ order
    (--order zorder for Z-order). The scene is generated on the GPU;
    K timed steps after W warm-up steps (the full run is 1000 steps)."""
    import torch

    import reyn_b200 as rb
    from reyn_b200 import scenes
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)
    S = stream.cuda_stream
    h, rho0, nu = 0.004 * a.scale, 1000.0, 0.005
    e = 256 // a.scale
    box = np.array([3.0, 1.5, 1.5], np.float32)
    st = rb.Particles(e ** 3, rho0)
    o = np.float32(1.5 * h)
    rb.scene_fluid_block(st, (e, e, e), (o, o, o), h, scenes.rest_mass(h, rho0, "W6"), 0.05,
                         0.0, 5 + rank, stream=S)
    wx, wy, wz = rb.scene_box_walls((0, 0, 0), box, h, stream=S)
    center = (1.5, 0.2, 0.75)
    sx, sy, sz = rb.scene_sphere(center, 0.2, h, stream=S)
    bx, by, bz = (torch.cat([u, v]) for u, v in ((wx, sx), (wy, sy), (wz, sz)))
    bd = rb.Boundary(bx, by, bz, None, h=h, rho0=rho0, mass_iters=5)
    kept = rb.scene_cull(st, bd, h) # no fluid inside the walls' first layer
    n = kept
    grid = rb.Grid((0, 0, 0), box, 2 * h, 0.5, rb.ORDER_ZORDER if a.order == "zorder"
                   else rb.ORDER_XYZ)
    prm = rb.reference_params(rb.IISPH, rb.W6, h, rho0, nu)
    prm.convergence = rb.CONV_AVERAGE
    prm.eta = 0.001
    prm.max_iter = 1000
    # default: MIXED_POS16, the fastest mode here too (11.5 ms/step against
    # 13.4 MIXED and 13.3 FP32 on a B200)
    prm.precision = rb.PRECISION_MIXED if a.precision == "mixed" else (
        rb.PRECISION_FP32 if a.precision == "fp32" else rb.PRECISION_MIXED_POS16)
    sv = rb.Solver(rb.IISPH, prm, n)
    dt_visc = viscous_dt_limit(h, nu)
    state = {"dt": DT0, "it": 0, "k": 0}
    log = []

    def step():
        state["dt"] = min(sv.next_dt(st, state["it"], state["dt"], LAMBDA, h, (0.0, -9.81, 0.0),
                                     10, 0.001, stream=S), dt_visc)
        # the state is reordered every `reorder_every` steps; the steps
        # between run on a grid built by construct (Resort::no)
        if state["k"] % a.reorder_every == 0:
            grid.construct_and_reorder(st, stream=S)
        else:
            grid.construct_state(st, stream=S)
        state["k"] += 1
        try:
            state["it"] = sv.step(st, grid, bd, state["dt"], stream=S, bounds=((0, 0, 0), box))
        except rb.ReynError as err:
            if err.code != rb.ERR_ITER_LIMIT:
                raise
            state["it"] = sv.stats().iters
        log.append((state["it"], sv.stats().avg_density_error, state["dt"]))

    for _ in range(a.warmup):
        step()
    log.clear()
    torch.cuda.synchronize()
    gpu_uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    clocks = ClockSampler(gpu_uuid)
    time.sleep(0.3)
    rb.profile_reset()
    rb.profile_enable(True)
    barrier(world)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(a.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    rb.profile_enable(False)
    prof = rb.profile_read()
    ck_clocks = clocks.stop()
    ms = max_over_ranks(world, e0.elapsed_time(e1))
    out = {
        "metric": "particle-steps/s, 16.7M IISPH column collapse onto a sphere",
        "value": round(world * n * a.steps / (ms / 1e3), 1), "unit": UNIT, "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(ms / a.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded lattice + jitter column, Akinci box walls and "
                "Fibonacci sphere, generated on the GPU)",
        "config": {"workload": "column_16m", "particles": n, "boundary_particles": bd.nb,
                   "kernel": "W6", "h": h, "nu": nu,
                   "precision": ("fp32", "mixed", "mixed_pos16")[prm.precision],
                   "cell_order": a.order, "convergence": "avg density error <= 0.1%",
                   "reorder_every": a.reorder_every},
        "clocks": ck_clocks, "gpu_launches": sum(v[0] for v in prof.values()),
        "iters_per_step": [x[0] for x in log],
        "avg_density_error_per_step": [round(x[1], 7) for x in log],
        "dt_per_step": [float(f"{x[2]:.4e}") for x in log],
        "kernels": {k: {"launches": v[0], "ms": round(v[1], 3)} for k, v in
                    sorted(prof.items(), key=lambda kv: -kv[1][1])},
    }
    if rank == 0:
        print(json.dumps(out), flush=True)
    for obj in (sv, grid, bd, st):
        obj.close()


def mesh_traffic(n_queries: int):
    """DRAM bytes of one k_mesh_query launch over n queries, from the
    committed ncu summary (profiles/k_mesh_query_mesh_lbvh.txt, captured at
    2M queries; the traffic grows with the query count)."""
    path = os.path.join(ROOT, "profiles", "k_mesh_query_mesh_lbvh.txt")
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_query:"):
                return float(line.split(":", 1)[1].split()[0]) * n_queries
    except OSError:
        pass
    return None


def mesh_workload(scale: int = 1):
    """A closed 327,680-face mesh: a level-7 icosphere of radius 1 with its
    vertices moved by a seeded uniform +-0.001 (a generic surface: no
    centroid on a Morton cell boundary)."""
    from reyn_b200 import meshes
    v, f = meshes.icosphere(max(7 - (scale - 1), 3), 1.0, (0.0, 0.0, 0.0))
    return meshes.perturb(v, 0.001, 21), f


def run_mesh(a, world, rank, local):
    """LBVH closest-point queries (LBVH::project, lbvh.cuh:726-741) of 16.7M
    seeded uniform points in the mesh's bounding box (+10 %) against a
    327,680-face mesh; the tree build; and sample_mesh (uniform sampling at
    h_bdy = 0.002, 50 relaxation sweeps, Akinci masses). A step re-copies the
    pristine points (3 device copies) and projects them."""
    import torch

    import reyn_b200 as rb
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)
    S = stream.cuda_stream
    v, f = mesh_workload(a.scale)
    torch.cuda.synchronize()
    b0 = time.perf_counter()
    mesh = rb.Mesh(v, f, stream=S)  # synchronises
    build_ms = (time.perf_counter() - b0) * 1e3
    b0 = time.perf_counter()
    rb.Mesh(v, f, stream=S).close()  # warm: the build again, modules loaded
    build_ms = min(build_ms, (time.perf_counter() - b0) * 1e3)
    info = mesh.info()
    n = (1 << 24) // (a.scale ** 3)
    lo = np.array(info.bounds_min) - 0.1
    hi = np.array(info.bounds_max) + 0.1
    g = torch.Generator(device=dev)
    g.manual_seed(1234 + rank)
    pristine = [torch.rand(n, generator=g, device=dev, dtype=torch.float32) * float(hi[k] - lo[k])
                + float(lo[k]) for k in range(3)]
    work = [t.clone() for t in pristine]

    def step():
        for w_, p_ in zip(work, pristine):
            w_.copy_(p_)
        mesh.project(*work, stream=S)

    for _ in range(max(a.warmup, 3)):
        step()
    torch.cuda.synchronize()
    gpu_uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    clocks = ClockSampler(gpu_uuid)
    time.sleep(0.3)
    rb.profile_reset()
    rb.profile_enable(True)
    barrier(world)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(a.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    rb.profile_enable(False)
    prof = rb.profile_read()
    ck_clocks = clocks.stop()
    ms = max_over_ranks(world, e0.elapsed_time(e1))
    k_ms = prof.get("k_mesh_project", (0, 0.0))[1] / max(a.steps, 1)
    peak, peak_kind = peaks()
    algo = 24.0 * n  # 12 B read + 12 B written per query; the tree stays in L2
    roof = {"kernel": "k_mesh_project", "bound": "hbm",
            "achieved": round(algo / (k_ms / 1e3) / 1e9, 1) if k_ms else None,
            "peak": peak, "unit": "GB/s", "peak_kind": peak_kind,
            "frac": round(algo / (k_ms / 1e3) / 1e9 / peak, 4) if k_ms else None,
            "traffic": mesh_traffic(n), "bytes_per_query": 24,
            "note": "a latency-bound stack traversal: ~log2(F) dependent 64-byte node loads "
                    "per query from the L2-resident tree"}
    # end to end through the public call with host buffers: pinned upload,
    # project, download
    e2e = None
    if not a.no_e2e:
        host = [p_.cpu().pin_memory() for p_ in pristine]
        back = [torch.empty_like(h_).pin_memory() for h_ in host]
        torch.cuda.synchronize()
        e2 = torch.cuda.Event(enable_timing=True)
        e3 = torch.cuda.Event(enable_timing=True)
        e2.record(stream)
        for _ in range(a.steps):
            for w_, h_ in zip(work, host):
                w_.copy_(h_, non_blocking=True)
            mesh.project(*work, stream=S)
            for b_, w_ in zip(back, work):
                b_.copy_(w_, non_blocking=True)
        e3.record(stream)
        torch.cuda.synchronize()
        t = max_over_ranks(world, e2.elapsed_time(e3))
        e2e = {"value": round(world * n * a.steps / (t / 1e3), 1), "unit": "queries/s",
               "h2d_bytes_per_step": 12 * n, "d2h_bytes_per_step": 12 * n}
    # sample_mesh: uniform samples, 50 relaxation sweeps, boundary masses
    torch.cuda.synchronize()
    e4 = torch.cuda.Event(enable_timing=True)
    e5 = torch.cuda.Event(enable_timing=True)
    e4.record(stream)
    bdy, (sx, _, _), rstats = rb.sample_mesh(mesh, 0.004 * a.scale, 1000.0, 2.0,
                                             relaxation_iters=50, stream=S)
    e5.record(stream)
    torch.cuda.synchronize()
    sample_ms = e4.elapsed_time(e5)
    n_samples = int(sx.numel())
    cpu = None
    if rank == 0 and not a.no_cpu_baseline:
        import oracle
        m = 2000000 // (a.scale ** 3)
        q = [p_[:m].cpu().numpy() for p_ in pristine]
        t0 = time.perf_counter()
        oracle.lbvh_project(v, f, q[0][:1], q[1][:1], q[2][:1])  # tree build alone
        tb = time.perf_counter() - t0
        t0 = time.perf_counter()
        oracle.lbvh_project(v, f, *q)
        tq = max(time.perf_counter() - t0 - tb, 1e-9)
        cpu = {"value": round(m / tq, 1), "unit": "queries/s", "cores": oracle.threads(),
               "kind": "port",
               "sample": f"{m} of the {n} queries (tree build of {tb:.2f} s excluded)"}
    out = {
        "metric": "LBVH closest-point queries/s, 327,680-face mesh",
        "value": round(world * n * a.steps / (ms / 1e3), 1), "unit": "queries/s",
        "n_gpus": world, "steps": a.steps, "warmup": max(a.warmup, 3),
        "ms_per_step": round(ms / a.steps, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (perturbed level-7 icosphere; seeded uniform query points)",
        "config": {"workload": "mesh_lbvh", "faces": info.n_faces, "queries": n,
                   "tree_height": info.tree_height,
                   "l2": "inputs (192 MB of points) larger than L2"},
        "kernel_ms_per_step": round(k_ms, 3), "build_ms": round(build_ms, 2),
        "sample_mesh": {"samples": n_samples, "ms": round(sample_ms, 2),
                        "relaxation_iters": 50,
                        "ratio_first_last": [round(float(rstats[0, 0]), 4),
                                             round(float(rstats[-1, 0]), 4)]},
        "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "clocks": ck_clocks,
        "gpu_launches": sum(v_[0] for v_ in prof.values()),
        "kernels": {k: {"launches": v_[0], "ms": round(v_[1], 3)} for k, v_ in
                    sorted(prof.items(), key=lambda kv: -kv[1][1])},
    }
    if rank == 0:
        print(json.dumps(out), flush=True)
    bdy.close()
    mesh.close()


def main():
    a = parse_args()
    world, rank, local = dist_setup()
    try:
        if a.impl == "reference":
            run_reference(a, world, rank)
        elif a.workload == "batched_pcisph":
            run_batched(a, world, rank, local)
        elif a.workload == "batched_iisph":
            run_batched_iisph(a, world, rank, local)
        elif a.workload == "column_16m":
            run_column(a, world, rank, local)
        elif a.workload == "mesh_lbvh":
            run_mesh(a, world, rank, local)
        else:
            run_engine(a, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
