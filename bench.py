#!/usr/bin/env python
"""Benchmark of the B200 SPH step engine on the IISPH dam break with
4,194,304 fluid particles (256 x 128 x 128 lattice, spacing 0.005, jitter
+-0.05 h, 2 x 1 x 1 box with one layer of Akinci wall particles, Wendland C2,
rest density 1000, viscosity 0.01, relaxed Jacobi omega = 0.5 to 0.1 % average
density error, adaptive dt from the reference's CFL controller with
lambda = 0.4).

A step is one iteration of the reference main loop (main.cu:60-78): dt
controller (CFL max-velocity reduction), uniform-grid build + reorder of the
state, IISPH step, hard bounds. Inputs are resident in HBM for `value`; `e2e`
repeats the step through the C ABI with the state uploaded from and downloaded
to pinned host memory inside the timed region.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]
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
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def scene_for(rank: int, scale: int):
    from reyn_b200 import scenes
    counts = (256 // scale, 128 // scale, 128 // scale)
    return scenes.dam_break(counts, 0.005 * scale, (2.0, 1.0, 1.0), 1000.0, 0.05,
                            seed=3 + rank, name=WORKLOAD, mass_kernel="C2")


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic(kernel: str):
    """DRAM bytes per launch of `kernel` on this workload, from the committed
    ncu summary (profiles/<kernel>_iisph_4m.txt, line 'traffic_bytes_per_launch:')."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_iisph_4m.txt")
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":", 1)[1])
    except OSError:
        pass
    return None


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
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
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
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---- engine arm ---------------------------------------------------------------

def run_engine(a, world, rank, local):
    import torch

    import reyn_b200 as rb

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    sc = scene_for(rank, a.scale)
    n = sc.n
    st = rb.Particles(n, sc.rho0)
    st.upload(sc.fluid)
    bd = rb.Boundary(*(torch.tensor(sc.bdy[k], device=dev) for k in ("x", "y", "z")), None,
                     h=sc.h, rho0=sc.rho0, mass_iters=5)
    grid = rb.Grid(sc.box_min, sc.box_max, 2 * sc.h)
    prm = rb.reference_params(rb.IISPH, rb.C2, sc.h, sc.rho0, 0.01)
    prm.convergence = rb.CONV_AVERAGE
    prm.eta = 0.001
    prm.max_iter = 1000
    sv = rb.Solver(rb.IISPH, prm, n)
    g = (0.0, -9.81, 0.0)
    lam = 0.4
    stream = torch.cuda.current_stream(dev)
    S = stream.cuda_stream
    state = {"dt": 5e-4, "iters": 0, "errs": [], "iters_log": [], "limit": 0}

    def step():
        # main.cu:64-75 with lambda = 0.4: dt controller, grid, solver, bounds
        state["dt"] = rb.dt_controller(st, state["iters"], state["dt"], lam, sc.h, g, 10,
                                       0.001, stream=S)
        grid.construct_and_reorder(st, stream=S)
        try:
            it = sv.step(st, grid, bd, state["dt"], stream=S)
        except rb.ReynError as e:
            if e.code != rb.ERR_ITER_LIMIT:
                raise
            it = sv.stats().iters
            state["limit"] += 1
        state["iters"] = it
        s = sv.stats()
        state["errs"].append(s.avg_density_error)
        state["iters_log"].append(it)
        rb.enforce_bounds(st, sc.box_min, sc.box_max, stream=S)

    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()
    state["errs"].clear()
    state["iters_log"].clear()

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
    ck = clocks.stop()
    ms = e0.elapsed_time(e1)
    ms_max = max_over_ranks(world, ms)
    value = world * n * a.steps / (ms_max / 1e3)
    iters_log = list(state["iters_log"])
    errs = list(state["errs"])
    dt_last = state["dt"]

    # dominant kernel and its roofline (live CUDA-event timing)
    launches = sum(v[0] for v in prof.values())
    dom = max(prof.items(), key=lambda kv: kv[1][1])
    dom_name, (dom_launches, dom_ms) = dom
    per_launch_s = dom_ms / 1e3 / max(dom_launches, 1)
    alg = ALG_BYTES.get(dom_name, 0) * n + (16 * sc.nb if dom_name == "k_density" else 0)
    peak, peak_kind = peaks()
    achieved = alg / per_launch_s / 1e9 if per_launch_s > 0 else 0.0
    traffic = profile_traffic(dom_name)
    roofline = {"bound": "hbm", "kernel": dom_name, "achieved": round(achieved, 1),
                "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
                "traffic": traffic, "peak_source": peak_kind,
                "alg_bytes_per_launch": alg, "ms_per_launch": round(per_launch_s * 1e3, 4),
                "share_of_step": round(dom_ms / ms, 4)}
    kernels = {k: {"launches": v[0], "ms": round(v[1], 3)} for k, v in
               sorted(prof.items(), key=lambda kv: -kv[1][1])}

    # e2e: same steps through the C ABI with the state in pinned host memory
    e2e = None
    if not a.no_e2e:
        host = {k: torch.empty(n, dtype=torch.float32, pin_memory=True).numpy()
                for k in ("x", "y", "z", "vx", "vy", "vz", "m")}
        st_host = st.download()
        for k in host:
            host[k][:] = st_host[k]
        L = rb.lib()
        hp = [host[k].ctypes.data for k in ("x", "y", "z", "vx", "vy", "vz", "m")]

        def e2e_step():
            rb.check(L.reyn_particles_upload(st.h, *hp, S))
            step()
            rb.check(L.reyn_particles_download(st.h, *hp[:6], None, S))

        barrier(world)
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for _ in range(a.steps):
            e2e_step()
        t1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        ems = max_over_ranks(world, t0.elapsed_time(t1))
        e2e = {"value": world * n * a.steps / (ems / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": 28 * n, "d2h_bytes_per_step": 24 * n,
               "ms_per_step": round(ems / a.steps, 3)}

    # CPU baseline: the oracle on one step of the same state (rank 0, N = 1)
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cpu = cpu_baseline_from(st, bd, sc, prm, dt_last)

    out = {
        "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(ms_max / a.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
        "data": "synthetic (seeded lattice + jitter dam break; Akinci box walls)",
        "config": {"workload": WORKLOAD, "particles_per_gpu": n, "boundary_particles": sc.nb,
                   "kernel": "C2", "h": sc.h, "rho0": sc.rho0, "nu": 0.01, "omega": 0.5,
                   "convergence": "avg density error <= 0.1% (FP64 reduction)",
                   "dt": "simple_dt_controller(lambda=0.4, target 10 iters, 0.1%/step) "
                         "from 5e-4",
                   "precision": "fp32", "parallelism": f"replicas{world}",
                   "l2": "inputs larger than L2 (state 4M x 28 B + grid 70 MB per step)"},
        "clocks": ck, "e2e": e2e, "gpu_launches": launches, "roofline": roofline,
        "cpu_baseline": cpu,
        "iters_per_step": iters_log, "avg_density_error_per_step": [round(e, 6) for e in errs],
        "iter_limit_hits": state["limit"], "dt_last": dt_last, "kernels": kernels,
    }
    if rank == 0:
        print(json.dumps(out), flush=True)
    for o in (sv, grid, bd, st):
        o.close()


def cpu_baseline_from(st, bd, sc, prm, dt):
    """One IISPH step of the oracle (C++/OpenMP, all host threads) from the
    engine's current state: the same workload point the GPU was timed on."""
    import oracle
    import reyn_b200 as rb

    fl = st.download()
    fl["id"] = np.arange(sc.n, dtype=np.float32)
    (px, py, pz, pm), nb = bd.arrays()
    bdy = {"x": rb.device_to_numpy(px, nb), "y": rb.device_to_numpy(py, nb),
           "z": rb.device_to_numpy(pz, nb), "m": rb.device_to_numpy(pm, nb)}
    op = oracle.reference_params(2, 0, sc.h, sc.rho0, 0.01)
    op.iisph_avg = 1
    op.eta = 0.001
    op.max_iter = 1000
    t0 = time.perf_counter()
    r = oracle.run(op, fl, bdy, sc.box_min, sc.box_max, dt, 1)
    secs = time.perf_counter() - t0
    return {"value": round(sc.n / secs, 1), "unit": UNIT, "cores": oracle.threads(),
            "kind": "port",
            "sample": f"1 IISPH step of the same 4M state (grid build, reorder, "
                      f"{int(r.iters[0])} Jacobi sweeps) on the C++/OpenMP oracle, {secs:.1f} s"}


# ---- reference arm -------------------------------------------------------------

def run_reference(a, world, rank):
    """The reference's path timed on the host cores. The reference has no CPU
    implementation of its step; its algorithm as restated in the C++/OpenMP
    oracle (every host thread) is timed on the same workload and config."""
    if rank != 0:
        return
    import oracle
    from reyn_b200 import scenes  # noqa: F401

    sc = scene_for(0, a.scale)
    t0 = time.perf_counter()
    bm = oracle.boundary_masses(sc.bdy["x"], sc.bdy["y"], sc.bdy["z"], sc.h, sc.rho0, 5)
    setup = time.perf_counter() - t0
    bdy = dict(sc.bdy, m=bm)
    op = oracle.reference_params(2, 0, sc.h, sc.rho0, 0.01)
    op.iisph_avg = 1
    op.eta = 0.001
    op.max_iter = 1000
    fl = {k: v.copy() for k, v in sc.fluid.items()}
    p = np.zeros(sc.n, np.float32)
    dt = 5e-4
    iters = 0
    g = [0.0, -9.81, 0.0]

    def one():
        nonlocal dt, iters, p
        dt = float(oracle.lib().orc_dt_controller(iters, dt, 0.4, sc.h, sc.n,
                                                  oracle.f32(fl["vx"]), oracle.f32(fl["vy"]),
                                                  oracle.f32(fl["vz"]), oracle.f32(g), 10,
                                                  0.001))
        r = oracle.run(op, fl, bdy, sc.box_min, sc.box_max, dt, 1, p0=p)
        for k in fl:
            fl[k] = r.state[k]
        p = r.p
        iters = int(r.iters[0])

    for _ in range(a.warmup):
        one()
    t0 = time.perf_counter()
    for _ in range(a.steps):
        one()
    secs = time.perf_counter() - t0
    v = sc.n * a.steps / secs
    out = {"impl": "reference", "metric": METRIC, "value": round(v, 1), "unit": UNIT,
           "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
           "ms_per_step": round(secs / a.steps * 1e3, 3), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
           "config": {"workload": WORKLOAD, "particles_per_gpu": sc.n,
                      "parallelism": "host threads", "setup_s": round(setup, 1)},
           "cpu_baseline": {"value": round(v, 1), "unit": UNIT, "cores": oracle.threads(),
                            "kind": "port",
                            "sample": f"{a.steps} timed steps of the full workload after "
                                      f"{a.warmup} warm-up steps, C++/OpenMP restatement"},
           "e2e": {"value": round(v, 1), "unit": UNIT, "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def main():
    a = parse_args()
    world, rank, local = dist_setup()
    try:
        if a.impl == "reference":
            run_reference(a, world, rank)
        else:
            run_engine(a, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
