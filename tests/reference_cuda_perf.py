"""Times the reference's own CUDA path (reyn src/, compiled unmodified for
sm_100a by oracle/ref/Makefile) and the engine on the same B200 and the same
inputs. Test infrastructure: the reference is the baseline being measured
against, not part of the product.

1. The reference's published grid benchmark (uniformgrid.cu:348-423):
   100^3 half-jittered lattice, spacing 1.1, r = 2.2, shuffled; construction
   with reordering of x, y, z + 4 extra arrays, then a B3 neighbour query.
   The engine's query is its neighbour-statistics pass (count, sum |x_ij|^2,
   density), comparable work per pair.
2. IISPH steps with the reference's own constants (any-particle 0.5 %
   criterion, omega 0.5, min 3 iterations, warm start) on the engine's
   benchmark scene at a fixed dt, same boundary masses. Both sides run once
   untimed first (kernel loading, buffer allocation), then the same steps
   from the same initial state are timed.

Usage: python tests/reference_cuda_perf.py [--iisph-steps K] [--out FILE]
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402

P = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
F32 = lambda a: np.ascontiguousarray(a, np.float32)  # noqa: E731


def grid_case(seed_lattice=161, seed_shuffle=1614201312, side=100, h=1.1):
    rng = np.random.Generator(np.random.PCG64(seed_lattice))
    i = np.arange(side, dtype=np.float32)
    X, Y, Z = np.meshgrid(i, i, i, indexing="ij")
    pts = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1) * np.float32(h)
    pts += np.float32(0.5 * h) * rng.random(pts.shape, dtype=np.float32)
    perm = np.random.Generator(np.random.PCG64(seed_shuffle)).permutation(pts.shape[0])
    pts = pts[perm]
    return F32(pts[:, 0]), F32(pts[:, 1]), F32(pts[:, 2]), np.float32(h * side)


def engine_grid(x, y, z, box, r, reps):
    import torch

    import reyn_b200 as rb
    n = x.size
    st = rb.Particles(n, 1.0)
    st.upload({"x": x, "y": y, "z": z, "vx": x, "vy": y, "vz": z, "m": np.ones(n, np.float32)})
    extra = [torch.empty(n, device="cuda") for _ in range(4)]
    grid = rb.Grid([0, 0, 0], [box] * 3, r)
    for _ in range(2):
        grid.construct_and_reorder(st, extra)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        grid.construct_and_reorder(st, extra)
    e1.record()
    torch.cuda.synchronize()
    t_build = e0.elapsed_time(e1) / reps
    soa = st.soa()
    tx = rb.device_tensor(soa.xx, n)
    ty = rb.device_tensor(soa.xy, n)
    tz = rb.device_tensor(soa.xz, n)
    tm = rb.device_tensor(soa.m, n)
    grid.neighbour_stats(tx, ty, tz, tm, rb.B3)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        grid.neighbour_stats(tx, ty, tz, tm, rb.B3)
    e1.record()
    torch.cuda.synchronize()
    t_query = e0.elapsed_time(e1) / reps
    return t_build, t_query


def reference_grid(x, y, z, box, r, reps):
    L = oracle.ref_cuda()
    ms = np.zeros(2, np.float32)
    rc = L.ref_grid_bench(ctypes.c_uint(x.size), P(x), P(y), P(z), P(F32([0, 0, 0])),
                          P(F32([box] * 3)), ctypes.c_float(r), ctypes.c_uint(reps), P(ms))
    if rc:
        raise RuntimeError(L.ref_last_error().decode())
    return float(ms[0]), float(ms[1])


def iisph_compare(steps: int, dt: float, scale: int):
    import torch

    import bench
    import reyn_b200 as rb

    sc = bench.scene_for(0, scale)
    bm = oracle.boundary_masses(sc.bdy["x"], sc.bdy["y"], sc.bdy["z"], sc.h, sc.rho0, 5)
    # reference
    L = oracle.ref_cuda()
    st = {k: F32(sc.fluid[k]).copy() for k in ("x", "y", "z", "vx", "vy", "vz", "m", "id")}
    iters = np.zeros(steps, np.uint32)
    ms = np.zeros(1, np.float32)
    bx, by, bz = F32(sc.bdy["x"]), F32(sc.bdy["y"]), F32(sc.bdy["z"])
    # twice: the first run loads the reference's kernels and allocates its
    # buffers, the second (from the same initial state) is the one timed
    for _ in range(2):
        st = {k: F32(sc.fluid[k]).copy() for k in ("x", "y", "z", "vx", "vy", "vz", "m", "id")}
        rc = L.ref_run_timed(2, 0, ctypes.c_uint(sc.n), *(P(st[k]) for k in
                                                           ("x", "y", "z", "vx", "vy", "vz",
                                                            "m", "id")),
                             ctypes.c_uint(sc.nb), P(bx), P(by), P(bz), P(F32(bm)),
                             P(F32(sc.box_min)), P(F32(sc.box_max)), ctypes.c_float(sc.h),
                             ctypes.c_float(sc.rho0), ctypes.c_float(bench.NU),
                             ctypes.c_float(dt), ctypes.c_uint(steps), P(iters), P(ms))
        if rc:
            raise RuntimeError(L.ref_last_error().decode())
    ref = {"ms_per_step": float(ms[0]), "iters": iters.tolist()}
    # engine, same constants
    dev = torch.device("cuda")
    pst = rb.Particles(sc.n, sc.rho0)
    pst.upload(sc.fluid)
    bd = rb.Boundary(*(torch.tensor(sc.bdy[k], device=dev) for k in ("x", "y", "z")),
                     torch.tensor(bm, device=dev), h=sc.h, rho0=sc.rho0)
    grid = rb.Grid(sc.box_min, sc.box_max, 2 * sc.h)
    sv = rb.Solver(rb.IISPH, rb.reference_params(rb.IISPH, rb.C2, sc.h, sc.rho0, bench.NU), sc.n)
    # one untimed step loads the engine's kernels and allocates its buffers;
    # then the same initial state (and a cold pressure) again
    grid.construct_and_reorder(pst)
    sv.step(pst, grid, bd, dt)
    pst.upload(sc.fluid)
    sv.set_pressure(pst, np.zeros(sc.n, np.float32))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    it = []
    torch.cuda.synchronize()
    e0.record()
    for _ in range(steps):
        grid.construct_and_reorder(pst)
        it.append(sv.step(pst, grid, bd, dt))
        rb.enforce_bounds(pst, sc.box_min, sc.box_max)
    e1.record()
    torch.cuda.synchronize()
    eng = {"ms_per_step": e0.elapsed_time(e1) / steps, "iters": it}
    return {"particles": sc.n, "dt": dt, "steps": steps, "reference_cuda": ref, "engine": eng,
            "speedup": ref["ms_per_step"] / eng["ms_per_step"]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--iisph-steps", type=int, default=5)
    ap.add_argument("--scale", type=int, default=1)
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    res = {}
    x, y, z, box = grid_case()
    r = 2.2
    rb_, rq = reference_grid(x, y, z, float(box), r, a.reps)
    eb, eq = engine_grid(x, y, z, float(box), r, a.reps)
    res["grid_benchmark_1M"] = {
        "reference_cuda_ms": {"construct_and_reorder": rb_, "query": rq},
        "engine_ms": {"construct_and_reorder": eb, "query_stats": eq},
        "published_rtx4060ti_ms": {"construct_and_reorder": 0.2065, "query": 0.6701}}
    print(json.dumps(res), flush=True)
    res["iisph_reference_constants"] = iisph_compare(a.iisph_steps, 2e-4, a.scale)
    print(json.dumps(res), flush=True)
    if a.out:
        with open(a.out, "w") as f:
            json.dump(res, f, indent=1)


if __name__ == "__main__":
    main()
