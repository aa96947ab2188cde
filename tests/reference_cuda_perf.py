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
3. (--mesh) The mesh path on bench.py's mesh_lbvh workload (327,680-face
   perturbed icosphere): the LBVH build, a device copy plus LBVH::project of
   16.7M seeded points, and sample_mesh at h = 0.004 with 50 relaxation
   sweeps. Each side builds once untimed first.

Usage: python tests/reference_cuda_perf.py [--iisph-steps K] [--mesh] [--out FILE]
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


def mesh_compare(reps: int, scale: int = 1) -> dict:
    import torch

    import bench
    import reyn_b200 as rb
    v, f = bench.mesh_workload(scale)
    v = np.ascontiguousarray(v, np.float64)
    f = np.ascontiguousarray(f, np.uint32)
    n = (1 << 24) // scale ** 3
    lo, hi = v.min(0) - 0.1, v.max(0) + 0.1
    rng = np.random.Generator(np.random.PCG64(1234))
    q = (lo + (hi - lo) * rng.random((n, 3))).astype(np.float32)
    qx, qy, qz = (np.ascontiguousarray(q[:, k]) for k in range(3))
    L = oracle.ref_cuda()
    d = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
    L.ref_mesh_bench.argtypes = [ctypes.c_uint, d, d, d, ctypes.c_uint, ctypes.c_void_p,
                                 ctypes.c_uint, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                 ctypes.c_uint, ctypes.c_float, ctypes.c_int, ctypes.c_void_p,
                                 ctypes.c_void_p]
    ms = np.zeros(4, np.float32)
    cnt = np.zeros(1, np.uint32)
    vx, vy, vz = (np.ascontiguousarray(v[:, k]) for k in range(3))
    rc = L.ref_mesh_bench(v.shape[0], vx, vy, vz, f.shape[0], P(f), n, P(qx), P(qy), P(qz), reps,
                          0.004 * scale, 50, P(ms), P(cnt))
    if rc:
        raise RuntimeError(L.ref_last_error().decode())
    # the engine, same inputs
    dev = torch.device("cuda")
    stream = torch.cuda.current_stream()
    S = stream.cuda_stream
    rb.Mesh(v, f, stream=S).close()  # untimed first build
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    torch.cuda.synchronize()
    ev[0].record(stream)
    mesh = rb.Mesh(v, f, stream=S)
    ev[1].record(stream)
    torch.cuda.synchronize()
    e_build = ev[0].elapsed_time(ev[1])
    pristine = [torch.from_numpy(a).to(dev) for a in (qx, qy, qz)]
    work = [t.clone() for t in pristine]

    def once():
        for w_, p_ in zip(work, pristine):
            w_.copy_(p_)
        mesh.project(*work, stream=S)

    once()
    torch.cuda.synchronize()
    ev[0].record(stream)
    for _ in range(reps):
        once()
    ev[1].record(stream)
    torch.cuda.synchronize()
    e_proj = ev[0].elapsed_time(ev[1]) / reps
    e_sample = 1e30
    for _ in range(2):  # best of two, as on the reference side
        torch.cuda.synchronize()
        ev[0].record(stream)
        bdy, (sx, _, _), _ = rb.sample_mesh(mesh, 0.004 * scale, 1000.0, 2.0,
                                            relaxation_iters=50, stream=S)
        ev[1].record(stream)
        torch.cuda.synchronize()
        e_sample = min(e_sample, ev[0].elapsed_time(ev[1]))
        bdy.close()
    out = {"faces": int(f.shape[0]), "queries": n,
           "reference_cuda_ms": {"build": float(ms[0]), "upload_and_build": float(ms[3]),
                                 "copy_and_project": float(ms[1]),
                                 "sample_mesh_50_sweeps": float(ms[2]),
                                 "samples": int(cnt[0])},
           "engine_ms": {"upload_and_build": e_build, "copy_and_project": e_proj,
                         "sample_mesh_50_sweeps": e_sample, "samples": int(sx.numel())}}
    mesh.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--iisph-steps", type=int, default=5)
    ap.add_argument("--scale", type=int, default=1)
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--out", default=None)
    ap.add_argument("--mesh", action="store_true", help="only the mesh comparison")
    a = ap.parse_args()
    res = {}
    if a.mesh:
        res["mesh_lbvh"] = mesh_compare(max(a.reps // 4, 2), a.scale)
        print(json.dumps(res), flush=True)
        if a.out:
            with open(a.out, "w") as f:
                json.dump(res, f, indent=1)
        return
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
