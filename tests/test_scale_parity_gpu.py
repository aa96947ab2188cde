"""Parity with the oracle on the benchmark workloads themselves, by particle
ID: the 4,194,304-particle IISPH dam break of bench.py (2 main-loop steps in
FP32 and in the mixed_pos16 headline mode), one in eight scenes of the
256-scene batched PCISPH workload stepped as a batch, and captured (CUDA
graph) IISPH and PCISPH steps. The oracle is the C++/OpenMP restatement of
the reference's step (oracle/oracle.cpp)."""
import numpy as np
import pytest

import oracle
from reyn_b200 import scenes
from tests.helpers import STEP_TOL, compare_steps, run_engine, run_oracle

pytestmark = pytest.mark.gpu

# aggregate bounds of the developed collapse, about 5x the MIXED_POS16
# differences measured on a B200 (FP32: 3e-6 m, 5e-5 rho0, 4e-6, 0 sweeps;
# MIXED_POS16: 1.1e-5 m, 3.2e-4 rho0, 7.5e-4, 0 sweeps of 1,203)
DEV_COM_TOL = 5e-5  # metres, per axis
DEV_RHO_TOL = 1.5e-3  # of rho0, mean density
DEV_KE_TOL = 4e-3  # relative, kinetic energy
DEV_ITER_TOL = 0.02  # relative, total sweeps


def _bench_params(rb, sc, precision):
    import bench
    prm = bench.EngineRun.params(rb, sc, precision)
    return prm


@pytest.mark.parametrize("precision,scale", [("fp32", 1), ("mixed_pos16", 20)])
def test_iisph_4m_steps_vs_oracle(cuda, precision, scale):
    """The benchmark scene (host generator, bit-identical to the device one),
    2 steps at dt 2e-4 with the benchmark's solver settings (average density
    error <= 0.1 %, FP64 reduction). FP32 at the step tolerances; the mixed
    mode at `scale` times them (its FP16 records); equal sweep counts."""
    import bench
    import reyn_b200 as rb

    sc = bench.scene_for(0, 1)
    bm = oracle.boundary_masses(sc.bdy["x"], sc.bdy["y"], sc.bdy["z"], sc.h, sc.rho0, 5)
    bdy = dict(sc.bdy, m=bm)
    steps, dt = 2, 2e-4
    prm = _bench_params(rb, sc, precision)
    got = run_engine(2, rb.C2, sc.fluid, bdy, sc.box_min, sc.box_max, sc.h, sc.rho0, bench.NU,
                     dt, steps, params=prm)
    want = run_oracle(2, 0, sc.fluid, bdy, sc.box_min, sc.box_max, sc.h, sc.rho0, bench.NU, dt,
                      steps, params=bench.oracle_params(sc.h, sc.rho0))
    assert got["iters"] == want["iters"]
    tol = {k: (r * steps * scale, a * steps * scale) for k, (r, a) in STEP_TOL.items()}
    compare_steps(got, want, 2, tol, f"iisph_4m/{precision}")


def test_batched_pcisph_workload_scenes_vs_oracle(cuda):
    """The batched PCISPH workload (256 cubes of log-uniform 2,000-200,000
    particles, cubic B-spline, 1 % average density tolerance, dt 2e-4)
    stepped as one batch for 3 steps; every eighth scene against the oracle
    stepped alone in its own box, with equal sweep counts."""
    import torch

    import reyn_b200 as rb

    b = scenes.batched_pcisph(n_scenes=256, seed=4)
    n = int(b.first[-1])
    steps, dt = 3, 2e-4

    def params():
        prm = rb.reference_params(rb.PCISPH, rb.B3, b.h, b.rho0, 0.01)
        prm.eta = 0.01
        prm.max_iter = 100
        return prm

    dev = torch.device("cuda")
    st = rb.Particles(n, b.rho0)
    st.upload(b.fluid)
    ids = torch.tensor(b.fluid["id"], device=dev)
    bd = rb.Boundary(*(torch.tensor(b.bdy[k], device=dev) for k in ("x", "y", "z")), None,
                     h=b.h, rho0=b.rho0, scene_first=b.bfirst)
    grid = rb.Grid(b.frame_min, b.frame_max, 2 * b.h, 0.5, 0, scene_first=b.first,
                   scene_min=b.box_min, scene_max=b.box_max)
    sv = rb.Solver(rb.PCISPH, params(), n)
    its = []
    for _ in range(steps):
        grid.construct_and_reorder(st, [ids])
        its.append(sv.step_batched(st, grid, bd, dt))
    out = st.download()
    out["id"] = ids.cpu().numpy()
    buf = sv.buffers()
    for k in ("rho", "p", "aii", "sii", "ax", "ay", "az"):
        out[k] = rb.device_to_numpy(getattr(buf, k), n)
    for o in (sv, grid, bd, st):
        o.close()
    its = np.array(its)
    ids_all = out["id"].astype(np.int64)
    tol = {k: (r * steps * 10, a * steps * 10) for k, (r, a) in STEP_TOL.items()}
    oprm = oracle.reference_params(1, 1, b.h, b.rho0, 0.01)
    oprm.eta = 0.01
    oprm.max_iter = 100
    for s in range(0, 256, 8):
        a0, a1 = int(b.first[s]), int(b.first[s + 1])
        c0, c1 = int(b.bfirst[s]), int(b.bfirst[s + 1])
        fl = {k: v[a0:a1] for k, v in b.fluid.items()}
        wall = {k: b.bdy[k][c0:c1] for k in ("x", "y", "z")}
        wall["m"] = oracle.boundary_masses(wall["x"], wall["y"], wall["z"], b.h, b.rho0, 5)
        want = run_oracle(1, 1, fl, wall, b.box_min[s], b.box_max[s], b.h, b.rho0, 0.01, dt,
                          steps, params=oprm)
        sel = (ids_all >= int(fl["id"].min())) & (ids_all <= int(fl["id"].max()))
        got = {k: v[sel] for k, v in out.items()}
        assert sel.sum() == a1 - a0
        assert list(its[:, s]) == list(want["iters"]), (s, its[:, s], want["iters"])
        compare_steps(got, want, 1, tol, f"batched_pcisph scene {s}")


@pytest.mark.parametrize("scheme,kind,precision", [("IISPH", "C2", "FP32"),
                                                   ("IISPH", "C2", "MIXED_POS16"),
                                                   ("PCISPH", "B3", "FP32")])
def test_captured_steps_vs_oracle(cuda, scheme, kind, precision):
    """Steps replayed from a captured step graph (grid build + reorder +
    bounded solver step at a fixed dt, the pressure loop decided on the
    device) against the oracle; particles are matched by position (the
    graph carries no ID array), which the step tolerances leave unambiguous
    at this spacing."""
    import torch
    from scipy.spatial import cKDTree

    import reyn_b200 as rb

    sch, knd = getattr(rb, scheme), getattr(rb, kind)
    sc = scenes.dam_break((16, 14, 12), 0.02, (0.5, 0.5, 0.5), velocity_noise=0.05, seed=8)
    bm = oracle.boundary_masses(sc.bdy["x"], sc.bdy["y"], sc.bdy["z"], sc.h, sc.rho0, 5)
    bdy = dict(sc.bdy, m=bm)
    steps, dt = 3, 1e-3
    st = rb.Particles(sc.n, sc.rho0)
    st.upload(sc.fluid)
    bd = rb.Boundary(*(torch.tensor(sc.bdy[k], device="cuda") for k in ("x", "y", "z")),
                     torch.tensor(bm, device="cuda"), h=sc.h, rho0=sc.rho0)
    grid = rb.Grid(sc.box_min, sc.box_max, 2 * sc.h)
    prm = rb.reference_params(sch, knd, sc.h, sc.rho0, 0.01)
    prm.precision = getattr(rb, "PRECISION_" + precision)
    sv = rb.Solver(sch, prm, sc.n)
    g = rb.StepGraph(sv, st, grid, bd, dt, bounds=(sc.box_min, sc.box_max))
    iters = []
    for _ in range(steps):
        g.launch()
        iters.append(g.stats().iters)
    got = st.download()
    g.close()
    for o in (sv, grid, bd, st):
        o.close()
    want = run_oracle(sch, 0 if kind == "C2" else 1, sc.fluid, bdy, sc.box_min, sc.box_max,
                      sc.h, sc.rho0, 0.01, dt, steps)
    assert iters == [int(x) for x in want["iters"]]
    gp = np.stack([got[k] for k in ("x", "y", "z")], 1).astype(np.float64)
    wp = np.stack([want[k] for k in ("x", "y", "z")], 1).astype(np.float64)
    d, idx = cKDTree(wp).query(gp)
    assert d.max() < 1e-3 * sc.h
    assert np.unique(idx).size == sc.n
    scale = 20 if precision != "FP32" else 1
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        rtol, af = STEP_TOL[k]
        w = np.asarray(want[k])[idx]
        err = np.abs(got[k] - w)
        lim = steps * scale * (af * np.abs(w).max() + rtol * np.abs(w))
        assert np.all(err <= lim), (k, float(err.max()))


def test_sesph_config_gravity_z_vs_oracle(cuda):
    """The SESPH dam break as its configuration states it: 32^3 particles at
    spacing 0.02, cubic B-spline, stiffness 1000, viscosity 0.01, gravity
    -9.81 along z, dt 5e-4. Five steps by particle ID at the step
    tolerances, then 200 steps in aggregate (per-particle paths diverge
    chaotically over long runs): centre of mass, mean density, kinetic
    energy."""
    import reyn_b200 as rb

    sc = scenes.sesph_small()
    bm = oracle.boundary_masses(sc.bdy["x"], sc.bdy["y"], sc.bdy["z"], sc.h, sc.rho0, 5)
    bdy = dict(sc.bdy, m=bm)
    prm = rb.reference_params(rb.SESPH, rb.B3, sc.h, sc.rho0, 0.01)
    prm.k_sesph = 1000.0
    prm.g[0], prm.g[1], prm.g[2] = 0.0, 0.0, -9.81
    oprm = oracle.reference_params(0, 1, sc.h, sc.rho0, 0.01)
    oprm.k_sesph = 1000.0
    oprm.g[0], oprm.g[1], oprm.g[2] = 0.0, 0.0, -9.81
    dt = 5e-4
    got = run_engine(0, 1, sc.fluid, bdy, sc.box_min, sc.box_max, sc.h, sc.rho0, 0.01, dt, 5,
                     params=prm)
    want = run_oracle(0, 1, sc.fluid, bdy, sc.box_min, sc.box_max, sc.h, sc.rho0, 0.01, dt, 5,
                      params=oprm)
    tol = {k: (r * 5, a * 5) for k, (r, a) in STEP_TOL.items()}
    compare_steps(got, want, 0, tol, "sesph_32k/gravity_z")
    got = run_engine(0, 1, sc.fluid, bdy, sc.box_min, sc.box_max, sc.h, sc.rho0, 0.01, dt, 200,
                     params=prm)
    want = run_oracle(0, 1, sc.fluid, bdy, sc.box_min, sc.box_max, sc.h, sc.rho0, 0.01, dt,
                      200, params=oprm)
    print({k: (float(got[k].mean()), float(want[k].mean())) for k in ("x", "y", "z", "rho")})
    # the block has fallen along z: its centre moved down by about two spacings
    assert want["z"].mean() < sc.fluid["z"].mean() - 0.02
    for k in ("x", "y", "z"):
        assert abs(got[k].mean() - want[k].mean()) < 2e-4, k
    assert abs(got["rho"].mean() - want["rho"].mean()) < 1e-3 * sc.rho0
    ke_g = float((got["vx"] ** 2 + got["vy"] ** 2 + got["vz"] ** 2).sum())
    ke_w = float((want["vx"] ** 2 + want["vy"] ** 2 + want["vz"] ** 2).sum())
    assert abs(ke_g - ke_w) < 0.02 * ke_w


@pytest.mark.parametrize("precision", ["FP32", "MIXED_POS16"])
def test_developed_collapse_vs_oracle(cuda, precision):
    """A column collapse run until the flow has developed (400 steps of 1 ms:
    the front reaches the far wall, cells hold 0 to several particles) with
    the benchmark's IISPH settings, against the oracle stepped alike.
    Per-particle paths separate over long runs, so the comparison is in
    aggregate: centre of mass, mean density, kinetic energy, and the total
    sweep count."""
    import bench
    import reyn_b200 as rb

    sc = scenes.dam_break((12, 20, 10), 0.02, (0.8, 0.5, 0.24), mass_kernel="C2", gap=1.5,
                          seed=12)
    bm = oracle.boundary_masses(sc.bdy["x"], sc.bdy["y"], sc.bdy["z"], sc.h, sc.rho0, 5)
    bdy = dict(sc.bdy, m=bm)
    steps, dt = 400, 1e-3
    prm = rb.reference_params(rb.IISPH, rb.C2, sc.h, sc.rho0, bench.NU)
    prm.convergence = rb.CONV_AVERAGE
    prm.eta = 0.001
    prm.max_iter = 1000
    prm.precision = getattr(rb, "PRECISION_" + precision)
    got = run_engine(2, rb.C2, sc.fluid, bdy, sc.box_min, sc.box_max, sc.h, sc.rho0, bench.NU,
                     dt, steps, params=prm)
    want = run_oracle(2, 0, sc.fluid, bdy, sc.box_min, sc.box_max, sc.h, sc.rho0, bench.NU, dt,
                      steps, params=bench.oracle_params(sc.h, sc.rho0))
    com = {k: (float(got[k].mean()), float(want[k].mean())) for k in ("x", "y", "z")}
    ke_g = float((got["vx"] ** 2 + got["vy"] ** 2 + got["vz"] ** 2).sum())
    ke_w = float((want["vx"] ** 2 + want["vy"] ** 2 + want["vz"] ** 2).sum())
    it_g, it_w = int(np.sum(got["iters"])), int(np.sum(want["iters"]))
    print(precision, com, float(got["rho"].mean()), float(want["rho"].mean()), ke_g, ke_w,
          it_g, it_w, float(want["x"].max()))
    # the front has crossed the box: the flow is developed
    assert want["x"].max() > 0.6
    for k, (g, w) in com.items():
        assert abs(g - w) < DEV_COM_TOL, (k, g, w)
    assert abs(got["rho"].mean() - want["rho"].mean()) < DEV_RHO_TOL * sc.rho0
    assert abs(ke_g - ke_w) < DEV_KE_TOL * ke_w
    assert abs(it_g - it_w) <= DEV_ITER_TOL * it_w


@pytest.mark.parametrize("precision,scale", [("FP32", 1), ("MIXED", 20)])
def test_column_16m_step_vs_oracle(cuda, precision, scale):
    """The 16,777,216-particle column collapse of bench.py (--workload
    column_16m: 256^3 lattice at 0.004 in a 3 x 1.5 x 1.5 box, box walls and a
    Fibonacci sphere of radius 0.2, fluid culled near the samples, Wendland C6,
    nu 0.005, 0.1 % average density error) generated on the GPU as the
    benchmark does; one step at dt 0.08 h^2 / nu by particle ID against the
    oracle, FP32 at the step tolerances and the benchmark's MIXED mode at
    `scale` times them, equal sweep counts."""
    import torch

    import bench
    import reyn_b200 as rb
    from reyn_b200 import scenes as sc_mod

    h, rho0, nu = 0.004, 1000.0, 0.005
    box = np.array([3.0, 1.5, 1.5], np.float32)
    st = rb.Particles(256 ** 3, rho0)
    o = np.float32(1.5 * h)
    rb.scene_fluid_block(st, (256, 256, 256), (o, o, o), h, sc_mod.rest_mass(h, rho0, "W6"),
                         0.05, 0.0, 5)
    wx, wy, wz = rb.scene_box_walls((0, 0, 0), box, h)
    sx, sy, sz = rb.scene_sphere((1.5, 0.2, 0.75), 0.2, h)
    bx, by, bz = (torch.cat([u, v]) for u, v in ((wx, sx), (wy, sy), (wz, sz)))
    bd = rb.Boundary(bx, by, bz, None, h=h, rho0=rho0, mass_iters=5)
    n = rb.scene_cull(st, bd, h)
    torch.cuda.synchronize()
    fluid = st.download()
    fluid["id"] = np.arange(n, dtype=np.float32)
    (px, py, pz, pm), nb = bd.arrays()
    bdy = {k: rb.device_to_numpy(p, nb) for k, p in zip(("x", "y", "z", "m"), (px, py, pz, pm))}
    for o_ in (bd, st):
        o_.close()
    del bx, by, bz, wx, wy, wz, sx, sy, sz
    dt = bench.viscous_dt_limit(h, nu)
    prm = rb.reference_params(rb.IISPH, rb.W6, h, rho0, nu)
    prm.convergence = rb.CONV_AVERAGE
    prm.eta = 0.001
    prm.max_iter = 1000
    prm.precision = getattr(rb, "PRECISION_" + precision)
    got = run_engine(2, rb.W6, fluid, bdy, (0, 0, 0), box, h, rho0, nu, dt, 1, params=prm)
    oprm = oracle.reference_params(2, 2, h, rho0, nu)
    oprm.iisph_avg = 1
    oprm.eta = 0.001
    oprm.max_iter = 1000
    want = run_oracle(2, 2, fluid, bdy, (0, 0, 0), box, h, rho0, nu, dt, 1, params=oprm)
    assert got["iters"] == [int(x) for x in want["iters"]]
    tol = {k: (r * scale, a * scale) for k, (r, a) in STEP_TOL.items()}
    compare_steps(got, want, 2, tol, f"column_16m/{precision}")
