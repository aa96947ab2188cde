"""GPU parity tests: the CUDA engine through its C ABI against the reference's
own CUDA outputs (golden fixtures) and the CPU oracle on the same inputs."""
import numpy as np
import pytest

import oracle
from reyn_b200 import scenes
from tests.helpers import (STEP_TOL, assert_close, compare_steps, fixture_inputs,
                           fixture_outputs, golden, run_engine, run_oracle)

pytestmark = pytest.mark.gpu

KERNELS = [("C2", 0), ("B3", 1), ("W6", 2), ("COS", 3)]


def T(a, dev="cuda"):
    import torch
    return torch.tensor(np.ascontiguousarray(a, np.float32), device=dev)


@pytest.mark.parametrize("name,kind", KERNELS)
def test_kernel_eval_vs_reference(cuda, name, kind):
    import reyn_b200 as rb
    g = golden("kernels_device.npz") or golden("kernels_host.npz")
    d = g["d"]
    w, gx, gy, gz = rb.kernel_eval(kind, float(g["h_bar"]), T(d[:, 0]), T(d[:, 1]), T(d[:, 2]))
    assert_close(w.cpu().numpy(), g[f"{name}_w"], 1e-5, 1e-6, f"{name} W")
    gg = np.stack([gx.cpu().numpy(), gy.cpu().numpy(), gz.cpu().numpy()], 1)
    assert_close(gg, g[f"{name}_g"], 1e-4, 1e-6, f"{name} dW")


def _engine_grid(x, y, z, bmin, bmax, r, ratio=0.5, kind=None, m=None, order=0):
    import reyn_b200 as rb
    grid = rb.Grid(bmin, bmax, r, ratio, order)
    tx, ty, tz = T(x), T(y), T(z)
    grid.construct(tx, ty, tz)
    info = grid.info()
    C = info.n_keys
    assert info.order == order
    prefix = rb.device_to_numpy(info.prefix, C + 1, np.uint32)
    srt = rb.device_to_numpy(info.sorted, x.size, np.uint32)
    tm = T(m) if m is not None else None
    count, len2, rho = grid.neighbour_stats(tx, ty, tz, tm, kind if kind is not None else 0)
    out = dict(info=info, prefix=prefix, sorted=srt, count=count.cpu().numpy().view(np.uint32),
               len2=len2.cpu().numpy(), rho=None if rho is None else rho.cpu().numpy())
    grid.close()
    return out


@pytest.mark.parametrize("name", ["grid_test.npz", "grid_cloud.npz"])
def test_grid_vs_reference_fixture(cuda, name):
    g = golden(name)
    if g is None:
        pytest.skip("device fixture not generated yet")
    for k in (0, 1, 2, 3):
        if f"rho_k{k}" not in g:
            continue
        e = _engine_grid(g["x"], g["y"], g["z"], g["bmin"], g["bmax"], float(g["r"]), kind=k,
                         m=np.ones(g["x"].size, np.float32))
        assert [e["info"].nx, e["info"].ny, e["info"].nz] == list(g["dims"])
        np.testing.assert_array_equal(e["prefix"][:-1], g["prefix"])   # bit-exact
        assert e["prefix"][-1] == g["x"].size
        np.testing.assert_array_equal(e["sorted"], g["sorted"])         # canonical order
        np.testing.assert_array_equal(e["count"], g["count"])           # exact counts
        assert_close(e["len2"], g["len2"], 1e-5, 1e-7, "len2")
        assert_close(e["rho"], g[f"rho_k{k}"], 1e-6, 1e-7, f"rho kernel {k}")


@pytest.mark.parametrize("ratio,order", [(0.5, 0), (1.0, 0), (0.5, 1), (1.0, 1)])
def test_grid_vs_oracle_microbench_full_size(cuda, ratio, order):
    """The neighbour-search + density microbenchmark at its full size:
    1,048,576 uniform points, r = 0.0196, Wendland C2, m = rho0 0.0098^3, in
    the reference's XYZ cell order and in Z-order: prefix and sorted
    bit-exact against the oracle's build in the same order, neighbour counts
    exact, densities within 1e-6."""
    x, y, z = scenes.uniform_cloud(1 << 20, seed=2)
    r = 0.0196
    m = np.full(x.size, np.float32(1000.0 * 0.0098 ** 3), np.float32)
    e = _engine_grid(x, y, z, [0, 0, 0], [1, 1, 1], r, ratio, kind=0, m=m, order=order)
    geom = oracle.geometry([0, 0, 0], [1, 1, 1], r, ratio, order=order)
    prefix, srt, _ = oracle.grid_build(geom, x, y, z)
    np.testing.assert_array_equal(e["prefix"], prefix)
    np.testing.assert_array_equal(e["sorted"], srt)
    c, l2, rho = oracle.neighbours(geom, x, y, z, prefix, srt, kind=0, m=m)
    np.testing.assert_array_equal(e["count"], c)
    assert_close(e["rho"], rho, 1e-6, 1e-7, "density")
    assert 25 < c.mean() < 40


def test_construct_and_reorder_permutes_state(cuda):
    import reyn_b200 as rb
    sc = scenes.dam_break((10, 9, 8), 0.02, (0.4, 0.4, 0.4), velocity_noise=0.1, seed=11)
    rng = np.random.Generator(np.random.PCG64(3))
    perm = rng.permutation(sc.n)
    fl = {k: v[perm] for k, v in sc.fluid.items()}
    st = rb.Particles(sc.n, 1000.0)
    st.upload(fl)
    ids = T(fl["id"])
    extra2 = T(fl["x"] * 2)
    grid = rb.Grid(sc.box_min, sc.box_max, 2 * sc.h)
    grid.construct_and_reorder(st, [ids, extra2])
    out = st.download()
    geom = oracle.geometry(sc.box_min, sc.box_max, 2 * sc.h)
    _, srt, _ = oracle.grid_build(geom, fl["x"], fl["y"], fl["z"])
    for k in ("x", "y", "z", "vx", "vy", "vz", "m"):
        np.testing.assert_array_equal(out[k], fl[k][srt])
    np.testing.assert_array_equal(ids.cpu().numpy(), fl["id"][srt])
    np.testing.assert_array_equal(extra2.cpu().numpy(), (fl["x"] * 2)[srt])
    assert grid.info().sorted is None  # Resort::yes: no indirection


def _solver_fixtures():
    import glob
    import os
    from tests.helpers import GOLDEN
    return sorted(os.path.basename(p) for p in glob.glob(os.path.join(GOLDEN, "solver_*.npz")))


@pytest.mark.parametrize("name", _solver_fixtures() or ["(none)"])
def test_solver_vs_reference_fixture(cuda, name):
    g = golden(name)
    if g is None:
        pytest.skip("solver fixtures not generated yet")
    fluid, bdy = fixture_inputs(g)
    scheme = int(g["scheme"])
    got = run_engine(scheme, int(g["kind"]), fluid, bdy, g["box_min"], g["box_max"],
                     float(g["h"]), 1000.0, float(g["nu"]), float(g["dt"]), int(g["steps"]))
    assert got["iters"] == list(g["iters"]), (got["iters"], list(g["iters"]))
    tol = dict(STEP_TOL)
    if int(g["steps"]) > 1:
        tol = {k: (r * 10, a * 10) for k, (r, a) in STEP_TOL.items()}
    compare_steps(got, fixture_outputs(g), scheme, tol, name)


@pytest.mark.parametrize("scheme,kind,steps,dt,order", [(0, 1, 5, 5e-4, 0), (1, 1, 2, 1e-3, 0),
                                                        (2, 0, 3, 1e-3, 0), (2, 2, 2, 1e-3, 0),
                                                        (1, 3, 1, 1e-3, 0), (2, 0, 3, 1e-3, 1),
                                                        (1, 1, 2, 1e-3, 1), (0, 1, 5, 5e-4, 1)])
def test_solver_vs_oracle(cuda, scheme, kind, steps, dt, order):
    """Every scheme against the oracle (the reference's XYZ order); with the
    engine's grid in Z-order (order 1) only the summation order differs."""
    sc = scenes.dam_break((20, 18, 16), 0.02, (0.6, 0.6, 0.6), velocity_noise=0.05, seed=5)
    bm = oracle.boundary_masses(sc.bdy["x"], sc.bdy["y"], sc.bdy["z"], sc.h, sc.rho0, 5)
    bdy = dict(sc.bdy, m=bm)
    got = run_engine(scheme, kind, sc.fluid, bdy, sc.box_min, sc.box_max, sc.h, sc.rho0, 0.01,
                     dt, steps, order=order)
    want = run_oracle(scheme, kind, sc.fluid, bdy, sc.box_min, sc.box_max, sc.h, sc.rho0, 0.01,
                      dt, steps)
    assert got["iters"] == want["iters"]
    tol = {k: (r * steps, a * steps) for k, (r, a) in STEP_TOL.items()}
    compare_steps(got, want, scheme, tol, f"scheme{scheme}/kernel{kind}")


def test_sesph_config_small_full_run_aggregates(cuda):
    """SESPH dam break, 32^3 particles, 200 steps at dt 5e-4: the engine and
    the oracle agree on aggregates (chaotic per-particle divergence is
    expected over long runs)."""
    import reyn_b200 as rb
    sc = scenes.sesph_small()
    bm = oracle.boundary_masses(sc.bdy["x"], sc.bdy["y"], sc.bdy["z"], sc.h, sc.rho0, 5)
    bdy = dict(sc.bdy, m=bm)
    prm = rb.reference_params(rb.SESPH, rb.B3, sc.h, sc.rho0, 0.01)
    prm.k_sesph = 1000.0
    got = run_engine(0, 1, sc.fluid, bdy, sc.box_min, sc.box_max, sc.h, sc.rho0, 0.01, 5e-4,
                     200, params=prm)
    oprm = oracle.reference_params(0, 1, sc.h, sc.rho0, 0.01)
    oprm.k_sesph = 1000.0
    want = run_oracle(0, 1, sc.fluid, bdy, sc.box_min, sc.box_max, sc.h, sc.rho0, 0.01, 5e-4,
                      200, params=oprm)
    for k in ("x", "y", "z"):
        assert abs(got[k].mean() - want[k].mean()) < 2e-3
    assert abs(got["rho"].mean() - want["rho"].mean()) < 2e-3 * sc.rho0
    ke_g = float((got["vx"] ** 2 + got["vy"] ** 2 + got["vz"] ** 2).sum())
    ke_w = float((want["vx"] ** 2 + want["vy"] ** 2 + want["vz"] ** 2).sum())
    assert abs(ke_g - ke_w) < 0.05 * ke_w


def test_boundary_masses_vs_oracle(cuda):
    import reyn_b200 as rb
    sc = scenes.dam_break((4, 4, 4), 0.02, (0.3, 0.3, 0.3))
    want = oracle.boundary_masses(sc.bdy["x"], sc.bdy["y"], sc.bdy["z"], sc.h, sc.rho0, 5)
    b = rb.Boundary(T(sc.bdy["x"]), T(sc.bdy["y"]), T(sc.bdy["z"]), None, h=sc.h, rho0=sc.rho0,
                    mass_iters=5)
    (px, py, pz, pm), nb = b.arrays()
    bx = rb.device_to_numpy(px, nb)
    by = rb.device_to_numpy(py, nb)
    bz = rb.device_to_numpy(pz, nb)
    m = rb.device_to_numpy(pm, nb)
    # match samples by position
    key = lambda x, y, z: np.lexsort((z, y, x))  # noqa: E731
    a = key(bx, by, bz)
    w = key(sc.bdy["x"], sc.bdy["y"], sc.bdy["z"])
    assert_close(m[a], want[w], 1e-5, 1e-6, "boundary mass")


def test_cfl_and_bounds_vs_oracle(cuda):
    import reyn_b200 as rb
    sc = scenes.dam_break((6, 6, 6), 0.02, (0.2, 0.2, 0.2), velocity_noise=1.0, seed=9)
    fl = dict(sc.fluid)
    fl["x"] = fl["x"] + np.float32(0.1)  # push some particles through the wall
    st = rb.Particles(sc.n, 1000.0)
    st.upload(fl)
    g = [0.0, -9.81, 0.0]
    dt = rb.cfl_time_step(st, 0.4, sc.h, g)
    want = oracle.cfl(fl["vx"], fl["vy"], fl["vz"], 0.4, sc.h, g)
    assert dt == pytest.approx(want, rel=1e-6)
    dt2 = rb.dt_controller(st, 3, 1e-3, 0.4, sc.h, g, 5, 0.01)
    assert dt2 == pytest.approx(min(want, 1e-3 * 1.01), rel=1e-6)
    rb.enforce_bounds(st, sc.box_min, sc.box_max)
    out = st.download()
    lo, hi = sc.box_min, sc.box_max
    px = np.clip(fl["x"], lo[0], hi[0])
    np.testing.assert_array_equal(out["x"], px)
    touch = ((fl["x"] <= lo[0]) | (fl["y"] <= lo[1]) | (fl["z"] <= lo[2]) |
             (fl["x"] >= hi[0]) | (fl["y"] >= hi[1]) | (fl["z"] >= hi[2]))
    assert touch.any()
    np.testing.assert_array_equal(out["vx"][touch], fl["vx"][touch] * np.float32(-0.1))
    np.testing.assert_array_equal(out["vx"][~touch], fl["vx"][~touch])


# ---- failure surfaces: errors come back as status codes, the GPU context
# stays usable (no trap, no fault) ----------------------------------------

def test_out_of_bounds_particle_is_reported(cuda):
    import reyn_b200 as rb
    x = np.array([0.5, 0.5, 5.0], np.float32)
    y = np.array([0.5, 0.6, 0.5], np.float32)
    grid = rb.Grid([0, 0, 0], [1, 1, 1], 0.1)
    with pytest.raises(rb.ReynError) as e:
        grid.construct(T(x), T(y), T(y))
    assert e.value.code == rb.ERR_OUT_OF_BOUNDS
    # the context is still usable
    grid.construct(T(x[:2]), T(y[:2]), T(y[:2]))


def test_nonfinite_particle_is_reported(cuda):
    import reyn_b200 as rb
    x = np.array([0.5, np.nan], np.float32)
    grid = rb.Grid([0, 0, 0], [1, 1, 1], 0.1)
    with pytest.raises(rb.ReynError) as e:
        grid.construct(T(x), T([0.5, 0.5]), T([0.5, 0.5]))
    assert e.value.code == rb.ERR_NONFINITE


def test_empty_inputs(cuda):
    import reyn_b200 as rb
    grid = rb.Grid([0, 0, 0], [1, 1, 1], 0.1)
    e = np.zeros(0, np.float32)
    grid.construct(T(e), T(e), T(e))
    info = grid.info()
    prefix = rb.device_to_numpy(info.prefix, info.nx * info.ny * info.nz + 1, np.uint32)
    assert not prefix.any()
    st = rb.Particles(0, 1000.0)
    grid.construct_and_reorder(st)
    sv = rb.Solver(rb.IISPH, rb.reference_params(rb.IISPH, rb.C2, 0.01, 1000.0, 0.01), 0)
    assert sv.step(st, grid, None, 1e-3) == 0


def test_step_requires_reordered_grid(cuda):
    import reyn_b200 as rb
    sc = scenes.dam_break((4, 4, 4), 0.02, (0.2, 0.2, 0.2))
    st = rb.Particles(sc.n, 1000.0)
    st.upload(sc.fluid)
    grid = rb.Grid(sc.box_min, sc.box_max, 2 * sc.h)
    grid.construct(T(sc.fluid["x"]), T(sc.fluid["y"]), T(sc.fluid["z"]))
    sv = rb.Solver(rb.SESPH, rb.reference_params(rb.SESPH, rb.B3, sc.h, 1000.0, 0.01), sc.n)
    with pytest.raises(rb.ReynError) as e:
        sv.step(st, grid, None, 1e-4)
    assert e.value.code == rb.ERR_NOT_READY


def test_iteration_limit_is_reported(cuda):
    import reyn_b200 as rb
    sc = scenes.dam_break((8, 8, 8), 0.02, (0.3, 0.3, 0.3))
    st = rb.Particles(sc.n, 1000.0)
    st.upload(sc.fluid)
    grid = rb.Grid(sc.box_min, sc.box_max, 2 * sc.h)
    prm = rb.reference_params(rb.IISPH, rb.C2, sc.h, 1000.0, 0.01)
    prm.eta = 0.0  # unreachable
    prm.max_iter = 4
    sv = rb.Solver(rb.IISPH, prm, sc.n)
    grid.construct_and_reorder(st)
    with pytest.raises(rb.ReynError) as e:
        sv.step(st, grid, None, 1e-3)
    assert e.value.code == rb.ERR_ITER_LIMIT
    assert sv.stats().iters == 4


@pytest.mark.parametrize("scheme,kind", [(0, 1), (1, 1), (2, 0)])
def test_bounded_step_equals_step_then_bounds(cuda, scheme, kind):
    """The step with its tail fused (bounds applied and max |v| reduced in the
    integrating kernel, next dt from that maximum) reproduces the reference's
    main loop of separate passes (dt controller, reorder, step, bounds) bit
    for bit, over steps where particles are clamped by the bounds."""
    import torch

    import reyn_b200 as rb
    sc = scenes.dam_break((16, 14, 12), 0.02, (0.6, 0.6, 0.6), velocity_noise=0.3, seed=21)
    bm = oracle.boundary_masses(sc.bdy["x"], sc.bdy["y"], sc.bdy["z"], sc.h, sc.rho0, 5)
    dev = torch.device("cuda")
    fx = np.asarray(sc.fluid["x"])
    # bounds that cut through the fluid block: its outer layers get clamped
    lo = [float(np.quantile(fx, 0.1)), float(sc.box_min[1]), float(sc.box_min[2])]
    hi = [float(sc.box_max[0]), float(sc.box_max[1]), float(sc.box_max[2])]
    g = (0.0, -9.81, 0.0)
    out = []
    for fused in (False, True):
        st = rb.Particles(sc.n, sc.rho0)
        st.upload(sc.fluid)
        bd = rb.Boundary(*(torch.tensor(sc.bdy[k], device=dev) for k in ("x", "y", "z")),
                         torch.tensor(bm, device=dev), h=sc.h, rho0=sc.rho0)
        grid = rb.Grid(sc.box_min, sc.box_max, 2 * sc.h)
        prm = rb.reference_params(scheme, kind, sc.h, sc.rho0, 0.01)
        if scheme == 0:
            prm.k_sesph = 1000.0
        sv = rb.Solver(scheme, prm, sc.n)
        dt, it, dts = 5e-4, 0, []
        for _ in range(4):
            if fused:
                dt = sv.next_dt(st, it, dt, 0.4, sc.h, g, 10, 0.001)
            else:
                dt = rb.dt_controller(st, it, dt, 0.4, sc.h, g, 10, 0.001)
            dts.append(dt)
            grid.construct_and_reorder(st)
            if fused:
                it = sv.step(st, grid, bd, dt, bounds=(lo, hi))
            else:
                it = sv.step(st, grid, bd, dt)
                rb.enforce_bounds(st, lo, hi)
        torch.cuda.synchronize()
        out.append((st.download(), dts))
        for o in (sv, grid, bd, st):
            o.close()
    (a, dta), (b, dtb) = out
    assert dta == dtb
    clamped = np.sum(a["x"] == np.float32(lo[0]))
    assert clamped > 0
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


@pytest.mark.parametrize("block", [64, 256, 512])
def test_block_size_gives_the_same_step(cuda, block):
    """The neighbour passes at any block size compute the same particles'
    sums in the same order; only the FP64 reductions may add in another
    order (iteration counts must agree)."""
    import reyn_b200 as rb
    sc = scenes.dam_break((20, 18, 16), 0.02, (0.6, 0.6, 0.6), velocity_noise=0.05, seed=5)
    bm = oracle.boundary_masses(sc.bdy["x"], sc.bdy["y"], sc.bdy["z"], sc.h, sc.rho0, 5)
    bdy = dict(sc.bdy, m=bm)
    out = []
    for b in (128, block):
        prm = rb.reference_params(rb.IISPH, rb.C2, sc.h, sc.rho0, 0.01)
        prm.block_size = b
        out.append(run_engine(2, 0, sc.fluid, bdy, sc.box_min, sc.box_max, sc.h, sc.rho0,
                              0.01, 1e-3, 3, params=prm))
    assert out[0]["iters"] == out[1]["iters"]
    compare_steps(out[1], out[0], 2, STEP_TOL, f"block {block}")


def test_autotune_covers_the_grid_and_restores_the_state(cuda):
    import torch

    import reyn_b200 as rb
    sc = scenes.dam_break((24, 20, 16), 0.02, (0.8, 0.6, 0.6), velocity_noise=0.05, seed=8)
    dev = torch.device("cuda")
    st = rb.Particles(sc.n, sc.rho0)
    st.upload(sc.fluid)
    bd = rb.Boundary(*(torch.tensor(sc.bdy[k], device=dev) for k in ("x", "y", "z")), None,
                     h=sc.h, rho0=sc.rho0)
    before = st.download()
    prm = rb.reference_params(rb.PCISPH, rb.B3, sc.h, sc.rho0, 0.01)
    best, pts = rb.autotune(rb.PCISPH, prm, st, bd, 1e-3, steps=2,
                            bounds=(sc.box_min, sc.box_max))
    after = st.download()
    for k in before:
        np.testing.assert_array_equal(before[k], after[k])
    combos = {(p.block_size, p.cell_ratio) for p in pts}
    assert combos == {(b, r) for b in (64, 128, 256, 512) for r in (0.5, 1.0)}
    assert all(p.ms_per_step > 0 for p in pts)
    assert best.ms_per_step == min(p.ms_per_step for p in pts)
    for o in (bd, st):
        o.close()


def test_fp64_diagnostics(cuda):
    import reyn_b200 as rb
    sc = scenes.dam_break((30, 20, 10), 0.02, (0.8, 0.6, 0.6), velocity_noise=0.5, seed=12)
    st = rb.Particles(sc.n, sc.rho0)
    st.upload(sc.fluid)
    d = rb.diagnostics(st)
    m = sc.fluid["m"].astype(np.float64)
    v = np.stack([sc.fluid[k].astype(np.float64) for k in ("vx", "vy", "vz")], 1)
    assert abs(d["mass"] - m.sum()) <= 1e-12 * m.sum()
    np.testing.assert_allclose(d["momentum"], (m[:, None] * v).sum(0), rtol=1e-10, atol=1e-14)
    assert abs(d["kinetic"] - 0.5 * (m * (v * v).sum(1)).sum()) <= 1e-10 * d["kinetic"]
    st.close()


def test_particles_reorder_by_permutation(cuda):
    """Particles::reorder (particles.cu:93-113) by a caller's permutation:
    every attribute gathered; a non-permutation is rejected before the state
    changes."""
    import torch

    import reyn_b200 as rb
    rng = np.random.default_rng(3)
    n = 10_001
    host = {k: rng.random(n, dtype=np.float32) for k in ("x", "y", "z", "vx", "vy", "vz", "m")}
    st = rb.Particles(n, 1000.0)
    st.upload(host)
    perm = rng.permutation(n).astype(np.int32)
    st.reorder(torch.tensor(perm, device="cuda"))
    got = st.download()
    for k in host:
        np.testing.assert_array_equal(got[k], host[k][perm], err_msg=k)
    for bad in (np.concatenate([perm[:-1], [n]]), np.concatenate([perm[:-1], perm[:1]])):
        with pytest.raises(rb.ReynError) as e:
            st.reorder(torch.tensor(bad.astype(np.int32), device="cuda"))
        assert e.value.code == rb.ERR_INVALID
        again = st.download()
        for k in host:
            np.testing.assert_array_equal(again[k], host[k][perm], err_msg=k)
    st.close()


def test_particles_resize(cuda):
    """resize_truncate keeps the first min(old, new) particles; resize_uninit
    keeps none; new particles are zero; a solver for the old count rejects
    the resized state."""
    import reyn_b200 as rb
    rng = np.random.default_rng(4)
    n = 5000
    host = {k: rng.random(n, dtype=np.float32) for k in ("x", "y", "z", "vx", "vy", "vz", "m")}
    st = rb.Particles(n, 1000.0)
    st.upload(host)
    sv = rb.Solver(rb.SESPH, rb.reference_params(rb.SESPH, rb.B3, 0.02, 1000.0, 0.01), n)
    st.resize(3000, keep=True)
    got = st.download()
    for k in host:
        np.testing.assert_array_equal(got[k], host[k][:3000], err_msg=k)
    st.resize(7000, keep=True)
    got = st.download()
    for k in host:
        np.testing.assert_array_equal(got[k][:3000], host[k][:3000], err_msg=k)
        assert not got[k][3000:].any()
    grid = rb.Grid((0, 0, 0), (1, 1, 1), 0.04)
    grid.construct_and_reorder(st)
    with pytest.raises(rb.ReynError) as e:
        sv.step(st, grid, None, 1e-3)
    assert e.value.code == rb.ERR_INVALID
    st.resize(100, keep=False)
    got = st.download()
    assert all(not got[k].any() for k in host) and got["x"].size == 100
    for o in (grid, sv, st):
        o.close()


def test_particles_download_async_per_field(cuda):
    """reyn_particles_download_async: single-field copies on a side stream
    into page-locked memory agree with the synchronous download."""
    import torch

    import reyn_b200 as rb
    rng = np.random.default_rng(5)
    n = 70_001
    keys = ("x", "y", "z", "vx", "vy", "vz", "m")
    host = {k: rng.random(n, dtype=np.float32) for k in keys}
    st = rb.Particles(n, 1000.0)
    st.upload(host)
    side = torch.cuda.Stream()
    out = [torch.empty(n, dtype=torch.float32, pin_memory=True) for _ in keys]
    for f in range(7):
        ptrs = [None] * 7
        ptrs[f] = out[f].data_ptr()
        rb.check(rb.lib().reyn_particles_download_async(st.h, *ptrs, side.cuda_stream))
    side.synchronize()
    for f, k in enumerate(keys):
        np.testing.assert_array_equal(out[f].numpy(), host[k], err_msg=k)
    st.close()
