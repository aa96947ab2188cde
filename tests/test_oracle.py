"""CPU tests of the oracle itself: it is pinned against the reference's own
kernel classes (host build, bit-exact), the reference's brute-force grid test
and, where present, the golden fixtures the reference's CUDA path produced."""
import numpy as np
import pytest

import oracle
from reyn_b200 import scenes
from tests.helpers import (STEP_TOL, assert_close, by_id, compare_steps, fixture_inputs,
                           fixture_outputs, golden, run_oracle)

KERNELS = [("C2", 0), ("B3", 1), ("W6", 2), ("COS", 3)]


@pytest.mark.parametrize("name,kind", KERNELS)
def test_oracle_kernels_bit_exact_vs_reference_host(name, kind):
    g = golden("kernels_host.npz")
    assert g is not None, "tests/golden/kernels_host.npz missing"
    d = g["d"]
    w, gx, gy, gz = oracle.kernel_eval(kind, float(g["h_bar"]), d[:, 0], d[:, 1], d[:, 2])
    np.testing.assert_array_equal(w.view(np.uint32), g[f"{name}_w"].view(np.uint32))
    np.testing.assert_array_equal(np.stack([gx, gy, gz], 1).view(np.uint32),
                                  g[f"{name}_g"].view(np.uint32))


@pytest.mark.parametrize("name,kind", KERNELS)
def test_oracle_kernels_vs_reference_device(name, kind):
    g = golden("kernels_device.npz")
    if g is None:
        pytest.skip("device fixture not generated yet")
    d = g["d"]
    w, gx, gy, gz = oracle.kernel_eval(kind, float(g["h_bar"]), d[:, 0], d[:, 1], d[:, 2])
    # host (sqrt of the dot) vs device (norm3df, contracted FMAs): a few ulp
    assert_close(w, g[f"{name}_w"], 1e-5, 1e-6, f"{name} W")
    assert_close(np.stack([gx, gy, gz], 1), g[f"{name}_g"], 1e-4, 1e-6, f"{name} dW")


@pytest.mark.parametrize("name,kind", KERNELS)
def test_oracle_kernel_properties(name, kind):
    """The reference's kernel property test (kernels.cu:19-190): W >= 0,
    compact support, dW(0) = 0, gradient antisymmetry on a lattice,
    sum W ~ 1/spacing^3 (0.5%), sum dW ~ 0."""
    h = 25.0
    n = 25
    sp = np.float32(2 * h / n)
    i = np.arange(n, dtype=np.float32)
    gx, gy, gz = np.meshgrid(i, i, i, indexing="ij")
    lat = np.stack([gx.ravel(), gy.ravel(), gz.ravel()], 1) * sp + np.float32(-h + sp / 2)
    w, dx, dy, dz = oracle.kernel_eval(kind, h, lat[:, 0], lat[:, 1], lat[:, 2])
    dw = np.stack([dx, dy, dz], 1)
    assert (w >= 0).all()
    r = np.linalg.norm(lat, axis=1)
    assert np.all(w[r >= h] == 0) or kind == 3
    np.testing.assert_allclose(-dw, dw[::-1], rtol=1e-5, atol=1e-9)
    assert abs(w.sum() * sp ** 3 - 1.0) < 5e-3
    assert np.all(np.abs(dw.sum(0)) < 1e-2 * np.abs(dw).sum(0))
    w0, g0x, g0y, g0z = oracle.kernel_eval(kind, h, [0.0], [0.0], [0.0])
    assert w0[0] > 0 and g0x[0] == 0 and g0y[0] == 0 and g0z[0] == 0


def test_oracle_grid_vs_brute_force():
    """uniformgrid.cu:247-346: neighbour counts equal the O(N^2) oracle."""
    side, h = 16, 1.1
    box = h * side
    rng = np.random.Generator(np.random.PCG64(161))
    x, y, z = (np.float32(box * rng.random(side ** 3)) for _ in range(3))
    g = oracle.geometry([0, 0, 0], [box] * 3, 2 * h)
    prefix, srt, _ = oracle.grid_build(g, x, y, z)
    c, l2, _ = oracle.neighbours(g, x, y, z, prefix, srt)
    cb, lb = oracle.brute_count(x, y, z, 2 * h)
    np.testing.assert_array_equal(c, cb)
    assert_close(l2, lb, 1e-5, 1e-7, "len2")


@pytest.mark.parametrize("ratio", [0.5, 1.0])
def test_oracle_grid_invariants(ratio):
    x, y, z = scenes.uniform_cloud(20000, seed=5)
    g = oracle.geometry([0, 0, 0], [1, 1, 1], 0.05, ratio)
    prefix, srt, keys = oracle.grid_build(g, x, y, z)
    assert prefix[0] == 0 and prefix[-1] == x.size
    assert np.all(np.diff(prefix.astype(np.int64)) >= 0)
    assert np.array_equal(np.sort(srt), np.arange(x.size))
    # keys along the sorted order are non-decreasing; indices ascend in a cell
    k = keys[srt]
    assert np.all(np.diff(k.astype(np.int64)) >= 0)
    same = np.diff(k.astype(np.int64)) == 0
    assert np.all(np.diff(srt.astype(np.int64))[same] > 0)
    c, _, _ = oracle.neighbours(g, x, y, z, prefix, srt)
    cb, _ = oracle.brute_count(x, y, z, 0.05)
    np.testing.assert_array_equal(c, cb)


def _zorder_key_spec(cx, cy, cz, nx, ny):
    """The Z-order key as documented (4^3-cell bricks, x fastest inside;
    bricks along the Morton curve inside 32^3-cell tiles; tiles in XYZ
    order), written independently of the oracle's C++ for a cross-check."""
    tx, ty = -(-nx // 32), -(-ny // 32)
    tile = (cz // 32 * ty + cy // 32) * tx + cx // 32
    bx, by, bz = (cx // 4) % 8, (cy // 4) % 8, (cz // 4) % 8
    brick = 0
    for bit in range(3):
        brick |= ((bx >> bit) & 1) << (3 * bit)
        brick |= ((by >> bit) & 1) << (3 * bit + 1)
        brick |= ((bz >> bit) & 1) << (3 * bit + 2)
    return (tile * 512 + brick) * 64 + cx % 4 + 4 * (cy % 4) + 16 * (cz % 4)


@pytest.mark.parametrize("ratio", [0.5, 1.0])
def test_oracle_zorder_grid(ratio):
    """Z-order: every cell gets its own key, the build sorts by it, and the
    cell-by-cell traversal finds exactly the brute-force neighbours."""
    x, y, z = scenes.uniform_cloud(20000, seed=6)
    g = oracle.geometry([0, 0, 0], [1, 1, 1], 0.05, ratio, order=1)
    assert g.order == 1 and g.n_keys >= g.n_cells
    prefix, srt, keys = oracle.grid_build(g, x, y, z)
    assert prefix.size == g.n_keys + 1 and prefix[-1] == x.size
    cell = np.float32(g.cell)
    c = [np.floor((a - np.float32(lo)) / cell).astype(np.int64)
         for a, lo in zip((x, y, z), g.bmin)]
    np.testing.assert_array_equal(keys, _zorder_key_spec(c[0], c[1], c[2], g.nx, g.ny))
    # a bijection from cells into the key space
    cx, cy, cz = np.meshgrid(np.arange(g.nx), np.arange(g.ny), np.arange(g.nz), indexing="ij")
    allk = _zorder_key_spec(cx.ravel(), cy.ravel(), cz.ravel(), g.nx, g.ny)
    assert np.unique(allk).size == allk.size and allk.max() < g.n_keys
    k = keys[srt]
    assert np.all(np.diff(k.astype(np.int64)) >= 0)
    same = np.diff(k.astype(np.int64)) == 0
    assert np.all(np.diff(srt.astype(np.int64))[same] > 0)
    cnt, _, _ = oracle.neighbours(g, x, y, z, prefix, srt)
    cb, _ = oracle.brute_count(x, y, z, 0.05)
    np.testing.assert_array_equal(cnt, cb)


@pytest.mark.parametrize("name", ["grid_test.npz", "grid_cloud.npz"])
def test_oracle_grid_vs_reference_fixture(name):
    g = golden(name)
    if g is None:
        pytest.skip("device fixture not generated yet")
    geom = oracle.geometry(g["bmin"], g["bmax"], float(g["r"]))
    assert [geom.nx, geom.ny, geom.nz] == list(g["dims"])
    prefix, srt, _ = oracle.grid_build(geom, g["x"], g["y"], g["z"])
    np.testing.assert_array_equal(prefix[:-1], g["prefix"])
    np.testing.assert_array_equal(srt, g["sorted"])
    for k in (0, 1, 2, 3):
        if f"rho_k{k}" not in g:
            continue
        c, l2, rho = oracle.neighbours(geom, g["x"], g["y"], g["z"], prefix, srt, kind=k,
                                       m=np.ones(g["x"].size, np.float32))
        np.testing.assert_array_equal(c, g["count"])
        assert_close(l2, g["len2"], 1e-5, 1e-7, "len2")
        assert_close(rho, g[f"rho_k{k}"], 1e-5, 1e-7, f"rho kernel {k}")


def test_oracle_boundary_masses_plausible():
    sc = scenes.dam_break((4, 4, 4), 0.02, (0.3, 0.3, 0.3))
    m = oracle.boundary_masses(sc.bdy["x"], sc.bdy["y"], sc.bdy["z"], sc.h, sc.rho0, 5)
    assert np.all(m > 0) and np.all(np.isfinite(m))
    # a flat wall sample carries roughly rho0 h^3 / (wall density factor)
    assert 0.05 * sc.rho0 * sc.h ** 3 < np.median(m) < 2 * sc.rho0 * sc.h ** 3


def _solver_fixtures():
    import glob
    import os
    from tests.helpers import GOLDEN
    return sorted(os.path.basename(p) for p in glob.glob(os.path.join(GOLDEN, "solver_*.npz")))


@pytest.mark.parametrize("name", _solver_fixtures() or ["(none)"])
def test_oracle_solver_vs_reference_fixture(name):
    g = golden(name)
    if g is None:
        pytest.skip("solver fixtures not generated yet")
    fluid, bdy = fixture_inputs(g)
    scheme = int(g["scheme"])
    got = run_oracle(scheme, int(g["kind"]), fluid, bdy, g["box_min"], g["box_max"],
                     float(g["h"]), 1000.0, float(g["nu"]), float(g["dt"]), int(g["steps"]))
    want = fixture_outputs(g)
    assert got["iters"] == list(g["iters"]), (got["iters"], list(g["iters"]))
    tol = dict(STEP_TOL)
    if int(g["steps"]) > 1:
        tol = {k: (r * 10, a * 10) for k, (r, a) in STEP_TOL.items()}
    compare_steps(got, want, scheme, tol, name)


def test_oracle_sesph_conserves_ids_and_mass():
    sc = scenes.dam_break((8, 8, 8), 0.02, (0.3, 0.3, 0.3), velocity_noise=0.01)
    bm = oracle.boundary_masses(sc.bdy["x"], sc.bdy["y"], sc.bdy["z"], sc.h, sc.rho0, 5)
    out = run_oracle(0, 1, sc.fluid, dict(sc.bdy, m=bm), sc.box_min, sc.box_max, sc.h,
                     sc.rho0, 0.01, 5e-4, 3)
    assert np.array_equal(np.sort(out["id"]), np.arange(sc.n, dtype=np.float32))
    assert abs(out["m"].sum() - sc.fluid["m"].sum()) < 1e-6 * sc.fluid["m"].sum()
    s = by_id({k: v for k, v in out.items() if k != "iters"}, out["id"])
    assert np.all(np.isfinite(s["x"])) and np.all(s["rho"] > 0)


def test_oracle_cfl():
    v = np.zeros((3, 100), np.float32)
    dt = oracle.cfl(*v, 0.4, 0.01, [0, -9.81, 0])
    assert abs(dt - np.sqrt(2 * 0.4 * 0.01 / 9.81)) < 1e-6
    v[0, 3] = 2.0
    dt = oracle.cfl(*v, 0.4, 0.01, [0, -9.81, 0])
    assert abs(dt - 0.4 * 0.01 / 2.0) < 1e-7
