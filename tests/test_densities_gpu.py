"""reyn_compute_densities (the reference's compute_densities<K, R>,
solver.cuh:19-38): fluid neighbours plus boundary samples, on a grid built by
construct (caller's order) and by construct_and_reorder (grid order), against
the oracle's densities of the same state and the solver's own first pass."""
import ctypes

import numpy as np
import pytest

import oracle
from reyn_b200 import scenes
from tests.helpers import assert_close, by_id, run_oracle

pytestmark = pytest.mark.gpu


def _scene():
    sc = scenes.dam_break((20, 18, 16), 0.02, (0.6, 0.6, 0.6), velocity_noise=0.05, seed=5)
    bm = oracle.boundary_masses(sc.bdy["x"], sc.bdy["y"], sc.bdy["z"], sc.h, sc.rho0, 5)
    return sc, dict(sc.bdy, m=bm)


def _boundary(rb, sc, bdy):
    import torch
    return rb.Boundary(*(torch.tensor(np.asarray(bdy[k], np.float32), device="cuda")
                         for k in ("x", "y", "z", "m")), h=sc.h, rho0=sc.rho0)


@pytest.mark.parametrize("kind", [0, 1, 2, 3])
def test_densities_unsorted_vs_oracle(cuda, kind):
    import torch

    import reyn_b200 as rb
    sc, bdy = _scene()
    # SESPH's rho after one step is the density of the initial state
    want = run_oracle(0, kind, sc.fluid, bdy, sc.box_min, sc.box_max, sc.h, sc.rho0, 0.01,
                      5e-4, 1)
    w = by_id({"rho": want["rho"]}, want["id"])["rho"]
    t = {k: torch.tensor(np.asarray(sc.fluid[k], np.float32), device="cuda")
         for k in ("x", "y", "z", "m")}
    bd = _boundary(rb, sc, bdy)
    grid = rb.Grid(sc.box_min, sc.box_max, 2 * sc.h)
    grid.construct(t["x"], t["y"], t["z"])
    rho = grid.compute_densities(t["x"], t["y"], t["z"], t["m"], bd, kind).cpu().numpy()
    got = by_id({"rho": rho}, np.asarray(sc.fluid["id"]))["rho"]
    assert_close(got, w, 1e-6, 1e-7, f"density kernel {kind}")
    # fluid only: the neighbour-statistics density
    rho_f = grid.compute_densities(t["x"], t["y"], t["z"], t["m"], None, kind)
    _, _, rho_s = grid.neighbour_stats(t["x"], t["y"], t["z"], t["m"], kind)
    np.testing.assert_array_equal(rho_f.cpu().numpy(), rho_s.cpu().numpy())
    assert (rho > rho_f.cpu().numpy()).any()  # the boundary contributes
    grid.close()
    bd.close()


def test_densities_reordered_match_solver_pass(cuda):
    import torch

    import reyn_b200 as rb
    sc, bdy = _scene()
    st = rb.Particles(sc.n, sc.rho0)
    st.upload(sc.fluid)
    bd = _boundary(rb, sc, bdy)
    grid = rb.Grid(sc.box_min, sc.box_max, 2 * sc.h)
    grid.construct_and_reorder(st)
    v = st.soa()
    rho = torch.empty(sc.n, device="cuda", dtype=torch.float32)
    rb.check(rb.lib().reyn_compute_densities(grid.h, v.xx, v.xy, v.xz, v.m, bd.h, rb.C2,
                                             ctypes.c_void_p(rho.data_ptr()), None))
    prm = rb.reference_params(rb.SESPH, rb.C2, sc.h, sc.rho0, 0.01)
    sv = rb.Solver(rb.SESPH, prm, sc.n)
    sv.step(st, grid, bd, 5e-4)
    want = rb.device_to_numpy(sv.buffers().rho, sc.n)
    assert_close(rho.cpu().numpy(), want, 1e-6, 1e-7, "density vs the solver's pass")
    for o in (sv, grid, bd, st):
        o.close()


def test_densities_reject_a_narrow_boundary(cuda):
    import torch

    import reyn_b200 as rb
    sc, bdy = _scene()
    t = {k: torch.tensor(np.asarray(sc.fluid[k], np.float32), device="cuda")
         for k in ("x", "y", "z", "m")}
    bt = [torch.tensor(np.asarray(bdy[k], np.float32), device="cuda") for k in ("x", "y", "z", "m")]
    bd = rb.Boundary(*bt, h=0.5 * sc.h, rho0=sc.rho0)  # its grid covers radius h only
    grid = rb.Grid(sc.box_min, sc.box_max, 2 * sc.h)
    grid.construct(t["x"], t["y"], t["z"])
    with pytest.raises(rb.ReynError) as e:
        grid.compute_densities(t["x"], t["y"], t["z"], t["m"], bd, rb.C2)
    assert e.value.code == rb.ERR_INVALID
    grid.close()
    bd.close()
