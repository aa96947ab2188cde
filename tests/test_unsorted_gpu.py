"""Solver steps on a grid built by construct (the reference's Resort::no
solvers, IISPH.cu:264-266): the particles keep the caller's order, neighbours
come through the grid's permutation. Checked against the oracle like the
reordered steps, bit for bit against a reordered step from the same start,
and for the carried IISPH pressure, the dt controller's max |v|, the
iteration-limit error and the rejection of a grid over other positions."""
import numpy as np
import pytest

import oracle
from reyn_b200 import scenes
from tests.helpers import STEP_TOL, by_id, compare_steps, run_engine, run_oracle

pytestmark = pytest.mark.gpu

OUT = ("x", "y", "z", "vx", "vy", "vz", "m", "rho", "p", "aii", "sii", "ax", "ay", "az")


def _scene():
    sc = scenes.dam_break((20, 18, 16), 0.02, (0.6, 0.6, 0.6), velocity_noise=0.05, seed=5)
    bm = oracle.boundary_masses(sc.bdy["x"], sc.bdy["y"], sc.bdy["z"], sc.h, sc.rho0, 5)
    return sc, dict(sc.bdy, m=bm)


@pytest.mark.parametrize("scheme,kind,steps,dt", [(0, 1, 5, 5e-4), (1, 1, 2, 1e-3),
                                                  (2, 0, 3, 1e-3), (2, 2, 2, 1e-3)])
def test_unsorted_solver_vs_oracle(cuda, scheme, kind, steps, dt):
    sc, bdy = _scene()
    got = run_engine(scheme, kind, sc.fluid, bdy, sc.box_min, sc.box_max, sc.h, sc.rho0, 0.01,
                     dt, steps, resort=False)
    # the caller's order is kept
    np.testing.assert_array_equal(got["id"], np.asarray(sc.fluid["id"], np.float32))
    np.testing.assert_array_equal(got["m"], np.asarray(sc.fluid["m"], np.float32))
    want = run_oracle(scheme, kind, sc.fluid, bdy, sc.box_min, sc.box_max, sc.h, sc.rho0, 0.01,
                      dt, steps)
    assert got["iters"] == want["iters"]
    tol = {k: (r * steps, a * steps) for k, (r, a) in STEP_TOL.items()}
    compare_steps(got, want, scheme, tol, f"unsorted scheme{scheme}/kernel{kind}")


@pytest.mark.parametrize("scheme,kind,precision", [(0, 1, "FP32"), (1, 1, "FP32"),
                                                   (2, 0, "FP32"), (2, 0, "MIXED"),
                                                   (2, 0, "MIXED_POS16")])
def test_unsorted_first_step_equals_reordered_step(cuda, scheme, kind, precision):
    """From one start both forms sum every neighbour in the same order, so one
    step agrees bit for bit per particle, solver buffers included."""
    import reyn_b200 as rb
    sc, bdy = _scene()
    prm = rb.reference_params(scheme, kind, sc.h, sc.rho0, 0.01)
    if scheme == rb.SESPH:
        prm.k_sesph = 1000.0
    prm.precision = getattr(rb, "PRECISION_" + precision)
    a = run_engine(scheme, kind, sc.fluid, bdy, sc.box_min, sc.box_max, sc.h, sc.rho0, 0.01,
                   1e-3, 1, params=prm, resort=True)
    b = run_engine(scheme, kind, sc.fluid, bdy, sc.box_min, sc.box_max, sc.h, sc.rho0, 0.01,
                   1e-3, 1, params=prm, resort=False)
    assert a["iters"] == b["iters"]
    a = by_id({k: a[k] for k in OUT + ("id",)}, a["id"])
    b = by_id({k: b[k] for k in OUT + ("id",)}, b["id"])
    for k in OUT:
        np.testing.assert_array_equal(b[k], a[k], err_msg=k)


def _setup(rb, sc, bdy, scheme=2, kind=0, params=None):
    import torch
    st = rb.Particles(sc.n, sc.rho0)
    st.upload(sc.fluid)
    bd = rb.Boundary(*(torch.tensor(np.asarray(bdy[k], np.float32), device="cuda")
                       for k in ("x", "y", "z", "m")), h=sc.h, rho0=sc.rho0)
    grid = rb.Grid(sc.box_min, sc.box_max, 2 * sc.h)
    prm = params or rb.reference_params(scheme, kind, sc.h, sc.rho0, 0.01)
    sv = rb.Solver(scheme, prm, sc.n)
    return st, bd, grid, sv


def _close(*objs):
    for o in objs:
        o.close()


def test_unsorted_then_reordered_step_carries_pressure(cuda):
    """The carried IISPH pressure stays in the caller's order across unsorted
    steps; a reordered step next re-permutes it like any carried pressure.
    Two unsorted steps + one reordered step reach, per particle, bit for bit
    what three unsorted steps reach (step 3 starts from the same state in
    the same order either way), with the same sweep counts and max |v|."""
    import torch

    import reyn_b200 as rb
    sc, bdy = _scene()
    res = []
    for last_reordered in (False, True):
        st, bd, grid, sv = _setup(rb, sc, bdy)
        ids = torch.tensor(np.asarray(sc.fluid["id"], np.float32), device="cuda")
        iters = []
        for k in range(3):
            if k == 2 and last_reordered:
                grid.construct_and_reorder(st, [ids])
            else:
                grid.construct_state(st)
            iters.append(sv.step(st, grid, bd, 1e-3, bounds=(sc.box_min, sc.box_max)))
        out = st.download()
        out["p"] = sv.pressure()
        out["rho"] = rb.device_to_numpy(sv.buffers().rho, sc.n)
        out["id"] = ids.cpu().numpy()
        dt = sv.next_dt(st, iters[-1], 1e-3, 0.4, sc.h, (0.0, -9.81, 0.0), 10, 1e-3)
        res.append((by_id(out, out["id"]), iters, dt))
        _close(sv, grid, bd, st)
    (a, ia, da), (b, ib, db) = res
    assert ia == ib and da == db
    for k in ("x", "y", "z", "vx", "vy", "vz", "p", "rho"):
        np.testing.assert_array_equal(b[k], a[k], err_msg=k)


def test_unsorted_iteration_limit_still_writes_back(cuda):
    import reyn_b200 as rb
    sc, bdy = _scene()
    prm = rb.reference_params(rb.IISPH, rb.C2, sc.h, sc.rho0, 0.01)
    prm.max_iter = 2
    prm.eta = 1e-9  # unreachable
    st, bd, grid, sv = _setup(rb, sc, bdy, params=prm)
    before = st.download()
    grid.construct_state(st)
    with pytest.raises(rb.ReynError) as e:
        sv.step(st, grid, bd, 2e-3)
    assert e.value.code == rb.ERR_ITER_LIMIT
    after = st.download()
    assert not np.array_equal(after["vy"], before["vy"])  # the step was applied
    np.testing.assert_array_equal(after["m"], before["m"])
    _close(sv, grid, bd, st)


def test_unsorted_grid_over_other_positions_is_rejected(cuda):
    import torch

    import reyn_b200 as rb
    sc, bdy = _scene()
    st, bd, grid, sv = _setup(rb, sc, bdy)
    h = st.download()
    xyz = [torch.tensor(h[k], device="cuda") for k in ("x", "y", "z")]
    grid.construct(*xyz)  # same positions, but not the state's own arrays
    with pytest.raises(rb.ReynError) as e:
        sv.step(st, grid, bd, 1e-3)
    assert e.value.code == rb.ERR_NOT_READY
    _close(sv, grid, bd, st)


def test_autotune_reorder_interval(cuda):
    """reyn_autotune_reorder times every candidate interval from the same
    state and restores the state; each candidate's steps run (the unsorted
    ones included) and the best is one of the candidates."""
    import reyn_b200 as rb
    sc, bdy = _scene()
    st, bd, grid, sv = _setup(rb, sc, bdy)
    before = st.download()
    prm = rb.reference_params(rb.IISPH, rb.C2, sc.h, sc.rho0, 0.01)
    prm.block_size = 128
    best, ms = rb.autotune_reorder(rb.IISPH, prm, st, bd, 1e-3, (sc.box_min, sc.box_max),
                                   0.5, (1, 2, 4), steps=4)
    assert best in (1, 2, 4) and len(ms) == 3 and all(m > 0 for m in ms)
    after = st.download()
    for k in before:
        np.testing.assert_array_equal(after[k], before[k], err_msg=k)
    _close(sv, grid, bd, st)


def test_two_phase_construct_then_reorder(cuda):
    """reyn_grid_reorder after construct over the state's positions equals
    construct_and_reorder (state, extra arrays, and a step on the result),
    and is refused for a grid built over other positions."""
    import torch

    import reyn_b200 as rb
    sc, bdy = _scene()
    out = []
    for two_phase in (False, True):
        st, bd, grid, sv = _setup(rb, sc, bdy)
        ids = torch.tensor(np.asarray(sc.fluid["id"], np.float32), device="cuda")
        if two_phase:
            grid.construct_state(st)
            grid.reorder(st, [ids])
        else:
            grid.construct_and_reorder(st, [ids])
        it = sv.step(st, grid, bd, 1e-3)
        o = st.download()
        o["id"] = ids.cpu().numpy()
        out.append((o, it))
        if two_phase:
            h = st.download()
            xyz = [torch.tensor(h[k], device="cuda") for k in ("x", "y", "z")]
            grid.construct(*xyz)
            with pytest.raises(rb.ReynError) as e:
                grid.reorder(st)
            assert e.value.code == rb.ERR_NOT_READY
        _close(sv, grid, bd, st)
    (a, ia), (b, ib) = out
    assert ia == ib
    for k in a:
        np.testing.assert_array_equal(b[k], a[k], err_msg=k)
