"""Captured steps (reyn_step_graph) against the plain calls: the same scene
stepped K times through graph launches and through construct_and_reorder +
step must reach the same state bit for bit with the same sweep counts, for
SESPH, PCISPH and IISPH, FP32 and mixed precision, one scene and a batch;
graph launches and plain steps may be interleaved; iteration-limit hits are
reported like the plain step's."""
import numpy as np
import pytest

from reyn_b200 import scenes

pytestmark = pytest.mark.gpu


def _setup_single(rb, scheme, kind, precision, seed=7):
    import torch
    sc = scenes.dam_break((14, 12, 10), 0.02, (0.5, 0.5, 0.5), velocity_noise=0.02, seed=seed)
    st = rb.Particles(sc.n, sc.rho0)
    st.upload(sc.fluid)
    bd = rb.Boundary(*(torch.tensor(sc.bdy[k], device="cuda") for k in ("x", "y", "z")), None,
                     h=sc.h, rho0=sc.rho0)
    grid = rb.Grid(sc.box_min, sc.box_max, 2 * sc.h)
    prm = rb.reference_params(scheme, kind, sc.h, sc.rho0, 0.01)
    if scheme == rb.SESPH:
        prm.k_sesph = 1000.0
    prm.precision = precision
    sv = rb.Solver(scheme, prm, sc.n)
    return st, bd, grid, sv, (sc.box_min, sc.box_max)


def _setup_batch(rb, scheme, kind, seed=11):
    import torch
    counts = [(9, 8, 7), (5, 5, 5), (12, 10, 9), (7, 7, 7), (3, 3, 3)]
    batch = scenes.batched_dam_breaks(counts, 0.02, seed=seed)
    n = int(batch.first[-1])
    st = rb.Particles(n, batch.rho0)
    st.upload(batch.fluid)
    bd = rb.Boundary(*(torch.tensor(batch.bdy[k], device="cuda") for k in ("x", "y", "z")), None,
                     h=batch.h, rho0=batch.rho0, scene_first=batch.bfirst)
    grid = rb.Grid(batch.frame_min, batch.frame_max, 2 * batch.h, 0.5, 0,
                   scene_first=batch.first, scene_min=batch.box_min, scene_max=batch.box_max)
    prm = rb.reference_params(scheme, kind, batch.h, batch.rho0, 0.01)
    if scheme == rb.SESPH:
        prm.k_sesph = 1000.0
    sv = rb.Solver(scheme, prm, n)
    return st, bd, grid, sv, batch


def _close(*objs):
    for o in objs:
        o.close()


CASES = [("SESPH", "B3", "FP32"), ("PCISPH", "B3", "FP32"), ("PCISPH", "C2", "FP32"),
         ("IISPH", "C2", "FP32"), ("IISPH", "W6", "FP32"), ("IISPH", "C2", "MIXED"),
         ("IISPH", "C2", "MIXED_POS16")]


@pytest.mark.parametrize("scheme,kind,precision", CASES)
def test_graph_steps_equal_plain_steps(cuda, scheme, kind, precision):
    import reyn_b200 as rb
    sch, knd = getattr(rb, scheme), getattr(rb, kind)
    prec = getattr(rb, "PRECISION_" + precision)
    dt, steps = 1e-3, 4
    # plain
    st, bd, grid, sv, box = _setup_single(rb, sch, knd, prec)
    plain_iters = []
    for _ in range(steps):
        grid.construct_and_reorder(st)
        plain_iters.append(sv.step(st, grid, bd, dt, bounds=box))
    want = st.download()
    _close(sv, grid, bd, st)
    # captured
    st, bd, grid, sv, box = _setup_single(rb, sch, knd, prec)
    g = rb.StepGraph(sv, st, grid, bd, dt, bounds=box)
    step_k, sweep_k = g.info()
    assert step_k > 0 and (sweep_k > 0) == (sch != rb.SESPH)
    graph_iters = []
    for _ in range(steps):
        g.launch()
        graph_iters.append(g.stats().iters)
    got = st.download()
    assert graph_iters == plain_iters
    for k in ("x", "y", "z", "vx", "vy", "vz", "m"):
        np.testing.assert_array_equal(got[k], want[k], err_msg=k)
    g.close()
    _close(sv, grid, bd, st)


def test_graph_and_plain_steps_interleave(cuda):
    import reyn_b200 as rb
    dt = 1e-3
    st, bd, grid, sv, box = _setup_single(rb, rb.IISPH, rb.C2, rb.PRECISION_FP32)
    for _ in range(3):
        grid.construct_and_reorder(st)
        sv.step(st, grid, bd, dt, bounds=box)
    want = st.download()
    _close(sv, grid, bd, st)
    st, bd, grid, sv, box = _setup_single(rb, rb.IISPH, rb.C2, rb.PRECISION_FP32)
    g = rb.StepGraph(sv, st, grid, bd, dt, bounds=box)
    g.launch()
    grid.construct_and_reorder(st)
    sv.step(st, grid, bd, dt, bounds=box)
    g.launch()
    got = st.download()
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        np.testing.assert_array_equal(got[k], want[k], err_msg=k)
    # max |v| of the last (captured) step feeds the dt controller
    dt_g = sv.next_dt(st, 3, dt, 0.4, 0.02, (0.0, -9.81, 0.0), 10, 0.001)
    assert 0 < dt_g < 1.0
    g.close()
    _close(sv, grid, bd, st)


@pytest.mark.parametrize("scheme,kind", [("PCISPH", "B3"), ("IISPH", "C2"), ("SESPH", "B3")])
def test_batched_graph_steps_equal_plain_steps(cuda, scheme, kind):
    import reyn_b200 as rb
    sch, knd = getattr(rb, scheme), getattr(rb, kind)
    dt, steps = 5e-4, 3
    st, bd, grid, sv, batch = _setup_batch(rb, sch, knd)
    plain = []
    for _ in range(steps):
        grid.construct_and_reorder(st)
        plain.append(sv.step_batched(st, grid, bd, dt))
    want = st.download()
    _close(sv, grid, bd, st)
    st, bd, grid, sv, batch = _setup_batch(rb, sch, knd)
    g = rb.StepGraph(sv, st, grid, bd, dt, bounds=((0, 0, 0), (0, 0, 0)))
    for k in range(steps):
        g.launch()
        g.stats()
        its = np.array([s.iters for s in sv.scene_stats(grid.n_scenes)])
        np.testing.assert_array_equal(its, plain[k])
    got = st.download()
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        np.testing.assert_array_equal(got[k], want[k], err_msg=k)
    g.close()
    _close(sv, grid, bd, st)


def test_graph_reports_iteration_limit(cuda):
    import reyn_b200 as rb
    st, bd, grid, sv, box = _setup_single(rb, rb.IISPH, rb.C2, rb.PRECISION_FP32)
    prm = rb.reference_params(rb.IISPH, rb.C2, 0.02, 1000.0, 0.01)
    prm.max_iter = 3
    prm.eta = 1e-9  # unreachable: every step stops at max_iter
    sv.close()
    sv = rb.Solver(rb.IISPH, prm, st.n)
    g = rb.StepGraph(sv, st, grid, bd, 2e-3, bounds=box)
    g.launch()
    with pytest.raises(rb.ReynError) as e:
        g.stats()
    assert e.value.code == rb.ERR_ITER_LIMIT
    g.close()
    _close(sv, grid, bd, st)
