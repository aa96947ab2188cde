"""Batched scenes: every scene of a batch, stepped together (one launch per
phase over all scenes, per-scene convergence), against the same scene
stepped alone (its own grid over its box, its own boundary), by particle
ID. Each scene of a batch gets exactly the grids it would get alone, so
the results agree bit for bit except where FP64 atomics sum in another
order; per-scene iteration counts must agree."""
import numpy as np
import pytest

from reyn_b200 import scenes
from tests.helpers import STEP_TOL, compare_steps

pytestmark = pytest.mark.gpu


def _small_batch(seed=11):
    counts = [(9, 8, 7), (5, 5, 5), (12, 10, 9), (7, 7, 7), (3, 3, 3)]
    return scenes.batched_dam_breaks(counts, 0.02, seed=seed)


def _params(rb, scheme, kind, h, precision=0):
    prm = rb.reference_params(scheme, kind, h, 1000.0, 0.01)
    if scheme == rb.SESPH:
        prm.k_sesph = 1000.0
    prm.precision = precision
    return prm


def _run_batched(batch, scheme, kind, steps, dt, precision=0):
    import torch

    import reyn_b200 as rb
    dev = torch.device("cuda")
    n = int(batch.first[-1])
    st = rb.Particles(n, batch.rho0)
    st.upload(batch.fluid)
    ids = torch.tensor(batch.fluid["id"], device=dev)
    bd = rb.Boundary(*(torch.tensor(batch.bdy[k], device=dev) for k in ("x", "y", "z")), None,
                     h=batch.h, rho0=batch.rho0, scene_first=batch.bfirst)
    grid = rb.Grid(batch.frame_min, batch.frame_max, 2 * batch.h, 0.5, 0,
                   scene_first=batch.first, scene_min=batch.box_min, scene_max=batch.box_max)
    sv = rb.Solver(scheme, _params(rb, scheme, kind, batch.h, precision), n)
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
    return out, np.array(its)


def _run_alone(batch, s, scheme, kind, steps, dt, precision=0):
    import torch

    import reyn_b200 as rb
    dev = torch.device("cuda")
    a, b = int(batch.first[s]), int(batch.first[s + 1])
    c, d = int(batch.bfirst[s]), int(batch.bfirst[s + 1])
    fl = {k: v[a:b] for k, v in batch.fluid.items()}
    st = rb.Particles(b - a, batch.rho0)
    st.upload(fl)
    ids = torch.tensor(fl["id"], device=dev)
    bd = rb.Boundary(*(torch.tensor(batch.bdy[k][c:d], device=dev) for k in ("x", "y", "z")),
                     None, h=batch.h, rho0=batch.rho0)
    grid = rb.Grid(batch.box_min[s], batch.box_max[s], 2 * batch.h)
    sv = rb.Solver(scheme, _params(rb, scheme, kind, batch.h, precision), b - a)
    its = []
    for _ in range(steps):
        grid.construct_and_reorder(st, [ids])
        its.append(sv.step(st, grid, bd, dt, bounds=(batch.box_min[s], batch.box_max[s])))
    out = st.download()
    out["id"] = ids.cpu().numpy()
    buf = sv.buffers()
    for k in ("rho", "p", "aii", "sii", "ax", "ay", "az"):
        out[k] = rb.device_to_numpy(getattr(buf, k), b - a)
    for o in (sv, grid, bd, st):
        o.close()
    return out, its


@pytest.mark.parametrize("scheme,kind,steps,dt", [(1, 1, 3, 1e-3), (2, 0, 3, 1e-3),
                                                  (0, 1, 4, 5e-4)])
def test_batch_matches_scenes_alone(cuda, scheme, kind, steps, dt):
    batch = _small_batch()
    got, its = _run_batched(batch, scheme, kind, steps, dt)
    tol = {k: (r * steps * 10, a * steps * 10) for k, (r, a) in STEP_TOL.items()}
    for s in range(batch.n_scenes):
        a, b = int(batch.first[s]), int(batch.first[s + 1])
        mine = {k: v[a:b] for k, v in got.items()}
        # a scene's particles stay in its own index range
        assert np.all((mine["id"] >= a) & (mine["id"] < b))
        want, wits = _run_alone(batch, s, scheme, kind, steps, dt)
        assert list(its[:, s]) == list(wits), (s, its[:, s], wits)
        compare_steps(mine, want, scheme, tol, f"scene {s}")


@pytest.mark.parametrize("precision", [1, 2])
def test_mixed_precision_batch_matches_scenes_alone(cuda, precision):
    """IISPH in MIXED (1) and MIXED_POS16 (2): each scene of the batch reads
    the same 16-bit records as when stepped alone (its own grid origin, the
    shared cell size and mass reference), so the per-scene results agree as
    in FP32"""
    batch = _small_batch()
    steps, dt = 3, 1e-3
    got, its = _run_batched(batch, 2, 0, steps, dt, precision)
    tol = {k: (r * steps * 10, a * steps * 10) for k, (r, a) in STEP_TOL.items()}
    for s in range(batch.n_scenes):
        a, b = int(batch.first[s]), int(batch.first[s + 1])
        mine = {k: v[a:b] for k, v in got.items()}
        want, wits = _run_alone(batch, s, 2, 0, steps, dt, precision)
        assert list(its[:, s]) == list(wits), (s, its[:, s], wits)
        compare_steps(mine, want, 2, tol, f"scene {s}")


def test_batched_scene_stats_and_errors(cuda):
    import reyn_b200 as rb
    batch = _small_batch()
    n = int(batch.first[-1])
    st = rb.Particles(n, batch.rho0)
    st.upload(batch.fluid)
    # a boundary over other scenes, or none, is refused
    grid = rb.Grid(batch.frame_min, batch.frame_max, 2 * batch.h, 0.5, 0,
                   scene_first=batch.first, scene_min=batch.box_min, scene_max=batch.box_max)
    sv = rb.Solver(rb.PCISPH, _params(rb, rb.PCISPH, rb.B3, batch.h), n)
    grid.construct_and_reorder(st)
    its = sv.step_batched(st, grid, None, 1e-3)
    stats = sv.scene_stats(batch.n_scenes)
    assert [s.iters for s in stats] == list(its)
    assert all(s.iters >= 3 for s in stats)
    with pytest.raises(rb.ReynError):
        rb.Grid(batch.frame_min, batch.frame_max, 2 * batch.h, 0.5, 0,
                scene_first=batch.first[::-1].copy(), scene_min=batch.box_min,
                scene_max=batch.box_max)
    for o in (sv, grid, st):
        o.close()
