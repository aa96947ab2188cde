"""The next grid build pre-keyed by a bounded solver step: the step's
integrating kernel computes the cell keys and the per-cell histogram of the
positions it stores, and the following construct_and_reorder of the same
grid over the unchanged state uses them instead of its own key pass. The
build must equal a build from scratch bit for bit, must drop the pre-keyed
histogram when the state changed in between, and must report positions
outside the grid found by the step."""
import numpy as np
import pytest

from reyn_b200 import scenes

pytestmark = pytest.mark.gpu


def _setup(rb, sc):
    import torch
    st = rb.Particles(sc.n, sc.rho0)
    st.upload(sc.fluid)
    bd = rb.Boundary(*(torch.tensor(sc.bdy[k], device="cuda") for k in ("x", "y", "z")), None,
                     h=sc.h, rho0=sc.rho0)
    grid = rb.Grid(sc.box_min, sc.box_max, 2 * sc.h)
    sv = rb.Solver(rb.IISPH, rb.reference_params(rb.IISPH, rb.C2, sc.h, sc.rho0, 0.01), sc.n)
    return st, bd, grid, sv


def _grid_arrays(rb, grid, n):
    """prefix and the permutation of the grid's last build (after
    construct_and_reorder `sorted` is not exposed; the permutation is)."""
    info = grid.info()
    C = info.nx * info.ny * info.nz
    perm = info.sorted if info.sorted else grid.permutation_ptr()
    return (rb.device_to_numpy(info.prefix, C + 1, np.uint32),
            rb.device_to_numpy(perm, n, np.uint32))


def _fresh_build(rb, sc, state):
    import torch
    g = rb.Grid(sc.box_min, sc.box_max, 2 * sc.h)
    g.construct(*(torch.tensor(state[k], device="cuda") for k in ("x", "y", "z")))
    out = _grid_arrays(rb, g, sc.n)
    g.close()
    return out


def test_prekeyed_build_equals_fresh_build(cuda):
    import reyn_b200 as rb
    sc = scenes.dam_break((14, 12, 10), 0.02, (0.5, 0.5, 0.5), velocity_noise=0.3, seed=31)
    st, bd, grid, sv = _setup(rb, sc)
    box = (sc.box_min, sc.box_max)
    for k in range(4):
        grid.construct_and_reorder(st)
        if k:
            prefix, srt = _grid_arrays(rb, grid, sc.n)
            np.testing.assert_array_equal(prefix, want_prefix)
            np.testing.assert_array_equal(srt, want_sorted)
        sv.step(st, grid, bd, 1e-3, bounds=box)
        # what a build from scratch over the stored positions gives
        want_prefix, want_sorted = _fresh_build(rb, sc, st.download())
    for o in (sv, grid, bd, st):
        o.close()


def test_prekey_dropped_when_state_changes(cuda):
    import reyn_b200 as rb
    sc = scenes.dam_break((14, 12, 10), 0.02, (0.5, 0.5, 0.5), velocity_noise=0.3, seed=32)
    st, bd, grid, sv = _setup(rb, sc)
    box = (sc.box_min, sc.box_max)
    grid.construct_and_reorder(st)
    sv.step(st, grid, bd, 1e-3, bounds=box)
    # new positions uploaded after the pre-keyed step
    moved = dict(sc.fluid)
    moved["x"] = np.asarray(sc.fluid["x"], np.float32)[::-1].copy()
    st.upload(moved)
    grid.construct_and_reorder(st)
    want_prefix, want_sorted = _fresh_build(rb, sc, moved)
    prefix, srt = _grid_arrays(rb, grid, sc.n)
    np.testing.assert_array_equal(prefix, want_prefix)
    np.testing.assert_array_equal(srt, want_sorted)
    for o in (sv, grid, bd, st):
        o.close()


def test_prekey_dropped_after_writes_through_raw_pointers(cuda):
    """A caller that takes the state's device pointers (Particles'
    DeviceBuffer::ptr()) and moves the particles with its own kernel between
    a pre-keyed step and the next build must get the build of the new
    positions."""
    import torch

    import reyn_b200 as rb
    sc = scenes.dam_break((14, 12, 10), 0.02, (0.5, 0.5, 0.5), velocity_noise=0.3, seed=34)
    st, bd, grid, sv = _setup(rb, sc)
    grid.construct_and_reorder(st)
    sv.step(st, grid, bd, 1e-3, bounds=(sc.box_min, sc.box_max))
    moved = st.download()
    moved["x"] = np.asarray(moved["x"], np.float32)[::-1].copy()
    v = st.soa()

    class _Dev:  # a device array at a raw pointer
        def __init__(self, ptr, n):
            self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f4",
                                             "data": (int(ptr), False), "version": 3}

    xs = torch.as_tensor(_Dev(v.xx, sc.n), device="cuda")
    xs.copy_(torch.tensor(moved["x"], device="cuda"))
    torch.cuda.synchronize()
    grid.construct_and_reorder(st)
    want_prefix, want_sorted = _fresh_build(rb, sc, moved)
    prefix, srt = _grid_arrays(rb, grid, sc.n)
    np.testing.assert_array_equal(prefix, want_prefix)
    np.testing.assert_array_equal(srt, want_sorted)
    for o in (sv, grid, bd, st):
        o.close()


def test_prekey_reports_positions_outside_the_grid(cuda):
    import reyn_b200 as rb
    sc = scenes.dam_break((10, 8, 8), 0.02, (0.5, 0.5, 0.5), seed=33)
    fast = dict(sc.fluid)
    fast["vx"] = np.full(sc.n, 2000.0, np.float32)  # leaves the grid within one step
    st, bd, grid, sv = _setup(rb, sc)
    st.upload(fast)
    far = ([-10.0, -10.0, -10.0], [10.0, 10.0, 10.0])  # bounds far beyond the grid
    grid.construct_and_reorder(st)
    try:
        sv.step(st, grid, bd, 1e-3, bounds=far)
    except rb.ReynError:
        pass
    with pytest.raises(rb.ReynError) as e:
        grid.construct_and_reorder(st)
    assert e.value.code == rb.ERR_OUT_OF_BOUNDS
    # the next build over valid positions succeeds again
    st.upload(sc.fluid)
    grid.construct_and_reorder(st)
    for o in (sv, grid, bd, st):
        o.close()
