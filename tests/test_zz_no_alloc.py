"""reyn_grid_construct_noalloc: the grid build for callers that cannot
allocate device memory (real-time loops that must not wait on the device
allocator, hosts whose device memory belongs to another runtime's pool). It
must produce exactly what reyn_grid_construct produces — the prefix over all
cells and the canonical sorted indices — from its file-scope scratch array,
on consecutive calls that reuse that array, must leave the device's free
memory unchanged, must report particles outside the grid and non-finite
positions like the allocating build, and must refuse sizes beyond the
scratch limit.

This file is collected last, so that a run stopping at the first failure has
already run every other test; it also passes on its own in a fresh process.
"""
import numpy as np
import pytest

from reyn_b200 import scenes

pytestmark = pytest.mark.gpu


def _t(a):
    import torch
    return torch.tensor(np.ascontiguousarray(a, np.float32), device="cuda")


def _existing(x, y, z, bmin, bmax, r):
    """prefix and sorted from the allocating entry point."""
    import reyn_b200 as rb
    g = rb.Grid(bmin, bmax, r)
    g.construct(_t(x), _t(y), _t(z))
    info = g.info()
    C = info.nx * info.ny * info.nz
    prefix = rb.device_to_numpy(info.prefix, C + 1, np.uint32)
    srt = rb.device_to_numpy(info.sorted, x.size, np.uint32)
    g.close()
    return (info.nx, info.ny, info.nz), prefix, srt


def test_noalloc_matches_allocating_build_on_consecutive_calls(cuda):
    import torch

    import reyn_b200 as rb

    bmin, bmax, r = [0, 0, 0], [1, 1, 1], 0.04
    clouds = [scenes.uniform_cloud(200_000, seed=41), scenes.uniform_cloud(150_000, seed=42)]
    dims = rb.grid_construct_noalloc(bmin, bmax, r, None, None, None, None, None)
    C = dims[0] * dims[1] * dims[2]
    prefix = torch.empty(C + 1, dtype=torch.int32, device="cuda")
    for x, y, z in clouds:  # two calls in a row on the same scratch array
        sorted_ = torch.empty(x.size, dtype=torch.int32, device="cuda")
        got_dims = rb.grid_construct_noalloc(bmin, bmax, r, _t(x), _t(y), _t(z), prefix, sorted_)
        want_dims, want_prefix, want_sorted = _existing(x, y, z, bmin, bmax, r)
        assert got_dims == want_dims
        np.testing.assert_array_equal(prefix.cpu().numpy().view(np.uint32), want_prefix)
        np.testing.assert_array_equal(sorted_.cpu().numpy().view(np.uint32), want_sorted)


def test_noalloc_rejects_sizes_beyond_its_scratch(cuda):
    import torch

    import reyn_b200 as rb

    # 4M particles need 8M words for keys and slots alone
    n = 4 * 1024 * 1024
    x = torch.full((n,), 0.5, device="cuda")
    bmin, bmax, r = [0, 0, 0], [1, 1, 1], 0.04
    dims = rb.grid_construct_noalloc(bmin, bmax, r, None, None, None, None, None)
    prefix = torch.empty(dims[0] * dims[1] * dims[2] + 1, dtype=torch.int32, device="cuda")
    sorted_ = torch.empty(n, dtype=torch.int32, device="cuda")
    with pytest.raises(rb.ReynError) as e:
        rb.grid_construct_noalloc(bmin, bmax, r, x, x, x, prefix, sorted_)
    assert e.value.code == rb.ERR_INVALID
    assert "scratch" in str(e.value)
    # a prefix buffer that is too small is refused as well
    with pytest.raises(rb.ReynError):
        rb.grid_construct_noalloc(bmin, bmax, r, x[:10], x[:10], x[:10], prefix[:5],
                                  sorted_[:10])


def test_noalloc_allocates_nothing_and_reports_bad_positions(cuda):
    import torch

    import reyn_b200 as rb

    bmin, bmax, r = [0, 0, 0], [1, 1, 1], 0.04
    x, y, z = scenes.uniform_cloud(100_000, seed=43)
    tx, ty, tz = _t(x), _t(y), _t(z)
    dims = rb.grid_construct_noalloc(bmin, bmax, r, None, None, None, None, None)
    C = dims[0] * dims[1] * dims[2]
    prefix = torch.empty(C + 1, dtype=torch.int32, device="cuda")
    sorted_ = torch.empty(x.size, dtype=torch.int32, device="cuda")
    bad = tx.clone()
    rb.grid_construct_noalloc(bmin, bmax, r, tx, ty, tz, prefix, sorted_)  # warm
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    rb.grid_construct_noalloc(bmin, bmax, r, tx, ty, tz, prefix, sorted_)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0, "a warm call changed the free device memory"

    # a non-finite position and a position outside the grid are reported
    bad[123] = float("nan")
    with pytest.raises(rb.ReynError) as e:
        rb.grid_construct_noalloc(bmin, bmax, r, bad, ty, tz, prefix, sorted_)
    assert e.value.code == rb.ERR_NONFINITE
    bad[123] = 5.0
    with pytest.raises(rb.ReynError) as e:
        rb.grid_construct_noalloc(bmin, bmax, r, bad, ty, tz, prefix, sorted_)
    assert e.value.code == rb.ERR_OUT_OF_BOUNDS

    # the next valid call starts from cleared counters and status
    rb.grid_construct_noalloc(bmin, bmax, r, tx, ty, tz, prefix, sorted_)
    want_dims, want_prefix, want_sorted = _existing(x, y, z, bmin, bmax, r)
    assert dims == want_dims
    np.testing.assert_array_equal(prefix.cpu().numpy().view(np.uint32), want_prefix)
    np.testing.assert_array_equal(sorted_.cpu().numpy().view(np.uint32), want_sorted)
