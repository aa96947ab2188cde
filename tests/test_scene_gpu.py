"""On-device scene generation against the host generator (bit for bit for
the lattice, jitter and walls), the Fibonacci sphere against its formula,
and the boundary cull against a brute-force CPU check."""
import numpy as np
import pytest
from scipy.spatial import cKDTree

from reyn_b200 import scenes

pytestmark = pytest.mark.gpu


def test_fluid_blocks_match_host_generator(cuda):
    import reyn_b200 as rb
    a = scenes.fluid_block((40, 30, 20), 0.01, (0.015, 0.02, 0.025), 1000.0, 0.05, 9,
                           velocity_noise=0.3)
    b = scenes.fluid_block((7, 5, 3), 0.02, (0.5, 0.1, 0.2), 1000.0, 0.1, 9, first=24000,
                           mass_kernel="C2")
    n = a["x"].size + b["x"].size
    st = rb.Particles(n, 1000.0)
    rb.scene_fluid_block(st, (40, 30, 20), (0.015, 0.02, 0.025), 0.01, mass=0.0, jitter=0.05,
                         velocity_noise=0.3, seed=9)
    rb.scene_fluid_block(st, (7, 5, 3), (0.5, 0.1, 0.2), 0.02, mass=float(b["m"][0]),
                         jitter=0.1, seed=9, first=24000)
    got = st.download()
    for k in ("x", "y", "z", "vx", "vy", "vz", "m"):
        np.testing.assert_array_equal(got[k], np.concatenate([a[k], b[k]]), err_msg=k)
    st.close()


@pytest.mark.parametrize("box,spacing", [((2.0, 1.0, 1.0), 0.005), ((0.6, 0.6, 0.6), 0.02),
                                         ((1.0, 0.5, 0.25), 0.05)])
def test_box_walls_match_host_generator(cuda, box, spacing):
    import reyn_b200 as rb
    x, y, z = rb.scene_box_walls((0, 0, 0), box, spacing)
    want = scenes.box_walls((0, 0, 0), box, spacing)
    np.testing.assert_array_equal(x.cpu().numpy(), want["x"])
    np.testing.assert_array_equal(y.cpu().numpy(), want["y"])
    np.testing.assert_array_equal(z.cpu().numpy(), want["z"])


def test_fibonacci_sphere(cuda):
    import reyn_b200 as rb
    c, r, sp = (1.5, 0.2, 0.75), 0.2, 0.004
    x, y, z = (t.cpu().numpy().astype(np.float64) for t in rb.scene_sphere(c, r, sp))
    n = int(np.rint(4 * np.pi * r * r / (sp * sp)))
    assert x.size == n
    k = np.arange(n)
    t = 1.0 - (2.0 * k + 1.0) / n
    ring = np.sqrt(np.maximum(0.0, 1.0 - t * t))
    ph = k * np.pi * (3.0 - np.sqrt(5.0))
    np.testing.assert_allclose(x, c[0] + r * ring * np.cos(ph), atol=2e-7)
    np.testing.assert_allclose(y, c[1] + r * t, atol=2e-7)
    np.testing.assert_allclose(z, c[2] + r * ring * np.sin(ph), atol=2e-7)
    # roughly one sample per spacing^2: nearest-neighbour distance ~ spacing
    d, _ = cKDTree(np.stack([x, y, z], 1)).query(np.stack([x, y, z], 1), k=2)
    assert 0.7 * sp < np.median(d[:, 1]) < 1.3 * sp


def test_cull_removes_particles_near_the_boundary(cuda):
    import torch

    import reyn_b200 as rb
    h = 0.02
    fl = scenes.fluid_block((30, 30, 30), h, (0.0, 0.0, 0.0), 1000.0, 0.2, 4)
    walls = scenes.box_walls((0.1, 0.1, 0.1), (0.5, 0.5, 0.5), h)
    st = rb.Particles(fl["x"].size, 1000.0)
    st.upload(fl)
    dev = torch.device("cuda")
    bd = rb.Boundary(*(torch.tensor(walls[k], device=dev) for k in ("x", "y", "z")), None,
                     h=h, rho0=1000.0)
    radius = 1.0 * h
    kept = rb.scene_cull(st, bd, radius)
    got = st.download()
    tree = cKDTree(np.stack([walls["x"], walls["y"], walls["z"]], 1).astype(np.float64))
    p = np.stack([fl["x"], fl["y"], fl["z"]], 1).astype(np.float64)
    # the engine decides in float32: only particles within 1e-6 of the radius
    # may go either way
    far = np.array([len(v) == 0 for v in tree.query_ball_point(p, radius * (1 + 1e-6))])
    close = np.array([len(v) > 0 for v in tree.query_ball_point(p, radius * (1 - 1e-6))])
    assert kept == got["x"].size and 0 < far.sum() <= kept <= (~close).sum()
    src = {v: i for i, v in enumerate(zip(fl["x"].tolist(), fl["y"].tolist(),
                                          fl["z"].tolist()))}
    order = np.array([src[v] for v in zip(got["x"].tolist(), got["y"].tolist(),
                                          got["z"].tolist())])
    assert np.all(np.diff(order) > 0)          # survivors keep their order
    assert set(np.flatnonzero(far)) <= set(order.tolist())
    assert not set(np.flatnonzero(close)) & set(order.tolist())
    for o in (st, bd):
        o.close()


def test_jitter_matches_host_generator(cuda):
    """reyn_scene_jitter: particle q of [first, first + count) moves by the
    uniform [-a, a] of streams 0..2 at counter q, as the fluid blocks' jitter;
    particles outside the range stay; the boundary reports its samples'
    bounds."""
    import torch

    import reyn_b200 as rb
    rng = np.random.default_rng(9)
    n, first, count = 5000, 700, 3000
    host = {k: rng.random(n, dtype=np.float32) for k in ("x", "y", "z", "vx", "vy", "vz", "m")}
    st = rb.Particles(n, 1000.0)
    st.upload(host)
    a = np.float32(0.0123)
    rb.scene_jitter(st, float(a), seed=77, first=first, count=count)
    got = st.download()
    idx = np.arange(first, first + count, dtype=np.uint64)
    for t, k in enumerate(("x", "y", "z")):
        want = host[k].copy()
        want[first:first + count] = host[k][first:first + count] + scenes._symmetric(
            scenes.uniform01(77, t, idx), a)
        np.testing.assert_array_equal(got[k], want, err_msg=k)
    for k in ("vx", "vy", "vz", "m"):
        np.testing.assert_array_equal(got[k], host[k], err_msg=k)
    st.close()
    b = [torch.tensor(rng.random(300, dtype=np.float32) * 2 - 0.5, device="cuda")
         for _ in range(3)]
    bd = rb.Boundary(*b, torch.ones(300, device="cuda"), h=0.05, rho0=1000.0)
    lo, hi = bd.bounds()
    for ax in range(3):
        v = b[ax].cpu().numpy()
        assert lo[ax] == v.min() and hi[ax] == v.max()
    bd.close()
