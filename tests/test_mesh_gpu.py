"""The engine's mesh path on the GPU against the mesh oracle: the LBVH (leaf
order, children, boxes, height) and its queries (closest points, inside
flags) bit for bit, the surface measures, the samples of the area-stratified
sampler bit for bit, relaxation sweeps within float tolerance, the fluid
fill bit for bit, the OBJ reader's shape filters, and sample_mesh end to
end."""
import os

import numpy as np
import pytest

import oracle
from reyn_b200 import meshes

pytestmark = pytest.mark.gpu


def cases():
    ico = meshes.icosphere(3, 0.7, (0.1, -0.2, 0.3))
    big = meshes.icosphere(6, 0.9, (0.0, 0.0, 0.0))  # 81920 faces: 40 radix tiles
    return {
        "ico": ico,
        "ico_perturbed": (meshes.perturb(ico[0], 0.01, 3), ico[1]),
        "box": meshes.box((-1.0, -0.5, 0.0), (1.0, 0.5, 0.75), 4),
        "torus_perturbed": (meshes.perturb(meshes.torus(1.0, 0.3, 40, 20, (0.5,) * 3)[0], 0.005,
                                           5), meshes.torus(1.0, 0.3, 40, 20)[1]),
        "ico6_perturbed": (meshes.perturb(big[0], 0.0005, 9), big[1]),
        "one_triangle": (np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.2]]),
                         np.array([[0, 1, 2]], np.uint32)),
    }


CASES = cases()


def points(v, n, seed, pad=0.2):
    rng = np.random.Generator(np.random.PCG64(seed))
    lo, hi = v.min(0) - pad, v.max(0) + pad
    p = (lo + (hi - lo) * rng.random((n, 3))).astype(np.float32)
    return p[:, 0].copy(), p[:, 1].copy(), p[:, 2].copy()


def dev(*arrs):
    import torch
    return [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in arrs]


@pytest.mark.parametrize("name", list(CASES))
def test_tree_matches_oracle(cuda, name):
    import reyn_b200 as rb
    v, f = CASES[name]
    m = rb.Mesh(v, f)
    info = m.info()
    want = oracle.lbvh_build(v, f)
    got = {k: t.cpu().numpy() for k, t in m.tree().items()}
    np.testing.assert_array_equal(got["order"].astype(np.uint32), want["order"])
    np.testing.assert_array_equal(got["children_l"].astype(np.uint32), want["children_l"])
    np.testing.assert_array_equal(got["children_r"].astype(np.uint32), want["children_r"])
    np.testing.assert_array_equal(got["leaf_box"], want["leaf_box"])
    np.testing.assert_array_equal(got["node_box"], want["node_box"])
    if len(f) > 1:
        assert info.tree_height == want["height"]
    area, vol, _ = oracle.mesh_measure(v, f)
    assert info.area == pytest.approx(area, rel=1e-12)
    assert info.volume == pytest.approx(vol, rel=1e-9, abs=1e-15)
    np.testing.assert_array_equal(np.array(info.bounds_min), v.min(0))
    np.testing.assert_array_equal(np.array(info.bounds_max), v.max(0))
    assert (info.n_vertices, info.n_faces) == (len(v), len(f))
    m.close()


@pytest.mark.parametrize("name", list(CASES))
def test_project_and_inside_match_oracle(cuda, name):
    import reyn_b200 as rb
    v, f = CASES[name]
    m = rb.Mesh(v, f)
    x, y, z = points(v, 20000, 17)
    want = oracle.lbvh_project(v, f, x, y, z)
    dx, dy, dz = dev(x, y, z)
    flags = m.inside(dx, dy, dz).cpu().numpy()
    np.testing.assert_array_equal(flags, oracle.lbvh_inside(v, f, x, y, z))
    m.project(dx, dy, dz)
    for g, w in zip((dx, dy, dz), want):
        np.testing.assert_array_equal(g.cpu().numpy(), w)
    m.close()


def test_sampling_matches_oracle(cuda):
    import reyn_b200 as rb
    for name in ("ico_perturbed", "box", "torus_perturbed"):
        v, f = CASES[name]
        m = rb.Mesh(v, f)
        for h, ov, seed in ((0.05, 2.0, 1614201312), (0.02, 1.0, 7)):
            x, y, z = m.sample_uniform(h, ov, seed)
            wx, wy, wz = oracle.mesh_sample(v, f, h, ov, seed)
            assert x.numel() == wx.size
            got = np.stack([t.cpu().numpy() for t in (x, y, z)], 1)
            want = np.stack([wx, wy, wz], 1)
            # the area sums are associated differently on the GPU: a sample
            # whose stratum position falls within an ulp of a face boundary
            # may pick the neighbouring face; none do here
            np.testing.assert_array_equal(got, want)
        m.close()


def test_relaxation_sweep_matches_oracle(cuda):
    import reyn_b200 as rb
    import torch
    v, f = CASES["ico_perturbed"]
    m = rb.Mesh(v, f)
    x, y, z = m.sample_uniform(0.08, 2.0, 3)
    hb = 0.04
    x0, y0, z0 = (t.cpu().numpy() for t in (x, y, z))
    nd = torch.empty_like(x)
    st = m.relax(x, y, z, hb, 1.0, 1, num_den=nd)
    wx, wy, wz, wnd = oracle.mesh_relax_sweep(v, f, x0, y0, z0, hb, 1.0)
    # number densities: float sums in another order (and rsqrt-based |x|)
    np.testing.assert_allclose(nd.cpu().numpy(), wnd, rtol=2e-5)
    got = np.stack([t.cpu().numpy() for t in (x, y, z)], 1)
    want = np.stack([wx, wy, wz], 1)
    assert np.abs(got - want).max() < 1e-4 * hb
    assert st[0, 0] == pytest.approx(wnd.max() / wnd.min(), rel=1e-4)
    assert st[0, 1] == pytest.approx(wnd.mean(), rel=1e-4)
    m.close()


def test_relaxation_evens_out_the_sampling(cuda):
    import reyn_b200 as rb
    v, f = CASES["ico6_perturbed"]
    m = rb.Mesh(v, f)
    x, y, z = m.sample_uniform(0.03, 2.0, 5)
    st = m.relax(x, y, z, 0.015, 1.0, 20)
    assert st[-1, 0] < 0.8 * st[0, 0]
    # the samples stay on the mesh: projecting them again moves none
    px, py, pz = (t.clone() for t in (x, y, z))
    m.project(px, py, pz)
    for a, b in zip((px, py, pz), (x, y, z)):
        assert (a - b).abs().max().item() < 1e-5
    m.close()


@pytest.mark.parametrize("name,h,jitter", [("ico", 0.05, 0.0), ("torus_perturbed", 0.04, 0.1),
                                           ("box", 0.1, 0.25)])
def test_fill_matches_oracle(cuda, name, h, jitter):
    import reyn_b200 as rb
    v, f = CASES[name]
    m = rb.Mesh(v, f)
    x, y, z = m.fill(h, jitter, 11)
    wx, wy, wz = oracle.mesh_fill(v, f, h, jitter, 11)
    assert x.numel() == wx.size > 0
    for g, w in zip((x, y, z), (wx, wy, wz)):
        np.testing.assert_array_equal(g.cpu().numpy(), w)
    m.close()


def test_obj_reader_shape_filters(cuda, tmp_path):
    import reyn_b200 as rb
    tv, tf = CASES["torus_perturbed"]
    bv, bf = CASES["box"]
    path = os.path.join(str(tmp_path), "scene.obj")
    meshes.write_obj(path, [("Fluid_volume", tv, tf), ("walls", bv, bf)])
    allv = np.concatenate([tv, bv])
    fluid = rb.Mesh.from_obj(path, only="fluid")
    walls = rb.Mesh.from_obj(path, ignore=["fluid"])
    both = rb.Mesh.from_obj(path)
    assert fluid.info().n_faces == len(tf) and walls.info().n_faces == len(bf)
    assert both.info().n_faces == len(tf) + len(bf)
    # every vertex of the file is kept, as load_mesh_from_obj does
    assert fluid.info().n_vertices == len(allv)
    want = oracle.lbvh_build(allv, tf)
    got = fluid.tree()
    np.testing.assert_array_equal(got["children_l"].cpu().numpy().astype(np.uint32),
                                  want["children_l"])
    np.testing.assert_array_equal(got["node_box"].cpu().numpy(), want["node_box"])
    wf = oracle.lbvh_build(allv, bf.astype(np.int64) + len(tv))
    np.testing.assert_array_equal(walls.tree()["order"].cpu().numpy().astype(np.uint32),
                                  wf["order"])
    for mm in (fluid, walls, both):
        mm.close()


def test_sample_mesh_builds_a_boundary(cuda):
    import reyn_b200 as rb
    v, f = CASES["box"]
    m = rb.Mesh(v, f)
    bdy, (x, y, z), st = rb.sample_mesh(m, 0.05, 1000.0, 2.0, relaxation_iters=5)
    area, _, _ = oracle.mesh_measure(v, f)
    assert x.numel() == oracle.mesh_sample_count(area, 0.05, 2.0) == bdy.nb
    assert st.shape == (5, 2)
    ptrs, nb = bdy.arrays()
    mass = rb.device_to_numpy(ptrs[3], nb)
    assert np.all(mass > 0) and np.all(np.isfinite(mass))
    bdy.close()
    m.close()


def test_size_queries_and_capacity(cuda):
    import ctypes
    import reyn_b200 as rb
    import torch
    v, f = CASES["ico"]
    m = rb.Mesh(v, f)
    L = rb.lib()
    cnt = ctypes.c_uint32()
    assert L.reyn_mesh_fill(m.h, 0.05, 0.0, 1, None, None, None, 0, ctypes.byref(cnt), None) == 0
    small = torch.empty(max(cnt.value - 1, 1), device="cuda")
    assert L.reyn_mesh_fill(m.h, 0.05, 0.0, 1, small.data_ptr(), small.data_ptr(),
                            small.data_ptr(), cnt.value - 1, ctypes.byref(cnt),
                            None) == rb.ERR_INVALID
    assert L.reyn_mesh_sample_uniform(m.h, 0.05, 2.0, 1, None, None, None, 0, ctypes.byref(cnt),
                                      None) == 0
    assert L.reyn_mesh_sample_uniform(m.h, 0.05, 2.0, 1, small.data_ptr(), small.data_ptr(),
                                      small.data_ptr(), 1, ctypes.byref(cnt),
                                      None) == rb.ERR_INVALID
    m.close()


@pytest.mark.parametrize("name", ["ico3", "ico4_perturbed", "box4", "torus_perturbed"])
def test_tree_matches_reference_fixture(cuda, name):
    """the engine's LBVH against the reference's own (tests/golden/mesh_*.npz)"""
    import reyn_b200 as rb
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                             f"mesh_{name}.npz"))
    m = rb.Mesh(g["verts"], g["faces"])
    t = {k: v.cpu().numpy() for k, v in m.tree().items()}
    np.testing.assert_array_equal(g["faces"][t["order"]], g["faces_sorted"])
    np.testing.assert_array_equal(t["children_l"].astype(np.uint32), g["children_l"])
    np.testing.assert_array_equal(t["children_r"].astype(np.uint32), g["children_r"])
    np.testing.assert_array_equal(t["leaf_box"], g["leaf_box"])
    np.testing.assert_array_equal(t["node_box"], g["node_box"])
    assert m.info().tree_height == int(g["height"])
    assert m.info().volume == pytest.approx(float(g["volume"]), rel=1e-12)
    m.close()


@pytest.mark.parametrize("name", ["ico6_perturbed", "torus_perturbed"])
def test_large_query_batches_match_oracle(cuda, name):
    """batches of 2^15 points and more run in Morton order; results return to
    the callers' slots unchanged"""
    import reyn_b200 as rb
    v, f = CASES[name]
    m = rb.Mesh(v, f)
    x, y, z = points(v, 100003, 29)
    dx, dy, dz = dev(x, y, z)
    np.testing.assert_array_equal(m.inside(dx, dy, dz).cpu().numpy(),
                                  oracle.lbvh_inside(v, f, x, y, z))
    m.project(dx, dy, dz)
    for g, w in zip((dx, dy, dz), oracle.lbvh_project(v, f, x, y, z)):
        np.testing.assert_array_equal(g.cpu().numpy(), w)
    m.close()


def test_relaxation_stiffness_sweep(cuda, tmp_path):
    """The reference's stiffness study (sample_boundary.cu:472-504): sample_mesh
    on a unit cube at h_bdy in {5e-3, 5e-2, 5e-1} (oversampling 2) with 20
    relaxation sweeps at relaxation factors k in {0.01, 0.1, 0.5, 1, 1.5, 2};
    per-sweep traces written as CSV with a JSON description, as the study
    does. Every trace is finite, the sample count follows the area formula,
    and at the two finer spacings the moderate factors (0.1 .. 1) even out
    the number density."""
    import json

    import reyn_b200 as rb
    v, f = meshes.box((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), 1)
    m = rb.Mesh(v, f)
    area = oracle.mesh_measure(v, f)[0]
    traces = []
    for hb in (5e-3, 5e-2, 5e-1):
        for k in (0.01, 0.1, 0.5, 1.0, 1.5, 2.0):
            bd, (x, y, z), st = rb.sample_mesh(m, hb, 1.0, 2.0, 20, k)
            n = x.numel()
            assert n == oracle.mesh_sample_count(area, hb, 2.0)
            assert st.shape == (20, 2) and np.isfinite(st).all()
            name = f"{k}-{hb}.csv"
            np.savetxt(os.path.join(str(tmp_path), name), st, delimiter=",",
                       header="max_over_min,average", comments="")
            traces.append({"k": k, "h_bdy": hb, "filename": name, "count": n})
            if hb < 0.1 and 0.1 <= k <= 1.0:
                assert st[-1, 0] < st[0, 0], (hb, k, st[0, 0], st[-1, 0])
            bd.close()
    with open(os.path.join(str(tmp_path), "description.json"), "w") as fh:
        json.dump({"traces": traces}, fh)
    assert len(traces) == 18
    m.close()
