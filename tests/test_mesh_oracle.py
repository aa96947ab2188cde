"""CPU tests of the mesh oracle (oracle/mesh.cpp): the LBVH checks of the
reference's own test (lbvh.cu:308-440: every child box inside its parent,
every leaf box around its triangle, every leaf and internal node referenced
once, LBVH projection equal to the brute force), an independent top-down
restatement of the radix tree and of the Morton codes, surface measures,
sampling, relaxation and the fluid fill; plus the host-side argument checks
of the engine's mesh entry points (no GPU needed)."""
import ctypes
import os

import numpy as np
import pytest

import oracle
import reyn_b200 as rb
from reyn_b200 import meshes

F32_EPS = np.finfo(np.float32).eps


def mesh_cases():
    ico = meshes.icosphere(3, 0.7, (0.1, -0.2, 0.3))
    ico_p = (meshes.perturb(ico[0], 0.01, 3), ico[1])
    box = meshes.box((-1.0, -0.5, 0.0), (1.0, 0.5, 0.75), 4)
    tor = meshes.torus(1.0, 0.3, 40, 20, (0.5, 0.5, 0.5))
    tor_p = (meshes.perturb(tor[0], 0.005, 5), tor[1])
    return {"ico": ico, "ico_perturbed": ico_p, "box": box, "torus_perturbed": tor_p}


CASES = mesh_cases()


def test_generators_are_outward_and_closed():
    for name, (v, f) in CASES.items():
        vol = meshes.signed_volume(v, f)
        assert vol > 0, name
        # closed: every edge shared by exactly two faces, in opposite directions
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]]).astype(np.int64)
        fwd = set(map(tuple, e))
        assert len(fwd) == len(e), name
        assert all((b, a) in fwd for a, b in e), name


def spread10_np(v):
    r = np.zeros_like(v, dtype=np.uint32)
    for b in range(10):
        r |= ((v >> b) & 1).astype(np.uint32) << (3 * b)
    return r


@pytest.mark.parametrize("name", list(CASES))
def test_morton_codes_independent(name):
    v, f = CASES[name]
    lo, hi = v.min(0), v.max(0)
    inv = 1.0 / (hi - lo)
    a, b, c = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    cen = ((a + b) + c) * (1.0 / 3.0) - lo
    q = np.minimum(np.maximum(cen * inv * 1024.0, 0.0), 1023.0).astype(np.float32).astype(np.uint32)
    want = (spread10_np(q[:, 0]) << 2) | (spread10_np(q[:, 1]) << 1) | spread10_np(q[:, 2])
    np.testing.assert_array_equal(oracle.mesh_morton(v, f), want)


def topdown_tree(keys):
    """The binary radix tree by recursive top-down splitting at the highest
    differing key bit; Karras' numbering: the children of a node split at g
    are g (left) and g + 1 (right)."""
    n = len(keys)
    cl = np.zeros(n - 1, np.uint32)
    cr = np.zeros(n - 1, np.uint32)

    def clz(x):
        return 64 - int(x).bit_length()

    stack = [(0, 0, n - 1)]
    while stack:
        idx, first, last = stack.pop()
        common = clz(keys[first] ^ keys[last])
        g = first
        for j in range(first, last):
            if clz(keys[first] ^ keys[j]) > common:
                g = j
        cl[idx] = (g << 1) | (0 if g == first else 1)
        cr[idx] = ((g + 1) << 1) | (0 if g + 1 == last else 1)
        if g != first:
            stack.append((g, first, g))
        if g + 1 != last:
            stack.append((g + 1, g + 1, last))
    return cl, cr


@pytest.mark.parametrize("name", ["ico", "box", "torus_perturbed"])
def test_lbvh_topology_matches_topdown_restatement(name):
    v, f = CASES[name]
    t = oracle.lbvh_build(v, f)
    codes = oracle.mesh_morton(v, f)
    order = np.argsort(codes, kind="stable")
    np.testing.assert_array_equal(t["order"], order)
    keys = [(int(codes[order[j]]) << 32) | j for j in range(len(order))]
    cl, cr = topdown_tree(keys)
    np.testing.assert_array_equal(t["children_l"], cl)
    np.testing.assert_array_equal(t["children_r"], cr)


def box_contains(outer, inner):
    return np.all(outer[:3] <= inner[:3]) and np.all(inner[3:] <= outer[3:])


@pytest.mark.parametrize("name", list(CASES))
def test_lbvh_reference_checks(name):
    """lbvh.cu:308-370: boxes nest, leaves hold their triangles, and every
    leaf and internal node (but the root) is referenced exactly once."""
    v, f = CASES[name]
    t = oracle.lbvh_build(v, f)
    nf = len(f)
    leaf, node = t["leaf_box"], t["node_box"]
    for i in range(nf - 1):
        for c in (t["children_l"][i], t["children_r"][i]):
            child = node[c >> 1] if c & 1 else leaf[c >> 1]
            assert np.all(child[:3] < child[3:] + 0)  # mini < maxi per axis
            assert box_contains(node[i], child)
    vf = v.astype(np.float32)
    for j in range(nf):
        tri = vf[f[t["order"][j]]]
        assert np.all(tri >= leaf[j][:3]) and np.all(tri <= leaf[j][3:])
    links = np.concatenate([t["children_l"], t["children_r"]])
    leaves = np.sort(links[(links & 1) == 0] >> 1)
    np.testing.assert_array_equal(leaves, np.arange(nf))
    internal = np.sort(links[(links & 1) == 1] >> 1)
    np.testing.assert_array_equal(internal, np.arange(1, nf - 1))
    assert 1 <= t["height"] < 64


def random_points(v, n, seed, pad=0.0):
    rng = np.random.Generator(np.random.PCG64(seed))
    lo, hi = v.min(0) - pad, v.max(0) + pad
    p = (lo + (hi - lo) * rng.random((n, 3))).astype(np.float32)
    return p[:, 0].copy(), p[:, 1].copy(), p[:, 2].copy()


@pytest.mark.parametrize("name", list(CASES))
def test_lbvh_projection_equals_brute_force(name):
    """lbvh.cu:372-433: the traversal finds the brute force's closest point
    (the distance exactly; the point up to ties between faces)."""
    v, f = CASES[name]
    x, y, z = random_points(v, 4000, 420, pad=0.2)
    a = np.stack(oracle.lbvh_project(v, f, x, y, z), 1)
    b = np.stack(oracle.project_brute(v, f, x, y, z), 1)
    q = np.stack([x, y, z], 1)
    da = ((a - q) ** 2).sum(1)
    db = ((b - q) ** 2).sum(1)
    np.testing.assert_allclose(da, db, rtol=1e-5, atol=1e-12)
    # the reference test's bound on the squared point difference (375 FLT_EPS)
    assert np.all(((a - b) ** 2).sum(1) <= 375 * F32_EPS)
    # projected points lie on the mesh: projecting again moves nothing much
    a2 = np.stack(oracle.lbvh_project(v, f, a[:, 0], a[:, 1], a[:, 2]), 1)
    assert np.abs(a2 - a).max() < 1e-5


def test_inside_matches_analytic_sphere():
    v, f = CASES["ico"]
    x, y, z = random_points(v, 6000, 7, pad=0.3)
    inside = oracle.lbvh_inside(v, f, x, y, z).astype(bool)
    r = np.sqrt((x - 0.1) ** 2 + (y + 0.2) ** 2 + (z - 0.3) ** 2)
    # an icosphere of level 3 deviates from the sphere by < 0.5 % of r
    clear = np.abs(r - 0.7) > 0.02
    np.testing.assert_array_equal(inside[clear], r[clear] < 0.7)


def test_measures():
    v, f = CASES["box"]
    area, vol, cdf = oracle.mesh_measure(v, f)
    assert area == pytest.approx(2 * (2 * 1 + 2 * 0.75 + 1 * 0.75), rel=1e-12)
    assert vol == pytest.approx(2 * 1 * 0.75, rel=1e-12)
    assert cdf[-1] == area and np.all(np.diff(cdf) > 0)
    v, f = CASES["ico"]
    area, vol, _ = oracle.mesh_measure(v, f)
    assert vol == pytest.approx(meshes.signed_volume(v, f), rel=1e-12)
    assert area == pytest.approx(4 * np.pi * 0.49, rel=0.02)


def test_sample_count_formula():
    # sample_boundary.cu:339-346, in float for the area per sample
    for area, h, ov in [(6.0, 0.05, 2.0), (1.2345, 0.01, 1.0), (3.3, 0.02, 3.0)]:
        hb = np.float32(np.float64(h) / np.float64(ov))
        per = np.float32(np.float32(1.5) * np.sqrt(np.float32(3.0))) * hb * hb
        assert oracle.mesh_sample_count(area, h, ov) == int(np.ceil(area / np.float64(per)))


def test_samples_on_surface_and_stratified():
    v, f = CASES["box"]
    x, y, z = oracle.mesh_sample(v, f, 0.05, 2.0, 1614201312)
    area, _, _ = oracle.mesh_measure(v, f)
    assert x.size == oracle.mesh_sample_count(area, 0.05, 2.0)
    q = np.stack([x, y, z], 1)
    p = np.stack(oracle.project_brute(v, f, x, y, z), 1)
    assert np.abs(p - q).max() < 1e-6
    # samples per box side follow the side areas (stratification keeps the
    # counts within a few samples of the expectation)
    sides = {(0, -1.0): 0.75, (0, 1.0): 0.75, (1, -0.5): 1.5, (1, 0.5): 1.5, (2, 0.0): 2.0,
             (2, 0.75): 2.0}
    for (ax, val), a in sides.items():
        n = int(np.sum(np.abs(q[:, ax] - val) < 1e-6))
        assert abs(n - a / area * x.size) <= 4, (ax, val, n)


def test_hex_plane_density_is_b3_sum():
    hb = 0.05
    d = []
    for qq in range(-2, 3):
        for rr in range(-2, 3):
            d.append(np.float32(qq) * np.array([hb, 0, 0], np.float32)
                     + np.float32(rr) * np.array([hb * 0.5, hb * np.float32(np.sqrt(3) * 0.5), 0],
                                                 np.float32))
    d = np.array(d, np.float32)
    w, _, _, _ = oracle.kernel_eval(oracle.B3, 2 * hb, d[:, 0], d[:, 1], d[:, 2])
    assert oracle.hex_plane_density(hb) == pytest.approx(float(w.astype(np.float64).sum()),
                                                         rel=1e-6)


def test_relaxation_sweeps_even_out_a_sphere_sampling():
    v, f = CASES["ico"]
    x, y, z = oracle.mesh_sample(v, f, 0.1, 2.0, 11)
    hb = 0.05
    ratios = []
    for _ in range(6):
        x, y, z, nd = oracle.mesh_relax_sweep(v, f, x, y, z, hb, 1.0)
        ratios.append(nd.max() / nd.min())
    assert ratios[-1] < 0.8 * ratios[0]
    # still on the mesh
    p = np.stack(oracle.project_brute(v, f, x, y, z), 1)
    assert np.abs(p - np.stack([x, y, z], 1)).max() < 1e-6


def test_fill_counts_volume_and_keeps_lattice_order():
    v, f = CASES["ico"]
    h = 0.05
    x, y, z = oracle.mesh_fill(v, f, h)
    vol = meshes.signed_volume(v, f)
    assert abs(x.size * h ** 3 - vol) < 0.05 * vol
    # lattice order: z, then y, then x non-decreasing
    x64, y64, z64 = (a.astype(np.float64) for a in (x, y, z))
    key = np.round((z64 - z64.min()) / h) * 1e6 + np.round((y64 - y64.min()) / h) * 1e3 + \
        np.round((x64 - x64.min()) / h)
    assert np.all(np.diff(key) > 0)
    xj, yj, zj = oracle.mesh_fill(v, f, h, jitter=0.1, seed=3)
    assert xj.size == x.size
    assert 0 < np.abs(xj - x).max() <= 0.1 * h * (1 + 1e-6)


def test_mesh_entry_points_reject_bad_arguments(tmp_path):
    """host-side checks run before any device work"""
    L = rb.lib()
    h = ctypes.c_void_p()
    v = np.zeros(3)
    f = np.array([0, 1, 5], np.uint32)
    ptr = v.ctypes.data
    assert L.reyn_mesh_create(ptr, ptr, ptr, 3, f.ctypes.data, 1, None, ctypes.byref(h)) == \
        rb.ERR_INVALID
    assert b"index" in L.reyn_last_error()
    assert L.reyn_mesh_create(ptr, ptr, ptr, 3, f.ctypes.data, 0, None, ctypes.byref(h)) == \
        rb.ERR_INVALID
    assert L.reyn_mesh_create(None, ptr, ptr, 3, f.ctypes.data, 1, None, ctypes.byref(h)) == \
        rb.ERR_INVALID
    missing = os.path.join(str(tmp_path), "missing.obj")
    assert L.reyn_mesh_load_obj(missing.encode(), None, 0, None, None, ctypes.byref(h)) == \
        rb.ERR_INVALID
    quad = os.path.join(str(tmp_path), "quad.obj")
    with open(quad, "w") as fh:
        fh.write("v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nf 1 2 3 4\n")
    assert L.reyn_mesh_load_obj(quad.encode(), None, 0, None, None, ctypes.byref(h)) == \
        rb.ERR_INVALID
    assert b"non-triangulated" in L.reyn_last_error()
    bad = os.path.join(str(tmp_path), "bad.obj")
    with open(bad, "w") as fh:
        fh.write("v 0 0 0\nv 1 0 0\nf 1 2 7\n")
    assert L.reyn_mesh_load_obj(bad.encode(), None, 0, None, None, ctypes.byref(h)) == \
        rb.ERR_INVALID
    assert L.reyn_mesh_project(None, None, None, None, 0, None) == rb.ERR_INVALID
    assert L.reyn_mesh_fill(None, 0.1, 0.0, 1, None, None, None, 0, None, None) == rb.ERR_INVALID


GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("name", ["ico3", "ico4_perturbed", "box4", "torus_perturbed"])
def test_oracle_matches_reference_lbvh(name):
    """Pinned against the reference's own LBVH (tests/golden/make_golden.py
    --mesh ran lbvh.cuh's LBVH on a B200): the sorted faces, children, boxes
    and height bit for bit, the volume, LBVH::project's results, and the
    sample counts of uniform_sample_mesh."""
    g = np.load(os.path.join(GOLDEN, f"mesh_{name}.npz"))
    v, f = g["verts"], g["faces"]
    t = oracle.lbvh_build(v, f)
    np.testing.assert_array_equal(f[t["order"]], g["faces_sorted"])
    np.testing.assert_array_equal(t["children_l"], g["children_l"])
    np.testing.assert_array_equal(t["children_r"], g["children_r"])
    np.testing.assert_array_equal(t["leaf_box"], g["leaf_box"])
    np.testing.assert_array_equal(t["node_box"], g["node_box"])
    assert t["height"] == int(g["height"])
    area, vol, _ = oracle.mesh_measure(v, f)
    assert vol == pytest.approx(float(g["volume"]), rel=1e-12)
    q = g["points"]
    a = np.stack(oracle.lbvh_project(v, f, q[:, 0], q[:, 1], q[:, 2]), 1)
    b = g["projected"]
    # the reference's device code may contract multiply-adds: distances agree
    # to float rounding, points within its own test's bound (lbvh.cu:420-426)
    a64, b64, q64 = (t.astype(np.float64) for t in (a, b, q))
    np.testing.assert_allclose(np.sqrt(((a64 - q64) ** 2).sum(1)),
                               np.sqrt(((b64 - q64) ** 2).sum(1)), rtol=1e-5, atol=1e-6)
    assert np.all(((a64 - b64) ** 2).sum(1) <= 375 * F32_EPS)
    # within 2 ulps but for near-ties between faces (same distance, another
    # face's point): at most 0.5 % of the points
    close = np.all(np.abs(a - b) <= 2.4e-7, 1)
    assert np.mean(close) >= 0.995
    for (h, ov), want in zip(g["sample_cases"], g["sample_counts"]):
        assert oracle.mesh_sample_count(area, float(h), float(ov)) == int(want)
