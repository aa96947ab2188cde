"""The C++ adapter layer (include/reyn_b200.hpp): the reference's main loop
(main.cu:60-78) written against reyn::Particles / UniformGridBuilder /
IISPH<C2> / simple_dt_controller / hard_enforce_bounds must drive the engine
to exactly the state the C ABI reaches when called directly, and that state
must agree with the CPU oracle."""
import os
import shutil
import struct
import subprocess

import numpy as np
import pytest

import oracle
from reyn_b200 import scenes
from tests.helpers import assert_close

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def compile_main_loop(tmp):
    exe = os.path.join(tmp, "main_loop")
    cxx = shutil.which("g++") or "g++"
    subprocess.run([cxx, "-std=c++17", "-O2", "-I" + os.path.join(ROOT, "include"),
                    "-I/usr/local/cuda/include", os.path.join(ROOT, "tests", "cpp", "main_loop.cpp"),
                    "-L" + os.path.join(ROOT, "reyn_b200"), "-lreyn_b200",
                    "-L/usr/local/cuda/lib64", "-lcudart",
                    "-Wl,-rpath," + os.path.join(ROOT, "reyn_b200"), "-o", exe], check=True)
    return exe


def write_scene(path, sc, bm, steps, dt0, lam, nu):
    with open(path, "wb") as f:
        f.write(struct.pack("<3I", sc.n, sc.nb, steps))
        f.write(struct.pack("<11f", sc.h, sc.rho0, nu, dt0, lam, *sc.box_min, *sc.box_max))
        for k in ("x", "y", "z", "vx", "vy", "vz", "m", "id"):
            f.write(np.ascontiguousarray(sc.fluid[k], np.float32).tobytes())
        for a in (sc.bdy["x"], sc.bdy["y"], sc.bdy["z"], bm):
            f.write(np.ascontiguousarray(a, np.float32).tobytes())


def read_out(path, n):
    raw = open(path, "rb").read()
    steps = struct.unpack("<I", raw[:4])[0]
    iters = np.frombuffer(raw[4:4 + 4 * steps], np.uint32)
    dts = np.frombuffer(raw[4 + 4 * steps:4 + 8 * steps], np.float32)
    body = np.frombuffer(raw[4 + 8 * steps:], np.float32).reshape(7, n)
    return iters, dts, dict(zip(("x", "y", "z", "vx", "vy", "vz", "id"), body))


@pytest.mark.parametrize("mode", [[], ["unsorted"]])
def test_cpp_main_loop_matches_oracle(cuda, tmp_path, mode):
    """The main loop with the solver on reordered state and, with
    "unsorted", on grids built by construct (IISPH<C2, Resort::no>)."""
    exe = compile_main_loop(str(tmp_path))
    sc = scenes.dam_break((14, 12, 10), 0.02, (0.5, 0.5, 0.5), velocity_noise=0.02, seed=21)
    bm = oracle.boundary_masses(sc.bdy["x"], sc.bdy["y"], sc.bdy["z"], sc.h, sc.rho0, 5)
    steps, dt0, lam, nu = 3, 1e-3, 0.4, 0.01
    inp = os.path.join(str(tmp_path), "in.bin")
    out = os.path.join(str(tmp_path), "out.bin")
    write_scene(inp, sc, bm, steps, dt0, lam, nu)
    subprocess.run([exe, inp, out] + mode, check=True)
    iters, dts, got = read_out(out, sc.n)
    if mode:  # the particles kept their order
        np.testing.assert_array_equal(got["id"], np.asarray(sc.fluid["id"], np.float32))

    # the same loop on the oracle
    fl = {k: v.copy() for k, v in sc.fluid.items()}
    p = np.zeros(sc.n, np.float32)
    prm = oracle.reference_params(2, 0, sc.h, sc.rho0, nu)
    it, dt = 0, dt0
    want_iters, want_dts = [], []
    for _ in range(steps):
        dt = float(oracle.lib().orc_dt_controller(it, dt, lam, sc.h, sc.n, fl["vx"], fl["vy"],
                                                  fl["vz"], oracle.f32([0, -9.81, 0]), 10,
                                                  0.001))
        r = oracle.run(prm, fl, dict(sc.bdy, m=bm), sc.box_min, sc.box_max, dt, 1, p0=p)
        fl, p, it = dict(r.state), r.p, int(r.iters[0])
        want_iters.append(it)
        want_dts.append(dt)
    assert list(iters) == want_iters
    np.testing.assert_allclose(dts, want_dts, rtol=1e-5)
    go = np.argsort(got["id"])
    wo = np.argsort(fl["id"])
    for k in ("x", "y", "z"):
        assert_close(got[k][go], fl[k][wo], 1e-6, 1e-6, k)
    for k in ("vx", "vy", "vz"):
        assert_close(got[k][go], fl[k][wo], 1e-3, 1e-3, k)


def test_cpp_main_loop_fused_tail_is_bit_identical(cuda, tmp_path):
    """The same C++ loop with the fused tail (next_dt + step_bounded)
    reproduces the separate calls bit for bit."""
    exe = compile_main_loop(str(tmp_path))
    sc = scenes.dam_break((14, 12, 10), 0.02, (0.5, 0.5, 0.5), velocity_noise=0.02, seed=22)
    bm = oracle.boundary_masses(sc.bdy["x"], sc.bdy["y"], sc.bdy["z"], sc.h, sc.rho0, 5)
    inp = os.path.join(str(tmp_path), "in.bin")
    write_scene(inp, sc, bm, 4, 1e-3, 0.4, 0.01)
    res = []
    for mode in ([], ["fused"]):
        out = os.path.join(str(tmp_path), f"out{len(mode)}.bin")
        subprocess.run([exe, inp, out] + mode, check=True)
        res.append(read_out(out, sc.n))
    (ia, da, a), (ib, db, b) = res
    assert list(ia) == list(ib)
    np.testing.assert_array_equal(da, db)
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


def test_cpp_step_graph_is_bit_identical(cuda, tmp_path):
    """The fixed-dt loop as StepGraph replays reproduces the plain calls bit
    for bit, with the same sweep counts."""
    exe = compile_main_loop(str(tmp_path))
    sc = scenes.dam_break((14, 12, 10), 0.02, (0.5, 0.5, 0.5), velocity_noise=0.02, seed=23)
    bm = oracle.boundary_masses(sc.bdy["x"], sc.bdy["y"], sc.bdy["z"], sc.h, sc.rho0, 5)
    inp = os.path.join(str(tmp_path), "in.bin")
    write_scene(inp, sc, bm, 4, 1e-3, 0.4, 0.01)
    res = []
    for mode in ("fixed", "graph"):
        out = os.path.join(str(tmp_path), f"out_{mode}.bin")
        subprocess.run([exe, inp, out, mode], check=True)
        res.append(read_out(out, sc.n))
    (ia, _, a), (ib, _, b) = res
    assert list(ia) == list(ib) and min(ia) >= 3
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


def test_cpp_mesh_adapters(cuda, tmp_path):
    """DeviceMesh / uniform_sample_mesh / relax_sampling / LBVH::project /
    BoundarySamples in the reference's calling pattern (tests/cpp/mesh_adapter.cpp)"""
    exe = os.path.join(str(tmp_path), "mesh_adapter")
    cxx = shutil.which("g++") or "g++"
    subprocess.run([cxx, "-std=c++17", "-O2", "-I" + os.path.join(ROOT, "include"),
                    "-I/usr/local/cuda/include", os.path.join(ROOT, "tests", "cpp",
                                                              "mesh_adapter.cpp"),
                    "-L" + os.path.join(ROOT, "reyn_b200"), "-lreyn_b200",
                    "-L/usr/local/cuda/lib64", "-lcudart",
                    "-Wl,-rpath," + os.path.join(ROOT, "reyn_b200"), "-o", exe], check=True)
    out = subprocess.run([exe, "1.0"], capture_output=True, text=True, check=True).stdout.split()
    n = int(out[0])
    # octahedron of "radius" 1: 8 equilateral faces of side sqrt(2)
    area = 8 * np.sqrt(3) / 4 * 2.0
    assert n == oracle.mesh_sample_count(area, 0.05, 2.0)
    first, last = out[1].split(","), out[2].split(",")
    assert first[0] == "1" and last[0] == "10"
    assert float(last[1]) < float(first[1])       # max/min number density ratio falls
    assert float(out[3]) < 1e-5                    # every sample on the surface
    assert float(out[4]) == pytest.approx(4.0 / 3.0, rel=1e-12)


@pytest.mark.parametrize("order,ratio", [("xyz", "0.5"), ("xyz", "1.0"), ("zorder", "0.5")])
def test_cpp_user_kernel_ff_nbrs(cuda, tmp_path, order, ratio):
    """UniformGrid<R>::ff_nbrs from a user kernel (tests/cpp/ff_nbrs.cu),
    Resort::no and Resort::yes: neighbour counts exactly and |x_ij|^2 sums
    within 1e-5 of the engine's neighbour statistics."""
    exe = os.path.join(str(tmp_path), "ff_nbrs")
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    subprocess.run([nvcc, "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "ff_nbrs.cu"),
                    "-L" + os.path.join(ROOT, "reyn_b200"), "-lreyn_b200",
                    "-Xlinker", "-rpath," + os.path.join(ROOT, "reyn_b200"), "-o", exe],
                   check=True)
    r = subprocess.run([exe, order, ratio], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr


def _scene_obj(path):
    """A container (shape "walls") with a fluid block (shape "fluid") inside."""
    from reyn_b200 import meshes
    walls = meshes.box((0.0, 0.0, 0.0), (1.0, 0.6, 0.6), 2)
    fluid = meshes.box((0.05, 0.05, 0.05), (0.45, 0.4, 0.4), 1)
    meshes.write_obj(path, [("walls", *walls), ("fluid", *fluid)])
    return walls, fluid


def _read_scene(path):
    raw = open(path, "rb").read()
    n, nb, steps = struct.unpack("<3I", raw[:12])
    geo = np.frombuffer(raw[12:40], np.float32)
    off = 40
    arr = np.frombuffer(raw[off:off + 4 * 3 * n], np.float32).reshape(3, n)
    off += 12 * n
    bdy = np.frombuffer(raw[off:off + 12 * nb], np.float32).reshape(3, nb)
    off += 12 * nb
    iters = np.frombuffer(raw[off:off + 4 * steps], np.uint32)
    off += 4 * steps
    fin = np.frombuffer(raw[off:], np.float32).reshape(3, n)
    return n, float(geo[0]), geo[1:4], geo[4:7], arr.T, bdy.T, iters, fin.T


def _compile_scene_loop(tmp):
    exe = os.path.join(tmp, "scene_loop")
    cxx = shutil.which("g++") or "g++"
    subprocess.run([cxx, "-std=c++17", "-O2", "-I" + os.path.join(ROOT, "include"),
                    "-I/usr/local/cuda/include",
                    os.path.join(ROOT, "tests", "cpp", "scene_loop.cpp"),
                    "-L" + os.path.join(ROOT, "reyn_b200"), "-lreyn_b200",
                    "-L/usr/local/cuda/lib64", "-lcudart",
                    "-Wl,-rpath," + os.path.join(ROOT, "reyn_b200"), "-o", exe], check=True)
    return exe


@pytest.mark.parametrize("mode", ["obj", "box"])
def test_cpp_scene_main_loop(cuda, tmp_path, mode):
    """The reference's main loop with its Scene (Scene::from_obj, or the box
    constructor), oversampling 3 and cull radius 1h as main.cu:43-44 has it:
    spacing from the fluid volume (or the box) and the desired count, the
    fluid lattice filled inside the "fluid" shape, every particle with a
    boundary sample within h culled, the rest jittered by at most sqrt(3)
    0.01 h, scene bounds holding boundary and fluid; then IISPH steps keep
    every particle inside the bounds."""
    from scipy.spatial import cKDTree
    exe = _compile_scene_loop(str(tmp_path))
    obj = os.path.join(str(tmp_path), "scene.obj")
    walls, fluid = _scene_obj(obj)
    out = os.path.join(str(tmp_path), "out.bin")
    n_desired, steps = 20000, 3
    subprocess.run([exe, obj, out, mode, str(n_desired), str(steps)], check=True)
    n, h, lo, hi, x0, bdy, iters, x1 = _read_scene(out)
    if mode == "obj":
        # the "fluid" shape as loaded: the reference's loader keeps every
        # vertex of the file, so the mesh's (and its LBVH's) bounds span all
        # shapes and the fill lattice starts at the file's lowest vertex
        verts = np.concatenate([np.asarray(walls[0], float), np.asarray(fluid[0], float)])
        faces = np.asarray(fluid[1], np.int64) + len(walls[0])
        vol = oracle.mesh_measure(verts, faces)[1]
        assert h == pytest.approx(float(np.float32(np.cbrt(vol / n_desired))), rel=1e-6)
        lx, ly, lz = oracle.mesh_fill(verts, faces, h)
        lat = np.stack([lx, ly, lz], 1)
        fmin = verts.min(0).astype(np.float32)
        fmax = verts.max(0).astype(np.float32)
        np.testing.assert_allclose(lo, np.minimum(bdy.min(0), fmin - np.float32(0.5 * h)),
                                   rtol=1e-6)
        np.testing.assert_allclose(hi, np.maximum(bdy.max(0), fmax + np.float32(0.5 * h)),
                                   rtol=1e-6)
    else:
        f32 = np.float32
        ext = [f32(0.45) - f32(0.05), f32(0.4) - f32(0.05), f32(0.4) - f32(0.05)]
        assert h == pytest.approx(float(np.cbrt(ext[0] * ext[1] * ext[2] / f32(n_desired))),
                                  rel=1e-6)
        cnt = [int(np.floor(e / f32(h))) for e in ext]
        i, j, k = np.meshgrid(*(np.arange(c) for c in cnt), indexing="ij")
        lat = np.stack([np.float32(0.05) + i.T.ravel() * np.float32(h),
                        np.float32(0.05) + j.T.ravel() * np.float32(h),
                        np.float32(0.05) + k.T.ravel() * np.float32(h)], 1).astype(np.float32)
        np.testing.assert_array_equal(lo, bdy.min(0))
        np.testing.assert_array_equal(hi, bdy.max(0))
    d, _ = cKDTree(bdy.astype(np.float64)).query(lat.astype(np.float64))
    near = np.abs(d - h) < 1e-5 * h  # ties at the cull radius may go either way
    kept = d > h
    assert kept.sum() <= n <= (kept | near).sum()
    if not near.any():
        dev = np.abs(x0 - lat[kept])
        # the amplitude plus the rounding of the jittered coordinate
        assert dev.max() <= np.sqrt(3.0) * 0.01 * h + 4 * np.finfo(np.float32).eps * np.abs(
            lat).max()
        assert dev.max() > 0.5 * 0.01 * h  # jitter applied
    assert len(iters) == steps and min(iters) >= 3
    assert np.isfinite(x1).all()
    assert (x1 >= lo).all() and (x1 <= hi).all()
