"""CPU oracle — TEST INFRASTRUCTURE ONLY.

ctypes bindings for two checkers, never for the product:

* ``liboracle.so`` (oracle/oracle.cpp): a host C++/OpenMP restatement of the
  reference's (reyn) SPH hot path: smoothing kernels, counting-sort uniform
  grid, ``ff_nbrs`` traversal, SESPH/PCISPH/IISPH steps, CFL, bounds, Akinci
  boundary masses, and (oracle/mesh.cpp) the triangle-mesh path: LBVH build
  and queries, surface sampling, relaxation and the fluid fill. It is the
  checker for the CUDA engine and the timed CPU baseline.
* ``_ref/libreyn_ref*.so`` (oracle/ref/): the reference's OWN sources compiled
  unmodified (kernel classes on the host; the CUDA path for a B200), used to
  pin the oracle and to generate the golden fixtures in tests/golden/.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this package.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_HOST_PATH = os.path.join(HERE, "_ref", "libreyn_ref_host.so")
REF_CUDA_PATH = os.path.join(HERE, "_ref", "libreyn_ref.so")
# the reference checkout (its src/ is compiled into _ref/ when present);
# REYN_REFERENCE overrides the default location
REFERENCE_SRC = os.path.join(os.environ.get("REYN_REFERENCE", "/root/reference"), "src")

SESPH, PCISPH, IISPH = 0, 1, 2
C2, B3, W6, COS = 0, 1, 2, 3

_lib = None
_ref_host = None
_ref_cuda = None

_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")


def build(force: bool = False) -> None:
    """Compile liboracle.so (and, where the reference sources are present,
    the reference libraries under oracle/_ref)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.check_call(["make", "-s", "-C", HERE])
    if os.path.isdir(REFERENCE_SRC):
        subprocess.check_call(["make", "-s", "-j8", "-C", os.path.join(HERE, "ref"),
                               "REF=" + os.path.dirname(REFERENCE_SRC)])


class Geom(ctypes.Structure):
    _fields_ = [
        ("bmin", ctypes.c_float * 3),
        ("cell", ctypes.c_float),
        ("r2", ctypes.c_float),
        ("nx", ctypes.c_int32),
        ("ny", ctypes.c_int32),
        ("nz", ctypes.c_int32),
        ("range", ctypes.c_int32),
        ("order", ctypes.c_int32),
    ]

    @property
    def n_cells(self) -> int:
        return self.nx * self.ny * self.nz

    @property
    def n_keys(self) -> int:
        return int(lib().orc_keys(ctypes.byref(self)))


class Params(ctypes.Structure):
    _fields_ = [
        ("scheme", ctypes.c_int),
        ("kind", ctypes.c_int),
        ("h", ctypes.c_float),
        ("rho0", ctypes.c_float),
        ("nu", ctypes.c_float),
        ("g", ctypes.c_float * 3),
        ("k_sesph", ctypes.c_float),
        ("eta", ctypes.c_float),
        ("min_iter", ctypes.c_uint32),
        ("max_iter", ctypes.c_uint32),
        ("omega", ctypes.c_float),
        ("warmstart", ctypes.c_int),
        ("iisph_avg", ctypes.c_int),
        ("cell_ratio", ctypes.c_float),
        ("projected", ctypes.c_int),
    ]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.orc_geometry.argtypes = [_f32p, _f32p, ctypes.c_float, ctypes.c_float, ctypes.POINTER(Geom)]
        L.orc_geometry_order.argtypes = [_f32p, _f32p, ctypes.c_float, ctypes.c_float, ctypes.c_int,
                                         ctypes.POINTER(Geom)]
        L.orc_keys.argtypes = [ctypes.POINTER(Geom)]
        L.orc_keys.restype = ctypes.c_int64
        L.orc_kernel_eval.argtypes = [ctypes.c_int, ctypes.c_float, ctypes.c_uint32] + [_f32p] * 7
        L.orc_grid_build.argtypes = [ctypes.POINTER(Geom), ctypes.c_uint32, _f32p, _f32p, _f32p,
                                     _u32p, _u32p, ctypes.c_void_p]
        L.orc_neighbours.argtypes = [ctypes.POINTER(Geom), ctypes.c_uint32, _f32p, _f32p, _f32p,
                                     _u32p, _u32p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                     ctypes.c_void_p, ctypes.c_void_p]
        L.orc_brute_count.argtypes = [ctypes.c_uint32, _f32p, _f32p, _f32p, ctypes.c_float, _u32p,
                                      ctypes.c_void_p]
        L.orc_boundary_masses.argtypes = [ctypes.c_uint32, _f32p, _f32p, _f32p, ctypes.c_float,
                                          ctypes.c_float, ctypes.c_uint32, _f32p]
        L.orc_boundary_masses_kernel.argtypes = [ctypes.c_uint32, _f32p, _f32p, _f32p,
                                                 ctypes.c_float, ctypes.c_float, ctypes.c_uint32,
                                                 ctypes.c_int, _f32p]
        L.orc_cfl.argtypes = [ctypes.c_uint32, _f32p, _f32p, _f32p, ctypes.c_float, ctypes.c_float,
                              _f32p]
        L.orc_cfl.restype = ctypes.c_float
        L.orc_dt_controller.argtypes = [ctypes.c_uint32, ctypes.c_float, ctypes.c_float,
                                        ctypes.c_float, ctypes.c_uint32, _f32p, _f32p, _f32p,
                                        _f32p, ctypes.c_uint32, ctypes.c_float]
        L.orc_dt_controller.restype = ctypes.c_float
        L.orc_params_reference.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                           ctypes.c_float, ctypes.c_float, ctypes.POINTER(Params)]
        L.orc_run.argtypes = [ctypes.POINTER(Params), ctypes.c_uint32] + [_f32p] * 9 + [
            ctypes.c_uint32, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p, ctypes.c_float,
            ctypes.c_uint32] + [ctypes.c_void_p] * 6 + [_u32p]
        L.orc_threads.restype = ctypes.c_int
        _d = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
        mesh = [_d, _d, _d, ctypes.c_uint32, _u32p, ctypes.c_uint32]
        vp = ctypes.c_void_p
        L.orc_mesh_morton.argtypes = mesh + [_u32p]
        L.orc_lbvh_build.argtypes = mesh + [vp] * 6
        L.orc_lbvh_query.argtypes = mesh + [ctypes.c_uint32, _f32p, _f32p, _f32p, vp]
        L.orc_project_brute.argtypes = mesh + [ctypes.c_uint32, _f32p, _f32p, _f32p]
        L.orc_mesh_measure.argtypes = mesh + [vp, vp, vp]
        L.orc_mesh_sample_count.argtypes = [ctypes.c_double, ctypes.c_float, ctypes.c_float]
        L.orc_mesh_sample_count.restype = ctypes.c_uint32
        L.orc_mesh_sample.argtypes = mesh + [ctypes.c_float, ctypes.c_float, ctypes.c_uint64,
                                             ctypes.c_uint32, vp, vp, vp, _u32p]
        L.orc_hex_plane_density.argtypes = [ctypes.c_float]
        L.orc_hex_plane_density.restype = ctypes.c_float
        L.orc_mesh_relax_sweep.argtypes = mesh + [ctypes.c_uint32, _f32p, _f32p, _f32p,
                                                  ctypes.c_float, ctypes.c_float, _f32p]
        L.orc_mesh_fill.argtypes = mesh + [ctypes.c_float, ctypes.c_float, ctypes.c_uint64,
                                           ctypes.c_uint32, vp, vp, vp, _u32p]
        _lib = L
    return _lib


def _vp(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def geometry(bmin, bmax, r: float, cell_ratio: float = 0.5, order: int = 0) -> Geom:
    g = Geom()
    rc = lib().orc_geometry_order(f32(bmin), f32(bmax), r, cell_ratio, order, ctypes.byref(g))
    if rc:
        raise ValueError(f"orc_geometry failed ({rc})")
    return g


def kernel_eval(kind: int, h_bar: float, dx, dy, dz):
    dx, dy, dz = f32(dx), f32(dy), f32(dz)
    n = dx.size
    w, gx, gy, gz = (np.zeros(n, np.float32) for _ in range(4))
    rc = lib().orc_kernel_eval(kind, h_bar, n, dx, dy, dz, w, gx, gy, gz)
    if rc:
        raise ValueError(rc)
    return w, gx, gy, gz


def grid_build(g: Geom, x, y, z):
    x, y, z = f32(x), f32(y), f32(z)
    n = x.size
    prefix = np.zeros(g.n_keys + 1, np.uint32)
    sorted_ = np.zeros(max(n, 1), np.uint32)
    keys = np.zeros(max(n, 1), np.uint32)
    rc = lib().orc_grid_build(ctypes.byref(g), n, x, y, z, prefix, sorted_, _vp(keys))
    if rc:
        raise ValueError(f"orc_grid_build failed ({rc})")
    return prefix, sorted_[:n], keys[:n]


def neighbours(g: Geom, x, y, z, prefix, sorted_, kind=None, m=None):
    x, y, z = f32(x), f32(y), f32(z)
    n = x.size
    count = np.zeros(n, np.uint32)
    len2 = np.zeros(n, np.float32)
    rho = np.zeros(n, np.float32) if m is not None else None
    mm = f32(m) if m is not None else None
    rc = lib().orc_neighbours(ctypes.byref(g), n, x, y, z, np.ascontiguousarray(prefix, np.uint32),
                              np.ascontiguousarray(sorted_, np.uint32), _vp(count), _vp(len2),
                              -1 if kind is None else kind, _vp(mm), _vp(rho))
    if rc:
        raise ValueError(rc)
    return count, len2, rho


def brute_count(x, y, z, r: float):
    x, y, z = f32(x), f32(y), f32(z)
    count = np.zeros(x.size, np.uint32)
    len2 = np.zeros(x.size, np.float32)
    lib().orc_brute_count(x.size, x, y, z, r, count, _vp(len2))
    return count, len2


def boundary_masses(bx, by, bz, h: float, rho0: float, iters: int = 5, kind: int = B3):
    bx, by, bz = f32(bx), f32(by), f32(bz)
    m = np.zeros(bx.size, np.float32)
    rc = lib().orc_boundary_masses_kernel(bx.size, bx, by, bz, h, rho0, iters, kind, m)
    if rc:
        raise ValueError(rc)
    return m


def cfl(vx, vy, vz, lam: float, h: float, g) -> float:
    vx, vy, vz = f32(vx), f32(vy), f32(vz)
    return float(lib().orc_cfl(vx.size, vx, vy, vz, lam, h, f32(g)))


def reference_params(scheme: int, kind: int, h: float, rho0: float, nu: float) -> Params:
    p = Params()
    lib().orc_params_reference(scheme, kind, h, rho0, nu, ctypes.byref(p))
    return p


@dataclass
class RunResult:
    state: dict
    rho: np.ndarray
    p: np.ndarray
    aii: np.ndarray
    sii: np.ndarray
    a: np.ndarray
    iters: np.ndarray


def run(params: Params, fluid: dict, bdy: dict, scene_min, scene_max, dt: float, steps: int,
        p0=None) -> RunResult:
    """Runs `steps` reference main-loop iterations on copies of `fluid`
    (keys x,y,z,vx,vy,vz,m,id) with boundary `bdy` (keys x,y,z,m)."""
    st = {k: f32(fluid[k]).copy() for k in ("x", "y", "z", "vx", "vy", "vz", "m", "id")}
    n = st["x"].size
    p = f32(p0).copy() if p0 is not None else np.zeros(n, np.float32)
    out = {k: np.zeros(n, np.float32) for k in ("rho", "aii", "sii", "ax", "ay", "az")}
    iters = np.zeros(max(steps, 1), np.uint32)
    nb = f32(bdy["x"]).size
    e = np.zeros(1, np.float32)
    bx, by, bz, bm = (f32(bdy[k]) if nb else e for k in ("x", "y", "z", "m"))
    rc = lib().orc_run(ctypes.byref(params), n, st["x"], st["y"], st["z"], st["vx"], st["vy"],
                       st["vz"], st["m"], st["id"], p, nb, bx, by, bz, bm, f32(scene_min),
                       f32(scene_max), dt, steps, *(_vp(out[k]) for k in
                                                    ("rho", "aii", "sii", "ax", "ay", "az")),
                       iters)
    if rc:
        raise ValueError(f"orc_run failed ({rc})")
    return RunResult(st, out["rho"], p, out["aii"], out["sii"],
                     np.stack([out["ax"], out["ay"], out["az"]], 1), iters[:steps])


def threads() -> int:
    return int(lib().orc_threads())


# ---- the reference itself ---------------------------------------------------

def ref_host():
    """The reference's kernel classes compiled for the host (no GPU needed)."""
    global _ref_host
    if _ref_host is None:
        if not os.path.exists(REF_HOST_PATH):
            raise FileNotFoundError(REF_HOST_PATH)
        L = ctypes.CDLL(REF_HOST_PATH)
        L.ref_kernel_eval_host.argtypes = [ctypes.c_int, ctypes.c_float, ctypes.c_uint] + [_f32p] * 7
        _ref_host = L
    return _ref_host


def ref_kernel_eval_host(kind: int, h_bar: float, dx, dy, dz):
    dx, dy, dz = f32(dx), f32(dy), f32(dz)
    n = dx.size
    w, gx, gy, gz = (np.zeros(n, np.float32) for _ in range(4))
    if ref_host().ref_kernel_eval_host(kind, h_bar, n, dx, dy, dz, w, gx, gy, gz):
        raise ValueError(kind)
    return w, gx, gy, gz


def ref_cuda():
    """The reference's CUDA path compiled for sm_100a (needs a GPU to run)."""
    global _ref_cuda
    if _ref_cuda is None:
        if not os.path.exists(REF_CUDA_PATH):
            raise FileNotFoundError(REF_CUDA_PATH)
        L = ctypes.CDLL(REF_CUDA_PATH)
        L.ref_last_error.restype = ctypes.c_char_p
        _ref_cuda = L
    return _ref_cuda


# ---- triangle meshes (oracle/mesh.cpp) -------------------------------------------

def _mesh_args(verts, faces):
    v = np.ascontiguousarray(verts, np.float64).reshape(-1, 3)
    f = np.ascontiguousarray(faces, np.uint32).reshape(-1)
    return (np.ascontiguousarray(v[:, 0]), np.ascontiguousarray(v[:, 1]),
            np.ascontiguousarray(v[:, 2]), v.shape[0], f, f.size // 3)


def _ok(rc):
    if rc:
        raise ValueError(f"oracle mesh call failed ({rc})")


def mesh_morton(verts, faces) -> np.ndarray:
    a = _mesh_args(verts, faces)
    codes = np.zeros(a[5], np.uint32)
    _ok(lib().orc_mesh_morton(*a, codes))
    return codes


def lbvh_build(verts, faces) -> dict:
    """The LBVH of a mesh: leaf order, ChildNode-encoded children, boxes
    (n x 6: min xyz, max xyz) and height."""
    a = _mesh_args(verts, faces)
    nf = a[5]
    order = np.zeros(nf, np.uint32)
    cl = np.zeros(max(nf - 1, 1), np.uint32)
    cr = np.zeros(max(nf - 1, 1), np.uint32)
    leaf = np.zeros((nf, 6), np.float32)
    node = np.zeros((max(nf - 1, 1), 6), np.float32)
    height = np.zeros(1, np.uint32)
    _ok(lib().orc_lbvh_build(*a, _vp(order), _vp(cl), _vp(cr), _vp(leaf), _vp(node),
                             _vp(height)))
    return {"order": order, "children_l": cl[:nf - 1], "children_r": cr[:nf - 1],
            "leaf_box": leaf, "node_box": node[:nf - 1], "height": int(height[0])}


def lbvh_project(verts, faces, x, y, z):
    x, y, z = f32(x).copy(), f32(y).copy(), f32(z).copy()
    _ok(lib().orc_lbvh_query(*_mesh_args(verts, faces), x.size, x, y, z, None))
    return x, y, z


def lbvh_inside(verts, faces, x, y, z) -> np.ndarray:
    x, y, z = f32(x).copy(), f32(y).copy(), f32(z).copy()
    inside = np.zeros(x.size, np.uint8)
    _ok(lib().orc_lbvh_query(*_mesh_args(verts, faces), x.size, x, y, z, _vp(inside)))
    return inside


def project_brute(verts, faces, x, y, z):
    x, y, z = f32(x).copy(), f32(y).copy(), f32(z).copy()
    _ok(lib().orc_project_brute(*_mesh_args(verts, faces), x.size, x, y, z))
    return x, y, z


def mesh_measure(verts, faces):
    """(total area, volume, inclusive area sums)"""
    a = _mesh_args(verts, faces)
    area = np.zeros(1)
    vol = np.zeros(1)
    cdf = np.zeros(a[5])
    _ok(lib().orc_mesh_measure(*a, _vp(area), _vp(vol), _vp(cdf)))
    return float(area[0]), float(vol[0]), cdf


def mesh_sample_count(area: float, h: float, oversampling: float) -> int:
    return int(lib().orc_mesh_sample_count(area, h, oversampling))


def mesh_sample(verts, faces, h: float, oversampling: float, seed: int):
    a = _mesh_args(verts, faces)
    cnt = np.zeros(1, np.uint32)
    _ok(lib().orc_mesh_sample(*a, h, oversampling, seed, 0, None, None, None, cnt))
    n = int(cnt[0])
    x, y, z = (np.zeros(max(n, 1), np.float32) for _ in range(3))
    _ok(lib().orc_mesh_sample(*a, h, oversampling, seed, n, _vp(x), _vp(y), _vp(z), cnt))
    return x[:n], y[:n], z[:n]


def hex_plane_density(h_bdy: float) -> float:
    return float(lib().orc_hex_plane_density(h_bdy))


def mesh_relax_sweep(verts, faces, x, y, z, h_bdy: float, k: float):
    """One relaxation sweep; returns (x, y, z, number densities)."""
    x, y, z = f32(x).copy(), f32(y).copy(), f32(z).copy()
    nd = np.zeros(x.size, np.float32)
    _ok(lib().orc_mesh_relax_sweep(*_mesh_args(verts, faces), x.size, x, y, z, h_bdy, k, nd))
    return x, y, z, nd


def mesh_fill(verts, faces, h: float, jitter: float = 0.0, seed: int = 1):
    a = _mesh_args(verts, faces)
    cnt = np.zeros(1, np.uint32)
    _ok(lib().orc_mesh_fill(*a, h, jitter, seed, 0, None, None, None, cnt))
    n = int(cnt[0])
    x, y, z = (np.zeros(max(n, 1), np.float32) for _ in range(3))
    _ok(lib().orc_mesh_fill(*a, h, jitter, seed, n, _vp(x), _vp(y), _vp(z), cnt))
    return x[:n], y[:n], z[:n]
