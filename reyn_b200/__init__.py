"""reyn_b200 — Python binding of the B200 SPH step engine's C ABI
(include/reyn_b200.h) through ctypes.

The engine itself is CUDA C++ (reyn_b200/csrc, built in-tree into
libreyn_b200.so by ``python -m reyn_b200.build``). This module only marshals
arguments; device memory for inputs/outputs is owned by torch tensors or by
the engine's own handles. There is no CPU fallback: every call fails loudly if
the library or a GPU is missing.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libreyn_b200.so")

C2, B3, W6, COS = 0, 1, 2, 3
KERNELS = {"C2": C2, "B3": B3, "W6": W6, "COS": COS}
SESPH, PCISPH, IISPH = 0, 1, 2
CONV_REFERENCE, CONV_AVERAGE = 0, 1
PRECISION_FP32, PRECISION_MIXED, PRECISION_MIXED_POS16 = 0, 1, 2
ORDER_XYZ, ORDER_ZORDER = 0, 1

OK = 0
ERR_INVALID, ERR_OUT_OF_BOUNDS, ERR_NONFINITE, ERR_ITER_LIMIT = -1, -2, -3, -4
ERR_CUDA, ERR_ALLOC, ERR_NOT_READY = -5, -6, -7

_vp = ctypes.c_void_p
_f = ctypes.c_float
_u32 = ctypes.c_uint32


class ReynError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"reyn_b200 error {code}: {msg}")
        self.code = code


class Soa(ctypes.Structure):
    _fields_ = [("xx", _vp), ("xy", _vp), ("xz", _vp), ("vx", _vp), ("vy", _vp), ("vz", _vp),
                ("m", _vp), ("n", _u32), ("rho0", _f)]


class GridInfo(ctypes.Structure):
    _fields_ = [("bound_min", _f * 3), ("cell_size", _f), ("r_c_2", _f), ("nx", ctypes.c_int32),
                ("ny", ctypes.c_int32), ("nz", ctypes.c_int32), ("nxny", ctypes.c_int32),
                ("range", ctypes.c_int32), ("n", _u32), ("prefix", _vp), ("sorted", _vp),
                ("order", ctypes.c_int32), ("n_keys", _u32)]


class Params(ctypes.Structure):
    _fields_ = [("kernel", ctypes.c_int), ("h", _f), ("rho0", _f), ("nu", _f), ("g", _f * 3),
                ("k_sesph", _f), ("eta", _f), ("min_iter", _u32), ("max_iter", _u32),
                ("omega", _f), ("warmstart", ctypes.c_int32), ("convergence", ctypes.c_int),
                ("precision", ctypes.c_int), ("block_size", _u32)]


class TunePoint(ctypes.Structure):
    _fields_ = [("block_size", _u32), ("cell_ratio", _f), ("ms_per_step", _f)]


class Diag(ctypes.Structure):
    _fields_ = [("mass", ctypes.c_double), ("momentum", ctypes.c_double * 3),
                ("kinetic", ctypes.c_double)]


class SolverBuffers(ctypes.Structure):
    _fields_ = [("rho", _vp), ("p", _vp), ("aii", _vp), ("sii", _vp), ("ax", _vp), ("ay", _vp),
                ("az", _vp), ("n", _u32)]


class ProfileEntry(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 48), ("launches", ctypes.c_uint64),
                ("total_ms", ctypes.c_double)]


class MeshInfo(ctypes.Structure):
    _fields_ = [("n_vertices", _u32), ("n_faces", _u32), ("tree_height", _u32),
                ("reserved", _u32), ("bounds_min", ctypes.c_double * 3),
                ("bounds_max", ctypes.c_double * 3), ("area", ctypes.c_double),
                ("volume", ctypes.c_double)]


class StepStats(ctypes.Structure):
    _fields_ = [("iters", _u32), ("avg_density_error", ctypes.c_double),
                ("max_density_error", ctypes.c_double)]


_lib = None

# (name, argtypes) of every entry point in include/reyn_b200.h
_SIGNATURES = {
    "reyn_last_error": [],
    "reyn_abi_version": [],
    "reyn_kernel_eval": [ctypes.c_int, _f, _vp, _vp, _vp, _u32, _vp, _vp, _vp, _vp, _vp],
    "reyn_particles_create": [_u32, _f, ctypes.POINTER(_vp)],
    "reyn_particles_destroy": [_vp],
    "reyn_particles_soa": [_vp, ctypes.POINTER(Soa)],
    "reyn_particles_count": [_vp, ctypes.POINTER(_u32)],
    "reyn_particles_reorder": [_vp, _vp, _vp],
    "reyn_particles_resize": [_vp, _u32, ctypes.c_int, _vp],
    "reyn_boundary_bounds": [_vp, _vp, _vp],
    "reyn_scene_jitter": [_vp, _u32, _u32, _f, ctypes.c_uint64, _vp],
    "reyn_particles_upload": [_vp] + [_vp] * 7 + [_vp],
    "reyn_particles_download": [_vp] + [_vp] * 7 + [_vp],
    "reyn_particles_download_async": [_vp] + [_vp] * 7 + [_vp],
    "reyn_grid_create": [_f * 3, _f * 3, _f, _f, ctypes.c_int, ctypes.POINTER(_vp)],
    "reyn_grid_destroy": [_vp],
    "reyn_grid_construct": [_vp, _f, _vp, _vp, _vp, _u32, _vp],
    "reyn_grid_construct_and_reorder": [_vp, _f, _vp, ctypes.POINTER(_vp), _u32, _vp],
    "reyn_grid_info_get": [_vp, ctypes.POINTER(GridInfo)],
    "reyn_grid_reorder": [_vp, _vp, ctypes.POINTER(_vp), _u32, _vp],
    "reyn_grid_permutation": [_vp, ctypes.POINTER(_vp)],
    "reyn_grid_neighbour_stats": [_vp, _vp, _vp, _vp, _vp, ctypes.c_int, _vp, _vp, _vp, _vp],
    "reyn_compute_densities": [_vp, _vp, _vp, _vp, _vp, _vp, ctypes.c_int, _vp, _vp],
    "reyn_boundary_create": [_vp, _vp, _vp, _vp, _u32, _f, _f, _u32, _vp, ctypes.POINTER(_vp)],
    "reyn_boundary_destroy": [_vp],
    "reyn_boundary_arrays": [_vp] + [ctypes.POINTER(_vp)] * 4 + [ctypes.POINTER(_u32)],
    "reyn_params_reference": [ctypes.c_int, ctypes.c_int, _f, _f, _f, ctypes.POINTER(Params)],
    "reyn_solver_create": [ctypes.c_int, ctypes.POINTER(Params), _u32, ctypes.POINTER(_vp)],
    "reyn_solver_destroy": [_vp],
    "reyn_particles_save_ply": [_vp, ctypes.c_char_p, _vp],
    "reyn_particles_save_raw": [_vp, ctypes.c_char_p, _vp],
    "reyn_particles_load_raw": [_vp, ctypes.c_char_p, _vp],
    "reyn_scene_fluid_block": [_vp, _u32, _u32 * 3, _f * 3, _f, _f, _f, _f, ctypes.c_uint64,
                               _vp],
    "reyn_scene_box_walls": [_f * 3, _f * 3, _f, _vp, _vp, _vp, ctypes.c_uint64,
                             ctypes.POINTER(ctypes.c_uint64), _vp],
    "reyn_scene_sphere": [_f * 3, _f, _f, _vp, _vp, _vp, _u32, ctypes.POINTER(_u32), _vp],
    "reyn_scene_cull": [_vp, _vp, _f, ctypes.POINTER(_u32), _vp],
    "reyn_grid_create_batched": [_f, _f, ctypes.c_int, _u32, _vp, _vp, _vp, ctypes.POINTER(_vp)],
    "reyn_boundary_create_batched": [_vp, _vp, _vp, _vp, _u32, _u32, _vp, _f, _f, _u32, _vp,
                                     ctypes.POINTER(_vp)],
    "reyn_solver_step_batched": [_vp, _vp, _vp, _vp, _f, ctypes.c_int, _vp, _vp],
    "reyn_solver_scene_stats": [_vp, _u32, _vp],
    "reyn_autotune": [ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _u32, _vp, _vp, _vp, _f, _u32,
                      _vp, _vp, _vp],
    "reyn_autotune_reorder": [ctypes.c_int, _vp, _vp, _vp, _f * 3, _f * 3, _f, _f, _u32, _vp,
                              _u32, ctypes.POINTER(_u32), _vp, _vp],
    "reyn_diagnostics": [_vp, ctypes.POINTER(Diag), _vp],
    "reyn_solver_step": [_vp, _vp, _vp, _vp, _f, ctypes.POINTER(_u32), _vp],
    "reyn_solver_step_bounded": [_vp, _vp, _vp, _vp, _f, _f * 3, _f * 3, ctypes.POINTER(_u32),
                                 _vp],
    "reyn_solver_next_dt": [_vp, _vp, _u32, _f, _f, _f, _f * 3, _u32, _f, ctypes.POINTER(_f),
                            _vp],
    "reyn_solver_buffers_get": [_vp, ctypes.POINTER(SolverBuffers)],
    "reyn_solver_stats": [_vp, ctypes.POINTER(StepStats)],
    "reyn_cfl_time_step": [_vp, _f, _f, _f * 3, ctypes.POINTER(_f), _vp],
    "reyn_dt_controller": [_vp, _u32, _f, _f, _f, _f * 3, _u32, _f, ctypes.POINTER(_f), _vp],
    "reyn_enforce_bounds": [_vp, _f * 3, _f * 3, _vp],
    "reyn_solver_pressure_download": [_vp, _vp, _vp],
    "reyn_solver_pressure_upload": [_vp, _vp, _vp, _vp],
    "reyn_grid_construct_noalloc": [_f * 3, _f * 3, _f, _f, _vp, _vp, _vp, _u32, _vp,
                                    ctypes.c_uint64, _vp, ctypes.POINTER(ctypes.c_int32), _vp],
    "reyn_mesh_create": [_vp, _vp, _vp, _u32, _vp, _u32, _vp, ctypes.POINTER(_vp)],
    "reyn_mesh_load_obj": [ctypes.c_char_p, ctypes.POINTER(ctypes.c_char_p), _u32,
                           ctypes.c_char_p, _vp, ctypes.POINTER(_vp)],
    "reyn_mesh_destroy": [_vp],
    "reyn_mesh_info_get": [_vp, ctypes.POINTER(MeshInfo)],
    "reyn_mesh_tree": [_vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "reyn_mesh_project": [_vp, _vp, _vp, _vp, _u32, _vp],
    "reyn_mesh_inside": [_vp, _vp, _vp, _vp, _u32, _vp, _vp],
    "reyn_mesh_sample_uniform": [_vp, _f, _f, ctypes.c_uint64, _vp, _vp, _vp, _u32,
                                 ctypes.POINTER(_u32), _vp],
    "reyn_mesh_relax": [_vp, _vp, _vp, _vp, _u32, _f, _f, _u32, _vp, _vp, _vp],
    "reyn_mesh_fill": [_vp, _f, _f, ctypes.c_uint64, _vp, _vp, _vp, _u32, ctypes.POINTER(_u32),
                       _vp],
    "reyn_step_graph_create": [_vp, _vp, _vp, _vp, _f, ctypes.POINTER(_f), ctypes.POINTER(_f),
                               ctypes.POINTER(_vp)],
    "reyn_step_graph_launch": [_vp, _vp],
    "reyn_step_graph_stats": [_vp, ctypes.POINTER(StepStats), _vp],
    "reyn_step_graph_info": [_vp, ctypes.POINTER(_u32), ctypes.POINTER(_u32)],
    "reyn_step_graph_destroy": [_vp],
    "reyn_profile_enable": [ctypes.c_int],
    "reyn_profile_reset": [],
    "reyn_profile_read": [ctypes.POINTER(ProfileEntry), _u32, ctypes.POINTER(_u32)],
}


def declared_symbols() -> list[str]:
    """Entry points declared in include/reyn_b200.h."""
    return list(_SIGNATURES)


def lib():
    """The loaded engine library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m reyn_b200.build` "
                              "(the engine has no fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, args in _SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = ctypes.c_int
        L.reyn_last_error.restype = ctypes.c_char_p
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != OK:
        raise ReynError(rc, lib().reyn_last_error().decode())


def _f3(v) -> ctypes.Array:
    return (_f * 3)(*[float(x) for x in v])


def _ptr(t) -> Optional[int]:
    """Device pointer of a torch tensor (or None)."""
    if t is None:
        return None
    assert t.is_cuda and t.is_contiguous(), "expected a contiguous CUDA tensor"
    return t.data_ptr()


def _stream(stream) -> Optional[int]:
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    return int(stream)


def kernel_eval(kernel: int, h_bar: float, dx, dy, dz, stream=None):
    """W and grad W (device tensors in, device tensors out)."""
    import torch
    n = dx.numel()
    w, gx, gy, gz = (torch.empty(n, device=dx.device, dtype=torch.float32) for _ in range(4))
    check(lib().reyn_kernel_eval(kernel, h_bar, _ptr(dx), _ptr(dy), _ptr(dz), n, _ptr(w),
                                 _ptr(gx), _ptr(gy), _ptr(gz), _stream(stream)))
    return w, gx, gy, gz


class Particles:
    """Particles(N, rho0) (reference particles.cuh:25-75): 7 device SoA arrays."""

    FIELDS = ("xx", "xy", "xz", "vx", "vy", "vz", "m")

    def __init__(self, n: int, rho0: float):
        h = _vp()
        check(lib().reyn_particles_create(n, rho0, ctypes.byref(h)))
        self.h = h
        self.n = n
        self.rho0 = rho0

    def close(self):
        # at interpreter shutdown the module globals may already be gone
        if getattr(self, "h", None) and _lib is not None:
            _lib.reyn_particles_destroy(self.h)
        self.h = None

    __del__ = close

    def soa(self) -> Soa:
        s = Soa()
        check(lib().reyn_particles_soa(self.h, ctypes.byref(s)))
        return s

    def upload(self, host: dict, stream=None):
        arrs = [np.ascontiguousarray(host[k], np.float32) if k in host else None
                for k in ("x", "y", "z", "vx", "vy", "vz", "m")]
        ptrs = [a.ctypes.data if a is not None else None for a in arrs]
        check(lib().reyn_particles_upload(self.h, *ptrs, _stream(stream)))
        import torch
        torch.cuda.synchronize()

    def reorder(self, sorted_, stream=None) -> None:
        """Particles::reorder by a device permutation (uint32/int32 tensor):
        new[i] = old[sorted_[i]]; checked to be a permutation first."""
        check(lib().reyn_particles_reorder(self.h, _ptr(sorted_), _stream(stream)))

    def resize(self, n: int, keep: bool = True, stream=None) -> None:
        """resize_truncate (keep) / resize_uninit: new particles are zero."""
        check(lib().reyn_particles_resize(self.h, n, int(keep), _stream(stream)))
        self.n = n

    def download(self, stream=None) -> dict:
        out = {k: np.empty(self.n, np.float32) for k in ("x", "y", "z", "vx", "vy", "vz", "m")}
        check(lib().reyn_particles_download(self.h, *[out[k].ctypes.data for k in
                                                      ("x", "y", "z", "vx", "vy", "vz", "m")],
                                            _stream(stream)))
        return out

    def save_ply(self, path: str, stream=None) -> None:
        """save_to_ply (reference ply_io.cu:7-55): positions as binary PLY."""
        check(lib().reyn_particles_save_ply(self.h, os.fsencode(path), _stream(stream)))

    def save_raw(self, path: str, stream=None) -> None:
        check(lib().reyn_particles_save_raw(self.h, os.fsencode(path), _stream(stream)))

    def load_raw(self, path: str, stream=None) -> None:
        check(lib().reyn_particles_load_raw(self.h, os.fsencode(path), _stream(stream)))


class Grid:
    """UniformGridBuilder (reference uniformgrid.cuh:200-489)."""

    def __init__(self, bmin, bmax, search_radius: float, cell_ratio: float = 0.5,
                 order: int = 0, scene_first=None, scene_min=None, scene_max=None):
        """With scene_first (n_scenes + 1 offsets) and per-scene boxes
        scene_min/max (n_scenes x 3): a batched grid, each scene gridded over
        its own box (reyn_grid_create_batched; bmin and bmax are unused)."""
        h = _vp()
        self.n_scenes = 0
        if scene_first is None:
            check(lib().reyn_grid_create(_f3(bmin), _f3(bmax), search_radius, cell_ratio, order,
                                         ctypes.byref(h)))
        else:
            first = np.ascontiguousarray(scene_first, np.uint32)
            lo = np.ascontiguousarray(scene_min, np.float32).reshape(-1)
            hi = np.ascontiguousarray(scene_max, np.float32).reshape(-1)
            self.n_scenes = first.size - 1
            check(lib().reyn_grid_create_batched(search_radius, cell_ratio, order, self.n_scenes,
                                                 first.ctypes.data, lo.ctypes.data,
                                                 hi.ctypes.data, ctypes.byref(h)))
        self.h = h
        self.r = search_radius

    def close(self):
        # at interpreter shutdown the module globals may already be gone
        if getattr(self, "h", None) and _lib is not None:
            _lib.reyn_grid_destroy(self.h)
        self.h = None

    __del__ = close

    def construct(self, x, y, z, stream=None):
        check(lib().reyn_grid_construct(self.h, self.r, _ptr(x), _ptr(y), _ptr(z), x.numel(),
                                        _stream(stream)))

    def construct_state(self, state: Particles, stream=None):
        """construct over the state's own positions: a solver step on this
        grid keeps the caller's particle order (Resort::no)."""
        v = state.soa()
        check(lib().reyn_grid_construct(self.h, self.r, v.xx, v.xy, v.xz, v.n,
                                        _stream(stream)))

    def construct_and_reorder(self, state: Particles, extra: Sequence = (), stream=None):
        ptrs = (_vp * max(len(extra), 1))(*[_ptr(t) for t in extra])
        check(lib().reyn_grid_construct_and_reorder(self.h, self.r, state.h, ptrs, len(extra),
                                                    _stream(stream)))

    def reorder(self, state: Particles, extra: Sequence = (), stream=None):
        """after construct_state: permute the state (and extra arrays) by
        that build's permutation, as construct_and_reorder would have."""
        ptrs = (_vp * max(len(extra), 1))(*[_ptr(t) for t in extra])
        check(lib().reyn_grid_reorder(self.h, state.h, ptrs, len(extra), _stream(stream)))

    def info(self) -> GridInfo:
        g = GridInfo()
        check(lib().reyn_grid_info_get(self.h, ctypes.byref(g)))
        return g

    def permutation_ptr(self) -> int:
        p = _vp()
        check(lib().reyn_grid_permutation(self.h, ctypes.byref(p)))
        return p.value

    def neighbour_stats(self, x, y, z, m=None, kernel: int = C2, stream=None):
        import torch
        n = x.numel()
        count = torch.empty(n, device=x.device, dtype=torch.int32)
        len2 = torch.empty(n, device=x.device, dtype=torch.float32)
        rho = torch.empty(n, device=x.device, dtype=torch.float32) if m is not None else None
        check(lib().reyn_grid_neighbour_stats(self.h, _ptr(x), _ptr(y), _ptr(z), _ptr(m), kernel,
                                              _ptr(count), _ptr(len2), _ptr(rho),
                                              _stream(stream)))
        return count, len2, rho

    def compute_densities(self, x, y, z, m, bdy: Optional["Boundary"] = None, kernel: int = C2,
                          stream=None):
        """compute_densities (reference solver.cuh:19-38): fluid neighbours
        plus boundary samples, over the arrays the grid was built over; the
        result is in the order of those arrays."""
        import torch
        rho = torch.empty(x.numel(), device=x.device, dtype=torch.float32)
        check(lib().reyn_compute_densities(self.h, _ptr(x), _ptr(y), _ptr(z), _ptr(m),
                                           bdy.h if bdy is not None else None, kernel,
                                           _ptr(rho), _stream(stream)))
        return rho


class Boundary:
    """BoundarySamples (reference scene.cuh:14-46) with Akinci masses."""

    def __init__(self, bx, by, bz, bm=None, h: float = 1.0, rho0: float = 1.0,
                 mass_iters: int = 5, stream=None, scene_first=None):
        """scene_first (n_scenes + 1 offsets): a batched boundary, scene s
        owning samples scene_first[s] .. scene_first[s + 1] - 1."""
        hdl = _vp()
        nb = 0 if bx is None else bx.numel()
        if scene_first is None:
            check(lib().reyn_boundary_create(_ptr(bx), _ptr(by), _ptr(bz), _ptr(bm), nb, h,
                                             rho0, mass_iters, _stream(stream),
                                             ctypes.byref(hdl)))
        else:
            first = np.ascontiguousarray(scene_first, np.uint32)
            check(lib().reyn_boundary_create_batched(_ptr(bx), _ptr(by), _ptr(bz), _ptr(bm), nb,
                                                     first.size - 1, first.ctypes.data, h, rho0,
                                                     mass_iters, _stream(stream),
                                                     ctypes.byref(hdl)))
        self.h = hdl
        self.nb = nb

    def close(self):
        # at interpreter shutdown the module globals may already be gone
        if getattr(self, "h", None) and _lib is not None:
            _lib.reyn_boundary_destroy(self.h)
        self.h = None

    __del__ = close

    def bounds(self):
        """(bound_min, bound_max) of the samples."""
        lo, hi = (_f * 3)(), (_f * 3)()
        check(lib().reyn_boundary_bounds(self.h, lo, hi))
        return tuple(lo), tuple(hi)

    def arrays(self):
        """(x, y, z, m) device pointers of the reordered samples."""
        ps = [_vp() for _ in range(4)]
        nb = _u32()
        check(lib().reyn_boundary_arrays(self.h, *[ctypes.byref(p) for p in ps],
                                         ctypes.byref(nb)))
        return [p.value for p in ps], nb.value


class StepGraph:
    """One full step (construct_and_reorder + the solver step, bounded when
    `bounds` is given; a batched grid uses its scenes' boxes) captured as CUDA
    graphs at a fixed dt; launch() replays it."""

    def __init__(self, solver: "Solver", state: Particles, grid: Grid, bdy, dt: float,
                 bounds=None):
        hdl = _vp()
        lo = _f3(bounds[0]) if bounds is not None else None
        hi = _f3(bounds[1]) if bounds is not None else None
        check(lib().reyn_step_graph_create(solver.h, state.h, grid.h, bdy.h if bdy else None, dt,
                                           lo, hi, ctypes.byref(hdl)))
        self.h = hdl

    def launch(self, stream=None) -> None:
        check(lib().reyn_step_graph_launch(self.h, _stream(stream)))

    def stats(self, stream=None) -> StepStats:
        """The last launch's sweeps and errors; raises as the plain step would."""
        out = StepStats()
        check(lib().reyn_step_graph_stats(self.h, ctypes.byref(out), _stream(stream)))
        return out

    def info(self):
        """(kernels per step outside the pressure loop, kernels per sweep)"""
        a, b = _u32(), _u32()
        check(lib().reyn_step_graph_info(self.h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def close(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.reyn_step_graph_destroy(self.h)
        self.h = None

    __del__ = close


class Mesh:
    """A triangle mesh with its LBVH: DeviceMesh + LBVH (reference
    sample_boundary.cuh:13-60, lbvh.cuh:614-760). verts (V, 3) and faces
    (F, 3) are host arrays."""

    def __init__(self, verts=None, faces=None, stream=None, _handle=None):
        if _handle is None:
            v = np.ascontiguousarray(verts, np.float64).reshape(-1, 3)
            f = np.ascontiguousarray(faces, np.uint32).reshape(-1)
            cols = [np.ascontiguousarray(v[:, k]) for k in range(3)]
            hdl = _vp()
            check(lib().reyn_mesh_create(cols[0].ctypes.data, cols[1].ctypes.data,
                                         cols[2].ctypes.data, v.shape[0], f.ctypes.data,
                                         f.size // 3, _stream(stream), ctypes.byref(hdl)))
            _handle = hdl
        self.h = _handle

    @classmethod
    def from_obj(cls, path: str, ignore=(), only=None, stream=None) -> "Mesh":
        """load_mesh_from_obj(path, ignore, only_this_name) (loader.cpp)."""
        ig = (ctypes.c_char_p * max(len(ignore), 1))(*[s.encode() for s in ignore])
        hdl = _vp()
        check(lib().reyn_mesh_load_obj(path.encode(), ig, len(ignore),
                                       only.encode() if only else None, _stream(stream),
                                       ctypes.byref(hdl)))
        return cls(_handle=hdl)

    def close(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.reyn_mesh_destroy(self.h)
        self.h = None

    __del__ = close

    def info(self) -> MeshInfo:
        out = MeshInfo()
        check(lib().reyn_mesh_info_get(self.h, ctypes.byref(out)))
        return out

    def tree(self, stream=None) -> dict:
        """The LBVH in the reference's layout, as device tensors."""
        import torch
        nf = self.info().n_faces
        ni = max(nf - 1, 0)
        dev = "cuda"
        order = torch.empty(nf, dtype=torch.int32, device=dev)
        cl = torch.empty(max(ni, 1), dtype=torch.int32, device=dev)
        cr = torch.empty(max(ni, 1), dtype=torch.int32, device=dev)
        leaf = torch.empty((nf, 6), dtype=torch.float32, device=dev)
        node = torch.empty((max(ni, 1), 6), dtype=torch.float32, device=dev)
        check(lib().reyn_mesh_tree(self.h, _ptr(order), _ptr(cl), _ptr(cr), _ptr(leaf),
                                   _ptr(node), _stream(stream)))
        return {"order": order, "children_l": cl[:ni], "children_r": cr[:ni], "leaf_box": leaf,
                "node_box": node[:ni]}

    def project(self, x, y, z, stream=None) -> None:
        """LBVH::project: device tensors, in place."""
        check(lib().reyn_mesh_project(self.h, _ptr(x), _ptr(y), _ptr(z), x.numel(),
                                      _stream(stream)))

    def inside(self, x, y, z, stream=None):
        import torch
        flags = torch.empty(x.numel(), dtype=torch.uint8, device=x.device)
        check(lib().reyn_mesh_inside(self.h, _ptr(x), _ptr(y), _ptr(z), x.numel(), _ptr(flags),
                                     _stream(stream)))
        return flags

    def sample_uniform(self, h: float, oversampling: float = 2.0, seed: int = 1614201312,
                       stream=None):
        """uniform_sample_mesh: three device tensors."""
        cnt = _u32()
        check(lib().reyn_mesh_sample_uniform(self.h, h, oversampling, seed, None, None, None, 0,
                                             ctypes.byref(cnt), None))
        x, y, z = _device_f32(cnt.value)
        check(lib().reyn_mesh_sample_uniform(self.h, h, oversampling, seed, _ptr(x), _ptr(y),
                                             _ptr(z), cnt.value, ctypes.byref(cnt),
                                             _stream(stream)))
        return x[:cnt.value], y[:cnt.value], z[:cnt.value]

    def relax(self, x, y, z, h_bdy: float, relaxation_factor: float = 1.0, iters: int = 50,
              num_den=None, stream=None) -> np.ndarray:
        """relax_sampling, in place; returns per sweep (max/min number-density
        ratio, average number density)."""
        st = np.zeros((max(iters, 1), 2), np.float32)
        check(lib().reyn_mesh_relax(self.h, _ptr(x), _ptr(y), _ptr(z), x.numel(), h_bdy,
                                    relaxation_factor, iters, st.ctypes.data, _ptr(num_den),
                                    _stream(stream)))
        return st[:iters]

    def fill(self, h: float, jitter: float = 0.0, seed: int = 1, stream=None):
        """Scene::from_obj's fluid fill: three device tensors."""
        cnt = _u32()
        check(lib().reyn_mesh_fill(self.h, h, jitter, seed, None, None, None, 0,
                                   ctypes.byref(cnt), _stream(stream)))
        x, y, z = _device_f32(cnt.value)
        check(lib().reyn_mesh_fill(self.h, h, jitter, seed, _ptr(x), _ptr(y), _ptr(z), cnt.value,
                                   ctypes.byref(cnt), _stream(stream)))
        return x[:cnt.value], y[:cnt.value], z[:cnt.value]


def sample_mesh(mesh: Mesh, h: float, rho0: float, oversampling_factor: float = 2.0,
                relaxation_iters: int = 50, relaxation_factor: float = 1.0,
                mass_refinement_iterations: int = 5, seed: int = 1614201312, stream=None):
    """sample_mesh (reference sample_boundary.cu:391-439, defaults of
    sample_boundary.cuh:160-163): uniform samples at h / oversampling_factor,
    relaxed, then a Boundary with Akinci masses. Returns (Boundary, (x, y, z),
    relaxation statistics)."""
    x, y, z = mesh.sample_uniform(h, oversampling_factor, seed, stream)
    stats = np.zeros((0, 2), np.float32)
    if relaxation_iters > 0:
        stats = mesh.relax(x, y, z, h / oversampling_factor, relaxation_factor,
                           relaxation_iters, stream=stream)
    bdy = Boundary(x, y, z, None, h, rho0, mass_refinement_iterations, stream)
    return bdy, (x, y, z), stats


NOALLOC_SCRATCH_WORDS = 8 * 1024 * 1024


def grid_construct_noalloc(bmin, bmax, search_radius: float, x, y, z, prefix, sorted_,
                           cell_ratio: float = 0.5, stream=None):
    """Uniform-grid build into caller-owned device tensors without any device
    allocation (reyn_grid_construct_noalloc), for callers that cannot
    allocate device memory. prefix=None only returns dims. x, y, z are
    float32 tensors of n entries, sorted_ a 4-byte integer tensor of n
    entries, prefix a 4-byte integer tensor of at least nx*ny*nz + 1.
    Returns (nx, ny, nz)."""
    import torch

    dims = (ctypes.c_int32 * 3)()
    n = 0 if x is None else x.numel()
    cap = 0 if prefix is None else prefix.numel()
    if prefix is not None:
        if n and any(t is None for t in (x, y, z, sorted_)):
            raise ValueError("x, y, z and sorted_ are needed with prefix")
        for name, t in (("x", x), ("y", y), ("z", z)):
            if t is not None and (t.dtype != torch.float32 or t.numel() != n):
                raise ValueError(f"{name} must be float32 with {n} entries")
        ints = (torch.int32, getattr(torch, "uint32", torch.int32))
        if prefix.dtype not in ints:
            raise ValueError("prefix must hold 4-byte integers")
        if sorted_ is not None and (sorted_.dtype not in ints or sorted_.numel() != n):
            raise ValueError(f"sorted_ must hold {n} 4-byte integers")
        for t in (x, y, z, prefix, sorted_):
            if t is not None and not t.is_contiguous():
                raise ValueError("tensors must be contiguous")
    check(lib().reyn_grid_construct_noalloc(_f3(bmin), _f3(bmax), search_radius, cell_ratio,
                                            _ptr(x), _ptr(y), _ptr(z), n, _ptr(prefix), cap,
                                            _ptr(sorted_), dims, _stream(stream)))
    return tuple(dims)


def reference_params(scheme: int, kernel: int, h: float, rho0: float, nu: float) -> Params:
    p = Params()
    check(lib().reyn_params_reference(scheme, kernel, h, rho0, nu, ctypes.byref(p)))
    return p


class Solver:
    """SESPH / PCISPH / IISPH (reference solvers/*.cuh)."""

    def __init__(self, scheme: int, params: Params, n: int):
        h = _vp()
        check(lib().reyn_solver_create(scheme, ctypes.byref(params), n, ctypes.byref(h)))
        self.h = h
        self.n = n
        self.scheme = scheme

    def close(self):
        # at interpreter shutdown the module globals may already be gone
        if getattr(self, "h", None) and _lib is not None:
            _lib.reyn_solver_destroy(self.h)
        self.h = None

    __del__ = close

    def step(self, state: Particles, grid: Grid, bdy: Optional[Boundary], dt: float,
             stream=None, bounds=None) -> int:
        """One step; with bounds=(bmin, bmax) the step also applies the hard
        bounds in its integrating kernel and records max |v| for next_dt."""
        it = _u32()
        if bounds is None:
            check(lib().reyn_solver_step(self.h, state.h, grid.h, bdy.h if bdy else None, dt,
                                         ctypes.byref(it), _stream(stream)))
        else:
            check(lib().reyn_solver_step_bounded(self.h, state.h, grid.h,
                                                 bdy.h if bdy else None, dt, _f3(bounds[0]),
                                                 _f3(bounds[1]), ctypes.byref(it),
                                                 _stream(stream)))
        return it.value

    def step_batched(self, state: Particles, grid: Grid, bdy: Optional[Boundary], dt: float,
                     bounded: bool = True, stream=None) -> np.ndarray:
        """One step of every scene of a batched grid; returns per-scene
        iteration counts."""
        it = np.zeros(grid.n_scenes, np.uint32)
        check(lib().reyn_solver_step_batched(self.h, state.h, grid.h, bdy.h if bdy else None, dt,
                                             1 if bounded else 0, it.ctypes.data,
                                             _stream(stream)))
        return it

    def scene_stats(self, n_scenes: int) -> list:
        out = (StepStats * n_scenes)()
        check(lib().reyn_solver_scene_stats(self.h, n_scenes, out))
        return list(out)

    def next_dt(self, state: Particles, iter_last: int, dt_last: float, lam: float, h: float,
                g, iter_target: int = 5, change: float = 0.01, stream=None) -> float:
        """simple_dt_controller on the max |v| of the last bounded step."""
        dt = _f()
        check(lib().reyn_solver_next_dt(self.h, state.h, iter_last, dt_last, lam, h, _f3(g),
                                        iter_target, change, ctypes.byref(dt),
                                        _stream(stream)))
        return dt.value

    def buffers(self) -> SolverBuffers:
        b = SolverBuffers()
        check(lib().reyn_solver_buffers_get(self.h, ctypes.byref(b)))
        return b

    def pressure(self, stream=None) -> np.ndarray:
        """The carried IISPH pressure, in the particle order of the state."""
        p = np.empty(self.n, np.float32)
        check(lib().reyn_solver_pressure_download(self.h, p.ctypes.data, _stream(stream)))
        return p

    def set_pressure(self, state: "Particles", p: np.ndarray, stream=None) -> None:
        p = np.ascontiguousarray(p, np.float32)
        check(lib().reyn_solver_pressure_upload(self.h, state.h, p.ctypes.data, _stream(stream)))

    def stats(self) -> StepStats:
        s = StepStats()
        check(lib().reyn_solver_stats(self.h, ctypes.byref(s)))
        return s


def cfl_time_step(state: Particles, lam: float, h: float, g, stream=None) -> float:
    dt = _f()
    check(lib().reyn_cfl_time_step(state.h, lam, h, _f3(g), ctypes.byref(dt), _stream(stream)))
    return dt.value


def dt_controller(state: Particles, iter_last: int, dt_last: float, lam: float, h: float, g,
                  iter_target: int = 5, change: float = 0.01, stream=None) -> float:
    dt = _f()
    check(lib().reyn_dt_controller(state.h, iter_last, dt_last, lam, h, _f3(g), iter_target,
                                   change, ctypes.byref(dt), _stream(stream)))
    return dt.value


def diagnostics(state: Particles, stream=None) -> dict:
    """Total mass, momentum and kinetic energy of the state (FP64 sums)."""
    d = Diag()
    check(lib().reyn_diagnostics(state.h, ctypes.byref(d), _stream(stream)))
    return {"mass": d.mass, "momentum": tuple(d.momentum), "kinetic": d.kinetic}


def enforce_bounds(state: Particles, bmin, bmax, stream=None) -> None:
    check(lib().reyn_enforce_bounds(state.h, _f3(bmin), _f3(bmax), _stream(stream)))


# ---- scene generation on the device ---------------------------------------------

def scene_fluid_block(state: Particles, counts, origin, spacing: float, mass: float = 0.0,
                      jitter: float = 0.0, velocity_noise: float = 0.0, seed: int = 1,
                      first: int = 0, stream=None) -> None:
    """Lattice + seeded jitter into particles first .. first + prod(counts) - 1."""
    check(lib().reyn_scene_fluid_block(state.h, first, (_u32 * 3)(*counts), _f3(origin),
                                       spacing, mass, jitter, velocity_noise, seed,
                                       _stream(stream)))


def _device_f32(n: int):
    import torch
    return [torch.empty(max(n, 1), dtype=torch.float32, device="cuda") for _ in range(3)]


def scene_box_walls(bmin, bmax, spacing: float, stream=None):
    """Box-wall samples as three device tensors."""
    cnt = ctypes.c_uint64()
    check(lib().reyn_scene_box_walls(_f3(bmin), _f3(bmax), spacing, None, None, None, 0,
                                     ctypes.byref(cnt), None))
    x, y, z = _device_f32(cnt.value)
    check(lib().reyn_scene_box_walls(_f3(bmin), _f3(bmax), spacing, x.data_ptr(), y.data_ptr(),
                                     z.data_ptr(), cnt.value, ctypes.byref(cnt),
                                     _stream(stream)))
    return x[:cnt.value], y[:cnt.value], z[:cnt.value]


def scene_sphere(center, radius: float, spacing: float, stream=None):
    """Fibonacci-sphere samples as three device tensors."""
    cnt = _u32()
    check(lib().reyn_scene_sphere(_f3(center), radius, spacing, None, None, None, 0,
                                  ctypes.byref(cnt), None))
    x, y, z = _device_f32(cnt.value)
    check(lib().reyn_scene_sphere(_f3(center), radius, spacing, x.data_ptr(), y.data_ptr(),
                                  z.data_ptr(), cnt.value, ctypes.byref(cnt), _stream(stream)))
    return x[:cnt.value], y[:cnt.value], z[:cnt.value]


def scene_jitter(state: Particles, amplitude: float, seed: int = 1, first: int = 0,
                 count: Optional[int] = None, stream=None) -> None:
    """jitter_positions: uniform [-amplitude, amplitude] per axis, keyed by
    the particle index (sqrt(3) sigma matches the reference's normal sigma)."""
    n = state.n - first if count is None else count
    check(lib().reyn_scene_jitter(state.h, first, n, amplitude, seed, _stream(stream)))


def scene_cull(state: Particles, bdy: Boundary, radius: float, stream=None) -> int:
    """Removes fluid particles within `radius` of a boundary sample; returns
    the new particle count (the state shrinks)."""
    n = _u32()
    check(lib().reyn_scene_cull(state.h, bdy.h, radius, ctypes.byref(n), _stream(stream)))
    state.n = n.value
    return n.value


def autotune(scheme: int, params: Params, state: Particles, bdy, dt: float, steps: int = 3,
             bounds=None, scene_first=None, scene_min=None, scene_max=None, stream=None):
    """reyn_autotune: returns (best, all eight) as TunePoint records."""
    best = TunePoint()
    pts = (TunePoint * 8)()
    if scene_first is None:
        check(lib().reyn_autotune(scheme, ctypes.byref(params), state.h, bdy.h if bdy else None,
                                  _f3(bounds[0]), _f3(bounds[1]), 0, None, None, None, dt, steps,
                                  ctypes.byref(best), pts, _stream(stream)))
    else:
        first = np.ascontiguousarray(scene_first, np.uint32)
        lo = np.ascontiguousarray(scene_min, np.float32).reshape(-1)
        hi = np.ascontiguousarray(scene_max, np.float32).reshape(-1)
        check(lib().reyn_autotune(scheme, ctypes.byref(params), state.h, bdy.h if bdy else None,
                                  None, None, first.size - 1, first.ctypes.data, lo.ctypes.data,
                                  hi.ctypes.data, dt, steps, ctypes.byref(best), pts,
                                  _stream(stream)))
    return best, list(pts)


def autotune_reorder(scheme: int, params: Params, state: Particles, bdy, dt: float, bounds,
                     cell_ratio: float = 0.5, every=(1, 2, 5, 10), steps: int = 10,
                     stream=None):
    """reyn_autotune_reorder: returns (best interval, [ms per step for each
    candidate]); params.block_size is the block size timed."""
    ev = np.ascontiguousarray(every, np.uint32)
    ms = np.zeros(ev.size, np.float32)
    best = _u32()
    check(lib().reyn_autotune_reorder(scheme, ctypes.byref(params), state.h,
                                      bdy.h if bdy else None, _f3(bounds[0]), _f3(bounds[1]),
                                      cell_ratio, dt, steps, ev.ctypes.data, ev.size,
                                      ctypes.byref(best), ms.ctypes.data, _stream(stream)))
    return best.value, [float(x) for x in ms]


def profile_enable(on: bool = True) -> None:
    """Bracket every engine kernel launch with CUDA events (launches are
    always counted)."""
    check(lib().reyn_profile_enable(1 if on else 0))


def profile_reset() -> None:
    check(lib().reyn_profile_reset())


def profile_read() -> dict:
    """{kernel name: (launches, total device ms)} since the last reset."""
    cnt = _u32()
    check(lib().reyn_profile_read(None, 0, ctypes.byref(cnt)))
    arr = (ProfileEntry * max(cnt.value, 1))()
    check(lib().reyn_profile_read(arr, cnt.value, ctypes.byref(cnt)))
    return {arr[i].name.decode(): (int(arr[i].launches), float(arr[i].total_ms))
            for i in range(cnt.value)}


class _DeviceView:
    """__cuda_array_interface__ over an engine-owned device array."""

    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr,
                                         "data": (ptr, False), "version": 3}


def device_tensor(ptr: int, n: int, dtype=np.float32):
    """A torch view (no copy) of n elements at an engine device pointer."""
    import torch
    typestr = {np.float32: "<f4", np.uint32: "<u4", np.int32: "<i4"}[dtype]
    if n == 0:
        return torch.empty(0, dtype=torch.float32 if dtype == np.float32 else torch.int32,
                           device="cuda")
    t = torch.as_tensor(_DeviceView(ptr, n, typestr), device="cuda")
    return t


def device_to_numpy(ptr: int, n: int, dtype=np.float32) -> np.ndarray:
    """Copies n elements at an engine device pointer into a numpy array."""
    import torch
    torch.cuda.synchronize()
    return device_tensor(ptr, n, dtype).cpu().numpy().astype(dtype, copy=False)


@dataclass
class StepOutputs:
    state: dict
    rho: np.ndarray
    p: np.ndarray
    aii: np.ndarray
    sii: np.ndarray
    a: np.ndarray
    iters: list
