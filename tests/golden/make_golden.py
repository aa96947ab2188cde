"""Generates the golden fixtures in tests/golden/ from the REFERENCE ITSELF.

* ``--host``: the reference's smoothing-kernel classes (src/kernels.cuh),
  compiled unmodified for the host by oracle/ref/Makefile, evaluated on the
  reference's own kernel-test inputs (kernels.cu:31-52: edge cases, then
  seeded pseudo-random offsets in [0, 1.5 h]^3, h = 25). Runs without a GPU.
* ``--mesh``: the reference's LBVH (datastructure/lbvh.cuh, compiled
  unmodified for sm_100a) on a B200, over seeded procedural meshes
  (reyn_b200.meshes): the sorted faces, the tree's children and boxes, its
  height, the mesh volume, LBVH::project of seeded points, and the sample
  counts of uniform_sample_mesh.
* ``--device``: the reference's CUDA path (src/, compiled unmodified for
  sm_100a by oracle/ref/Makefile) on a B200: kernel values on the device, the
  uniform grid (prefix, canonicalised sorted indices, neighbour counts,
  sum |x_ij|^2, densities) and SESPH / PCISPH / IISPH steps on small seeded
  dam breaks, with boundary masses from the reference's own
  calculate_boundary_masses.

Inputs are regenerated deterministically (numpy PCG64 seeds) and stored with
the outputs so that the tests never need the reference at run time.

Usage: python tests/golden/make_golden.py --host|--device|--mesh [--out DIR]
"""
from __future__ import annotations

import argparse
import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from reyn_b200 import meshes, scenes  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
P = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
F32 = lambda a: np.ascontiguousarray(a, np.float32)  # noqa: E731

# solver fixtures: (name, scheme, kernel, counts, h, box, nu, dt, steps, velocity noise)
SOLVER_CASES = [
    ("sesph_b3_1", oracle.SESPH, oracle.B3, (16, 16, 16), 0.02, (0.5, 0.5, 0.5), 0.01, 5e-4, 1, 0.05),
    ("sesph_b3_5", oracle.SESPH, oracle.B3, (16, 16, 16), 0.02, (0.5, 0.5, 0.5), 0.01, 5e-4, 5, 0.05),
    ("pcisph_b3_1", oracle.PCISPH, oracle.B3, (16, 16, 16), 0.02, (0.5, 0.5, 0.5), 0.01, 1e-3, 1, 0.05),
    ("pcisph_c2_3", oracle.PCISPH, oracle.C2, (16, 16, 16), 0.02, (0.5, 0.5, 0.5), 0.01, 1e-3, 3, 0.05),
    ("iisph_c2_1", oracle.IISPH, oracle.C2, (16, 16, 16), 0.02, (0.5, 0.5, 0.5), 0.01, 1e-3, 1, 0.05),
    ("iisph_c2_5", oracle.IISPH, oracle.C2, (16, 16, 16), 0.02, (0.5, 0.5, 0.5), 0.01, 1e-3, 5, 0.05),
    ("iisph_w6_1", oracle.IISPH, oracle.W6, (16, 16, 16), 0.02, (0.5, 0.5, 0.5), 0.01, 1e-3, 1, 0.05),
    ("iisph_cos_1", oracle.IISPH, oracle.COS, (12, 12, 12), 0.02, (0.4, 0.4, 0.4), 0.01, 1e-3, 1, 0.05),
]


def kernel_inputs(seed_rand: int = 16142069, n: int = 4096):
    """The reference kernel test's offsets (kernels.cu:31-52): its edge
    cases, then n seeded offsets in [0, 1.5 h]^3 (a numpy-seeded stand-in
    for its std::rand() stream), plus its regular lattice (kernels.cu:54-66)."""
    h_bar = 25.0
    eps = np.finfo(np.float32).eps
    edge = [0.0, h_bar, h_bar - eps, h_bar + eps, eps, h_bar + 1e-20, h_bar - 1e-20, 1e-20,
            np.finfo(np.float32).max]
    rng = np.random.Generator(np.random.PCG64(seed_rand))
    d = (h_bar * 1.5 * rng.random((n, 3))).astype(np.float32)
    for k, v in enumerate(edge):
        d[k, :] = np.float32(v)
    # the regular lattice of kernels.cu:54-66 (antisymmetry and sum tests)
    sc = 25
    sp = np.float32(h_bar * 2.0 / sc)
    ii = np.arange(sc, dtype=np.float32)
    gx, gy, gz = np.meshgrid(ii, ii, ii, indexing="ij")
    lat = np.stack([gx.ravel(), gy.ravel(), gz.ravel()], 1) * sp + np.float32(-h_bar + sp / 2)
    return np.float32(h_bar), d, lat.astype(np.float32)


def make_host(out: str) -> None:
    h_bar, d, lat = kernel_inputs()
    res = {"h_bar": h_bar, "d": d}
    for name, k in (("C2", 0), ("B3", 1), ("W6", 2), ("COS", 3)):
        w, gx, gy, gz = oracle.ref_kernel_eval_host(k, float(h_bar), d[:, 0], d[:, 1], d[:, 2])
        res[f"{name}_w"], res[f"{name}_g"] = w, np.stack([gx, gy, gz], 1)
    np.savez_compressed(os.path.join(out, "kernels_host.npz"), **res)
    print("wrote kernels_host.npz")


def _ref():
    L = oracle.ref_cuda()
    return L


def _check(L, rc):
    if rc:
        raise RuntimeError(L.ref_last_error().decode())


def canonical_sorted(prefix: np.ndarray, sorted_: np.ndarray) -> np.ndarray:
    """Sorts the indices inside every cell segment ascending."""
    out = sorted_.copy()
    nz = np.nonzero(np.diff(prefix.astype(np.int64)))[0]
    for c in nz:
        a, b = int(prefix[c]), int(prefix[c + 1])
        if b - a > 1:
            out[a:b] = np.sort(out[a:b])
    return out


def ref_grid(L, x, y, z, bmin, bmax, r, kinds=(0, 1)):
    n = x.size
    dims = np.zeros(3, np.int32)
    _check(L, L.ref_grid(ctypes.c_uint(n), P(x), P(y), P(z), P(F32(bmin)), P(F32(bmax)),
                         ctypes.c_float(r), P(dims), None, None, None, None, 0, None, None))
    C = int(dims.prod())
    prefix = np.zeros(C, np.uint32)
    sorted_ = np.zeros(n, np.uint32)
    count = np.zeros(n, np.uint32)
    len2 = np.zeros(n, np.float32)
    out = {}
    m = np.ones(n, np.float32)
    for k in kinds:
        rho = np.zeros(n, np.float32)
        _check(L, L.ref_grid(ctypes.c_uint(n), P(x), P(y), P(z), P(F32(bmin)), P(F32(bmax)),
                             ctypes.c_float(r), P(dims), P(prefix), P(sorted_), P(count),
                             P(len2), k, P(m), P(rho)))
        out[f"rho_k{k}"] = rho
    full = np.concatenate([prefix, np.array([n], np.uint32)])
    out.update({"dims": dims.copy(), "prefix": prefix.copy(),
                "sorted": canonical_sorted(full, sorted_), "count": count.copy(),
                "len2": len2.copy()})
    return out


def make_device(out: str) -> None:
    L = _ref()
    # kernel values on the device
    h_bar, d, lat = kernel_inputs()
    res = {"h_bar": h_bar, "d": d}
    for name, k in (("C2", 0), ("B3", 1), ("W6", 2), ("COS", 3)):
        n = d.shape[0]
        w, gx, gy, gz = (np.zeros(n, np.float32) for _ in range(4))
        dx, dy, dz = F32(d[:, 0]), F32(d[:, 1]), F32(d[:, 2])
        _check(L, L.ref_kernel_eval_device(k, ctypes.c_float(h_bar), ctypes.c_uint(n), P(dx),
                                           P(dy), P(dz), P(w), P(gx), P(gy), P(gz)))
        res[f"{name}_w"], res[f"{name}_g"] = w, np.stack([gx, gy, gz], 1)
    np.savez_compressed(os.path.join(out, "kernels_device.npz"), **res)
    print("wrote kernels_device.npz", flush=True)

    # the reference grid test (uniformgrid.cu:247-346) at side 24, and the
    # neighbour-search microbenchmark geometry at 32768 points
    side, hh = 24, 1.1
    box = hh * side
    rng = np.random.Generator(np.random.PCG64(161))
    x, y, z = (F32(box * rng.random(side ** 3)) for _ in range(3))
    g = ref_grid(L, x, y, z, [0, 0, 0], [box] * 3, 2 * hh)
    np.savez_compressed(os.path.join(out, "grid_test.npz"), x=x, y=y, z=z, bmin=F32([0, 0, 0]),
                        bmax=F32([box] * 3), r=np.float32(2 * hh), **g)
    print("wrote grid_test.npz", flush=True)
    n = 32768
    x, y, z = scenes.uniform_cloud(n, seed=2)
    r = np.float32(0.0196 * (float(1 << 20) / n) ** (1.0 / 3.0))
    g = ref_grid(L, x, y, z, [0, 0, 0], [1, 1, 1], float(r), kinds=(0, 1, 2, 3))
    np.savez_compressed(os.path.join(out, "grid_cloud.npz"), x=x, y=y, z=z, bmin=F32([0, 0, 0]),
                        bmax=F32([1, 1, 1]), r=r, **g)
    print("wrote grid_cloud.npz", flush=True)

    # boundary masses and solver steps
    for (name, scheme, kind, counts, h, boxs, nu, dt, steps, vnoise) in SOLVER_CASES:
        sc = scenes.dam_break(counts, h, boxs, 1000.0, 0.1, seed=7, velocity_noise=vnoise)
        nb = sc.nb
        bx, by, bz = F32(sc.bdy["x"]), F32(sc.bdy["y"]), F32(sc.bdy["z"])
        ox, oy, oz, om = (np.zeros(nb, np.float32) for _ in range(4))
        _check(L, L.ref_boundary_masses(ctypes.c_uint(nb), P(bx), P(by), P(bz), ctypes.c_float(h),
                                        ctypes.c_float(1000.0), ctypes.c_uint(5), P(ox), P(oy),
                                        P(oz), P(om)))
        st = {k: F32(sc.fluid[k]).copy() for k in ("x", "y", "z", "vx", "vy", "vz", "m", "id")}
        inputs = {f"in_{k}": v.copy() for k, v in st.items()}
        N = sc.n
        outs = {k: np.zeros(N, np.float32) for k in ("rho", "p", "aii", "sii", "ax", "ay", "az")}
        iters = np.zeros(steps, np.uint32)
        _check(L, L.ref_run(scheme, kind, ctypes.c_uint(N), *(P(st[k]) for k in
                                                               ("x", "y", "z", "vx", "vy", "vz",
                                                                "m", "id")),
                            ctypes.c_uint(nb), P(ox), P(oy), P(oz), P(om), P(F32(sc.box_min)),
                            P(F32(sc.box_max)), ctypes.c_float(h), ctypes.c_float(1000.0),
                            ctypes.c_float(nu), ctypes.c_float(dt), ctypes.c_uint(steps),
                            *(P(outs[k]) for k in ("rho", "p", "aii", "sii", "ax", "ay", "az")),
                            P(iters)))
        np.savez_compressed(os.path.join(out, f"solver_{name}.npz"), scheme=scheme, kind=kind,
                            h=np.float32(h), nu=np.float32(nu), dt=np.float32(dt), steps=steps,
                            box_min=F32(sc.box_min), box_max=F32(sc.box_max), bx=ox, by=oy,
                            bz=oz, bm=om, iters=iters, **inputs,
                            **{f"out_{k}": v for k, v in st.items()},
                            **{f"out_{k}": v for k, v in outs.items()})
        print(f"wrote solver_{name}.npz iters={iters.tolist()}", flush=True)


# mesh fixtures: (name, builder); the builders are deterministic
MESH_CASES = [
    ("ico3", lambda: meshes.icosphere(3, 0.7, (0.1, -0.2, 0.3))),
    ("ico4_perturbed", lambda: (lambda v, f: (meshes.perturb(v, 0.004, 3), f))(
        *meshes.icosphere(4, 0.7, (0.1, -0.2, 0.3)))),
    ("box4", lambda: meshes.box((-1.0, -0.5, 0.0), (1.0, 0.5, 0.75), 4)),
    ("torus_perturbed", lambda: (lambda v, f: (meshes.perturb(v, 0.005, 5), f))(
        *meshes.torus(1.0, 0.3, 40, 20, (0.5, 0.5, 0.5)))),
]
# (h, oversampling) pairs for the sample counts
SAMPLE_CASES = [(0.05, 2.0), (0.02, 1.0), (0.1, 3.0)]


def make_mesh(out: str) -> None:
    L = _ref()
    u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
    d = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
    L.ref_lbvh.argtypes = [ctypes.c_uint, d, d, d, ctypes.c_uint, u32p, u32p, u32p, u32p,
                           oracle._f32p, oracle._f32p, u32p, d, ctypes.c_uint, oracle._f32p,
                           oracle._f32p, oracle._f32p]
    L.ref_mesh_sample.argtypes = [ctypes.c_uint, d, d, d, ctypes.c_uint, u32p, ctypes.c_float,
                                  ctypes.c_float, ctypes.c_uint, ctypes.c_void_p,
                                  ctypes.c_void_p, ctypes.c_void_p, u32p]
    for name, make in MESH_CASES:
        v, f = make()
        v = np.ascontiguousarray(v, np.float64)
        f = np.ascontiguousarray(f, np.uint32)
        vx, vy, vz = (np.ascontiguousarray(v[:, k]) for k in range(3))
        nv, nf = v.shape[0], f.shape[0]
        rng = np.random.Generator(np.random.PCG64(420))
        lo, hi = v.min(0) - 0.2, v.max(0) + 0.2
        q = (lo + (hi - lo) * rng.random((2000, 3))).astype(np.float32)
        px, py, pz = (np.ascontiguousarray(q[:, k]) for k in range(3))
        fs = np.zeros(3 * nf, np.uint32)
        cl = np.zeros(nf - 1, np.uint32)
        cr = np.zeros(nf - 1, np.uint32)
        lb = np.zeros(6 * nf, np.float32)
        nb = np.zeros(6 * (nf - 1), np.float32)
        height = np.zeros(1, np.uint32)
        vol = np.zeros(1, np.float64)
        _check(L, L.ref_lbvh(nv, vx, vy, vz, nf, f.ravel(), fs, cl, cr, lb, nb, height, vol,
                             2000, px, py, pz))
        counts = []
        for h, ov in SAMPLE_CASES:
            c = np.zeros(1, np.uint32)
            _check(L, L.ref_mesh_sample(nv, vx, vy, vz, nf, f.ravel(), h, ov, 0, None, None, None,
                                        c))
            counts.append(int(c[0]))
        np.savez_compressed(os.path.join(out, f"mesh_{name}.npz"), verts=v, faces=f,
                            faces_sorted=fs.reshape(-1, 3), children_l=cl, children_r=cr,
                            leaf_box=lb.reshape(-1, 6), node_box=nb.reshape(-1, 6),
                            height=height[0], volume=vol[0], points=q,
                            projected=np.stack([px, py, pz], 1),
                            sample_cases=np.array(SAMPLE_CASES, np.float32),
                            sample_counts=np.array(counts, np.uint32))
        print(f"wrote mesh_{name}.npz faces={nf} height={int(height[0])}", flush=True)


def main():
    ap = argparse.ArgumentParser()
    g = ap.add_mutually_exclusive_group(required=True)
    g.add_argument("--host", action="store_true")
    g.add_argument("--device", action="store_true")
    g.add_argument("--mesh", action="store_true")
    ap.add_argument("--out", default=HERE)
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    if a.host:
        make_host(a.out)
    elif a.mesh:
        make_mesh(a.out)
    else:
        make_device(a.out)


if __name__ == "__main__":
    main()
