"""Seeded synthetic scenes for the workloads the engine is measured on.

Each scene is a fluid block on a cubic lattice with seeded uniform jitter,
standing in the lower corner of a closed box whose six walls are sampled with
one layer of boundary particles on a square lattice. "Up" is +y: gravity is
(0, -9.81, 0), the reference solvers' hard-coded axis (PCISPH.cuh:27,
IISPH.cuh:37). Fluid masses are rho0 h^3 (the reference's _init_box_kernel,
scene.cu:14-37). Boundary masses are left to the Akinci refinement
(calculate_boundary_masses, sample_boundary.cu:267-297).

The generator is numpy with counter-based random numbers (SplitMix64 of the
seed and the particle index), so every machine builds the same scene bit for
bit, and the GPU generator (reyn_scene_fluid_block, reyn_scene_box_walls)
writes the same arrays on the device.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class Scene:
    name: str
    h: float                 # particle spacing
    rho0: float
    fluid: dict              # x, y, z, vx, vy, vz, m, id (float32)
    bdy: dict                # x, y, z (float32)
    box_min: np.ndarray
    box_max: np.ndarray
    meta: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return int(self.fluid["x"].size)

    @property
    def nb(self) -> int:
        return int(self.bdy["x"].size)


def box_walls(box_min, box_max, spacing: float) -> dict:
    """One layer of samples on the six faces of an axis-aligned box, on a
    square lattice of n = rint((hi - lo) / spacing) intervals per axis (no
    duplicates at edges/corners): the x faces (all j, k), the y faces
    (interior i), the z faces (interior i, j), the first index slowest;
    sample (i, j, k) at lo + (i, j, k) * step, step = (hi - lo) / n, in
    float32 arithmetic (the same samples reyn_scene_box_walls writes on the
    GPU)."""
    lo = np.asarray(box_min, np.float32)
    hi = np.asarray(box_max, np.float32)
    ext = hi - lo
    n = np.rint(ext.astype(np.float64) / float(spacing)).astype(np.int64)
    step = ext / n.astype(np.float32)
    axes = [np.arange(k + 1) for k in n]
    pts = []
    for ix in (0, n[0]):
        j, k = np.meshgrid(axes[1], axes[2], indexing="ij")
        pts.append(np.stack([np.full(j.size, ix), j.ravel(), k.ravel()], 1))
    for iy in (0, n[1]):
        i, k = np.meshgrid(axes[0][1:-1], axes[2], indexing="ij")
        pts.append(np.stack([i.ravel(), np.full(i.size, iy), k.ravel()], 1))
    for iz in (0, n[2]):
        i, j = np.meshgrid(axes[0][1:-1], axes[1][1:-1], indexing="ij")
        pts.append(np.stack([i.ravel(), j.ravel(), np.full(i.size, iz)], 1))
    p = np.concatenate(pts, 0).astype(np.float32)
    xyz = lo + p * step
    return {"x": xyz[:, 0].copy(), "y": xyz[:, 1].copy(), "z": xyz[:, 2].copy()}


# counter-based random numbers shared with the GPU scene generator: value k of
# stream t under seed s is SplitMix64(s + 0x9E3779B97F4A7C15 * (t * 2^40 + k + 1)),
# its top 24 bits an exact float in [0, 1)
_GOLDEN = np.uint64(0x9E3779B97F4A7C15)


def _splitmix64(z: np.ndarray) -> np.ndarray:
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def uniform01(seed: int, stream: int, k: np.ndarray) -> np.ndarray:
    """float32 uniforms in [0, 1) of `stream` at counters k."""
    with np.errstate(over="ignore"):
        c = (np.uint64(stream) << np.uint64(40)) + k.astype(np.uint64) + np.uint64(1)
        z = _splitmix64(np.uint64(seed) + _GOLDEN * c)
    return (z >> np.uint64(40)).astype(np.uint32).astype(np.float32) * np.float32(1.0 / 16777216.0)


def _symmetric(u: np.ndarray, a: np.float32) -> np.ndarray:
    return (np.float32(2.0) * u - np.float32(1.0)) * a


_ALPHA = {"C2": 21.0 / (2.0 * np.pi), "B3": 16.0 / np.pi, "W6": 1365.0 / (64.0 * np.pi),
          "COS": np.pi / (4.0 * np.pi ** 2 - 30.0)}


def _shape(kernel: str, q: np.ndarray) -> np.ndarray:
    """Kernel shape functions w(q) of the four smoothing kernels."""
    t = np.maximum(0.0, 1.0 - q)
    if kernel == "C2":
        return t ** 4 * (4 * q + 1)
    if kernel == "B3":
        return t ** 3 - 4 * np.clip(0.5 - q, 0, 1) ** 3
    if kernel == "W6":
        return t ** 8 * (32 * q ** 3 + 25 * q ** 2 + 8 * q + 1)
    qq = np.minimum(1.0, q)
    return 4 * np.cos(np.pi * qq) + np.cos(2 * np.pi * qq) + 3


def lattice_density_factor(kernel: str) -> float:
    """sum_j h^3 W(x_ij) over a cubic lattice of spacing h at support 2h: the
    SPH density of a perfect lattice of masses rho0 h^3, in units of rho0
    (C2 1.034, B3 1.000, W6 1.169, COS 0.988)."""
    r = np.arange(-2, 3, dtype=np.float64)
    X, Y, Z = np.meshgrid(r, r, r, indexing="ij")
    q = np.sqrt(X ** 2 + Y ** 2 + Z ** 2).ravel() / 2.0
    return float((_ALPHA[kernel] / 8.0 * _shape(kernel, np.minimum(q, 1.0))).sum())


def fluid_block(counts, h: float, origin, rho0: float, jitter: float, seed: int,
                velocity_noise: float = 0.0, mass_kernel: str | None = None,
                first: int = 0) -> dict:
    """counts[0] x counts[1] x counts[2] lattice at spacing h from `origin`,
    x fastest (the reference's _init_box_kernel, scene.cu:14-37), with
    uniform jitter in [-jitter, jitter] * h per axis and velocities uniform
    in [-velocity_noise, velocity_noise], drawn from the counter-based
    generator at the particle's index (first + q): bit for bit what
    reyn_scene_fluid_block writes on the GPU."""
    nx, ny, nz = counts
    q = np.arange(nx * ny * nz, dtype=np.int64)
    i, j, k = q % nx, (q // nx) % ny, q // (nx * ny)
    hh = np.float32(h)
    o = np.asarray(origin, np.float32)
    g = q + first
    pos = []
    for axis, idx in enumerate((i, j, k)):
        p = o[axis] + idx.astype(np.float32) * hh
        if jitter:
            p = p + _symmetric(uniform01(seed, axis, g), np.float32(jitter) * hh)
        pos.append(p.astype(np.float32))
    n = q.size
    vel = []
    for axis in range(3):
        if velocity_noise:
            vel.append(_symmetric(uniform01(seed, 3 + axis, g), np.float32(velocity_noise)))
        else:
            vel.append(np.zeros(n, np.float32))
    m = np.float32(np.float32(np.float32(rho0) * hh) * hh) * hh
    if mass_kernel:
        # calibrated so that the unjittered lattice sits exactly at rho0
        m = np.float32(float(m) / lattice_density_factor(mass_kernel))
    return {"x": pos[0], "y": pos[1], "z": pos[2], "vx": vel[0], "vy": vel[1], "vz": vel[2],
            "m": np.full(n, m, np.float32), "id": np.arange(first, first + n, dtype=np.float32)}


def dam_break(counts, h: float, box, rho0: float = 1000.0, jitter: float = 0.1,
              seed: int = 1, velocity_noise: float = 0.0, name: str = "dam_break",
              mass_kernel: str | None = None, gap: float = 1.0) -> Scene:
    """A fluid block `gap` spacings away from the lower corner of box
    [0, box]. Fluid masses are rho0 h^3 (the reference's), or calibrated to
    the lattice density of `mass_kernel` when given. A gap of one spacing puts
    the first fluid layer inside the walls' kernel support, where one layer of
    Akinci samples over-densifies it by 5-15 %; 1.5 spacings starts the block
    free of wall contact."""
    box_max = np.asarray(box, np.float32)
    box_min = np.zeros(3, np.float32)
    o = gap * h
    fl = fluid_block(counts, h, (o, o, o), rho0, jitter, seed, velocity_noise, mass_kernel)
    bd = box_walls(box_min, box_max, h)
    return Scene(name, h, rho0, fl, bd, box_min, box_max,
                 {"counts": list(counts), "box": list(map(float, box)), "jitter": jitter,
                  "seed": seed})


def rest_mass(h: float, rho0: float, mass_kernel: str | None = None) -> float:
    """rho0 h^3 in float32 (scene.cu:36), calibrated to the lattice density of
    `mass_kernel` when given."""
    hh = np.float32(h)
    m = np.float32(np.float32(np.float32(rho0) * hh) * hh) * hh
    if mass_kernel:
        m = np.float32(float(m) / lattice_density_factor(mass_kernel))
    return float(m)


def dam_break_on_device(counts, h: float, box, rho0: float = 1000.0, jitter: float = 0.1,
                        seed: int = 1, velocity_noise: float = 0.0,
                        mass_kernel: str | None = None, gap: float = 1.0, stream=None):
    """The dam_break scene generated on the GPU (reyn_scene_fluid_block and
    reyn_scene_box_walls): the same arrays, without a host copy. Returns the
    particle state, the wall samples as three device tensors, and the box."""
    import reyn_b200 as rb
    n = int(counts[0]) * int(counts[1]) * int(counts[2])
    st = rb.Particles(n, rho0)
    o = np.float32(gap * h)
    rb.scene_fluid_block(st, counts, (o, o, o), h, rest_mass(h, rho0, mass_kernel), jitter,
                         velocity_noise, seed, stream=stream)
    box_min = np.zeros(3, np.float32)
    box_max = np.asarray(box, np.float32)
    walls = rb.scene_box_walls(box_min, box_max, h, stream=stream)
    return st, walls, box_min, box_max


@dataclass
class Batch:
    """Independent scenes sharing spacing and kernel: scene s owns fluid
    particles first[s] .. first[s+1]-1 and wall samples bfirst[s] ..
    bfirst[s+1]-1, in its own box [0, box_max[s]] (all boxes share the
    origin; the frame is their union)."""
    h: float
    rho0: float
    fluid: dict
    bdy: dict
    first: np.ndarray
    bfirst: np.ndarray
    box_min: np.ndarray   # (n_scenes, 3)
    box_max: np.ndarray   # (n_scenes, 3)
    counts: list

    @property
    def n_scenes(self) -> int:
        return int(self.first.size - 1)

    @property
    def frame_min(self) -> np.ndarray:
        return self.box_min.min(0)

    @property
    def frame_max(self) -> np.ndarray:
        return self.box_max.max(0)


def batch_counts(n_scenes: int, nmin: int, nmax: int, seed: int) -> list:
    """Per-scene fluid cubes with particle counts drawn log-uniform from
    [nmin, nmax] (counter-based, stream 6): cube edges of round(N^(1/3))."""
    u = uniform01(seed, 6, np.arange(n_scenes)).astype(np.float64)
    n = np.exp(np.log(nmin) + u * (np.log(nmax) - np.log(nmin)))
    edge = np.maximum(2, np.rint(np.cbrt(n))).astype(int)
    return [(int(e), int(e), int(e)) for e in edge]


def batched_dam_breaks(counts, h: float, rho0: float = 1000.0, jitter: float = 0.05,
                       seed: int = 4, mass_kernel: str | None = None,
                       gap: float = 1.5) -> Batch:
    """One dam break per entry of `counts`: the block `gap` spacings from the
    corner of a box twice its width in x and 1.5 times in y and z."""
    fl, bd, first, bfirst, lo, hi = [], [], [0], [0], [], []
    for s, c in enumerate(counts):
        ext = np.asarray(c, np.float64) * h
        box = np.float32(np.array([2.0, 1.5, 1.5]) * ext + 2 * gap * h)
        o = gap * h
        f = fluid_block(c, h, (o, o, o), rho0, jitter, seed, mass_kernel=mass_kernel,
                        first=first[-1])
        w = box_walls((0, 0, 0), box, h)
        fl.append(f)
        bd.append(w)
        first.append(first[-1] + f["x"].size)
        bfirst.append(bfirst[-1] + w["x"].size)
        lo.append(np.zeros(3, np.float32))
        hi.append(box)
    fluid = {k: np.concatenate([f[k] for f in fl]) for k in fl[0]}
    bdy = {k: np.concatenate([w[k] for w in bd]) for k in ("x", "y", "z")}
    return Batch(h, rho0, fluid, bdy, np.asarray(first, np.uint32), np.asarray(bfirst, np.uint32),
                 np.asarray(lo, np.float32), np.asarray(hi, np.float32), list(counts))


def batched_pcisph(n_scenes: int = 256, seed: int = 4, nmin: int = 2000,
                   nmax: int = 200000) -> Batch:
    """The batched PCISPH workload: n_scenes fluid cubes of log-uniform
    particle counts in [nmin, nmax] at spacing 0.01, each a dam break in its
    own closed box."""
    return batched_dam_breaks(batch_counts(n_scenes, nmin, nmax, seed), 0.01, seed=seed)


def sesph_small(seed: int = 1) -> Scene:
    """SESPH dam break: 32^3 fluid particles at spacing 0.02, jitter +-0.1 h,
    unit box with Akinci walls at spacing 0.02."""
    return dam_break((32, 32, 32), 0.02, (1.0, 1.0, 1.0), 1000.0, 0.1, seed,
                     name="sesph_32k")


def iisph_4m(seed: int = 3) -> Scene:
    """IISPH dam break: 256 x 128 x 128 = 4,194,304 fluid particles at spacing
    0.005, jitter +-0.05 h, in a 2 x 1 x 1 box with Akinci walls; masses
    calibrated to the Wendland C2 lattice density, 1.5 h from the walls."""
    return dam_break((256, 128, 128), 0.005, (2.0, 1.0, 1.0), 1000.0, 0.05, seed,
                     name="iisph_4m", mass_kernel="C2", gap=1.5)


def uniform_cloud(n: int = 1 << 20, seed: int = 2):
    """Neighbour-search microbenchmark: n uniform-random points in [0,1)^3."""
    rng = np.random.Generator(np.random.PCG64(seed))
    p = rng.random((n, 3), dtype=np.float32)
    return p[:, 0].copy(), p[:, 1].copy(), p[:, 2].copy()


def scaled(counts, h: float, box, **kw) -> Scene:
    """A smaller dam break with the same structure (for parity tests)."""
    return dam_break(counts, h, box, **kw)
