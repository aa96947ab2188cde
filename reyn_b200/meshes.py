"""Procedural triangle meshes (host numpy arrays) for the mesh entry points:
an icosphere, a subdivided box and a torus, all wound so that
cross(b - a, c - a) points outward (the orientation the inside test of
scene.cu:120-130 assumes), plus a Wavefront OBJ writer.

Each generator returns (vertices (V, 3) float64, faces (F, 3) uint32).
"""
from __future__ import annotations

import numpy as np


def icosphere(subdivisions: int = 2, radius: float = 1.0, center=(0.0, 0.0, 0.0)):
    """A sphere from a subdivided icosahedron (each level splits every face
    into four and pushes the new vertices onto the sphere)."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t),
         (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
         (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
         (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    verts = [np.array(p, float) / np.linalg.norm(p) for p in v]
    faces = list(f)
    for _ in range(subdivisions):
        mid: dict = {}

        def midpoint(a, b):
            key = (min(a, b), max(a, b))
            if key not in mid:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                mid[key] = len(verts) - 1
            return mid[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = midpoint(a, b), midpoint(b, c), midpoint(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    V = np.array(verts) * radius + np.asarray(center, float)
    return V, np.array(faces, np.uint32)


def box(lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), divisions: int = 1):
    """The surface of an axis-aligned box, each face a divisions x divisions
    grid of quads split into two triangles."""
    lo = np.asarray(lo, float)
    hi = np.asarray(hi, float)
    n = int(divisions)
    verts: list = []
    faces: list = []
    for axis in range(3):
        u, w = (axis + 1) % 3, (axis + 2) % 3
        for side, val in ((0, lo[axis]), (1, hi[axis])):
            base = len(verts)
            for j in range(n + 1):
                for i in range(n + 1):
                    p = np.empty(3)
                    p[axis] = val
                    p[u] = lo[u] + (hi[u] - lo[u]) * i / n
                    p[w] = lo[w] + (hi[w] - lo[w]) * j / n
                    verts.append(p)
            for j in range(n):
                for i in range(n):
                    a = base + j * (n + 1) + i
                    b, c, d = a + 1, a + n + 1, a + n + 2
                    # (u, w, axis) is right-handed: counter-clockwise in (u, w)
                    # faces +axis; the low side is reversed
                    if side == 1:
                        faces += [(a, b, d), (a, d, c)]
                    else:
                        faces += [(a, d, b), (a, c, d)]
    # merge the copies of edge and corner vertices (computed identically)
    index: dict = {}
    remap = np.empty(len(verts), np.int64)
    for k, p in enumerate(verts):
        remap[k] = index.setdefault(tuple(p), len(index))
    uniq = np.empty((len(index), 3))
    for p, k in index.items():
        uniq[k] = p
    return uniq, remap[np.array(faces, np.int64)].astype(np.uint32)


def torus(major: float = 1.0, minor: float = 0.3, nu: int = 32, nv: int = 16,
          center=(0.0, 0.0, 0.0)):
    """A torus around the z axis, nu segments around it and nv around the tube."""
    verts = []
    for i in range(nu):
        a = 2 * np.pi * i / nu
        for j in range(nv):
            b = 2 * np.pi * j / nv
            r = major + minor * np.cos(b)
            verts.append((r * np.cos(a), r * np.sin(a), minor * np.sin(b)))
    faces = []
    for i in range(nu):
        for j in range(nv):
            a = i * nv + j
            b = ((i + 1) % nu) * nv + j
            c = ((i + 1) % nu) * nv + (j + 1) % nv
            d = i * nv + (j + 1) % nv
            faces += [(a, b, c), (a, c, d)]
    return np.array(verts) + np.asarray(center, float), np.array(faces, np.uint32)


def perturb(verts, amplitude: float, seed: int = 0):
    """Vertices moved by a seeded uniform offset in [-amplitude, amplitude]^3."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return np.asarray(verts, float) + rng.uniform(-amplitude, amplitude, np.shape(verts))


def signed_volume(verts, faces) -> float:
    """Sum of a . (b x c) / 6 over the faces: positive for outward winding."""
    v = np.asarray(verts, float)
    f = np.asarray(faces, np.int64)
    a, b, c = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    return float(np.einsum("ij,ij->i", a, np.cross(b, c)).sum() / 6.0)


def write_obj(path: str, shapes) -> None:
    """Writes shapes [(name, verts, faces), ...] to one OBJ file (1-based
    indices, one "o" record per shape)."""
    with open(path, "w") as fh:
        base = 0
        for name, v, f in shapes:
            fh.write(f"o {name}\n")
            for p in np.asarray(v, float):
                fh.write(f"v {float(p[0])!r} {float(p[1])!r} {float(p[2])!r}\n")
            for t in np.asarray(f, np.int64):
                fh.write(f"f {t[0] + base + 1} {t[1] + base + 1} {t[2] + base + 1}\n")
            base += len(v)
