"""FP64 restatement of the IISPH step — TEST INFRASTRUCTURE ONLY.

The error reference for the engine's precision modes: the same algorithm as
the FP32 oracle (oracle.cpp, which follows the reference's IISPH.cu), carried
out in double precision over explicit pair lists: scipy's k-d tree finds the
pairs on the host, and the arithmetic runs in torch float64 on the host or,
for large scenes, on a GPU (`device="cuda"`). The summation order differs
from any grid traversal, which FP64 makes irrelevant at the tolerances the
tests use. Both the FP32 engine
and the mixed-precision engine are measured against it, so the cost of FP16
storage is stated as an error against the exact arithmetic rather than
against another FP32 result.

Reference functions restated (reyn, src/):
* kernels.cuh:32-64 (W, nabla) and :78-165 (C2, B3, W6, COS shapes)
* solver.cuh:18-38 compute_densities, :40-69 write_non_prs_acc_ff
* solver.cu:3-32 integrate_a_v_only, integrate
* IISPH.cu:11-66 diagonal element and source term, :68-98 pressure
  accelerations, :108-162 Jacobi update, :165-262 the step
* scene.cu:466-483 hard_enforce_bounds

Only tests/ import this module.
"""
from __future__ import annotations

import numpy as np
from scipy.spatial import cKDTree

C2, B3, W6, COS = 0, 1, 2, 3

_ALPHA = {C2: 21.0 / 2.0 / np.pi, B3: 16.0 / np.pi, W6: 1365.0 / 64.0 / np.pi,
          COS: np.pi / (4.0 * np.pi * np.pi - 30.0)}


def _w(kind: int, q):
    """kernels.cuh:78-165, w(q) on [0, 1]."""
    import torch
    t1 = torch.clamp_min(1.0 - q, 0.0)
    if kind == C2:
        return t1 ** 4 * (4.0 * q + 1.0)
    if kind == B3:
        t2 = torch.clamp(0.5 - q, 0.0, 1.0)
        return t1 ** 3 - 4.0 * t2 ** 3
    if kind == W6:
        return t1 ** 8 * (32.0 * q ** 3 + 25.0 * q * q + 8.0 * q + 1.0)
    s = np.pi * torch.clamp_max(q, 1.0)
    return 4.0 * torch.cos(s) + torch.cos(2.0 * s) + 3.0


def _dw(kind: int, q):
    """kernels.cuh:78-165, dw/dq on [0, 1]."""
    import torch
    t1 = torch.clamp_min(1.0 - q, 0.0)
    if kind == C2:
        return t1 ** 3 * (-20.0 * q)
    if kind == B3:
        t2 = torch.clamp(0.5 - q, 0.0, 1.0)
        return -3.0 * t1 * t1 + 12.0 * t2 * t2
    if kind == W6:
        return t1 ** 7 * (16.0 * q * q + 7.0 * q + 1.0) * (-22.0 * q)
    s = np.pi * torch.clamp_max(q, 1.0)
    return -4.0 * np.pi * torch.sin(s) - 2.0 * np.pi * torch.sin(2.0 * s)


def _pairs_host(a, b, hbar: float, same: bool):
    """(i, j) with |a_i - b_j| <= hbar from scipy's k-d tree on the host."""
    import torch
    an = a.cpu().numpy()
    ta = cKDTree(an)
    tb = ta if same else cKDTree(b.cpu().numpy())
    sp = ta.sparse_distance_matrix(tb, hbar, output_type="ndarray")
    # for a tree against itself the pairs include i == j (distance 0)
    i = torch.from_numpy(sp["i"].astype(np.int64)).to(a.device)
    j = torch.from_numpy(sp["j"].astype(np.int64)).to(a.device)
    return i, j


def _pairs_cells(a, b, hbar: float, chunk: int = 1 << 18):
    """(i, j) with |a_i - b_j| <= hbar by bucketing b into cubes of side hbar
    (torch, on the tensors' device): every a_i is tested against the points
    of the 27 cubes around its own, in FP64, a chunk of a at a time. Used for
    scenes too large for the host k-d tree; the pair set is the same."""
    import torch
    dev = a.device
    lo = torch.minimum(a.min(0).values, b.min(0).values) - hbar
    n3 = ((torch.maximum(a.max(0).values, b.max(0).values) + hbar - lo) / hbar).floor().long() + 2
    nx, ny = int(n3[0]), int(n3[1])
    cb = ((b - lo) / hbar).floor().long()
    kb = (cb[:, 2] * ny + cb[:, 1]) * nx + cb[:, 0]
    kb_sorted, order = torch.sort(kb)
    offs = torch.tensor([(dz * ny + dy) * nx + dx for dz in (-1, 0, 1) for dy in (-1, 0, 1)
                         for dx in (-1, 0, 1)], device=dev, dtype=torch.long)
    ii, jj = [], []
    h2 = hbar * hbar
    for c0 in range(0, a.shape[0], chunk):
        ac = a[c0:c0 + chunk]
        ca = ((ac - lo) / hbar).floor().long()
        ka = (ca[:, 2] * ny + ca[:, 1]) * nx + ca[:, 0]
        keys = (ka[:, None] + offs[None, :]).reshape(-1)
        st = torch.searchsorted(kb_sorted, keys)
        en = torch.searchsorted(kb_sorted, keys, right=True)
        cnt = en - st
        total = int(cnt.sum())
        if total == 0:
            continue
        seg = torch.repeat_interleave(torch.arange(keys.numel(), device=dev), cnt)
        first = torch.cumsum(cnt, 0) - cnt
        pos = torch.arange(total, device=dev) - first[seg] + st[seg]
        i = seg // offs.numel() + c0
        j = order[pos]
        d = a[i] - b[j]
        keep = (d * d).sum(1) <= h2
        ii.append(i[keep])
        jj.append(j[keep])
        del seg, first, pos, i, j, d, keep
    if not ii:
        z = torch.zeros(0, dtype=torch.long, device=dev)
        return z, z
    return torch.cat(ii), torch.cat(jj)


class _Pairs:
    """All pairs (i, j) with |x_i - x_j| < r, i from `a`, j from `b`, with the
    kernel value and the gradient factor: grad W_ij = gf * x_ij. a, b: (N, 3)
    float64 tensors; the pairs are found on the host (k-d tree) or, for
    tensors on a GPU with many points, by cube bucketing on the GPU."""

    def __init__(self, kind: int, hbar: float, a, b, same: bool):
        import torch
        if a.device.type == "cuda" and a.shape[0] > 1_000_000:
            i, j = _pairs_cells(a, b, hbar)
        else:
            i, j = _pairs_host(a, b, hbar, same)
        x = a[i] - b[j]
        r = torch.sqrt((x * x).sum(1))
        q = torch.clamp_max(r / hbar, 1.0)
        alpha = _ALPHA[kind]
        self.i, self.j, self.x, self.r2 = i, j, x, r * r
        self.w = alpha / hbar ** 3 * _w(kind, q)
        gf = alpha / hbar ** 4 * _dw(kind, q) / r
        self.gf = torch.where(torch.isfinite(gf), gf, torch.zeros_like(gf))
        self.n = a.shape[0]

    def sum(self, v):
        """sum over j of v (per pair, scalar or (P, 3)) into i."""
        import torch
        if v.dim() == 1:
            return torch.bincount(self.i, weights=v, minlength=self.n)
        return torch.stack([torch.bincount(self.i, weights=v[:, c], minlength=self.n)
                            for c in range(v.shape[1])], 1)


def iisph_run(kind: int, fluid: dict, bdy: dict, box_min, box_max, h: float, rho0: float,
              nu: float, g, dt: float, steps: int, iters: int, omega: float = 0.5,
              warmstart: bool = True, p=None, device: str = "cpu"):
    """`steps` IISPH steps with exactly `iters` Jacobi sweeps each (the
    convergence test is left out, so that every precision runs the same
    arithmetic). fluid: x, y, z, vx, vy, vz, m (any order); bdy: x, y, z, m.
    Returns dict of float64 numpy arrays in the input order: x, y, z, vx, vy,
    vz, rho, p, aii, sii."""
    import torch
    f64 = torch.float64

    def t(a):
        return torch.as_tensor(np.asarray(a, np.float64), dtype=f64, device=device)

    X = torch.stack([t(fluid[k]) for k in ("x", "y", "z")], 1)
    V = torch.stack([t(fluid[k]) for k in ("vx", "vy", "vz")], 1)
    m = t(fluid["m"])
    B = torch.stack([t(bdy[k]) for k in ("x", "y", "z")], 1)
    mb = t(bdy["m"])
    n = m.numel()
    P = torch.zeros(n, dtype=f64, device=device) if p is None else t(p).clone()
    lo = t(box_min)
    hi = t(box_max)
    grav = t(g)
    hbar = 2.0 * h
    r0i = 1.0 / (rho0 * rho0)
    rho = aii = sii = None
    for _ in range(steps):
        F = _Pairs(kind, hbar, X, X, True)
        Bp = _Pairs(kind, hbar, X, B, False) if mb.numel() else None
        mj = m[F.j]
        # densities (solver.cuh:18-38)
        rho = F.sum(mj * F.w)
        gb = torch.zeros((n, 3), dtype=f64, device=device)
        if Bp is not None:
            rho = rho + Bp.sum(mb[Bp.j] * Bp.w)
            gb = Bp.sum((mb[Bp.j] * Bp.gf)[:, None] * Bp.x)
        # gravity + artificial viscosity (solver.cuh:40-69), then v*
        vij = V[F.i] - V[F.j]
        vx = (vij * F.x).sum(1)
        s = 10.0 * nu * mj / rho[F.j] * vx / (F.r2 + 0.01 * h * h) * F.gf
        V = V + dt * (grav + F.sum(s[:, None] * F.x))
        # diagonal element and source term (IISPH.cu:11-66)
        vij = V[F.i] - V[F.j]
        mg = mj * F.gf
        gff = F.sum(mg[:, None] * F.x)
        gsq = F.sum(mg * F.gf * F.r2)
        vdiv = F.sum(mg * (vij * F.x).sum(1))
        grad = gff + gb
        aii = -dt * ((grad * grad).sum(1) + m * gsq) * r0i
        sii = (rho0 - rho) / dt - (vdiv + (V * gb).sum(1))

        def jacobi(Ap):  # IISPH.cu:108-117
            small = torch.abs(aii) < 1e-6
            d = torch.clamp_min(omega * (sii - Ap) / aii, 0.0)
            return torch.where(small, torch.zeros_like(d), d)

        def pacc(P):  # IISPH.cu:68-98
            sp = mj * (P[F.i] + P[F.j]) * F.gf
            return -r0i * (F.sum(sp[:, None] * F.x) + P[:, None] * gb)

        P = 0.5 * P if warmstart else jacobi(torch.zeros(n, dtype=f64, device=device))
        for _ in range(iters):  # IISPH.cu:119-162
            A = pacc(P)
            aij = A[F.i] - A[F.j]
            Ap = dt * (F.sum(mj * F.gf * (aij * F.x).sum(1)) + (A * gb).sum(1))
            P = P + jacobi(Ap)
        A = pacc(P)
        # integrate (solver.cu:15-32)
        V = V + dt * A
        X = X + dt * V
        # hard_enforce_bounds (scene.cu:466-483)
        touch = ((X <= lo) | (X >= hi)).any(1)
        V = torch.where(touch[:, None], V * -0.1, V)
        X = torch.minimum(torch.maximum(X, lo), hi)
        del F, Bp
    out = {"x": X[:, 0], "y": X[:, 1], "z": X[:, 2], "vx": V[:, 0], "vy": V[:, 1],
           "vz": V[:, 2], "rho": rho, "p": P, "aii": aii, "sii": sii}
    return {k: v.cpu().numpy() for k, v in out.items()}
