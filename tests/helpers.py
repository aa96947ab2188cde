"""Shared test helpers: run the CUDA engine and the CPU oracle on the same
inputs and compare per particle by carried ID."""
from __future__ import annotations

import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIELDS = ("x", "y", "z", "vx", "vy", "vz", "m")


def golden(name: str):
    path = os.path.join(GOLDEN, name)
    if not os.path.exists(path):
        return None
    return np.load(path)


def assert_close(a, b, rtol: float, atol_frac: float = 0.0, what: str = ""):
    """|a - b| <= atol + rtol |b| elementwise, atol = atol_frac * max|b|."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    assert a.shape == b.shape, (what, a.shape, b.shape)
    scale = float(np.max(np.abs(b))) if b.size else 0.0
    atol = atol_frac * scale
    err = np.abs(a - b)
    bad = err > atol + rtol * np.abs(b)
    if bad.any():
        k = int(np.argmax(err - (atol + rtol * np.abs(b))))
        raise AssertionError(
            f"{what}: {int(bad.sum())}/{a.size} outside rtol={rtol} atol={atol:.3g}; "
            f"worst at {k}: {a.flat[k]!r} vs {b.flat[k]!r} (max|b|={scale:.4g})")


def by_id(arrs: dict, ids: np.ndarray) -> dict:
    order = np.argsort(ids.astype(np.int64))
    return {k: np.asarray(v)[order] for k, v in arrs.items()}


def run_engine(scheme: int, kind: int, fluid: dict, bdy: dict, box_min, box_max, h: float,
               rho0: float, nu: float, dt: float, steps: int, params=None, cell_ratio=0.5,
               order=0, resort=True):
    """The reference main loop on the engine: construct_and_reorder (with
    the particle ID as an extra array), solver step, hard bounds. With
    resort=False the grid is built by construct over the state's positions
    and the particles keep their order (the solvers' Resort::no form)."""
    import torch

    import reyn_b200 as rb

    dev = torch.device("cuda:0")
    n = int(np.asarray(fluid["x"]).size)
    st = rb.Particles(n, rho0)
    st.upload(fluid)
    ids = torch.tensor(np.asarray(fluid["id"], np.float32), device=dev)
    nb = int(np.asarray(bdy["x"]).size)
    bt = {k: torch.tensor(np.asarray(bdy[k], np.float32), device=dev) for k in ("x", "y", "z")}
    bm = torch.tensor(np.asarray(bdy["m"], np.float32), device=dev) if "m" in bdy else None
    bd = rb.Boundary(bt["x"], bt["y"], bt["z"], bm, h=h, rho0=rho0, mass_iters=5) if nb else None
    grid = rb.Grid(box_min, box_max, 2.0 * h, cell_ratio, order)
    prm = params or rb.reference_params(scheme, kind, h, rho0, nu)
    sv = rb.Solver(scheme, prm, n)
    iters = []
    for _ in range(steps):
        if resort:
            grid.construct_and_reorder(st, [ids])
        else:
            grid.construct_state(st)
        iters.append(sv.step(st, grid, bd, dt))
        rb.enforce_bounds(st, box_min, box_max)
    torch.cuda.synchronize()
    out = st.download()
    buf = sv.buffers()
    for k in ("rho", "p", "aii", "sii", "ax", "ay", "az"):
        out[k] = rb.device_to_numpy(getattr(buf, k), n)
    out["id"] = ids.cpu().numpy()
    out["iters"] = iters
    for o in (sv, grid, bd, st):
        if o is not None:
            o.close()
    return out


def run_oracle(scheme: int, kind: int, fluid: dict, bdy: dict, box_min, box_max, h: float,
               rho0: float, nu: float, dt: float, steps: int, params=None):
    import oracle

    prm = params or oracle.reference_params(scheme, kind, h, rho0, nu)
    r = oracle.run(prm, fluid, bdy, box_min, box_max, dt, steps)
    out = dict(r.state)
    out.update(rho=r.rho, p=r.p, aii=r.aii, sii=r.sii, ax=r.a[:, 0], ay=r.a[:, 1],
               az=r.a[:, 2], iters=list(r.iters))
    return out


def fixture_outputs(g) -> dict:
    keys = ("x", "y", "z", "vx", "vy", "vz", "m", "id", "rho", "p", "aii", "sii", "ax", "ay",
            "az")
    return {k: g[f"out_{k}"] for k in keys}


def fixture_inputs(g):
    fluid = {k: g[f"in_{k}"] for k in ("x", "y", "z", "vx", "vy", "vz", "m", "id")}
    bdy = {"x": g["bx"], "y": g["by"], "z": g["bz"], "m": g["bm"]}
    return fluid, bdy


# per-quantity tolerances of a solver step against the reference (FP32, a
# different summation order and norm evaluation): relative + absolute as a
# fraction of the field's largest magnitude
STEP_TOL = {
    "x": (1e-6, 1e-6), "y": (1e-6, 1e-6), "z": (1e-6, 1e-6),
    "vx": (1e-4, 1e-4), "vy": (1e-4, 1e-4), "vz": (1e-4, 1e-4),
    "m": (0.0, 0.0), "rho": (1e-5, 1e-6),
    "p": (1e-3, 1e-3), "aii": (1e-4, 1e-5), "sii": (1e-3, 1e-3),
    "ax": (1e-3, 1e-3), "ay": (1e-3, 1e-3), "az": (1e-3, 1e-3),
}


def compare_steps(got: dict, want: dict, scheme: int, tol=STEP_TOL, what: str = ""):
    g = by_id({k: v for k, v in got.items() if k != "iters"}, got["id"])
    w = by_id({k: v for k, v in want.items() if k != "iters"}, want["id"])
    np.testing.assert_array_equal(g["id"], w["id"])
    keys = ["x", "y", "z", "vx", "vy", "vz", "m", "rho", "ax", "ay", "az"]
    if scheme == 2:
        keys += ["p", "aii", "sii"]
    for k in keys:
        rtol, af = tol[k]
        assert_close(g[k], w[k], rtol, af, f"{what}:{k}")
