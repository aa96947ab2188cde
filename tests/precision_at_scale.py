"""States the precision modes' errors against the FP64 restatement of the
IISPH step (oracle/fp64.py, arithmetic in torch float64 on the GPU) on the
benchmark's scene at one eighth of its size: a 128 x 64 x 64 = 524,288
particle dam break at spacing 0.005 (the 4M scene's spacing, jitter, C2 lattice
masses and wall layout) in a 1 x 0.5 x 0.5 box. Each solver runs 3 steps of
exactly 4 Jacobi sweeps at dt 2e-4, as tests/test_mixed_precision_gpu.py does
at 5,760 particles; errors are per quantity relative to the field's largest
magnitude, plus the mean |rho - rho_FP64| / rho0. Test infrastructure: a
measurement run on a GPU, printed as one JSON line.

Usage: python tests/precision_at_scale.py [--scale K]  (K divides each axis)
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from oracle import fp64  # noqa: E402
from reyn_b200 import scenes  # noqa: E402
from tests.helpers import by_id, run_engine  # noqa: E402

FIELDS = ("x", "y", "z", "vx", "vy", "vz", "rho", "p", "aii", "sii")


def main():
    import reyn_b200 as rb
    ap = argparse.ArgumentParser()
    ap.add_argument("--scale", type=int, default=1)
    a = ap.parse_args()
    k = a.scale
    sc = scenes.dam_break((128 // k, 64 // k, 64 // k), 0.005, (1.0, 0.5, 0.5), 1000.0, 0.05, 3,
                          name="iisph_eighth", mass_kernel="C2", gap=1.5)
    bm = oracle.boundary_masses(sc.bdy["x"], sc.bdy["y"], sc.bdy["z"], sc.h, sc.rho0, 5)
    bdy = dict(sc.bdy, m=bm)
    steps, sweeps, dt = 3, 4, 2e-4
    t0 = time.perf_counter()
    prm0 = rb.reference_params(rb.IISPH, rb.C2, sc.h, sc.rho0, 0.01)
    want = fp64.iisph_run(rb.C2, sc.fluid, bdy, sc.box_min, sc.box_max, sc.h, sc.rho0, 0.01,
                          tuple(prm0.g), dt, steps, sweeps, prm0.omega, bool(prm0.warmstart),
                          device="cuda")
    t_fp64 = time.perf_counter() - t0
    order = np.argsort(np.asarray(sc.fluid["id"]).astype(np.int64))
    w = {f: v[order] for f, v in want.items()}
    res = {"particles": sc.n, "boundary_particles": int(sc.bdy["x"].size), "steps": steps,
           "sweeps_per_step": sweeps, "dt": dt, "fp64_seconds": round(t_fp64, 1)}
    for name, prec in (("fp32", rb.PRECISION_FP32), ("mixed", rb.PRECISION_MIXED),
                       ("mixed_pos16", rb.PRECISION_MIXED_POS16)):
        prm = rb.reference_params(rb.IISPH, rb.C2, sc.h, sc.rho0, 0.01)
        prm.min_iter = prm.max_iter = sweeps
        prm.eta = 1.0  # met after every sweep: exactly `sweeps` sweeps
        prm.precision = prec
        got = run_engine(2, rb.C2, sc.fluid, bdy, sc.box_min, sc.box_max, sc.h, sc.rho0, 0.01,
                         dt, steps, params=prm)
        assert got["iters"] == [sweeps] * steps
        g = by_id({f: v for f, v in got.items() if f != "iters"}, got["id"])
        err = {f: float(np.abs(g[f] - w[f]).max() / np.abs(w[f]).max()) for f in FIELDS}
        err["mean_abs_rho_rel"] = float(np.mean(np.abs(g["rho"] - w["rho"])) / sc.rho0)
        res[name] = {f: float(f"{v:.3g}") for f, v in err.items()}
    print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
