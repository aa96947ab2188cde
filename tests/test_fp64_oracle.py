"""The FP64 restatement of the IISPH step (oracle/fp64.py), the error
reference of the precision modes, pinned against the FP32 oracle (itself
pinned bit-exact against the reference's kernels and its CUDA fixtures): with
a fixed number of Jacobi sweeps both carry out the same arithmetic, so they
differ only by FP32 rounding."""
import numpy as np
import pytest

import oracle
from oracle import fp64
from reyn_b200 import scenes
from tests.helpers import by_id, run_oracle


@pytest.mark.parametrize("kind", [0, 1, 2, 3])
def test_fp64_step_matches_fp32_oracle(kind):
    sc = scenes.dam_break((20, 18, 16), 0.02, (0.6, 0.6, 0.6), velocity_noise=0.05, seed=5)
    bm = oracle.boundary_masses(sc.bdy["x"], sc.bdy["y"], sc.bdy["z"], sc.h, sc.rho0, 5)
    bdy = dict(sc.bdy, m=bm)
    prm = oracle.reference_params(2, kind, sc.h, sc.rho0, 0.01)
    prm.min_iter = prm.max_iter = 4
    steps, dt = 3, 1e-3
    want = fp64.iisph_run(kind, sc.fluid, bdy, sc.box_min, sc.box_max, sc.h, sc.rho0, 0.01,
                          prm.g, dt, steps, 4, prm.omega, bool(prm.warmstart))
    got = run_oracle(2, kind, sc.fluid, bdy, sc.box_min, sc.box_max, sc.h, sc.rho0, 0.01, dt,
                     steps, params=prm)
    assert got["iters"] == [4] * steps
    g = by_id({k: v for k, v in got.items() if k != "iters"}, got["id"])
    order = np.argsort(np.asarray(sc.fluid["id"]).astype(np.int64))
    w = {k: v[order] for k, v in want.items()}
    # FP32 rounding relative to the field's largest magnitude
    tol = {"x": 1e-6, "y": 1e-6, "z": 1e-6, "vx": 5e-5, "vy": 5e-5, "vz": 5e-5,
           "rho": 1e-5, "p": 1e-4, "aii": 5e-5, "sii": 5e-5}
    for k, t in tol.items():
        err = np.abs(g[k] - w[k]).max() / np.abs(w[k]).max()
        assert err <= t, (k, err)
