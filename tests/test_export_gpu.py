"""State export: the PLY point cloud against the reference's own save_to_ply
(ply_io.cu:7-55, compiled unmodified) on the same positions, and the raw SoA
checkpoint's save/load round trip."""
import ctypes
import os

import numpy as np
import pytest

import oracle
from reyn_b200 import scenes

pytestmark = pytest.mark.gpu


def _split_ply(blob: bytes):
    head, _, payload = blob.partition(b"end_header\n")
    lines = head.decode("ascii").splitlines()
    return [ln for ln in lines if not ln.startswith("comment")], payload


def _state(n, seed):
    import reyn_b200 as rb
    rng = np.random.Generator(np.random.PCG64(seed))
    fl = {k: rng.random(n, dtype=np.float32) for k in ("x", "y", "z", "vx", "vy", "vz")}
    fl["m"] = np.full(n, 0.125, np.float32)
    st = rb.Particles(n, 1000.0)
    st.upload(fl)
    return st, fl


@pytest.mark.parametrize("n", [1, 1000, 100_000])
def test_ply_matches_reference_save_to_ply(cuda, tmp_path, n):
    st, fl = _state(n, 7 + n)
    ours = tmp_path / "engine.ply"
    st.save_ply(str(ours))
    st.close()
    ref = tmp_path / "reference.ply"
    L = oracle.ref_cuda()
    P = lambda a: np.ascontiguousarray(a, np.float32).ctypes.data_as(ctypes.c_void_p)  # noqa
    rc = L.ref_save_ply(ctypes.c_uint(n), P(fl["x"]), P(fl["y"]), P(fl["z"]),
                        os.fsencode(str(ref)))
    assert rc == 0, L.ref_last_error()
    h_ours, p_ours = _split_ply(ours.read_bytes())
    h_ref, p_ref = _split_ply(ref.read_bytes())
    assert h_ours == h_ref  # same format line, vertex count and properties
    assert p_ours == p_ref  # byte-identical payload
    want = np.stack([fl["x"], fl["y"], fl["z"]], 1).astype("<f4").tobytes()
    assert p_ours == want


def test_raw_state_round_trip(cuda, tmp_path):
    import reyn_b200 as rb
    sc = scenes.dam_break((12, 10, 8), 0.02, (0.4, 0.4, 0.4), velocity_noise=0.1, seed=3)
    st = rb.Particles(sc.n, sc.rho0)
    st.upload(sc.fluid)
    path = tmp_path / "state.raw"
    st.save_raw(str(path))
    assert path.stat().st_size == 20 + 7 * 4 * sc.n
    back = rb.Particles(sc.n, sc.rho0)
    back.load_raw(str(path))
    a, b = st.download(), back.download()
    for k in a:
        np.testing.assert_array_equal(a[k], b[k])
    # a file for a different particle count, and a file that is not a state
    other = rb.Particles(sc.n + 1, sc.rho0)
    with pytest.raises(rb.ReynError):
        other.load_raw(str(path))
    bad = tmp_path / "bad.raw"
    bad.write_bytes(b"NOTASTATEFILE" + bytes(64))
    with pytest.raises(rb.ReynError):
        back.load_raw(str(bad))
    for o in (st, back, other):
        o.close()
