"""Host scene generator: its counter-based random numbers are SplitMix64,
pinned against the published output sequence for seed 1234567, and the
lattice/wall layouts hold the documented counts and spacing."""
import numpy as np

from reyn_b200 import scenes


def test_splitmix64_known_answer():
    # the first outputs of SplitMix64 seeded with 1234567 (Steele, Lea and
    # Flood's generator as published with its reference implementation)
    want = [6457827717110365317, 3203168211198807973, 9817491932198370423,
            4593380528125082431, 16408922859458223821]
    with np.errstate(over="ignore"):
        z = np.uint64(1234567) + scenes._GOLDEN * np.arange(1, 6, dtype=np.uint64)
    np.testing.assert_array_equal(scenes._splitmix64(z), np.array(want, np.uint64))


def test_uniforms_are_exact_24_bit_fractions():
    u = scenes.uniform01(7, 1, np.arange(100000))
    assert u.dtype == np.float32 and u.min() >= 0 and u.max() < 1
    assert np.all((u * np.float32(16777216.0)) % 1 == 0)
    assert abs(float(u.mean()) - 0.5) < 5e-3


def test_fluid_block_layout():
    fl = scenes.fluid_block((4, 3, 2), 0.1, (1.0, 2.0, 3.0), 1000.0, 0.0, 1)
    assert fl["x"].size == 24
    np.testing.assert_allclose(fl["x"][:4], [1.0, 1.1, 1.2, 1.3], rtol=1e-6)
    np.testing.assert_allclose(fl["y"][[0, 4, 8]], [2.0, 2.1, 2.2], rtol=1e-6)
    np.testing.assert_allclose(fl["z"][[0, 12]], [3.0, 3.1], rtol=1e-6)
    jit = scenes.fluid_block((4, 3, 2), 0.1, (1.0, 2.0, 3.0), 1000.0, 0.2, 1)
    d = np.abs(jit["x"] - fl["x"])
    assert d.max() <= 0.02 + 1e-6 and d.max() > 0


def test_box_walls_counts():
    w = scenes.box_walls((0, 0, 0), (1.0, 0.5, 0.25), 0.05)
    n = np.array([20, 10, 5])
    want = 2 * (n[1] + 1) * (n[2] + 1) + 2 * (n[0] - 1) * (n[2] + 1) + 2 * (n[0] - 1) * (n[1] - 1)
    assert w["x"].size == want
    pts = np.stack([w["x"], w["y"], w["z"]], 1)
    assert np.unique(pts, axis=0).shape[0] == want
