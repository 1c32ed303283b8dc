"""Body state on disk (gravity_b200/state_io.py): the reference's vec4 layout
(Scenario.kt:286-297, 571-580) round-trips bit for bit for every seeded
workload, and normalized() follows ScenarioBuilder.normalized() in FP32."""

import numpy as np
import pytest

from gravity_b200 import scenarios, state_io

WORKLOADS = {
    "uniform_torus": lambda: scenarios.uniform_torus(),
    "plummer_walls": lambda: scenarios.plummer_walls(),
    "lattice_scale_512x256": lambda: scenarios.lattice_scale(n=120_000, grid=(512, 256)),
    "adjoint_cluster": lambda: scenarios.adjoint_cluster(),
}


@pytest.mark.parametrize("name", sorted(WORKLOADS))
def test_seeded_workload_round_trips(tmp_path, name):
    sc = WORKLOADS[name]()
    st = state_io.from_scenario(sc, seed=7)
    p = tmp_path / f"{name}.grvs"
    state_io.save(p, st)
    assert p.stat().st_size == 32 + sc.n * 32
    back = state_io.load(p)
    assert back.viewport == (sc.config.viewport_width, sc.config.viewport_height)
    assert back.seed == 7 and back.n == sc.n and back.acceleration is None
    assert back.bodies.tobytes() == sc.bodies.astype(np.float32).tobytes()
    assert back.materials.tobytes() == sc.materials.astype(np.float32).tobytes()


def test_batch_simulations_round_trip_with_accelerations(tmp_path):
    rng = np.random.default_rng(3)
    for i, sc in enumerate(scenarios.batch(sims=6)):
        acc = rng.normal(0, 1e-3, (sc.n, 2)).astype(np.float32)
        st = state_io.BodyState(sc.bodies, None, acc,
                                (sc.config.viewport_width, sc.config.viewport_height), i)
        p = tmp_path / f"b{i}.grvs"
        state_io.save(p, st)
        back = state_io.load(p)
        assert back.materials is None
        assert back.bodies.tobytes() == sc.bodies.tobytes()
        assert back.acceleration.tobytes() == acc.tobytes()


def test_normalized_matches_the_reference_formula():
    w, h = 2560.0, 1440.0
    px = np.array([
        [0.0, 0.0, 5.0, -5.0],
        [2560.0, 1440.0, 0.0, 0.0],          # exactly the far edge: wraps to 0
        [-1.0, -0.5, 1.0, 1.0],              # negative: wraps below 1
        [2559.9998, 1439.9999, 0.0, 0.0],    # rounds to 1 after wrapping -> 0
        [5120.5, 2881.0, 0.0, 0.0],          # more than one period
    ], np.float32)
    got = state_io.normalized(px, w, h)
    for row, out in zip(px, got):
        for axis, size in ((0, np.float32(w)), (1, np.float32(h))):
            v = np.float32(row[axis]) / size
            f = np.float32(v - np.float32(np.floor(v)))
            exp = np.float32(0.0) if f >= np.float32(1.0) else f
            assert out[axis] == exp
            assert 0.0 <= out[axis] < 1.0
        assert out[2] == np.float32(row[2]) / np.float32(w)
        assert out[3] == np.float32(row[3]) / np.float32(h)


def test_corrupt_files_are_rejected(tmp_path):
    sc = scenarios.uniform_torus(n=100)
    p = tmp_path / "s.grvs"
    state_io.save(p, state_io.from_scenario(sc))
    data = p.read_bytes()
    for bad, what in ((b"XXXX" + data[4:], "magic"), (data[:-4], "truncated"),
                      (data + b"\0", "trailing")):
        q = tmp_path / "bad.grvs"
        q.write_bytes(bad)
        with pytest.raises(ValueError, match=what):
            state_io.load(q)
