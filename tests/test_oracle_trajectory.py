"""The oracle's restatement of the aim preview (S/trajectory.comp) on fields
whose paths are known in closed form."""

import numpy as np

import oracle

from helpers import small_torus


def preview(sim, n, origin, velocity, **kw):
    out = sim.trajectory(n, origin, velocity, **kw)
    return out.reshape(-1, 6, 4)


def test_straight_line_without_gravity():
    sc = small_torus(n=500)
    with oracle.OracleSim(sc.config) as sim:
        sim.upload(sc.bodies, sc.materials)
        sim.set_mutual_gravity(False)
        sim.initialize_acceleration(sc.n)
        w, h = sc.config.viewport_width, sc.config.viewport_height
        steps = preview(sim, sc.n, (100.0, 200.0), (300.0, 0.0), steps=64, segment_px=6.0)
    # Constant velocity: each step covers target_segment_pixels (dt = 6/300 s
    # is inside [time_step, maximum_time_step]) along +x.
    first = steps[:, 0, :]
    valid = first[:, 3] >= 0
    assert valid.all()
    x_px = first[:, 0] * w
    np.testing.assert_allclose(np.diff(x_px), 6.0, atol=1e-3)
    np.testing.assert_allclose(first[:, 1] * h, 200.0, atol=1e-3)
    # Distances along the path are fractions of the whole path, increasing.
    d = first[:, 3]
    assert np.all(np.diff(d) > 0) and d[0] == 0.0 and d[-1] < 1.0


def test_path_stops_at_the_length_limit_and_wraps():
    sc = small_torus(n=500)
    with oracle.OracleSim(sc.config) as sim:
        sim.upload(sc.bodies, sc.materials)
        sim.set_mutual_gravity(False)
        sim.initialize_acceleration(sc.n)
        w, h = sc.config.viewport_width, sc.config.viewport_height
        diag = float(np.hypot(w, h))
        steps = preview(sim, sc.n, (w - 10.0, 50.0), (400.0, 0.0), steps=1024, segment_px=6.0)
    used = (steps[:, :, 3] >= 0).any(axis=1)
    n_used = int(used.sum())
    assert 0 < n_used < 1024
    assert not used[n_used:].any()
    # The path length is one viewport diagonal: the last distance fraction is 1.
    last = steps[n_used - 1]
    assert abs(last[last[:, 3] >= 0][:, 3].max() - 1.0) < 1e-6
    # Crossing the right edge splits a step into two pieces (four vertices).
    pieces = (steps[:, :, 3] >= 0).sum(axis=1)
    assert (pieces == 4).sum() >= 1
    assert abs(n_used * 6.0 - diag) <= 6.0
