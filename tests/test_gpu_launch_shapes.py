"""Launch shapes of one context (p3m_set_launch_shape) and its autotuner
(p3m_autotune).

The FFT lines per CTA and the short-range block size change how the work is
cut, never what is computed: every shape must give the same bits. The
autotuner times steps under each shape and must put the context's state
(bodies, materials, accelerations, step counter, hence the reorder phase)
back, so that a tuned context continues exactly like an untuned one.
"""

import numpy as np
import pytest

from gravity_b200.pipeline import GravityPipeline, P3MArgumentError

from helpers import clustered, small_torus

pytestmark = pytest.mark.gpu

SHAPES = [(0, 256), (1, 64), (2, 128), (4, 256), (8, 64), (16, 128)]


def _run(sc, shape, steps):
    with GravityPipeline(sc.config) as p:
        p.upload(sc.bodies, sc.materials)
        p.set_launch_shape(*shape)
        p.initialize_acceleration(sc.n)
        p.step(sc.n, steps)
        return p.download(sc.n)


@pytest.mark.parametrize("scene", ["torus", "walls"])
def test_every_launch_shape_gives_the_same_bits(cuda_device, scene):
    sc = (small_torus(n=30_000, grid=(256, 128)) if scene == "torus"
          else clustered(n=20_000, grid=(128, 64), bounded=True))
    want = _run(sc, SHAPES[0], 5)
    for shape in SHAPES[1:]:
        got = _run(sc, shape, 5)
        for g, w, name in zip(got, want, ("bodies", "materials", "acceleration")):
            np.testing.assert_array_equal(g, w, err_msg=f"shape {shape}: {name}")


def test_autotune_puts_the_state_back(cuda_device):
    sc = small_torus(n=50_000, grid=(512, 256))
    n = sc.n
    with GravityPipeline(sc.config) as tuned, GravityPipeline(sc.config) as plain:
        for p in (tuned, plain):
            p.upload(sc.bodies, sc.materials)
            p.initialize_acceleration(n)
            p.step(n, 3)  # an odd count: the next step is not a reorder step
        before = tuned.download(n)
        fft_lines, threads = tuned.autotune(n, 2)
        assert fft_lines in (0, 1, 2, 4, 8) and threads in (64, 128, 256)
        after = tuned.download(n)
        for a, b, name in zip(after, before, ("bodies", "materials", "acceleration")):
            np.testing.assert_array_equal(a, b, err_msg=f"autotune changed the {name}")
        # Same step counter: both contexts reorder on the same later steps.
        for p in (tuned, plain):
            p.step(n, 4)
        for a, b, name in zip(tuned.download(n), plain.download(n),
                              ("bodies", "materials", "acceleration")):
            np.testing.assert_array_equal(a, b, err_msg=f"tuned vs untuned: {name}")
        assert tuned.wait_timeouts() == 0


def test_launch_shape_rejects_invalid_values(cuda_device):
    sc = small_torus(n=1000)
    with GravityPipeline(sc.config) as p:
        with pytest.raises(P3MArgumentError):
            p.set_launch_shape(17, 256)
        with pytest.raises(P3MArgumentError):
            p.set_launch_shape(-1, 256)
        with pytest.raises(P3MArgumentError):
            p.set_launch_shape(0, 100)
        with pytest.raises(P3MArgumentError):
            p.autotune(sc.n, 0)
