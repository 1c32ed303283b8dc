"""p3m_step_io: one step with its host copies pipelined against the
neighbouring steps. Over a sequence of steps whose inputs differ from step
to step, it must give the same bits as the serial calls it stands for —
p3m_upload_state, p3m_step, p3m_download_state — for every step's output,
with the reorder phases, the walls and NULL inputs or outputs."""

import numpy as np
import pytest

from gravity_b200.pipeline import GravityPipeline, PinnedArray

from helpers import clustered, small_torus

pytestmark = pytest.mark.gpu


def _inputs(sc, steps, seed=1):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(steps):
        b = sc.bodies.copy()
        # Move a few bodies per step (a host edit between steps).
        idx = rng.choice(sc.n, size=32, replace=False)
        b[idx, :2] = np.minimum(rng.uniform(0, 1, (32, 2)), 0.99999994).astype(np.float32)
        out.append(b)
    return out


@pytest.mark.parametrize("scene", ["torus", "walls"])
def test_pipelined_steps_equal_serial_steps(cuda_device, scene):
    sc = (small_torus(n=40_000, grid=(256, 128)) if scene == "torus"
          else clustered(n=20_000, grid=(128, 64), bounded=True))
    n, steps = sc.n, 6
    ins = _inputs(sc, steps)
    with GravityPipeline(sc.config) as serial:
        serial.upload(sc.bodies, sc.materials)
        serial.initialize_acceleration(n)
        want = []
        for b in ins:
            serial.upload_n(n, b)
            serial.step(n)
            want.append(serial.download(n)[0])
    pins = [PinnedArray((n, 4)) for _ in range(steps)]
    outs = [PinnedArray((n, 4)) for _ in range(steps)]
    try:
        for p, b in zip(pins, ins):
            p.array[:] = b
        with GravityPipeline(sc.config) as piped:
            piped.upload(sc.bodies, sc.materials)
            piped.initialize_acceleration(n)
            for k in range(steps):
                piped.step_io(n, pins[k].array, outs[k].array)
            piped.synchronize()
            for k in range(steps):
                np.testing.assert_array_equal(outs[k].array, want[k], err_msg=f"step {k}")
            # The context's state is the last step's.
            np.testing.assert_array_equal(piped.download(n)[0], want[-1])
    finally:
        for a in pins + outs:
            a.free()


def test_step_io_without_input_or_output(cuda_device):
    sc = small_torus(n=20_000, grid=(256, 128))
    n = sc.n
    with GravityPipeline(sc.config) as a, GravityPipeline(sc.config) as b:
        for p in (a, b):
            p.upload(sc.bodies, sc.materials)
            p.initialize_acceleration(n)
        out = PinnedArray((n, 4))
        try:
            a.step_io(n)                       # no copies: a plain step
            a.step_io(n, None, out.array)      # download only
            a.synchronize()
            b.step(n, 2)
            np.testing.assert_array_equal(out.array, b.download(n)[0])
            with pytest.raises(ValueError):
                a.step_io(n, np.zeros((n - 1, 4), np.float32))
        finally:
            out.free()
