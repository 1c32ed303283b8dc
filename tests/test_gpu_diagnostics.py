"""FP64 diagnostics and the stage profiler, on the GPU, through the C-ABI."""

import numpy as np
import pytest

import oracle
from gravity_b200 import _abi
from gravity_b200.pipeline import GravityPipeline, kernel_launches

from helpers import clustered, small_torus

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("bounded", [False, True])
def test_direct_accel_f64_matches_oracle(cuda_device, bounded):
    sc = clustered(n=5000, bounded=bounded)
    targets = np.arange(0, sc.n, 13, dtype=np.int32)
    with GravityPipeline(sc.config) as gpu:
        gpu.upload(sc.bodies, sc.materials)
        got = gpu.direct_accel_f64(sc.n, targets)
    ref = oracle.direct_sum_f64(sc.bodies, sc.materials, targets, sc.config.to_abi(),
                                float(sc.n), bounded)
    np.testing.assert_allclose(got, ref, rtol=1e-10, atol=1e-12 * np.abs(ref).max())


def test_conservation_diagnostics(cuda_device):
    sc = small_torus(n=3000)
    w, h = sc.config.viewport_width, sc.config.viewport_height
    with GravityPipeline(sc.config) as gpu:
        gpu.upload(sc.bodies, sc.materials)
        d1 = gpu.diagnostics_f64(sc.n)
        d2 = gpu.diagnostics_f64(sc.n)
    b = sc.bodies.astype(np.float64)
    m = sc.materials[:, 0].astype(np.float64)
    vx, vy = b[:, 2] * w, b[:, 3] * h
    assert d1 == d2, "the reduction is deterministic"
    assert d1["mass"] == pytest.approx(m.sum(), rel=1e-12)
    assert d1["momentum"][0] == pytest.approx((m * vx).sum(), rel=1e-9, abs=1e-9)
    assert d1["momentum"][1] == pytest.approx((m * vy).sum(), rel=1e-9, abs=1e-9)
    assert d1["kinetic_energy"] == pytest.approx((0.5 * m * (vx * vx + vy * vy)).sum(), rel=1e-10)
    assert d1["center_of_mass"][0] == pytest.approx((m * b[:, 0] * w).sum() / m.sum(), rel=1e-10)


def test_profiler_times_every_stage_and_launches_are_counted(cuda_device):
    sc = small_torus(n=4000)
    with GravityPipeline(sc.config) as gpu:
        gpu.upload(sc.bodies, sc.materials)
        gpu.initialize_acceleration(sc.n)
        gpu.profile_enable(True)
        k0 = kernel_launches()
        gpu.step(sc.n, 4)
        stages = gpu.profile_read()
        gpu.profile_enable(False)
        assert kernel_launches() - k0 > 4 * 8
    for name in _abi.STAGES:
        ms, count = stages[name]
        expected = 2 if name == "spatial_sort" else 4
        assert count == expected, (name, count)
        assert ms > 0.0


def test_nonfinite_bodies_are_counted(cuda_device):
    sc = small_torus(n=1000)
    bodies = sc.bodies.copy()
    bodies[5, 2] = np.inf
    with GravityPipeline(sc.config.with_(spatial_sort_interval=0)) as gpu:
        gpu.upload(bodies, sc.materials)
        gpu.initialize_acceleration(sc.n)
        assert gpu.nonfinite_count() == 0
        gpu.step(sc.n)
        assert gpu.nonfinite_count() >= 1
