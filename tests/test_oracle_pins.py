"""The oracle pinned against the reference's own tests and published numbers.

* FFT: Radix2FftLayoutTest.kt:17-188 — the shader's radix-2 layout checked
  bin by bin against an independent FFT (JTransforms 3.2 there; numpy's FP64
  FFT here, JTransforms is not available) at abs < 1e-9 and rel < 1e-10, on
  the test's sizes; periodic convolution against a direct circular sum.
* FFT precision: docs/performance-fft.md:44-49 — the FP32 density spectrum
  of 50,000 bodies on 512x256 against FP64: max rel 6.35e-8, RMS 4.52e-5.
* Morton keys and reorder invariants: SpatialSortIntegrationTest.kt:18-54
  and its independent CPU key (:177-186), via tests/golden/morton_keys.json.
* Config defaults: GravityConfigTest.kt:9-13 / GravityConfig.kt:641-654.
"""

import json
from pathlib import Path

import numpy as np
import pytest

import oracle
from gravity_b200 import scenarios
from gravity_b200.config import (GravityFieldConfig, P3MConfig, mass_scale_for, neighbor_radii,
                                 sort_axis_bits)

GOLDEN = Path(__file__).resolve().parent / "golden"
FFT_SIZES = [(16, 16), (32, 16), (16, 64), (128, 128), (512, 128), (128, 512), (2048, 128)]


def _assert_error(expected, actual, abs_tol, rel_tol):
    max_abs = float(np.abs(expected - actual).max())
    ref = max(float(np.abs(expected).max()), 1e-12)
    assert max_abs < abs_tol, max_abs
    assert max_abs / ref < rel_tol, max_abs / ref


@pytest.mark.parametrize("w,h", FFT_SIZES)
@pytest.mark.parametrize("inverse", [False, True])
def test_fp64_layout_agrees_with_independent_fft(w, h, inverse):
    rng = np.random.default_rng(73 + w * 31 + h)
    v = rng.uniform(-1, 1, (h, w)) + 1j * rng.uniform(-1, 1, (h, w))
    expected = np.fft.ifft2(v) * (w * h) if inverse else np.fft.fft2(v)
    _assert_error(expected, oracle.fft2d_f64(v, inverse), 1e-9, 1e-10)


@pytest.mark.parametrize("w,h", FFT_SIZES)
def test_fp32_mirror_of_shader_is_fp32_accurate(w, h):
    rng = np.random.default_rng(5 + w + h)
    v = rng.uniform(-1, 1, (h, w)) + 1j * rng.uniform(-1, 1, (h, w))
    for inverse in (False, True):
        expected = np.fft.ifft2(v) * (w * h) if inverse else np.fft.fft2(v)
        got = oracle.fft2d_f32(v.astype(np.complex64), inverse)
        rel = float(np.abs(got - expected).max() / np.abs(expected).max())
        assert rel < 2e-6, rel


def test_periodic_convolution_agrees_with_direct_circular_sum():
    """Radix2FftLayoutTest.kt:47-73 on a 16x8 grid."""
    w, h = 16, 8
    rng = np.random.default_rng(991)
    left = rng.uniform(-1, 1, (h, w)).astype(np.complex128)
    right = rng.uniform(-1, 1, (h, w)).astype(np.complex128)
    expected = np.zeros((h, w))
    for y in range(h):
        for x in range(w):
            s = 0.0
            for sy in range(h):
                for sx in range(w):
                    s += left[sy, sx].real * right[(y - sy) % h, (x - sx) % w].real
            expected[y, x] = s
    prod = oracle.fft2d_f64(left, False) * oracle.fft2d_f64(right, False)
    got = oracle.fft2d_f64(prod, True) / (w * h)
    _assert_error(expected.astype(np.complex128), got, 1e-9, 1e-10)


def test_density_spectrum_error_matches_published_magnitude():
    """docs/performance-fft.md:49: 512x256, 50,000 bodies, FP32 spectrum vs
    FP64: max rel 6.34766e-8, RMS 4.52413e-5. The oracle's FP32 mirror on a
    seeded uniform 50k scene must land in the same range."""
    sc = scenarios.uniform_torus(n=50_000, seed=1)
    sim = oracle.OracleSim(sc.config)
    sim.upload(sc.bodies, sc.materials)
    sim.initialize_acceleration(sc.n)
    total, scale = sim.normalization()
    rho = sim.density().astype(np.float64) / scale
    ref = oracle.fft2d_f64(rho.astype(np.complex128), False)
    got = sim.density_spectrum().astype(np.complex128)
    diff = np.concatenate([(got - ref).real.ravel(), (got - ref).imag.ravel()])
    refc = np.concatenate([ref.real.ravel(), ref.imag.ravel()])
    max_rel = float(np.abs(diff).max() / np.abs(refc).max())
    rms = float(np.sqrt(np.mean(diff ** 2)))
    assert max_rel < 2e-7, max_rel
    assert 1e-5 < rms < 2e-4, rms


def test_morton_keys_match_reference_test_key():
    g = json.loads((GOLDEN / "morton_keys.json").read_text())
    x = np.array(g["x_bits"], np.uint32).view(np.float32)
    y = np.array(g["y_bits"], np.uint32).view(np.float32)
    wb, hb = g["width_bits"], g["height_bits"]
    assert (wb, hb) == (sort_axis_bits(g["viewport"][0]), sort_axis_bits(g["viewport"][1]))
    assert (wb, hb) == (oracle.sort_axis_bits(g["viewport"][0]), oracle.sort_axis_bits(g["viewport"][1]))
    got = [oracle.morton_key(float(a), float(b), wb, hb) for a, b in zip(x, y)]
    assert got == g["keys"]
    assert len(set(got)) > 1000


def test_reorder_is_bit_exact_permutation_along_morton_curve():
    """SpatialSortIntegrationTest.kt:18-54 on the oracle."""
    g = json.loads((GOLDEN / "morton_keys.json").read_text())
    x = np.array(g["x_bits"], np.uint32).view(np.float32)
    y = np.array(g["y_bits"], np.uint32).view(np.float32)
    n = len(x)
    rng = np.random.default_rng(4242)
    order = rng.permutation(n)
    bodies = np.zeros((n, 4), np.float32)
    bodies[:, 0], bodies[:, 1] = x[order], y[order]
    bodies[:, 2] = rng.random(n)
    bodies[:, 3] = -rng.random(n)
    acc = rng.random((n, 2)).astype(np.float32) - 0.5
    cfg = P3MConfig(viewport_width=3440, viewport_height=1440,
                    gravity=GravityFieldConfig(grid_width=128, grid_height=128), capacity=n)
    sim = oracle.OracleSim(cfg)
    sim.upload(bodies, None, acc)
    sim.sort_bodies(n)
    b2, _, a2 = sim.download(n)

    def records(b, a):
        rows = np.concatenate([b.view(np.uint32), a.view(np.uint32)], axis=1)
        return rows[np.lexsort(rows.T[::-1])]

    np.testing.assert_array_equal(records(bodies, acc), records(b2, a2))
    wb, hb = g["width_bits"], g["height_bits"]
    keys = [oracle.morton_key(float(p[0]), float(p[1]), wb, hb) for p in b2]
    assert all(keys[i - 1] <= keys[i] for i in range(1, n))
    dest = sim.destinations(n)
    np.testing.assert_array_equal(b2[dest], bodies)


def test_config_defaults_match_reference():
    g = GravityFieldConfig()
    assert (g.grid_width, g.grid_height) == (512, 256)
    assert g.gravitational_constant == pytest.approx(0.035)
    assert g.softening_cells == pytest.approx(0.85)
    assert g.local_search_sigma_multiplier == 3.0
    assert (g.minimum_neighbor_radius_cells, g.maximum_neighbor_radius_cells) == (1, 6)
    assert (g.exact_neighbor_body_limit, g.maximum_home_body_interactions) == (2, 8)
    assert g.minimum_distance_cell_fraction == pytest.approx(0.05)
    assert g.minimum_assignment_window_power == pytest.approx(0.08)
    c = P3MConfig()
    assert c.time_step == pytest.approx(1 / 120)
    assert c.drift_substeps == 16
    assert c.spatial_sort_interval == 2


@pytest.mark.parametrize("kw", [dict(grid_width=100), dict(grid_height=8192),
                                dict(gravitational_constant=-1.0), dict(softening_cells=0.0),
                                dict(exact_neighbor_body_limit=0),
                                dict(minimum_assignment_window_power=1.5)])
def test_invalid_gravity_config_is_rejected(kw):
    with pytest.raises(ValueError):
        GravityFieldConfig(**kw)


def test_walls_need_the_doubled_mesh_to_fit():
    with pytest.raises(ValueError):
        P3MConfig(gravity=GravityFieldConfig(grid_width=4096, grid_height=2048), bounded=True)


@pytest.mark.parametrize("n,scale", [(50_000, 65536), (100_000, 40000), (400_000, 10000),
                                     (8_000_000, 500)])
def test_mass_scale(n, scale):
    """GravityPipeline.kt:1546-1547: the fixed-point mass scale falls as the
    body count grows, so the summed density stays inside 32 bits."""
    assert mass_scale_for(n) == scale
    assert oracle.mass_scale(n) == scale


@pytest.mark.parametrize("grid,viewport", [((512, 256), (2560, 1440)), ((1024, 512), (2560, 1440)),
                                           ((4096, 2048), (4096, 2048)), ((128, 128), (640, 640))])
def test_neighbor_radii(grid, viewport):
    cfg = P3MConfig(viewport_width=viewport[0], viewport_height=viewport[1],
                    gravity=GravityFieldConfig(grid_width=grid[0], grid_height=grid[1]))
    sim = oracle.OracleSim(cfg.with_(capacity=1))
    assert neighbor_radii(cfg) == sim.radii()
    if grid == (512, 256):
        assert neighbor_radii(cfg) == (3, 3)
