"""Shared helpers of the parity tests (comparison metrics, small scenes)."""

from __future__ import annotations

import numpy as np

from gravity_b200 import scenarios
from gravity_b200.config import GravityFieldConfig, P3MConfig

# Tolerance of forces, accelerations and positions against the oracle's FP32
# restatement: relative RMS of the difference.
REL_RMS_TOL = 1e-5


def rel_rms(actual, expected) -> float:
    a = np.asarray(actual, np.float64)
    e = np.asarray(expected, np.float64)
    den = np.sqrt(np.mean(e * e))
    return float(np.sqrt(np.mean((a - e) ** 2)) / max(den, 1e-300))


def small_torus(n=4000, seed=3, grid=(128, 64), viewport=(2560, 1440), **kw) -> scenarios.Scenario:
    rng = np.random.default_rng(seed)
    w, h = viewport
    x = rng.uniform(0, w, n)
    y = rng.uniform(0, h, n)
    vx = rng.normal(0, 5.0, n)
    vy = rng.normal(0, 5.0, n)
    b = np.empty((n, 4), np.float32)
    b[:, 0] = x / w
    b[:, 1] = y / h
    b[:, 2] = vx / w
    b[:, 3] = vy / h
    b[:, :2] = np.minimum(b[:, :2], np.float32(0.99999994))
    cfg = P3MConfig(viewport_width=w, viewport_height=h,
                    gravity=GravityFieldConfig(grid_width=grid[0], grid_height=grid[1]),
                    capacity=max(n, 1), **kw)
    return scenarios.Scenario("small", cfg, b, scenarios.unit_materials(n), 10)


def clustered(n=6000, seed=4, grid=(64, 32), bounded=False, **kw) -> scenarios.Scenario:
    """Dense clumps (cells far above the exact-body and home limits), seams,
    coincident bodies and the far corner, then uniform bodies."""
    rng = np.random.default_rng(seed)
    w, h = 2560, 1440
    pts = []
    for i in range(n):
        if i < n // 3:
            pts.append((1200 + rng.normal(0, 15), 700 + rng.normal(0, 15)))
        elif i < n // 3 + 100:
            pts.append((300.0, 300.0))
        elif i < n // 3 + 200:
            pts.append((0.0 if i % 2 == 0 else w - 0.01, (i % 97) * 14.0))
        elif i < n // 3 + 210:
            pts.append((w * 0.99999994, h * 0.99999994))
        else:
            pts.append((rng.uniform(0, w), rng.uniform(0, h)))
    p = np.array(pts)
    b = np.zeros((n, 4), np.float32)
    b[:, 0] = np.clip(p[:, 0] / w, 0, 0.99999994)
    b[:, 1] = np.clip(p[:, 1] / h, 0, 0.99999994)
    b[:, 2] = rng.normal(0, 3, n) / w
    b[:, 3] = rng.normal(0, 3, n) / h
    cfg = P3MConfig(viewport_width=w, viewport_height=h,
                    gravity=GravityFieldConfig(grid_width=grid[0], grid_height=grid[1]),
                    capacity=n, bounded=bounded, **kw)
    mats = scenarios.unit_materials(n)
    mats[::7, 0] = 2.5  # some heavier bodies: non-unit cell masses
    return scenarios.Scenario("clustered", cfg, b, mats, 10)
