"""Seeded initial conditions for the P3M workloads this library is measured on.

Bodies are float32 (n, 4) rows (x, y, vx, vy) in unit coordinates and unit/s,
the reference's body layout (GravityPipeline.kt:752-756: a pixel position is
divided by the viewport size). Materials are (mass, friction, solid, block).

Workloads (sizes as stated for this library's benchmarks):
  uniform_torus   50,000 equal masses uniform in 2560x1440 px, velocities
                  N(0, 5 px/s) per component, grid 512x256, torus, dt 1/60.
  plummer_walls   400,000 bodies in two projected Plummer spheres (scale radii
                  80 / 40 px, 300k / 100k unit masses), centres 600 px apart,
                  relative velocity 30 px/s perpendicular to the separation
                  (centre-of-mass frame), no internal velocities, walls,
                  physical grid 512x256 (FFT mesh 1024x512).
  lattice_scale   8,000,000 bodies: a seeded subset of a 4096x2048 lattice in a
                  4096x2048 px torus, displaced by an irrotational Gaussian
                  field whose displacement spectrum is P(k) ~ k^-2 with RMS
                  3 cells, velocities 0.5/s x displacement, int64 deposit.
  batch           256 simulations, N log-uniform in [1000, 65536], uniform in
                  their own domain (5 px per cell), grids drawn from
                  {128x128, 256x128, 256x256, 512x256}.
  adjoint_cluster Plummer 99,000 (r_s 100 px) + a 1,000-body disc of radius
                  20 px at 800 px offset, torus, grid 1024x512.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _abi
from .config import GravityFieldConfig, P3MConfig


@dataclass
class Scenario:
    name: str
    config: P3MConfig
    bodies: np.ndarray      # (n, 4) float32
    materials: np.ndarray   # (n, 4) float32
    steps: int

    @property
    def n(self) -> int:
        return self.bodies.shape[0]


def unit_materials(n: int) -> np.ndarray:
    m = np.zeros((n, 4), np.float32)
    m[:, 0] = 1.0
    return m


def _to_unit(xp, yp, vxp, vyp, w, h) -> np.ndarray:
    b = np.empty((len(xp), 4), np.float32)
    b[:, 0] = np.asarray(xp, np.float64) / w
    b[:, 1] = np.asarray(yp, np.float64) / h
    b[:, 2] = np.asarray(vxp, np.float64) / w
    b[:, 3] = np.asarray(vyp, np.float64) / h
    return b


def uniform_torus(n: int = 50_000, seed: int = 1, steps: int = 10) -> Scenario:
    w, h = 2560, 1440
    rng = np.random.default_rng(seed)
    x = rng.uniform(0.0, w, n)
    y = rng.uniform(0.0, h, n)
    vx = rng.normal(0.0, 5.0, n)
    vy = rng.normal(0.0, 5.0, n)
    b = _to_unit(x, y, vx, vy, w, h)
    b[:, :2] = np.minimum(b[:, :2], np.float32(0.99999994))
    cfg = P3MConfig(viewport_width=w, viewport_height=h,
                    gravity=GravityFieldConfig(grid_width=512, grid_height=256),
                    time_step=1.0 / 60.0, capacity=n, bounded=False)
    return Scenario("uniform_torus", cfg, b, unit_materials(n), steps)


def _plummer_2d(rng, n, a, cx, cy, rmax):
    """Projected Plummer sphere: M(<R) = R^2/(R^2+a^2), truncated at rmax."""
    umax = rmax * rmax / (rmax * rmax + a * a)
    u = rng.uniform(0.0, umax, n)
    r = a * np.sqrt(u / (1.0 - u))
    t = rng.uniform(0.0, 2.0 * np.pi, n)
    return cx + r * np.cos(t), cy + r * np.sin(t)


def plummer_walls(n: int = 400_000, seed: int = 2, steps: int = 100) -> Scenario:
    w, h = 2560, 1440
    rng = np.random.default_rng(seed)
    na = (3 * n) // 4
    nb = n - na
    cx, cy = w / 2.0, h / 2.0
    rmax = 0.45 * h
    xa, ya = _plummer_2d(rng, na, 80.0, cx - 300.0, cy, rmax)
    xb, yb = _plummer_2d(rng, nb, 40.0, cx + 300.0, cy, rmax)
    # 30 px/s relative velocity along y, zero total momentum (masses 3:1).
    va, vb = -30.0 * nb / n, 30.0 * na / n
    x = np.concatenate([xa, xb])
    y = np.concatenate([ya, yb])
    vx = np.zeros(n)
    vy = np.concatenate([np.full(na, va), np.full(nb, vb)])
    order = rng.permutation(n)
    b = _to_unit(x[order], y[order], vx[order], vy[order], w, h)
    b[:, :2] = np.clip(b[:, :2], 0.0, np.float32(0.99999994))
    cfg = P3MConfig(viewport_width=w, viewport_height=h,
                    gravity=GravityFieldConfig(grid_width=512, grid_height=256),
                    capacity=n, bounded=True)
    return Scenario("plummer_walls", cfg, b, unit_materials(n), steps)


def lattice_scale(n: int = 8_000_000, grid=(4096, 2048), seed: int = 7, steps: int = 50,
                  rms_cells: float = 3.0, deposit_mode: int = _abi.P3M_DEPOSIT_I64) -> Scenario:
    gw, gh = grid
    w, h = gw, gh  # one pixel per cell, a 2:1 domain
    rng = np.random.default_rng(seed)
    # Displacement psi = -grad(phi), |psi(k)|^2 ~ k^-2: phi(k) ~ noise / k^2.
    noise = rng.standard_normal((gh, gw)).astype(np.float32)
    nk = np.fft.rfft2(noise)
    ky = np.fft.fftfreq(gh)[:, None] * gh
    kx = np.fft.rfftfreq(gw)[None, :] * gw
    k2 = kx * kx + ky * ky
    k2[0, 0] = 1.0
    amp = 1.0 / k2
    amp[0, 0] = 0.0
    phi_k = nk * amp
    psix = np.fft.irfft2(-1j * (2 * np.pi * kx / gw) * phi_k, s=(gh, gw))
    psiy = np.fft.irfft2(-1j * (2 * np.pi * ky / gh) * phi_k, s=(gh, gw))
    rms = np.sqrt(np.mean(psix ** 2 + psiy ** 2))
    s = rms_cells / rms
    psix *= s
    psiy *= s
    sites = rng.choice(gw * gh, size=n, replace=False)
    sites.sort()
    sy, sx = np.divmod(sites, gw)
    x = (sx + 0.5 + psix.ravel()[sites]) % gw
    y = (sy + 0.5 + psiy.ravel()[sites]) % gh
    growth = 0.5
    b = _to_unit(x, y, growth * psix.ravel()[sites], growth * psiy.ravel()[sites], w, h)
    b[:, :2] = np.where(b[:, :2] >= 1.0, np.float32(0.0), b[:, :2])
    cfg = P3MConfig(viewport_width=w, viewport_height=h,
                    gravity=GravityFieldConfig(grid_width=gw, grid_height=gh),
                    capacity=n, bounded=False, deposit_mode=deposit_mode)
    return Scenario("lattice_scale", cfg, b, unit_materials(n), steps)


BATCH_GRIDS = ((128, 128), (256, 128), (256, 256), (512, 256))


def batch(sims: int = 256, seed: int = 11, steps: int = 60, nmin: int = 1000,
          nmax: int = 65536) -> list[Scenario]:
    rng = np.random.default_rng(seed)
    out = []
    for i in range(sims):
        n = int(round(np.exp(rng.uniform(np.log(nmin), np.log(nmax)))))
        gw, gh = BATCH_GRIDS[rng.integers(len(BATCH_GRIDS))]
        w, h = 5 * gw, 5 * gh
        x = rng.uniform(0, w, n)
        y = rng.uniform(0, h, n)
        b = _to_unit(x, y, np.zeros(n), np.zeros(n), w, h)
        b[:, :2] = np.minimum(b[:, :2], np.float32(0.99999994))
        cfg = P3MConfig(viewport_width=w, viewport_height=h,
                        gravity=GravityFieldConfig(grid_width=gw, grid_height=gh),
                        capacity=n, bounded=False)
        out.append(Scenario(f"batch_{i}", cfg, b, unit_materials(n), steps))
    return out


def adjoint_cluster(n_cluster: int = 99_000, n_disc: int = 1_000, seed: int = 5,
                    steps: int = 200, viewport=(2560, 1440), grid=(1024, 512)) -> Scenario:
    """The projectile disc is bodies n_cluster .. n-1. A smaller viewport
    scales the cluster, the disc and the offset with its width."""
    w, h = viewport
    k = w / 2560.0
    rng = np.random.default_rng(seed)
    cx, cy = w / 2.0, h / 2.0
    xc, yc = _plummer_2d(rng, n_cluster, 100.0 * k, cx, cy, 0.45 * h)
    r = 20.0 * k * np.sqrt(rng.uniform(0, 1, n_disc))
    t = rng.uniform(0, 2 * np.pi, n_disc)
    xd = (cx + 800.0 * k + r * np.cos(t)) % w
    yd = cy + r * np.sin(t)
    x = np.concatenate([xc, xd]) % w
    y = np.concatenate([yc, yd]) % h
    n = n_cluster + n_disc
    b = _to_unit(x, y, np.zeros(n), np.zeros(n), w, h)
    b[:, :2] = np.minimum(b[:, :2], np.float32(0.99999994))
    cfg = P3MConfig(viewport_width=w, viewport_height=h,
                    gravity=GravityFieldConfig(grid_width=grid[0], grid_height=grid[1]),
                    capacity=n, bounded=False, spatial_sort_interval=0)
    return Scenario("adjoint_cluster", cfg, b, unit_materials(n), steps)
