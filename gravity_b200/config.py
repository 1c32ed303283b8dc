"""Gravity configuration, mirroring the reference's Kotlin data classes.

``GravityFieldConfig`` follows GravityConfig.kt:641-674 (defaults and the
``require`` checks of its ``init``), ``time_step`` / ``drift_substeps`` follow
CollisionConfig (GravityConfig.kt:677-678) and ``spatial_sort_interval``
follows ParticleConfig (GravityConfig.kt:621). Invalid values raise
``ValueError``, as Kotlin's ``require`` raises IllegalArgumentException.

The one widened limit: the reference accepts grids of 128..2048 cells per
axis (GravityConfig.kt:655-660) because its FFT line lives in one 2048-entry
shared-memory array (fft_shared.comp:12-14). This library's FFT handles mesh
lines up to 4096, so grids of 16..4096 are accepted (walls still need the
doubled mesh to fit: 2 * max(grid) <= 4096).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field, replace

from . import _abi


def _pow2(v: int) -> bool:
    return v > 0 and (v & (v - 1)) == 0


@dataclass(frozen=True)
class GravityFieldConfig:
    grid_width: int = 512
    grid_height: int = 256
    gravitational_constant: float = 0.035
    softening_cells: float = 0.85
    local_search_sigma_multiplier: float = 3.0
    minimum_neighbor_radius_cells: int = 1
    maximum_neighbor_radius_cells: int = 6
    exact_neighbor_body_limit: int = 2
    maximum_home_body_interactions: int = 8
    minimum_distance_cell_fraction: float = 0.05
    minimum_assignment_window_power: float = 0.08

    def __post_init__(self) -> None:
        if not (_pow2(self.grid_width) and 16 <= self.grid_width <= 4096):
            raise ValueError("grid width must be a power of two in 16..4096")
        if not (_pow2(self.grid_height) and 16 <= self.grid_height <= 4096):
            raise ValueError("grid height must be a power of two in 16..4096")
        if not (self.gravitational_constant >= 0 and math.isfinite(self.gravitational_constant)):
            raise ValueError("gravitational constant must be finite and >= 0")
        if not (self.softening_cells > 0 and math.isfinite(self.softening_cells)):
            raise ValueError("softening must be finite and > 0")
        if not (self.local_search_sigma_multiplier > 0 and math.isfinite(self.local_search_sigma_multiplier)):
            raise ValueError("search multiplier must be finite and > 0")
        if self.minimum_neighbor_radius_cells < 1:
            raise ValueError("minimum neighbour radius must be >= 1")
        if self.maximum_neighbor_radius_cells < self.minimum_neighbor_radius_cells:
            raise ValueError("maximum neighbour radius below minimum")
        if self.exact_neighbor_body_limit < 1:
            raise ValueError("exact neighbour body limit must be >= 1")
        if self.maximum_home_body_interactions < 1:
            raise ValueError("home interactions must be >= 1")
        if not (self.minimum_distance_cell_fraction > 0 and math.isfinite(self.minimum_distance_cell_fraction)):
            raise ValueError("minimum distance fraction must be finite and > 0")
        if not (0 < self.minimum_assignment_window_power <= 1):
            raise ValueError("window power floor must be in (0, 1]")


@dataclass(frozen=True)
class P3MConfig:
    """Everything a P3M context needs (one ``p3m_config``)."""

    viewport_width: int = 2560
    viewport_height: int = 1440
    gravity: GravityFieldConfig = field(default_factory=GravityFieldConfig)
    time_step: float = 1.0 / 120.0
    drift_substeps: int = 16
    spatial_sort_interval: int = 2
    capacity: int = 400_000
    bounded: bool = False
    deposit_mode: int = _abi.P3M_DEPOSIT_U32
    mutual_gravity: bool = True

    def __post_init__(self) -> None:
        if self.viewport_width <= 0 or self.viewport_height <= 0:
            raise ValueError("viewport must be positive")
        if not (self.time_step > 0 and math.isfinite(self.time_step)):
            raise ValueError("time step must be finite and > 0")
        if self.drift_substeps < 1:
            raise ValueError("drift substeps must be >= 1")
        if self.spatial_sort_interval < 0:
            raise ValueError("sort interval must be non-negative")
        if self.capacity <= 0:
            raise ValueError("capacity must be positive")
        if self.deposit_mode not in (_abi.P3M_DEPOSIT_U32, _abi.P3M_DEPOSIT_I64):
            raise ValueError("unknown deposit mode")
        if self.bounded and not self.walls_supported:
            raise ValueError("walls need an FFT grid of at most 2048 cells per axis")

    @property
    def walls_supported(self) -> bool:
        return 2 * max(self.gravity.grid_width, self.gravity.grid_height) <= 4096

    def with_(self, **kw) -> "P3MConfig":
        return replace(self, **kw)

    def to_abi(self) -> _abi.P3MConfig:
        import ctypes

        c = _abi.P3MConfig()
        c.struct_size = ctypes.sizeof(_abi.P3MConfig)
        c.viewport_width = self.viewport_width
        c.viewport_height = self.viewport_height
        g = self.gravity
        c.grid_width = g.grid_width
        c.grid_height = g.grid_height
        c.gravitational_constant = g.gravitational_constant
        c.softening_cells = g.softening_cells
        c.local_search_sigma_multiplier = g.local_search_sigma_multiplier
        c.minimum_neighbor_radius_cells = g.minimum_neighbor_radius_cells
        c.maximum_neighbor_radius_cells = g.maximum_neighbor_radius_cells
        c.exact_neighbor_body_limit = g.exact_neighbor_body_limit
        c.maximum_home_body_interactions = g.maximum_home_body_interactions
        c.minimum_distance_cell_fraction = g.minimum_distance_cell_fraction
        c.minimum_assignment_window_power = g.minimum_assignment_window_power
        c.time_step = self.time_step
        c.drift_substeps = self.drift_substeps
        c.spatial_sort_interval = self.spatial_sort_interval
        c.capacity = self.capacity
        c.bounded = 1 if self.bounded else 0
        c.deposit_mode = self.deposit_mode
        c.mutual_gravity = 1 if self.mutual_gravity else 0
        return c


def neighbor_radii(cfg: P3MConfig) -> tuple[int, int]:
    """GravityPipeline.kt:153-169 in float32 arithmetic, like the Kotlin code."""
    import numpy as np

    f = np.float32
    g = cfg.gravity
    aspect = f(cfg.viewport_width) / f(cfg.viewport_height)
    vx = f(g.local_search_sigma_multiplier) * f(g.softening_cells) * f(g.grid_width) / (
        f(g.grid_height) * aspect)
    vy = f(g.softening_cells) * f(g.local_search_sigma_multiplier)
    lo, hi = g.minimum_neighbor_radius_cells, g.maximum_neighbor_radius_cells
    rx = min(max(int(math.ceil(float(vx))), lo), hi)
    ry = min(max(int(math.ceil(float(vy))), lo), hi)
    return rx, ry


def mass_scale_for(total_mass: float) -> int:
    """GravityPipeline.kt:1546-1547 massScaleFor (uint32 fixed point)."""
    import numpy as np

    v = int(4_000_000_000.0 / float(np.float32(total_mass)))
    return min(max(v, 1), 65536)


def sort_axis_bits(extent: int) -> int:
    """GravityPipeline.kt:1649-1650 sortAxisBits."""
    tiles = max(1, extent // 4)
    return min(10, tiles.bit_length() - 1)
