"""Body state on disk in the reference's vec4 layout.

The reference hands bodies to its GPU pipeline as a FloatArray of count x 4
floats (x, y, vx, vy): positions in unit coordinates wrapped onto [0, 1),
velocities in screens per second. ``Scenario.bodies`` builds it with
``ScenarioBuilder.normalized()`` (src/main/kotlin/dev/gravity/Scenario.kt:
286-297, 571-580) from pixel coordinates. This module keeps that layout on
disk so that a seeded workload, or a state read back from a context, can be
stored and loaded bit for bit:

    offset  type                    content
    0       4 bytes                 magic b"GRVS"
    4       uint32                  format version (1)
    8       uint32                  body count n
    12      uint32                  flags: bit 0 materials, bit 1 accelerations
    16      uint32                  viewport width in px
    20      uint32                  viewport height in px
    24      uint64                  seed of the generator (0: none)
    32      float32[n][4]           bodies (x, y, vx, vy), the reference's layout
    ...     float32[n][4]           materials (mass, friction, solid, block), if flagged
    ...     float32[n][2]           accelerations (unit/s^2), if flagged

All numbers are little-endian. A JVM host reads the body block with a
``ByteBuffer.order(LITTLE_ENDIAN).asFloatBuffer()`` straight into the array
it uploads.
"""

from __future__ import annotations

import os
import struct
from dataclasses import dataclass
from typing import Optional

import numpy as np

MAGIC = b"GRVS"
VERSION = 1
_HEADER = struct.Struct("<4sIIIIIQ")  # 32 bytes
FLAG_MATERIALS = 1
FLAG_ACCELERATION = 2


@dataclass
class BodyState:
    bodies: np.ndarray                      # (n, 4) float32
    materials: Optional[np.ndarray] = None  # (n, 4) float32
    acceleration: Optional[np.ndarray] = None  # (n, 2) float32
    viewport: tuple[int, int] = (2560, 1440)
    seed: int = 0

    @property
    def n(self) -> int:
        return int(self.bodies.shape[0])


def normalized(pixels: np.ndarray, width_px: float, height_px: float) -> np.ndarray:
    """ScenarioBuilder.normalized() (Scenario.kt:286-297) in FP32: positions
    divided by the viewport and wrapped onto [0, 1) (a wrapped value that
    rounds to 1 becomes 0), velocities divided by the viewport."""
    p = np.ascontiguousarray(pixels, np.float32).reshape(-1, 4)
    w, h = np.float32(width_px), np.float32(height_px)
    out = np.empty_like(p)
    for axis, size in ((0, w), (1, h)):
        v = p[:, axis] / size
        f = v - np.floor(v)
        out[:, axis] = np.where(f >= np.float32(1.0), np.float32(0.0), f)
    out[:, 2] = p[:, 2] / w
    out[:, 3] = p[:, 3] / h
    return out


def save(path: str | os.PathLike, state: BodyState) -> None:
    b = np.ascontiguousarray(state.bodies, "<f4").reshape(-1, 4)
    n = b.shape[0]
    flags = 0
    blocks = [b]
    if state.materials is not None:
        flags |= FLAG_MATERIALS
        blocks.append(np.ascontiguousarray(state.materials, "<f4").reshape(n, 4))
    if state.acceleration is not None:
        flags |= FLAG_ACCELERATION
        blocks.append(np.ascontiguousarray(state.acceleration, "<f4").reshape(n, 2))
    w, h = state.viewport
    with open(path, "wb") as f:
        f.write(_HEADER.pack(MAGIC, VERSION, n, flags, int(w), int(h), int(state.seed)))
        for a in blocks:
            f.write(a.tobytes())


def load(path: str | os.PathLike) -> BodyState:
    with open(path, "rb") as f:
        head = f.read(_HEADER.size)
        if len(head) != _HEADER.size:
            raise ValueError("truncated body-state header")
        magic, version, n, flags, w, h, seed = _HEADER.unpack(head)
        if magic != MAGIC:
            raise ValueError("not a body-state file (bad magic)")
        if version != VERSION:
            raise ValueError(f"unsupported body-state version {version}")
        if flags & ~(FLAG_MATERIALS | FLAG_ACCELERATION):
            raise ValueError(f"unknown body-state flags {flags:#x}")

        def block(width: int) -> np.ndarray:
            data = f.read(4 * width * n)
            if len(data) != 4 * width * n:
                raise ValueError("truncated body-state data")
            return np.frombuffer(data, "<f4").astype(np.float32).reshape(n, width)

        bodies = block(4)
        materials = block(4) if flags & FLAG_MATERIALS else None
        accel = block(2) if flags & FLAG_ACCELERATION else None
        if f.read(1):
            raise ValueError("trailing bytes after the body-state data")
    return BodyState(bodies, materials, accel, (w, h), seed)


def from_scenario(sc, seed: int = 0) -> BodyState:
    """The state of a seeded workload of gravity_b200.scenarios."""
    return BodyState(sc.bodies, sc.materials, None,
                     (sc.config.viewport_width, sc.config.viewport_height), seed)
