"""Generates the golden fixtures under tests/golden/ (run from the repo root:
``python tests/golden/make_golden.py``).

morton_keys.json
    Positions and their Morton tile keys computed by an independent
    restatement of the CPU key that the reference's own test uses to check
    the GPU reorder (SpatialSortIntegrationTest.kt:177-186: a bit-by-bit
    interleave, written differently from the shader's spreadBits). The scene
    follows that test's layout (SpatialSortIntegrationTest.kt:23-31): a dense
    block, coincident bodies, both seams, the far corner and uniform bodies,
    on its 3440x1440 viewport; Kotlin's Random is not available here, so the
    positions come from numpy with a fixed seed.

oracle_small.npz
    A regression fixture of the CPU oracle on a small clustered torus scene:
    inputs, sorted cell keys and IDs, occupancy, cell masses, the uint32
    density, the force mesh and accelerations after initializeAcceleration,
    and the bodies after three steps. It pins the oracle against accidental
    change; the tests compare the CUDA path with it as well.
"""

from __future__ import annotations

import json
import math
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
sys.path.insert(0, str(REPO))
sys.path.insert(0, str(REPO / "tests"))


def morton_key_bitwise(x: float, y: float, wbits: int, hbits: int) -> int:
    """SpatialSortIntegrationTest.kt:177-186 restated: interleave bit by bit."""
    f32 = np.float32
    tx = int(math.floor(float(f32(x) * f32(1 << wbits))))
    ty = int(math.floor(float(f32(y) * f32(1 << hbits))))
    tx = min(max(tx, 0), (1 << wbits) - 1)
    ty = min(max(ty, 0), (1 << hbits) - 1)
    common = min(wbits, hbits)
    key = 0
    for bit in range(common):
        key |= ((tx >> bit) & 1) << (2 * bit)
        key |= ((ty >> bit) & 1) << (2 * bit + 1)
    return key | (((tx | ty) >> common) << (2 * common))


def sort_axis_bits(extent: int) -> int:
    return min(10, max(1, extent // 4).bit_length() - 1)


def morton_scene(count: int = 6000, seed: int = 4242):
    width, height = 3440, 1440
    rng = np.random.default_rng(seed)
    pts = []
    for i in range(count):
        if i < 2500:
            pts.append((1200 + (i % 50) * 0.9, 700 + (i // 50) * 0.9))
        elif i < 2600:
            pts.append((300.0, 300.0))
        elif i < 2700:
            pts.append((0.0 if i % 2 == 0 else width - 0.01, (i % 97) * 14.0))
        elif i < 2710:
            pts.append((width * 0.99999994, height * 0.99999994))
        else:
            pts.append((rng.random() * width, rng.random() * height))
    p = np.array(pts, dtype=np.float64)
    x = (p[:, 0] / width).astype(np.float32)
    y = (p[:, 1] / height).astype(np.float32)
    return width, height, x, y


def make_morton():
    width, height, x, y = morton_scene()
    wb, hb = sort_axis_bits(width), sort_axis_bits(height)
    keys = [morton_key_bitwise(float(a), float(b), wb, hb) for a, b in zip(x, y)]
    out = {
        "source": "SpatialSortIntegrationTest.kt:177-186 (independent CPU key)",
        "viewport": [width, height], "width_bits": wb, "height_bits": hb,
        "x_bits": [int(v) for v in x.view(np.uint32)],
        "y_bits": [int(v) for v in y.view(np.uint32)],
        "keys": keys,
    }
    (HERE / "morton_keys.json").write_text(json.dumps(out))


def make_oracle_small():
    import oracle
    from helpers import clustered

    sc = clustered(n=3000, grid=(64, 32), seed=9)
    sim = oracle.OracleSim(sc.config)
    sim.upload(sc.bodies, sc.materials)
    sim.initialize_acceleration(sc.n)
    keys, ids, start, count, mass = sim.cell_lists(sc.n)
    _, _, accel0 = sim.download(sc.n)
    density = sim.density()
    force = sim.force()
    sim.step(sc.n, 3)
    bodies3, mats3, accel3 = sim.download(sc.n)
    np.savez_compressed(
        HERE / "oracle_small.npz", bodies=sc.bodies, materials=sc.materials, keys=keys, ids=ids,
        start=start, count=count, mass=mass, density=density, force=force, accel0=accel0,
        bodies3=bodies3, materials3=mats3, accel3=accel3,
        grid=np.array([64, 32]), viewport=np.array([sc.config.viewport_width, sc.config.viewport_height]))


if __name__ == "__main__":
    os.chdir(REPO)
    make_morton()
    make_oracle_small()
    print("golden fixtures written to", HERE)
