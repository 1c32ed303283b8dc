"""The mesh-tile deposit (2^21 bodies and more) against the oracle, bit for bit.

Above 2^21 bodies the deposit switches from chunks of the cell order to mesh
tiles that own their cells, with heavy tiles handed to a second kernel. These
scenes reach every branch of that path: uniform bodies (light tiles), a
cluster (heavy tiles, walls with the padded mesh), a small mesh whose tiles
span all of its columns (every tile heavy), both fixed-point forms, and
bodies on the last column / row (wrapped runs).
"""

import numpy as np
import pytest

from gravity_b200 import _abi, scenarios
from gravity_b200.config import GravityFieldConfig, P3MConfig

from test_gpu_parity import pair

pytestmark = pytest.mark.gpu

N = (1 << 21) + 4099


def uniform(grid, deposit, seed=1, bounded=False):
    rng = np.random.default_rng(seed)
    b = np.zeros((N, 4), np.float32)
    b[:, :2] = rng.uniform(0.0, 1.0, (N, 2)).astype(np.float32)
    b[:, :2] = np.minimum(b[:, :2], np.float32(0.99999994))
    # Bodies on the seams: first and last column / row.
    b[:64, 0] = 0.0
    b[64:128, 0] = np.float32(0.99999994)
    b[128:192, 1] = 0.0
    b[192:256, 1] = np.float32(0.99999994)
    m = scenarios.unit_materials(N)
    m[::7, 0] = 2.5
    cfg = P3MConfig(viewport_width=2 * grid[0], viewport_height=2 * grid[1],
                    gravity=GravityFieldConfig(grid_width=grid[0], grid_height=grid[1]),
                    capacity=N, bounded=bounded, deposit_mode=deposit)
    return scenarios.Scenario("tiles", cfg, b, m, 1)


def clustered(deposit):
    rng = np.random.default_rng(5)
    w, h = 2560, 1440
    x, y = scenarios._plummer_2d(rng, N, 60.0, w / 2, h / 2, 0.45 * h)
    b = np.zeros((N, 4), np.float32)
    b[:, 0] = np.clip(x / w, 0.0, 0.99999994)
    b[:, 1] = np.clip(y / h, 0.0, 0.99999994)
    cfg = P3MConfig(viewport_width=w, viewport_height=h,
                    gravity=GravityFieldConfig(grid_width=512, grid_height=256),
                    capacity=N, bounded=True, deposit_mode=deposit)
    return scenarios.Scenario("tiles_cluster", cfg, b, scenarios.unit_materials(N), 1)


CASES = {
    "uniform_i64_2048x1024": lambda: uniform((2048, 1024), _abi.P3M_DEPOSIT_I64),
    "uniform_u32_1024x512": lambda: uniform((1024, 512), _abi.P3M_DEPOSIT_U32),
    "uniform_walls_u32_512x256": lambda: uniform((512, 256), _abi.P3M_DEPOSIT_U32, bounded=True),
    "small_mesh_i64_64x32": lambda: uniform((64, 32), _abi.P3M_DEPOSIT_I64),
    "tiny_mesh_u32_16x16": lambda: uniform((16, 16), _abi.P3M_DEPOSIT_U32),
    "cluster_walls_u32": lambda: clustered(_abi.P3M_DEPOSIT_U32),
    "cluster_walls_i64": lambda: clustered(_abi.P3M_DEPOSIT_I64),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_tile_deposit_matches_oracle(cuda_device, name):
    sc = CASES[name]()
    gpu, ref = pair(sc)
    with gpu, ref:
        # initializeAcceleration normalises the mass scale, then deposits.
        gpu.initialize_acceleration(sc.n)
        ref.initialize_acceleration(sc.n)
        d = gpu.density()
        np.testing.assert_array_equal(d, ref.density(), err_msg="density mesh")
        # Run to run: the same mesh again (heavy tiles add with atomics).
        gpu.build_force(sc.n)
        np.testing.assert_array_equal(gpu.density(), d)
