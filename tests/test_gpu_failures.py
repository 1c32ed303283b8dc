"""Failure detection on the device, without a GPU fault.

The cell and Morton sorts find each tile's output offsets by looking back at
the tiles before it; every such wait is bounded. The test hook
p3m_set_lookback_fault lowers the poll limit and keeps one tile from ever
publishing its counts (a flag that nothing sets), so the waits behind it run
out: the kernels end, the waits are counted, and the next synchronising call
returns P3M_ERR_TIMEOUT. The context stays usable: with the hook cleared the
next sort is correct again.
"""

import numpy as np
import pytest

from gravity_b200 import _abi, scenarios
from gravity_b200.config import GravityFieldConfig, P3MConfig
from gravity_b200.pipeline import GravityPipeline

pytestmark = pytest.mark.gpu


def _scene(n=200_000, grid=(512, 256), seed=12):
    rng = np.random.default_rng(seed)
    b = np.zeros((n, 4), np.float32)
    b[:, :2] = np.minimum(rng.uniform(0, 1, (n, 2)), np.float32(0.99999994))
    cfg = P3MConfig(gravity=GravityFieldConfig(grid_width=grid[0], grid_height=grid[1]),
                    capacity=n)
    return cfg, b


def _expected_lists(b, W, H):
    hx = np.floor(b[:, 0] * np.float32(W)).astype(np.int64) % W
    hy = np.floor(b[:, 1] * np.float32(H)).astype(np.int64) % H
    cell = (hx + hy * W).astype(np.uint32)
    order = np.lexsort((-np.arange(len(b)), cell))
    return cell[order], order.astype(np.int32)


def test_lookback_wait_that_runs_out_is_reported_and_recovers(cuda_device):
    cfg, b = _scene()
    n = len(b)
    W, H = cfg.gravity.grid_width, cfg.gravity.grid_height
    with GravityPipeline(cfg) as gpu:
        gpu.upload(b, scenarios.unit_materials(n))
        gpu.build_cell_lists(n)
        gpu.synchronize()
        assert gpu.wait_timeouts() == 0

        # 49 tiles of 4096 keys: tile 0 never publishes, the waits behind it
        # give up after 64 polls each.
        gpu.set_lookback_fault(poll_limit=64, withheld_tile=0)
        gpu.build_cell_lists(n)
        with pytest.raises(_abi.P3MError) as err:
            gpu.synchronize()
        assert err.value.status == _abi.P3M_ERR_TIMEOUT
        timeouts = gpu.wait_timeouts()
        assert timeouts > 0
        gpu.synchronize()  # reported once

        # The stepping path reports through the download as well.
        gpu.step(n)
        with pytest.raises(_abi.P3MError) as err:
            gpu.download(n)
        assert err.value.status == _abi.P3M_ERR_TIMEOUT
        assert gpu.wait_timeouts() > timeouts

        # Cleared: the same context sorts correctly again.
        gpu.set_lookback_fault()
        gpu.upload(b, scenarios.unit_materials(n))
        before = gpu.wait_timeouts()
        gpu.build_cell_lists(n)
        gpu.synchronize()
        assert gpu.wait_timeouts() == before
        keys, ids, _, count, _ = gpu.cell_lists(n)
    ek, ei = _expected_lists(b, W, H)
    np.testing.assert_array_equal(keys, ek)
    np.testing.assert_array_equal(ids, ei)
    np.testing.assert_array_equal(count, np.bincount(ek, minlength=W * H))


def test_nonfinite_bodies_are_reported_once(cuda_device):
    cfg, b = _scene(n=5000)
    b[7, 3] = np.nan
    with GravityPipeline(cfg.with_(spatial_sort_interval=0)) as gpu:
        gpu.upload(b, scenarios.unit_materials(len(b)))
        gpu.initialize_acceleration(len(b))
        gpu.synchronize()
        gpu.step(len(b))
        with pytest.raises(_abi.P3MError) as err:
            gpu.synchronize()
        assert err.value.status == _abi.P3M_ERR_NON_FINITE
        assert gpu.nonfinite_count() >= 1
        gpu.synchronize()


def test_fault_hook_rejects_invalid_arguments(cuda_device):
    cfg, b = _scene(n=1000)
    with GravityPipeline(cfg) as gpu:
        with pytest.raises(ValueError):
            gpu.set_lookback_fault(poll_limit=0)
        with pytest.raises(ValueError):
            gpu.set_lookback_fault(withheld_tile=-2)
