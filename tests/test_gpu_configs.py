"""GPU parity at the three single-simulation workloads the library is
benchmarked on, at their full sizes, through the C-ABI:

  uniform_torus   50,000 bodies, 512x256 torus, dt 1/60, seed 1, 10 steps
  plummer_walls   400,000 bodies in two Plummer spheres inside walls,
                  physical grid 512x256 (Hockney mesh 1024x512), 10 steps
  lattice_scale   8,000,000 bodies from a displaced 4096x2048 lattice, torus,
                  int64 deposit, 3 steps

Two comparisons per workload.

Per step, from the same state: the oracle is handed the CUDA path's state
(bodies, materials, accelerations) before each step, and both take one step
(reorder every second step, half kick + drift, lists, deposit, FFT, kick).
The sorted cell keys, the list order, cell starts, occupancy and masses, the
fixed-point density mesh, the Morton permutation and the drifted positions
are then bit-exact (GravityPipeline.kt:445-494; build_grid.comp:49-76;
collision_build.comp:40-51); the long-range force mesh, the accelerations and
the kicked velocities agree to REL_RMS_TOL (1e-5 relative RMS).

Free-running: the oracle steps from the initial state on its own; after the
last step positions, velocities and accelerations agree to REL_RMS_TOL.
"""

import numpy as np
import pytest

import oracle
from gravity_b200 import scenarios
from gravity_b200.pipeline import GravityPipeline

from helpers import REL_RMS_TOL, rel_rms

pytestmark = pytest.mark.gpu


def _assert_lists_equal(gpu, ref, n, label):
    gk, gi, gs, gc, gm = gpu.cell_lists(n)
    rk, ri, rs, rc, rm = ref.cell_lists(n)
    np.testing.assert_array_equal(gc, rc, err_msg=f"{label}: cell occupancy")
    np.testing.assert_array_equal(gm, rm, err_msg=f"{label}: cell masses")
    np.testing.assert_array_equal(gk, rk, err_msg=f"{label}: sorted cell keys")
    np.testing.assert_array_equal(gi, ri, err_msg=f"{label}: list order (body IDs)")
    occupied = rc > 0
    np.testing.assert_array_equal(gs[occupied], rs[occupied], err_msg=f"{label}: cell starts")


def _assert_mesh(gpu, ref, label):
    np.testing.assert_array_equal(gpu.density(), ref.density(), err_msg=f"{label}: density mesh")
    e = rel_rms(gpu.force(), ref.force())
    assert e < REL_RMS_TOL, f"{label}: force mesh rel RMS {e:.3e}"


def _run(sc, steps):
    n = sc.n
    cfg = sc.config
    with GravityPipeline(cfg) as gpu, oracle.OracleSim(cfg) as ref, \
            oracle.OracleSim(cfg) as free:
        for s in (gpu, ref, free):
            s.upload(sc.bodies, sc.materials)
            s.initialize_acceleration(n)
        _assert_lists_equal(gpu, ref, n, "initial pass")
        _assert_mesh(gpu, ref, "initial pass")
        b_g, _, a_g = gpu.download(n)
        _, _, a_r = ref.download(n)
        np.testing.assert_array_equal(b_g, sc.bodies, err_msg="the initial pass moved bodies")
        assert rel_rms(a_g, a_r) < REL_RMS_TOL, rel_rms(a_g, a_r)

        for k in range(steps):
            label = f"step {k}"
            bg, mg, ag = gpu.download(n)
            ref.upload(bg, mg, ag)
            gpu.step(n)
            ref.step(n)
            free.step(n)
            _assert_lists_equal(gpu, ref, n, label)
            _assert_mesh(gpu, ref, label)
            bg, mg, ag = gpu.download(n)
            br, mr, ar = ref.download(n)
            np.testing.assert_array_equal(mg, mr, err_msg=f"{label}: materials (permutation)")
            if k % max(1, cfg.spatial_sort_interval) == 0 and cfg.spatial_sort_interval > 0:
                np.testing.assert_array_equal(gpu.destinations(n), ref.destinations(n),
                                              err_msg=f"{label}: reorder destinations")
            np.testing.assert_array_equal(bg[:, :2], br[:, :2], err_msg=f"{label}: drifted positions")
            ev = rel_rms(bg[:, 2:], br[:, 2:])
            ea = rel_rms(ag, ar)
            assert ev < REL_RMS_TOL, f"{label}: velocities rel RMS {ev:.3e}"
            assert ea < REL_RMS_TOL, f"{label}: accelerations rel RMS {ea:.3e}"
        assert gpu.wait_timeouts() == 0
        gpu.synchronize()

        bg, _, ag = gpu.download(n)
        bf, _, af = free.download(n)
        # Positions on the torus: compare the minimum-image difference.
        d = bg[:, :2].astype(np.float64) - bf[:, :2].astype(np.float64)
        if not cfg.bounded:
            d -= np.round(d)
        ep = float(np.sqrt(np.mean(d * d) / np.mean(bf[:, :2].astype(np.float64) ** 2)))
        assert ep < REL_RMS_TOL, f"free-running positions rel RMS {ep:.3e}"
        ev = rel_rms(bg[:, 2:], bf[:, 2:])
        ea = rel_rms(ag, af)
        assert ev < REL_RMS_TOL, f"free-running velocities rel RMS {ev:.3e}"
        assert ea < REL_RMS_TOL, f"free-running accelerations rel RMS {ea:.3e}"


def test_uniform_torus_50k_ten_steps(cuda_device):
    sc = scenarios.uniform_torus()
    assert sc.n == 50_000 and sc.config.time_step == pytest.approx(1 / 60)
    _run(sc, 10)


def test_plummer_walls_400k_ten_steps(cuda_device):
    sc = scenarios.plummer_walls()
    assert sc.n == 400_000 and sc.config.bounded
    _run(sc, 10)


def test_lattice_scale_8m_int64_three_steps(cuda_device):
    sc = scenarios.lattice_scale()
    assert sc.n == 8_000_000 and sc.config.deposit_mode == 1
    _run(sc, 3)
