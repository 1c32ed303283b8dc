"""The batched form (p3m_batch_*) against simulations stepped one by one.

In every form of a batch step — per-stage (one launch per stage for every
simulation, the default), persistent (one cooperative launch per step
running all stages of all simulations phase by phase) and per-simulation
(one graph over the simulations' streams) — each simulation must come out
bit for bit as the same simulation stepped alone in its own context, before
and after the autotuner changes launch shapes, and across the reorder
phases (a batch cycles through several captured plans). The persistent
step's grid barrier is bounded: a CTA that never arrives makes the waits run
out, which the next synchronising call reports as P3M_ERR_TIMEOUT.
"""

from dataclasses import replace

import numpy as np
import pytest

from gravity_b200 import _abi, scenarios
from gravity_b200.batch import GravityBatch
from gravity_b200.pipeline import GravityPipeline

pytestmark = pytest.mark.gpu


def mixed_batch():
    scs = scenarios.batch(sims=7, seed=21, nmin=300, nmax=9000)
    # One simulation with walls, one with a field, one without mutual gravity.
    scs[1] = replace(scs[1], config=scs[1].config.with_(bounded=True))
    scs[3] = replace(scs[3], config=scs[3].config.with_(mutual_gravity=False))
    return scs


def step_alone(sc, steps, field=(0.0, 0.0)):
    with GravityPipeline(sc.config) as p:
        p.upload(sc.bodies, sc.materials)
        if field != (0.0, 0.0):
            p.set_field_acceleration(*field)
        p.initialize_acceleration(sc.n)
        p.step(sc.n, steps)
        return p.download(sc.n)


MODES = ("persistent", "per_stage", "per_simulation")


def set_mode(batch, mode):
    if mode == "persistent":
        batch.set_persistent(True)
    elif mode == "per_stage":
        batch.set_persistent(False)
    elif mode == "per_simulation":
        batch.set_fused(False)


def assert_same(got, want, what):
    for g, w, name in zip(got, want, ("bodies", "materials", "acceleration")):
        np.testing.assert_array_equal(g, w, err_msg=f"{what}: {name}")


@pytest.mark.parametrize("mode", MODES)
def test_batch_matches_individual_steps(cuda_device, mode):
    scs = mixed_batch()
    field = (0.0, 3.5)
    with GravityBatch([sc.config for sc in scs]) as batch:
        set_mode(batch, mode)
        for i, sc in enumerate(scs):
            batch.upload(i, sc.bodies, sc.materials)
        batch.simulation(5).set_field_acceleration(*field)
        batch.initialize_acceleration()
        batch.step(5)
        for i, sc in enumerate(scs):
            want = step_alone(sc, 5, field if i == 5 else (0.0, 0.0))
            assert_same(batch.download(i), want, f"simulation {i}")


@pytest.mark.parametrize("mode", MODES)
def test_batch_after_autotune_is_unchanged(cuda_device, mode):
    scs = mixed_batch()
    with GravityBatch([sc.config for sc in scs]) as batch:
        set_mode(batch, mode)
        for i, sc in enumerate(scs):
            batch.upload(i, sc.bodies, sc.materials)
        batch.initialize_acceleration()
        batch.step(3)
        rows = batch.autotune(trial_steps=2)
        grids = {(sc.config.gravity.grid_width, sc.config.gravity.grid_height) for sc in scs}
        assert {(r[0], r[1]) for r in rows} == grids
        assert all(r[2] in (0, 1, 2, 4, 8) and r[3] in (64, 128, 256) for r in rows)
        batch.step(4)
        if mode != "per_simulation":
            assert batch.plan_info()["launches"] >= 1  # a fused plan ran (either form)
        for i, sc in enumerate(scs):
            assert_same(batch.download(i), step_alone(sc, 7), f"simulation {i}")


def test_batch_with_an_empty_simulation(cuda_device):
    scs = scenarios.batch(sims=3, seed=5, nmin=200, nmax=2000)
    with GravityBatch([sc.config for sc in scs]) as batch:
        for i, sc in enumerate(scs):
            if i != 1:
                batch.upload(i, sc.bodies, sc.materials)
        batch.initialize_acceleration()
        batch.step(3)
        for i in (0, 2):
            assert_same(batch.download(i), step_alone(scs[i], 3), f"simulation {i}")


def test_batch_rejects_bad_arguments(cuda_device):
    scs = scenarios.batch(sims=2, seed=6, nmin=100, nmax=200)
    with GravityBatch([sc.config for sc in scs]) as batch:
        with pytest.raises(ValueError):
            batch.upload(2, scs[0].bodies)
        with pytest.raises(ValueError):
            batch.step(-1)
        with pytest.raises(ValueError):
            batch.upload(0, np.zeros((scs[0].config.capacity + 1, 4), np.float32))


def test_persistent_step_is_one_launch_and_matches_per_stage_launches(cuda_device):
    scs = scenarios.batch(sims=24, seed=8, nmin=500, nmax=40000)
    got = {}
    for mode in ("persistent", "per_stage"):
        with GravityBatch([sc.config for sc in scs]) as batch:
            set_mode(batch, mode)
            for i, sc in enumerate(scs):
                batch.upload(i, sc.bodies, sc.materials)
            batch.initialize_acceleration()
            batch.step(4)
            info = batch.plan_info()
            if mode == "persistent":
                assert info["persistent"] and info["launches"] == 1, info
                assert info["phases"] >= 8 and info["ctas"] > 0, info
                times = batch.phase_times()
                assert len(times) == info["phases"] and all(t >= 0.0 for t in times)
            else:
                assert not info["persistent"] and info["launches"] > 10, info
                assert batch.phase_times() == []
            got[mode] = [batch.download(i) for i in range(len(scs))]
    for i in range(len(scs)):
        assert_same(got["persistent"][i], got["per_stage"][i], f"simulation {i}")


def test_batch_workload_scale_matches_individual_steps(cuda_device):
    """The trajectory-preview batch at its benchmark size: 256 simulations of
    1,000 to 65,536 bodies on mixed grids, four steps (both reorder phases,
    every captured plan of the cycle)."""
    scs = scenarios.batch()
    assert len(scs) == 256
    got = {}
    for mode in ("per_stage", "persistent"):
        with GravityBatch([sc.config for sc in scs]) as batch:
            set_mode(batch, mode)
            for i, sc in enumerate(scs):
                batch.upload(i, sc.bodies, sc.materials)
            batch.initialize_acceleration()
            batch.step(4)
            assert batch.plan_info()["persistent"] == (mode == "persistent")
            got[mode] = [batch.download(i) for i in range(len(scs))]
    for i, sc in enumerate(scs):
        want = step_alone(sc, 4)
        for mode in got:
            assert_same(got[mode][i], want, f"{mode}: simulation {i}")


def test_persistent_barrier_that_runs_out_is_reported(cuda_device):
    scs = scenarios.batch(sims=6, seed=9, nmin=500, nmax=8000)
    with GravityBatch([sc.config for sc in scs]) as batch:
        batch.set_persistent(True)
        with pytest.raises(ValueError):
            batch.set_barrier_fault(poll_limit=0)
        with pytest.raises(ValueError):
            batch.set_barrier_fault(withheld_cta=-2)
        for i, sc in enumerate(scs):
            batch.upload(i, sc.bodies, sc.materials)
        batch.initialize_acceleration()
        batch.step(1)
        batch.synchronize()
        # CTA 0 never arrives at the barrier after phase 2; every other CTA's
        # wait gives up after 2,000 polls and its CTA ends.
        batch.set_barrier_fault(poll_limit=2000, withheld_cta=0, phase=2)
        batch.step(1)
        with pytest.raises(_abi.P3MError) as err:
            batch.synchronize()
        assert err.value.status == _abi.P3M_ERR_TIMEOUT
        batch.synchronize()  # reported once
        # Cleared: the same batch steps correctly from a fresh upload.
        batch.set_barrier_fault()
        for i, sc in enumerate(scs):
            batch.upload(i, sc.bodies, sc.materials)
        batch.initialize_acceleration()
        batch.step(3)
        batch.synchronize()
        for i, sc in enumerate(scs):
            assert_same(batch.download(i), step_alone(sc, 3), f"simulation {i}")


@pytest.mark.parametrize("mode", MODES)
def test_pipelined_batch_steps_equal_serial_steps(cuda_device, mode):
    """p3m_batch_step_io over steps whose inputs change from step to step
    gives every step's bodies bit for bit as uploading each simulation,
    stepping the batch and downloading each simulation would."""
    from gravity_b200.pipeline import PinnedArray

    scs = mixed_batch()
    steps = 5
    rng = np.random.default_rng(7)
    ins = []
    for _ in range(steps):
        per = []
        for sc in scs:
            b = sc.bodies.copy()
            idx = rng.choice(sc.n, size=min(16, sc.n), replace=False)
            b[idx, :2] = np.minimum(rng.uniform(0, 1, (len(idx), 2)), 0.99999994).astype(np.float32)
            per.append(b)
        ins.append(per)
    with GravityBatch([sc.config for sc in scs]) as serial:
        set_mode(serial, mode)
        for i, sc in enumerate(scs):
            serial.upload(i, sc.bodies, sc.materials)
        serial.initialize_acceleration()
        want = []
        for k in range(steps):
            for i in range(len(scs)):
                serial.upload(i, ins[k][i])
            serial.step(1)
            want.append(np.concatenate([serial.download(i)[0] for i in range(len(scs))]))
    total = sum(sc.n for sc in scs)
    cin = [PinnedArray((total, 4)) for _ in range(steps)]
    cout = [PinnedArray((total, 4)) for _ in range(steps)]
    try:
        for k in range(steps):
            cin[k].array[:] = np.concatenate(ins[k])
        with GravityBatch([sc.config for sc in scs]) as piped:
            set_mode(piped, mode)
            for i, sc in enumerate(scs):
                piped.upload(i, sc.bodies, sc.materials)
            piped.initialize_acceleration()
            for k in range(steps):
                piped.step_io(cin[k].array, cout[k].array)
            piped.synchronize()
            for k in range(steps):
                np.testing.assert_array_equal(cout[k].array, want[k], err_msg=f"{mode}: step {k}")
    finally:
        for a in cin + cout:
            a.free()
