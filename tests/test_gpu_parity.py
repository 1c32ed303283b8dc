"""GPU parity of the P3M path against the CPU oracle, through the C-ABI.

Bit-exact: cell keys, cell lists (IDs in walk order), cell occupancy and
cell masses, the fixed-point density mesh (uint32 and int64 forms), the
Morton reorder. Within REL_RMS_TOL (1e-5 relative RMS): the long-range force
mesh, accelerations, velocities and positions.
"""

import numpy as np
import pytest

import oracle
from gravity_b200 import _abi
from gravity_b200.pipeline import GravityPipeline

from helpers import REL_RMS_TOL, clustered, rel_rms, small_torus

pytestmark = pytest.mark.gpu


def pair(sc, **overrides):
    cfg = sc.config.with_(**overrides) if overrides else sc.config
    gpu = GravityPipeline(cfg)
    ref = oracle.OracleSim(cfg)
    gpu.upload(sc.bodies, sc.materials)
    ref.upload(sc.bodies, sc.materials)
    return gpu, ref


def assert_lists_equal(gpu, ref, n):
    gk, gi, gs, gc, gm = gpu.cell_lists(n)
    rk, ri, rs, rc, rm = ref.cell_lists(n)
    np.testing.assert_array_equal(gc, rc, err_msg="cell occupancy")
    np.testing.assert_array_equal(gm, rm, err_msg="cell masses")
    np.testing.assert_array_equal(gk, rk, err_msg="sorted cell keys")
    np.testing.assert_array_equal(gi, ri, err_msg="cell list order (body IDs)")
    occupied = rc > 0
    np.testing.assert_array_equal(gs[occupied], rs[occupied], err_msg="cell starts")


SCENES = {
    "uniform": lambda: small_torus(n=4000),
    "clustered": lambda: clustered(n=6000),
    "clustered_walls": lambda: clustered(n=6000, bounded=True),
    "wide_grid": lambda: small_torus(n=20000, grid=(512, 256)),
}


@pytest.mark.parametrize("name", sorted(SCENES))
def test_initial_acceleration_matches_oracle(cuda_device, name):
    sc = SCENES[name]()
    n = sc.n
    gpu, ref = pair(sc)
    with gpu, ref:
        gpu.initialize_acceleration(n)
        ref.initialize_acceleration(n)
        assert_lists_equal(gpu, ref, n)
        np.testing.assert_array_equal(gpu.density(), ref.density(), err_msg="density mesh")
        f_gpu, f_ref = gpu.force(), ref.force()
        assert rel_rms(f_gpu, f_ref) < REL_RMS_TOL, rel_rms(f_gpu, f_ref)
        b_gpu, _, a_gpu = gpu.download(n)
        b_ref, _, a_ref = ref.download(n)
        np.testing.assert_array_equal(b_gpu, b_ref, err_msg="initial pass must not move bodies")
        assert rel_rms(a_gpu, a_ref) < REL_RMS_TOL, rel_rms(a_gpu, a_ref)


def test_int64_deposit_bit_exact_and_reproducible(cuda_device):
    sc = clustered(n=6000)
    gpu, ref = pair(sc, deposit_mode=_abi.P3M_DEPOSIT_I64)
    with gpu, ref:
        gpu.initialize_acceleration(sc.n)
        ref.initialize_acceleration(sc.n)
        d1 = gpu.density()
        np.testing.assert_array_equal(d1, ref.density())
        # The total mass is conserved exactly up to rounding of each weight.
        total = d1.astype(np.float64).sum() / 2.0 ** 32
        assert abs(total - sc.materials[:, 0].sum()) < 1e-3
        gpu.build_force(sc.n)
        np.testing.assert_array_equal(gpu.density(), d1, err_msg="run-to-run bit reproducibility")
        assert rel_rms(gpu.force(), ref.force()) < REL_RMS_TOL


@pytest.mark.parametrize("name", ["uniform", "clustered", "clustered_walls"])
def test_steps_match_oracle(cuda_device, name):
    sc = SCENES[name]()
    n = sc.n
    gpu, ref = pair(sc)
    with gpu, ref:
        gpu.initialize_acceleration(n)
        ref.initialize_acceleration(n)
        for _ in range(5):
            gpu.step(n)
            ref.step(n)
        b_gpu, m_gpu, a_gpu = gpu.download(n)
        b_ref, m_ref, a_ref = ref.download(n)
        # Morton reorders happened at steps 0, 2, 4: same permutation.
        np.testing.assert_array_equal(m_gpu, m_ref, err_msg="materials follow the same permutation")
        np.testing.assert_array_equal(gpu.destinations(n), ref.destinations(n))
        assert rel_rms(b_gpu[:, :2], b_ref[:, :2]) < REL_RMS_TOL
        assert rel_rms(b_gpu[:, 2:], b_ref[:, 2:]) < REL_RMS_TOL
        assert rel_rms(a_gpu, a_ref) < REL_RMS_TOL
        assert gpu.wait_timeouts() == 0


def _numpy_cell_lists(bodies, W, H):
    """Home cells (build_grid.comp:71-72 in float32) and the list order:
    cell ascending, body ID descending."""
    x = bodies[:, 0].astype(np.float32)
    y = bodies[:, 1].astype(np.float32)
    hx = np.floor(x * np.float32(W)).astype(np.int64) % W
    hy = np.floor(y * np.float32(H)).astype(np.int64) % H
    cell = (hx + hy * W).astype(np.uint32)
    ids = np.arange(len(bodies), dtype=np.int64)
    order = np.lexsort((-ids, cell))
    return cell[order], order.astype(np.int32)


@pytest.mark.parametrize("n,grid,seed", [
    (400_000, (512, 256), 3),        # 17 key bits: 3 passes, 98 tiles
    (3_000_000, (2048, 1024), 4),    # 21 bits: 3 passes, 733 tiles
    (1_500_000, (4096, 4096), 5),    # 24 bits (the largest grid): 3 passes of 8
    (70_000, (256, 128), 6),         # 15 bits: 2 passes
])
def test_cell_lists_many_tiles_match_a_stable_sort(cuda_device, n, grid, seed):
    """Cell lists from the sort whose tiles find their offsets by looking
    back at earlier tiles: bit-exact against numpy's stable sort, with
    clustered bodies (long runs of one cell) mixed with uniform ones, and no
    look-back wait given up."""
    from gravity_b200.config import GravityFieldConfig, P3MConfig
    from gravity_b200 import scenarios

    rng = np.random.default_rng(seed)
    b = np.zeros((n, 4), np.float32)
    b[:, :2] = rng.uniform(0.0, 1.0, (n, 2))
    k = n // 3
    b[:k, :2] = np.clip(rng.normal(0.5, 0.01, (k, 2)), 0.0, 0.99999994)
    b[:, :2] = np.minimum(b[:, :2], np.float32(0.99999994))
    cfg = P3MConfig(viewport_width=grid[0], viewport_height=grid[1],
                    gravity=GravityFieldConfig(grid_width=grid[0], grid_height=grid[1]),
                    capacity=n)
    with GravityPipeline(cfg) as gpu:
        gpu.upload(b, scenarios.unit_materials(n))
        for _ in range(2):  # twice: the look-back words are cleared per sort
            gpu.build_cell_lists(n)
        keys, ids, start, count, _ = gpu.cell_lists(n)
        assert gpu.wait_timeouts() == 0
    ek, ei = _numpy_cell_lists(b, *grid)
    np.testing.assert_array_equal(keys, ek)
    np.testing.assert_array_equal(ids, ei)
    np.testing.assert_array_equal(count, np.bincount(ek, minlength=grid[0] * grid[1]))


def test_sort_bodies_is_bit_exact_permutation(cuda_device):
    sc = clustered(n=6000)
    n = sc.n
    gpu, ref = pair(sc)
    with gpu, ref:
        acc = np.random.default_rng(1).uniform(-0.5, 0.5, (n, 2)).astype(np.float32)
        gpu.upload(sc.bodies, sc.materials, acc)
        ref.upload(sc.bodies, sc.materials, acc)
        gpu.sort_bodies(n)
        ref.sort_bodies(n)
        bg, mg, ag = gpu.download(n)
        br, mr, ar = ref.download(n)
        np.testing.assert_array_equal(bg, br)
        np.testing.assert_array_equal(mg, mr)
        np.testing.assert_array_equal(ag, ar)
        dest = gpu.destinations(n)
        np.testing.assert_array_equal(np.sort(dest), np.arange(n, dtype=np.uint32))
        np.testing.assert_array_equal(bg[dest], sc.bodies)


def test_mutual_gravity_off_uses_field_only(cuda_device):
    sc = small_torus(n=3000)
    gpu, ref = pair(sc)
    with gpu, ref:
        for s in (gpu, ref):
            s.set_field_acceleration(0.0, -300.0)
        gpu.mutual_gravity = False
        ref.set_mutual_gravity(False)
        gpu.initialize_acceleration(sc.n)
        ref.initialize_acceleration(sc.n)
        gpu.step(sc.n, 3)
        ref.step(sc.n, 3)
        bg, _, ag = gpu.download(sc.n)
        br, _, ar = ref.download(sc.n)
        np.testing.assert_array_equal(bg, br)
        np.testing.assert_array_equal(ag, ar)


def test_edge_sizes(cuda_device):
    """Empty, single-body and tiny systems. With one or two bodies the exact
    mesh self-force is zero and both sides hold FFT round-off, so the
    accelerations are compared against the scale of the force mesh."""
    sc = small_torus(n=5)
    gpu, ref = pair(sc)
    with gpu, ref:
        for n in (0, 1, 2, 5):
            gpu.initialize_acceleration(n)
            ref.initialize_acceleration(n)
            gpu.step(n, 2)
            ref.step(n, 2)
            bg, _, ag = gpu.download(n)
            br, _, ar = ref.download(n)
            if n:
                assert rel_rms(bg, br) < REL_RMS_TOL
                scale = float(np.abs(ref.force()).max())
                assert float(np.abs(ag - ar).max()) <= REL_RMS_TOL * scale


def test_capacity_and_arguments_fail_loudly(cuda_device):
    sc = small_torus(n=100)
    with GravityPipeline(sc.config) as gpu:
        with pytest.raises(ValueError):
            gpu.step(sc.n + 1)
        with pytest.raises(ValueError):
            gpu.step(-1)
    with pytest.raises(ValueError):
        GravityPipeline(sc.config.with_(capacity=0))


def test_inactive_slots_survive_reorder_and_range_upload(cuda_device):
    """Bodies beyond the active count keep their slots across Morton
    reorders; a ranged upload adds bodies the way spawnProjectile does."""
    sc = small_torus(n=3000)
    gpu, ref = pair(sc)
    with gpu, ref:
        active = 2000
        gpu.initialize_acceleration(active)
        ref.initialize_acceleration(active)
        gpu.step(active, 3)
        ref.step(active, 3)
        bg, _, _ = gpu.download(sc.n)
        np.testing.assert_array_equal(bg[active:], sc.bodies[active:])
        extra = sc.bodies[active:active + 100].copy()
        extra[:, 2:] = 0.0
        gpu.upload_range(active, extra)
        full_b, full_m, full_a = ref.download(sc.n)
        full_b[active:active + 100] = extra
        ref.upload(full_b, full_m, full_a)
        gpu.step(active + 100, 2)
        ref.step(active + 100, 2)
        bg, _, ag = gpu.download(active + 100)
        br, _, ar = ref.download(active + 100)
        assert rel_rms(bg, br) < REL_RMS_TOL
        assert rel_rms(ag, ar) < REL_RMS_TOL


def test_graph_replay_equals_direct_launches(cuda_device):
    """Captured-and-replayed steps produce the same bits as kernels launched
    one by one (same kernels, same order), across reorder and non-reorder
    steps and both ping-pong buffers."""
    sc = clustered(n=5000)
    a = GravityPipeline(sc.config)
    b = GravityPipeline(sc.config)
    with a, b:
        b._check(b._lib.p3m_set_graphs(b.handle, 0))
        for p in (a, b):
            p.upload(sc.bodies, sc.materials)
            p.initialize_acceleration(sc.n)
            p.step(sc.n, 7)
        ba, ma, aa = a.download(sc.n)
        bb, mb, ab = b.download(sc.n)
        np.testing.assert_array_equal(ba, bb)
        np.testing.assert_array_equal(ma, mb)
        np.testing.assert_array_equal(aa, ab)


def test_against_committed_golden_fixture(cuda_device):
    """The CUDA path against tests/golden/oracle_small.npz (made by
    tests/golden/make_golden.py from the oracle)."""
    from pathlib import Path

    g = np.load(Path(__file__).resolve().parent / "golden" / "oracle_small.npz")
    sc = clustered(n=3000, grid=(64, 32), seed=9)
    with GravityPipeline(sc.config) as gpu:
        gpu.upload(g["bodies"], g["materials"])
        gpu.initialize_acceleration(sc.n)
        keys, ids, start, count, mass = gpu.cell_lists(sc.n)
        np.testing.assert_array_equal(keys, g["keys"])
        np.testing.assert_array_equal(ids, g["ids"])
        np.testing.assert_array_equal(count, g["count"])
        np.testing.assert_array_equal(mass, g["mass"])
        np.testing.assert_array_equal(gpu.density(), g["density"])
        assert rel_rms(gpu.force(), g["force"]) < REL_RMS_TOL
        assert rel_rms(gpu.acceleration(sc.n), g["accel0"]) < REL_RMS_TOL
        gpu.step(sc.n, 3)
        b3, m3, a3 = gpu.download(sc.n)
        np.testing.assert_array_equal(m3, g["materials3"])
        assert rel_rms(b3, g["bodies3"]) < REL_RMS_TOL
        assert rel_rms(a3, g["accel3"]) < REL_RMS_TOL
