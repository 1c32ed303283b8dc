"""Physics checks of the oracle itself (CPU): the P3M force against the FP64
direct sum it approximates, the structure of the Green's function, and the
committed regression fixture."""

from pathlib import Path

import numpy as np
import pytest

import oracle
from helpers import clustered, small_torus

GOLDEN = Path(__file__).resolve().parent / "golden"


def _force_error(sc):
    sim = oracle.OracleSim(sc.config)
    sim.upload(sc.bodies, sc.materials)
    sim.initialize_acceleration(sc.n)
    _, _, acc = sim.download(sc.n)
    total, _ = sim.normalization()
    targets = np.arange(0, sc.n, 7, dtype=np.int32)
    ref = oracle.direct_sum_f64(sc.bodies, sc.materials, targets, sc.config.to_abi(), total,
                                sc.config.bounded)
    diff = acc[targets] - ref
    return float(np.sqrt(np.sum(diff ** 2) / np.sum(ref ** 2))), float(np.sqrt(np.mean(diff ** 2)))


def test_p3m_force_approximates_fp64_direct_sum_inside_walls():
    rel, _ = _force_error(small_torus(n=4000, grid=(128, 64), bounded=True))
    assert rel < 0.02, rel


def test_torus_force_error_shrinks_with_resolution():
    """On the torus a uniform background cancels, so the net force is ~10x
    smaller than inside walls while the mesh's absolute error is the same;
    the relative error falls as the grid refines."""
    errs = [_force_error(small_torus(n=4000, grid=g))[0] for g in ((64, 32), (128, 64), (256, 128))]
    assert errs[0] > errs[1] > errs[2], errs
    assert errs[2] < 0.08, errs
    _, abs_torus = _force_error(small_torus(n=4000, grid=(128, 64)))
    _, abs_walls = _force_error(small_torus(n=4000, grid=(128, 64), bounded=True))
    assert 0.5 < abs_torus / abs_walls < 2.0


def test_kernel_spectra_are_imaginary_and_odd():
    """kernel_init.comp zeroes the Nyquist component so the real, odd force
    kernels have purely imaginary spectra (what the library's one-float
    Green's table relies on)."""
    sc = small_torus(n=10, grid=(64, 32))
    sim = oracle.OracleSim(sc.config)
    kx, ky = sim.kernel_spectra()
    for k in (kx, ky):
        assert np.abs(k.real).max() < 1e-5 * np.abs(k.imag).max()
        mirrored = k[(-np.arange(k.shape[0])) % k.shape[0]][:, (-np.arange(k.shape[1])) % k.shape[1]]
        np.testing.assert_allclose(mirrored.imag, -k.imag, atol=1e-5 * np.abs(k.imag).max())


def test_momentum_is_nearly_conserved_on_the_torus():
    sc = small_torus(n=3000, grid=(64, 32))
    sim = oracle.OracleSim(sc.config)
    sim.upload(sc.bodies, sc.materials)
    sim.initialize_acceleration(sc.n)
    _, _, acc = sim.download(sc.n)
    # Pairwise forces are nearly antisymmetric; the net force is tiny
    # compared with the typical one.
    assert np.abs(acc.sum(axis=0)).max() < 0.02 * np.abs(acc).sum(axis=0).max()


def test_regression_fixture():
    g = np.load(GOLDEN / "oracle_small.npz")
    sc = clustered(n=3000, grid=(64, 32), seed=9)
    np.testing.assert_array_equal(sc.bodies, g["bodies"])
    sim = oracle.OracleSim(sc.config)
    sim.upload(sc.bodies, sc.materials)
    sim.initialize_acceleration(sc.n)
    keys, ids, start, count, mass = sim.cell_lists(sc.n)
    np.testing.assert_array_equal(keys, g["keys"])
    np.testing.assert_array_equal(ids, g["ids"])
    np.testing.assert_array_equal(count, g["count"])
    np.testing.assert_array_equal(mass, g["mass"])
    np.testing.assert_array_equal(sim.density(), g["density"])
    np.testing.assert_array_equal(sim.force(), g["force"])
    _, _, acc = sim.download(sc.n)
    np.testing.assert_array_equal(acc, g["accel0"])
    sim.step(sc.n, 3)
    b3, m3, a3 = sim.download(sc.n)
    np.testing.assert_array_equal(b3, g["bodies3"])
    np.testing.assert_array_equal(a3, g["accel3"])


def test_cell_lists_run_in_descending_id():
    sc = clustered(n=2000, grid=(32, 16))
    sim = oracle.OracleSim(sc.config)
    sim.upload(sc.bodies, sc.materials)
    sim.initialize_acceleration(sc.n)
    keys, ids, start, count, _ = sim.cell_lists(sc.n)
    assert count.sum() == sc.n
    for c in np.nonzero(count)[0][:200]:
        seg = ids[start[c]:start[c] + count[c]]
        assert (np.diff(seg) < 0).all()
        assert (keys[start[c]:start[c] + count[c]] == c).all()
