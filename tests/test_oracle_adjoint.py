"""The FP64 reference adjoint of the oracle against central finite
differences of its own FP64 forward (pins the reference the CUDA adjoint is
checked against)."""

import numpy as np

import oracle
from gravity_b200 import scenarios


def scene():
    sc = scenarios.adjoint_cluster(n_cluster=1200, n_disc=100, seed=13, steps=12,
                                   viewport=(640, 360), grid=(64, 32))
    group = np.arange(1200, 1300)
    b = sc.bodies.astype(np.float64)
    b[group, 2] = 25.0 / 640.0
    b[group, 3] = 10.0 / 360.0
    return sc, group, b


def centroid_loss(ref, b, group, steps, target):
    final, _ = ref.forward(b, steps)
    c = final[group, :2].mean(axis=0) * np.array([640.0, 360.0])
    return float(((c - target) ** 2).sum()), c


def test_fp64_adjoint_matches_central_differences():
    sc, group, b = scene()
    target = np.array([560.0, 150.0])
    ref = oracle.Adjoint64(sc.config, sc.materials)
    loss, c = centroid_loss(ref, b, group, sc.steps, target)
    seed = np.zeros((sc.n, 4))
    seed[group, 0] = 2 * (c[0] - target[0]) * 640.0 / len(group)
    seed[group, 1] = 2 * (c[1] - target[1]) * 360.0 / len(group)
    g, ga = ref.backward(seed)
    np.testing.assert_array_equal(ga, 0.0)
    # Launch velocity (px/s). The step is small enough that no body changes
    # cell or mesh node between the two runs (with h = 1e-2 px/s a few do
    # here, and the difference quotient then differs by ~1%: the loss is
    # only piecewise smooth).
    gv = np.array([g[group, 2].sum() / 640.0, g[group, 3].sum() / 360.0])
    h = 1e-3
    for k, extent in ((0, 640.0), (1, 360.0)):
        bp, bm = b.copy(), b.copy()
        bp[group, 2 + k] += h / extent
        bm[group, 2 + k] -= h / extent
        fd = (centroid_loss(ref, bp, group, sc.steps, target)[0]
              - centroid_loss(ref, bm, group, sc.steps, target)[0]) / (2 * h)
        assert abs(gv[k] - fd) <= 1e-6 * abs(fd), (k, gv[k], fd)
    # Single positions (cluster and projectile bodies); the step (0.006 px)
    # is far below a cell so the topology stays put, and large enough that
    # the loss's round-off (~1e-11 of ~1e5 px^2) stays below 1e-6 of the
    # quotient.
    for i in (3, 700, 1250):
        for k in range(2):
            e = 1e-5
            bp, bm = b.copy(), b.copy()
            bp[i, k] += e
            bm[i, k] -= e
            fd = (centroid_loss(ref, bp, group, sc.steps, target)[0]
                  - centroid_loss(ref, bm, group, sc.steps, target)[0]) / (2 * e)
            assert abs(g[i, k] - fd) <= 1e-3 * abs(fd) + 1e-8 * np.abs(g[:, :2]).max(), (i, k, g[i, k], fd)


def test_fp64_force_is_linear_in_mass_layout():
    # The reference force of two bodies is equal and opposite (momentum):
    # the mesh kernel is odd and the short-range pair antisymmetric.
    sc, group, b = scene()
    ref = oracle.Adjoint64(sc.config, sc.materials[:2] * 0 + np.array([1.0, 0, 0, 0]))
    pos = np.array([[0.30, 0.40], [0.33, 0.42]])
    a = ref.force(pos)
    np.testing.assert_allclose(a[0], -a[1], rtol=1e-9, atol=1e-12 * np.abs(a).max())
