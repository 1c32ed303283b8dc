"""The differentiated rollout (p3m_adjoint_forward / p3m_adjoint_backward).

Against the FP64 reference adjoint of the oracle (same initial state, each
side running its own forward): the gradient with respect to the initial
positions and velocities for a generic cotangent, and the projectile's
launch-velocity gradient. Against central finite differences of the FP64
forward (h = 1e-3 px/s): the launch-velocity gradient of the
projectile-centroid loss, within 1e-3; against those of the CUDA forward at
h = 1e-2 px/s, within the spread that the force's cell-boundary
discontinuities give the difference quotient.
"""

from dataclasses import replace

import numpy as np
import pytest

import oracle
from gravity_b200 import scenarios
from gravity_b200.adjoint import Rollout, launch_velocity_objective, optimise_launch_velocity
from gravity_b200.pipeline import GravityPipeline, P3MArgumentError

pytestmark = pytest.mark.gpu

FD_TOL = 1e-3


def small_scene(n_cluster=3000, n_disc=200, steps=24, viewport=(1280, 720), grid=(256, 128),
                seed=9):
    sc = scenarios.adjoint_cluster(n_cluster=n_cluster, n_disc=n_disc, seed=seed, steps=steps,
                                   viewport=viewport, grid=grid)
    group = np.arange(n_cluster, n_cluster + n_disc)
    return sc, group


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def gpu_and_fp64(sc, bodies, steps, seed, seed_a=None, interval=8, initial=True,
                 along_gpu=False):
    with GravityPipeline(sc.config) as p:
        p.upload(bodies, sc.materials)
        a0 = None
        if not initial:
            p.initialize_acceleration(sc.n)
            a0 = p.acceleration(sc.n).astype(np.float64)
        r = Rollout(p, sc.n, steps, checkpoint_interval=interval, initial_acceleration=initial)
        final = r.forward()
        ga = np.empty((sc.n, 2), np.float32)
        g = r.backward(seed, seed_a, out_accel=ga)
    ref = oracle.Adjoint64(sc.config, sc.materials)
    final64, _ = ref.forward(bodies.astype(np.float64), steps, acceleration=a0)
    if along_gpu:
        assert steps == 1
        ref.set_positions(1, final[:, :2])
    g64, ga64 = ref.backward(seed.astype(np.float64),
                             None if seed_a is None else seed_a.astype(np.float64))
    return final, g, ga, final64, g64, ga64


def launched(sc, group, v_px):
    b = sc.bodies.copy()
    b[group, 2] = v_px[0] / sc.config.viewport_width
    b[group, 3] = v_px[1] / sc.config.viewport_height
    return b


@pytest.mark.parametrize("deposit, tol", [(1, 2e-4), (0, 5e-3)])
def test_one_step_adjoint_matches_fp64_reference(cuda_device, deposit, tol):
    # One step, with the FP64 reverse pass evaluated along the CUDA
    # trajectory (close pairs in the cluster turn the ~1e-7 FP32 / FP64
    # position difference into ~1e-3 of their Jacobians), so this measures
    # the adjoint's arithmetic. With the int64 deposit (2^-32 mass quanta)
    # the FP32 mesh is the continuous model up to round-off; with the uint32
    # deposit the mass quanta (1/massScale per node) move the mesh force by
    # up to ~1e-3 relative on these scenes, and the cotangents follow.
    sc, group = small_scene(steps=1)
    sc = replace(sc, config=sc.config.with_(deposit_mode=deposit))
    b = launched(sc, group, (60.0, -25.0))
    rng = np.random.default_rng(3)
    seed = rng.standard_normal((sc.n, 4)).astype(np.float32)
    seed_a = rng.standard_normal((sc.n, 2)).astype(np.float32) * 0.1
    final, g, ga, final64, g64, ga64 = gpu_and_fp64(sc, b, 1, seed, seed_a, along_gpu=True)
    assert rel_l2(final[:, :2], final64[:, :2]) < 1e-6
    assert rel_l2(g[:, :2], g64[:, :2]) < tol, "position cotangents"
    assert rel_l2(g[:, 2:], g64[:, 2:]) < tol, "velocity cotangents"
    np.testing.assert_array_equal(ga, 0.0)  # a0 came from initializeAcceleration


def test_rollout_adjoint_matches_fp64_reference(cuda_device):
    sc, group = small_scene(steps=24)
    v0, target = np.array([60.0, -25.0]), np.array([1200.0, 300.0])
    scale = np.array([sc.config.viewport_width, sc.config.viewport_height], np.float64)
    with GravityPipeline(sc.config) as p:
        p.upload(sc.bodies, sc.materials)
        obj = launch_velocity_objective(Rollout(p, sc.n, sc.steps, checkpoint_interval=8),
                                        sc.bodies, group, v0, target)
    ref = oracle.Adjoint64(sc.config, sc.materials)
    b = launched(sc, group, v0).astype(np.float64)
    f, _ = ref.forward(b, sc.steps)
    c = f[group, :2].mean(axis=0) * scale
    seed = np.zeros((sc.n, 4))
    seed[group, :2] = 2.0 * (c - target) * scale / len(group)
    g64, _ = ref.backward(seed)
    gv64 = np.array([g64[group, 2].sum(), g64[group, 3].sum()]) / scale
    # The launch-velocity gradient of the centroid loss.
    assert rel_l2(obj.grad_velocity_px, gv64) < 1e-3
    # Per body, the cluster's close encounters amplify the FP32 / FP64
    # trajectory difference (~3e-6 after 24 steps) into a few percent.
    assert rel_l2(obj.grad_bodies, g64) < 5e-2


def test_adjoint_without_initial_acceleration(cuda_device):
    # a0 given (not recomputed): its cotangent is returned, not folded.
    sc, group = small_scene(steps=2)
    sc = replace(sc, config=sc.config.with_(deposit_mode=1))
    rng = np.random.default_rng(4)
    seed = rng.standard_normal((sc.n, 4)).astype(np.float32)
    final, g, ga, final64, g64, ga64 = gpu_and_fp64(sc, sc.bodies, 2, seed, interval=1,
                                                    initial=False)
    assert rel_l2(g, g64) < 1e-3
    assert rel_l2(ga, ga64) < 1e-3


def test_launch_velocity_gradient_matches_fp64_finite_differences(cuda_device):
    # Central differences of the FP64 forward with h = 1e-3 px/s: small
    # enough that no body changes cell or mesh node between the two runs,
    # which the FP32 forward cannot resolve (its round-off at that h is ~10%).
    sc, group = small_scene(steps=24)
    v0, target, h = np.array([60.0, -25.0]), np.array([1200.0, 300.0]), 1e-3
    with GravityPipeline(sc.config) as p:
        p.upload(sc.bodies, sc.materials)
        obj = launch_velocity_objective(Rollout(p, sc.n, sc.steps, checkpoint_interval=8),
                                        sc.bodies, group, v0, target)
    ref = oracle.Adjoint64(sc.config, sc.materials)
    scale = np.array([sc.config.viewport_width, sc.config.viewport_height], np.float64)

    def loss(v):
        b = sc.bodies.astype(np.float64)  # velocities set in FP64: h is ~300 float32 ulps
        b[group, 2:] = np.asarray(v) / scale
        f, _ = ref.forward(b, sc.steps)
        c = f[group, :2].mean(axis=0) * scale
        return float(((c - target) ** 2).sum())

    fd = np.array([(loss(v0 + e) - loss(v0 - e)) / (2 * h) for e in np.eye(2) * h])
    err = np.linalg.norm(obj.grad_velocity_px - fd) / np.linalg.norm(fd)
    assert err < FD_TOL, (obj.grad_velocity_px, fd)


def test_launch_velocity_gradient_against_fp32_finite_differences(cuda_device):
    # h = 1e-2 px/s on the CUDA forward. The reference's P3M force is only
    # piecewise smooth in the positions (home cells, monopole switches, CIC
    # nodes); between the +h and -h runs a few projectile bodies cross such
    # a boundary at a different step, which moves the difference quotient by
    # ~1% here (the FP64 model shows the same at this h). Bound: 3e-2.
    sc, group = small_scene(steps=24)
    v0, target, h = np.array([60.0, -25.0]), np.array([1200.0, 300.0]), 1e-2
    with GravityPipeline(sc.config) as p:
        p.upload(sc.bodies, sc.materials)
        r = Rollout(p, sc.n, sc.steps, checkpoint_interval=8)
        obj = launch_velocity_objective(r, sc.bodies, group, v0, target)
        fd = np.array([
            (launch_velocity_objective(r, sc.bodies, group, v0 + e, target, False).loss
             - launch_velocity_objective(r, sc.bodies, group, v0 - e, target, False).loss) / (2 * h)
            for e in np.eye(2) * h])
    err = np.linalg.norm(obj.grad_velocity_px - fd) / np.linalg.norm(fd)
    assert err < 3e-2, (obj.grad_velocity_px, fd)


def test_launch_velocity_optimisation_reduces_the_loss(cuda_device):
    sc, group = small_scene(steps=40)
    with GravityPipeline(sc.config) as p:
        p.upload(sc.bodies, sc.materials)
        r = Rollout(p, sc.n, sc.steps, checkpoint_interval=16)
        target = np.array([1050.0, 300.0])
        v, hist = optimise_launch_velocity(r, sc.bodies, group, [0.0, 0.0], target, iterations=12)
    assert hist[-1] < 0.05 * hist[0]


def test_adjoint_rejects_unsupported_setups(cuda_device):
    sc, _ = small_scene(steps=4)
    with GravityPipeline(sc.config.with_(spatial_sort_interval=2)) as p:
        p.upload(sc.bodies, sc.materials)
        with pytest.raises(P3MArgumentError):
            Rollout(p, sc.n, 4).forward()
    with GravityPipeline(sc.config) as p:
        p.upload(sc.bodies, sc.materials)
        with pytest.raises(RuntimeError):
            Rollout(p, sc.n, 4).backward(np.zeros((sc.n, 4), np.float32))


def test_autograd_function_matches_the_rollout(cuda_device):
    import torch

    from gravity_b200.adjoint import rollout_function

    sc, group = small_scene(steps=12)
    with GravityPipeline(sc.config) as p:
        p.upload(sc.bodies, sc.materials)
        r = Rollout(p, sc.n, sc.steps, checkpoint_interval=5)
        x0 = torch.tensor(sc.bodies, device="cuda", requires_grad=True)
        final = rollout_function().apply(x0, r)
        w = torch.linspace(-1.0, 1.0, sc.n * 4, device="cuda").reshape(sc.n, 4)
        (final * w).sum().backward()
        g_torch = x0.grad.cpu().numpy()
        final_np = r.forward(sc.bodies)
        g_np = r.backward(w.cpu().numpy())
    np.testing.assert_array_equal(final.detach().cpu().numpy(), final_np)
    assert rel_l2(g_torch, g_np) < 1e-5  # float atomics: not bitwise run to run


def test_workload_launch_velocity_gradient_matches_fp64_adjoint(cuda_device):
    """The differentiation workload itself: 100,000 bodies (a 99,000-body
    Plummer cluster and a 1,000-body projectile disc), torus 1024x512, 200
    steps, checkpoints every 16. The loss there is not differentiable at any
    usable finite-difference step (the disc's bodies cross cell and node
    boundaries between the +h and -h runs), so the CUDA adjoint's
    launch-velocity gradient is checked against the FP64 adjoint of the same
    rollout, each side running its own forward: within 1% (the FP32 / FP64
    trajectories part through the cluster's close encounters)."""
    sc = scenarios.adjoint_cluster()
    assert sc.n == 100_000 and sc.steps == 200
    group = np.arange(99_000, 100_000)
    v0, target = np.array([-60.0, 45.0]), np.array([1900.0, 760.0])
    scale = np.array([sc.config.viewport_width, sc.config.viewport_height], np.float64)
    with GravityPipeline(sc.config) as p:
        p.upload(sc.bodies, sc.materials)
        obj = launch_velocity_objective(Rollout(p, sc.n, sc.steps, checkpoint_interval=16),
                                        sc.bodies, group, v0, target)
    ref = oracle.Adjoint64(sc.config, sc.materials)
    b = launched(sc, group, v0).astype(np.float64)
    f, _ = ref.forward(b, sc.steps)
    c = f[group, :2].mean(axis=0) * scale
    seed = np.zeros((sc.n, 4))
    seed[group, :2] = 2.0 * (c - target) * scale / len(group)
    g64, _ = ref.backward(seed)
    gv64 = np.array([g64[group, 2].sum(), g64[group, 3].sum()]) / scale
    assert rel_l2(obj.grad_velocity_px, gv64) < 1e-2, (obj.grad_velocity_px, gv64)
