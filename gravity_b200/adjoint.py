"""Differentiated P3M rollouts: forward/backward through the C-ABI.

``Rollout`` drives p3m_adjoint_forward / p3m_adjoint_backward (include/p3m.h)
on a :class:`GravityPipeline`; ``RolloutFunction`` is the same pair as a
``torch.autograd.Function`` (initial bodies -> final bodies, CUDA tensors);
``launch_velocity_objective`` and ``optimise_launch_velocity`` aim a group of
bodies (the application's projectile, GravityPipeline.kt:621-718
spawnProjectile) at a target point by gradient descent on its launch
velocity. The reference has no adjoint; the differentiated step is its
gravity-only step (GravityPipeline.kt:445-494 without collisions).

Units: bodies are (x, y, vx, vy) in unit coordinates and unit/s (a pixel
position divided by the viewport size), as everywhere in this library;
velocities and targets of the objective are in px/s and px.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _abi
from .pipeline import GravityPipeline


def _pointer(a):
    """Address of a contiguous float32 numpy array or CUDA tensor (or None)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if a.dtype != np.float32 or not a.flags.c_contiguous:
            raise ValueError("arrays must be contiguous float32")
        return a.ctypes.data_as(ctypes.c_void_p)
    if str(a.dtype) != "torch.float32" or not a.is_contiguous():
        raise ValueError("tensors must be contiguous float32")
    return ctypes.c_void_p(a.data_ptr())


class Rollout:
    """`steps` gravity-only steps of `pipeline` with checkpoints every
    `checkpoint_interval` steps; `initial_acceleration` computes a0 from the
    initial positions (initializeAcceleration) and differentiates through it."""

    def __init__(self, pipeline: GravityPipeline, n: int, steps: int, checkpoint_interval: int = 16,
                 initial_acceleration: bool = True):
        self.pipeline = pipeline
        self.n = int(n)
        self.steps = int(steps)
        self.interval = int(checkpoint_interval)
        self.flags = _abi.P3M_ADJOINT_INITIAL_ACCELERATION if initial_acceleration else 0
        self._lib = pipeline._lib

    def forward(self, bodies=None, out=None):
        """Runs the rollout (from `bodies` when given, else the current
        state) and returns the final bodies ((n, 4) float32; written into
        `out` when given, a host array or CUDA tensor)."""
        p = self.pipeline
        if bodies is not None:
            p._check(self._lib.p3m_upload_state(p.handle, _pointer(bodies), None, None, self.n))
        p._check(self._lib.p3m_adjoint_forward(p.handle, self.n, self.steps, self.interval, self.flags))
        if out is None:
            out = np.empty((self.n, 4), np.float32)
        p._check(self._lib.p3m_download_state(p.handle, _pointer(out), None, None, self.n))
        return out

    def backward(self, seed, seed_accel=None, out=None, out_accel=None):
        """dL/d(initial bodies) from dL/d(final bodies) [and dL/d(final a)]."""
        p = self.pipeline
        if out is None:
            out = np.empty((self.n, 4), np.float32)
        if isinstance(seed, np.ndarray):
            seed = np.ascontiguousarray(seed, np.float32).reshape(self.n, 4)
        if isinstance(seed_accel, np.ndarray):
            seed_accel = np.ascontiguousarray(seed_accel, np.float32).reshape(self.n, 2)
        p._check(self._lib.p3m_adjoint_backward(p.handle, _pointer(seed), _pointer(seed_accel),
                                                _pointer(out), _pointer(out_accel)))
        return out

    def release(self) -> None:
        self.pipeline._check(self._lib.p3m_adjoint_release(self.pipeline.handle))


def _autograd_function():
    import torch

    class RolloutFunction(torch.autograd.Function):
        """final_bodies = RolloutFunction.apply(initial_bodies, rollout):
        CUDA float32 (n, 4) tensors on the pipeline's device."""

        @staticmethod
        def forward(ctx, bodies, rollout):
            torch.cuda.current_stream().synchronize()
            out = torch.empty_like(bodies)
            rollout.forward(bodies.detach().contiguous(), out)
            ctx.rollout = rollout
            return out

        @staticmethod
        def backward(ctx, grad_out):
            torch.cuda.current_stream().synchronize()
            grad = torch.empty_like(grad_out)
            ctx.rollout.backward(grad_out.contiguous(), out=grad)
            return grad, None

    return RolloutFunction


_fn = None


def rollout_function():
    """The ``torch.autograd.Function`` over a :class:`Rollout`."""
    global _fn
    if _fn is None:
        _fn = _autograd_function()
    return _fn


@dataclass
class LaunchObjective:
    loss: float                 # squared distance of the group's centroid to the target, px^2
    centroid_px: np.ndarray     # (2,)
    grad_velocity_px: np.ndarray  # dL/d(launch velocity) in px^2 / (px/s)
    grad_bodies: np.ndarray     # dL/d(initial bodies), (n, 4), unit coordinates


def launch_velocity_objective(rollout: Rollout, bodies: np.ndarray, group: np.ndarray,
                              velocity_px, target_px, with_gradient: bool = True) -> LaunchObjective:
    """Loss |centroid(group at the last step) - target|^2 with every body of
    `group` starting at velocity `velocity_px`, and the loss's gradient
    through the adjoint."""
    cfg = rollout.pipeline.config
    scale = np.array([cfg.viewport_width, cfg.viewport_height], np.float64)
    b = np.array(bodies, np.float32, copy=True)
    b[group, 2] = np.float32(velocity_px[0] / scale[0])
    b[group, 3] = np.float32(velocity_px[1] / scale[1])
    final = rollout.forward(b)
    # Centroid of the unwrapped displacement (the group moves less than half
    # the domain), in px.
    d = final[group, :2].astype(np.float64) - b[group, :2]
    d -= np.round(d)
    c = (b[group, :2].astype(np.float64) + d).mean(axis=0) * scale
    t = np.asarray(target_px, np.float64)
    loss = float(((c - t) ** 2).sum())
    if not with_gradient:
        return LaunchObjective(loss, c, None, None)
    seed = np.zeros((rollout.n, 4), np.float32)
    seed[group, 0] = 2.0 * (c[0] - t[0]) * scale[0] / len(group)
    seed[group, 1] = 2.0 * (c[1] - t[1]) * scale[1] / len(group)
    g = rollout.backward(seed)
    gv = np.array([g[group, 2].astype(np.float64).sum() / scale[0],
                   g[group, 3].astype(np.float64).sum() / scale[1]])
    return LaunchObjective(loss, c, gv, g)


def optimise_launch_velocity(rollout: Rollout, bodies: np.ndarray, group: np.ndarray,
                             velocity_px, target_px, iterations: int = 20,
                             step_px: float = 20.0):
    """Gradient descent on the launch velocity (px/s): each iteration moves
    against the gradient by at most `step_px` px/s (a normalised step that
    shrinks when the loss rises). Returns (velocity, history of losses)."""
    v = np.asarray(velocity_px, np.float64).copy()
    history = []
    step = float(step_px)
    best = None
    for _ in range(iterations):
        obj = launch_velocity_objective(rollout, bodies, group, v, target_px)
        history.append(obj.loss)
        if best is not None and obj.loss > best[0]:
            v = best[1].copy()
            step *= 0.5
            continue
        best = (obj.loss, v.copy())
        gnorm = float(np.linalg.norm(obj.grad_velocity_px))
        if gnorm == 0.0:
            break
        # Newton-like length for a quadratic in v, capped at `step`.
        length = min(step, obj.loss / gnorm)
        v = v - length * obj.grad_velocity_px / gnorm
    return best[1] if best else v, history
