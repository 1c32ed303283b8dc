"""``GravityPipeline``: the host-side mirror of the reference's P3M seam.

The reference's gravity solver is the Kotlin class ``GravityPipeline``
(src/main/kotlin/dev/gravity/GravityPipeline.kt:73-81). This class keeps the
names and meaning of its P3M surface — ``initialize_acceleration(n)``
(:366-370), ``step(n)`` (:445-494), the ``bounded`` / ``field_acceleration_*``
/ ``mutual_gravity`` properties (:97-121) and the private stages
``build_force`` (:907), ``apply_kick`` (:1213), ``sort_bodies`` (:1269) — and
runs every one of them through the C-ABI of include/p3m.h on the GPU.

Errors follow the reference: invalid arguments raise ``ValueError``
(Kotlin ``require``), invalid state raises ``RuntimeError`` (``check``).
There is no CPU path: without the CUDA library or a GPU, construction fails.
"""

from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from . import _abi
from .config import P3MConfig


class P3MArgumentError(_abi.P3MError, ValueError):
    """Invalid argument, capacity or unsupported configuration."""


_ARG_STATUSES = {_abi.P3M_ERR_INVALID_ARGUMENT, _abi.P3M_ERR_CAPACITY, _abi.P3M_ERR_UNSUPPORTED}


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


class GravityPipeline:
    """A P3M gravity context on the current CUDA device."""

    def __init__(self, config: P3MConfig | None = None):
        self.config = config or P3MConfig()
        self._lib = _abi.load()
        self._ctx = ctypes.c_void_p()
        abi_cfg = self.config.to_abi()
        rc = self._lib.p3m_create(ctypes.byref(abi_cfg), ctypes.byref(self._ctx))
        if rc != _abi.P3M_OK:
            msg = self._lib.p3m_last_error(None).decode()
            raise (P3MArgumentError if rc in _ARG_STATUSES else _abi.P3MError)(rc, msg)
        self._bounded = bool(self.config.bounded)
        self._mutual = bool(self.config.mutual_gravity)
        self._field = (0.0, 0.0)
        self._mass_excess = 0.0
        self._owned = True

    @classmethod
    def borrow(cls, handle: ctypes.c_void_p, config: P3MConfig) -> "GravityPipeline":
        """A view of a context owned elsewhere (a simulation of a batch);
        closing the view leaves the context alive."""
        self = cls.__new__(cls)
        self.config = config
        self._lib = _abi.load()
        self._ctx = handle
        self._bounded = bool(config.bounded)
        self._mutual = bool(config.mutual_gravity)
        self._field = (0.0, 0.0)
        self._mass_excess = 0.0
        self._owned = False
        return self

    # ------------------------------------------------------------ plumbing
    def _check(self, rc: int) -> None:
        if rc != _abi.P3M_OK:
            msg = self._lib.p3m_last_error(self._ctx).decode()
            raise (P3MArgumentError if rc in _ARG_STATUSES else _abi.P3MError)(rc, msg)

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._ctx

    def close(self) -> None:
        if self._ctx and getattr(self, "_owned", True):
            self._lib.p3m_destroy(self._ctx)
        self._ctx = ctypes.c_void_p()

    def __enter__(self) -> "GravityPipeline":
        return self

    def __exit__(self, *exc) -> None:
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---------------------------------------------------------- properties
    @property
    def bounded(self) -> bool:
        return self._bounded

    @bounded.setter
    def bounded(self, value: bool) -> None:
        self._check(self._lib.p3m_set_bounded(self._ctx, 1 if value else 0))
        self._bounded = bool(value)

    @property
    def mutual_gravity(self) -> bool:
        return self._mutual

    @mutual_gravity.setter
    def mutual_gravity(self, value: bool) -> None:
        self._check(self._lib.p3m_set_mutual_gravity(self._ctx, 1 if value else 0))
        self._mutual = bool(value)

    @property
    def field_acceleration_x(self) -> float:
        return self._field[0]

    @field_acceleration_x.setter
    def field_acceleration_x(self, value: float) -> None:
        self.set_field_acceleration(value, self._field[1])

    @property
    def field_acceleration_y(self) -> float:
        return self._field[1]

    @field_acceleration_y.setter
    def field_acceleration_y(self, value: float) -> None:
        self.set_field_acceleration(self._field[0], value)

    def set_field_acceleration(self, ax_px: float, ay_px: float) -> None:
        """Uniform field in px/s^2 (GravityPipeline.kt:105-107)."""
        self._check(self._lib.p3m_set_field_acceleration(self._ctx, float(ax_px), float(ay_px)))
        self._field = (float(ax_px), float(ay_px))

    @property
    def mass_excess(self) -> float:
        return self._mass_excess

    @mass_excess.setter
    def mass_excess(self, value: float) -> None:
        self._check(self._lib.p3m_set_mass_excess(self._ctx, float(value)))
        self._mass_excess = float(value)

    # --------------------------------------------------------------- state
    def upload(self, bodies: np.ndarray, materials: np.ndarray | None = None,
               acceleration: np.ndarray | None = None) -> None:
        """Upload float32 (n, 4) bodies [, (n, 4) materials, (n, 2) accelerations]."""
        b = np.ascontiguousarray(bodies, dtype=np.float32).reshape(-1, 4)
        n = b.shape[0]
        m = None if materials is None else np.ascontiguousarray(materials, dtype=np.float32).reshape(n, 4)
        a = None if acceleration is None else np.ascontiguousarray(acceleration, dtype=np.float32).reshape(n, 2)
        self._check(self._lib.p3m_upload_state(self._ctx, _ptr(b), _ptr(m), _ptr(a), n))

    def upload_range(self, first: int, bodies: np.ndarray, materials: np.ndarray | None = None,
                     acceleration: np.ndarray | None = None) -> None:
        """Write bodies into slots [first, first + len) (spawnProjectile's
        glBufferSubData at an offset, GravityPipeline.kt:621-718)."""
        b = np.ascontiguousarray(bodies, dtype=np.float32).reshape(-1, 4)
        k = b.shape[0]
        m = None if materials is None else np.ascontiguousarray(materials, dtype=np.float32).reshape(k, 4)
        a = None if acceleration is None else np.ascontiguousarray(acceleration, dtype=np.float32).reshape(k, 2)
        self._check(self._lib.p3m_upload_range(self._ctx, first, k, _ptr(b), _ptr(m), _ptr(a)))

    def download(self, n: int):
        """(bodies (n,4), materials (n,4), acceleration (n,2)) as float32."""
        b = np.empty((n, 4), np.float32)
        m = np.empty((n, 4), np.float32)
        a = np.empty((n, 2), np.float32)
        self._check(self._lib.p3m_download_state(self._ctx, _ptr(b), _ptr(m), _ptr(a), n))
        return b, m, a

    def download_into(self, n: int, bodies: np.ndarray | None = None,
                      materials: np.ndarray | None = None,
                      acceleration: np.ndarray | None = None) -> None:
        """Read state into caller-owned (e.g. page-locked) float32 arrays."""
        for a, w in ((bodies, 4), (materials, 4), (acceleration, 2)):
            if a is not None and (a.dtype != np.float32 or a.size < n * w or not a.flags.c_contiguous):
                raise ValueError("output arrays must be contiguous float32 with room for n rows")
        self._check(self._lib.p3m_download_state(self._ctx, _ptr(bodies), _ptr(materials),
                                                  _ptr(acceleration), n))

    def upload_n(self, n: int, bodies: np.ndarray | None = None,
                 materials: np.ndarray | None = None,
                 acceleration: np.ndarray | None = None) -> None:
        """Upload the first n rows of caller-owned float32 arrays as they are."""
        for a, w in ((bodies, 4), (materials, 4), (acceleration, 2)):
            if a is not None and (a.dtype != np.float32 or a.size < n * w or not a.flags.c_contiguous):
                raise ValueError("input arrays must be contiguous float32 with n rows")
        self._check(self._lib.p3m_upload_state(self._ctx, _ptr(bodies), _ptr(materials),
                                                _ptr(acceleration), n))

    def bodies(self, n: int) -> np.ndarray:
        return self.download(n)[0]

    def acceleration(self, n: int) -> np.ndarray:
        return self.download(n)[2]

    def debug_get(self, which: int, dtype, count: int) -> np.ndarray:
        out = np.empty(count, dtype=dtype)
        self._check(self._lib.p3m_debug_get(self._ctx, which, _ptr(out), out.nbytes))
        return out

    def synchronize(self) -> None:
        self._check(self._lib.p3m_synchronize(self._ctx))

    # ----------------------------------------------------------- the step
    def initialize_acceleration(self, active_bodies: int) -> None:
        self._check(self._lib.p3m_initialize_acceleration(self._ctx, active_bodies))

    def step(self, active_bodies: int, steps: int = 1) -> None:
        self._check(self._lib.p3m_step(self._ctx, active_bodies, steps))

    def step_io(self, n: int, bodies_in: np.ndarray | None = None,
                bodies_out: np.ndarray | None = None) -> None:
        """One step with its host copies pipelined (p3m_step_io): bodies_in
        becomes the first n bodies before the step, the stepped bodies go to
        bodies_out. Asynchronous: keep both arrays (page-locked for overlap)
        alive and bodies_in unchanged until synchronize()."""
        for a, what in ((bodies_in, "input"), (bodies_out, "output")):
            if a is not None and (a.dtype != np.float32 or a.size < n * 4 or not a.flags.c_contiguous):
                raise ValueError(f"{what} array must be contiguous float32 with n rows of 4")
        self._check(self._lib.p3m_step_io(self._ctx, n, _ptr(bodies_in), _ptr(bodies_out)))

    def set_launch_shape(self, fft_lines: int = 0, short_range_threads: int = 256) -> None:
        """FFT lines per CTA (0: automatic) and short-range block size; the
        results do not depend on them."""
        self._check(self._lib.p3m_set_launch_shape(self._ctx, fft_lines, short_range_threads))

    def autotune(self, active_bodies: int, trial_steps: int = 3) -> tuple[int, int]:
        """Times steps under each launch shape, keeps the fastest and puts the
        state back; returns (fft_lines, short_range_threads)."""
        out = (ctypes.c_int32 * 2)()
        self._check(self._lib.p3m_autotune(self._ctx, active_bodies, trial_steps, out))
        return int(out[0]), int(out[1])

    def build_force(self, active_bodies: int) -> None:
        self._check(self._lib.p3m_build_force(self._ctx, active_bodies))

    def apply_kick(self, active_bodies: int, initial: bool) -> None:
        self._check(self._lib.p3m_apply_kick(self._ctx, active_bodies, 1 if initial else 0))

    def sort_bodies(self, active_bodies: int) -> None:
        self._check(self._lib.p3m_sort_bodies(self._ctx, active_bodies))

    def drift(self, active_bodies: int, kick_dt: float, drift_dt: float) -> None:
        self._check(self._lib.p3m_drift(self._ctx, active_bodies, float(kick_dt), float(drift_dt)))

    def build_cell_lists(self, active_bodies: int) -> None:
        self._check(self._lib.p3m_build_cell_lists(self._ctx, active_bodies))

    # -------------------------------------------------- profiling, diagnostics
    def profile_enable(self, enabled: bool = True) -> None:
        self._check(self._lib.p3m_profile_enable(self._ctx, 1 if enabled else 0))

    def profile_read(self) -> dict:
        """{stage: (total device ms, intervals)} since profiling was enabled."""
        ms = np.zeros(len(_abi.STAGES), np.float64)
        cnt = np.zeros(len(_abi.STAGES), np.int64)
        self._check(self._lib.p3m_profile_read(self._ctx, _ptr(ms), _ptr(cnt)))
        return {name: (float(ms[i]), int(cnt[i])) for i, name in enumerate(_abi.STAGES)}

    def stream_handle(self) -> int:
        s = ctypes.c_void_p()
        self._check(self._lib.p3m_get_stream(self._ctx, ctypes.byref(s)))
        return s.value or 0

    def trajectories(self, n: int, origins_px, velocities_px, steps: int = 1024,
                     maximum_time_step: float = 1.0, target_segment_pixels: float = 6.0,
                     maximum_path_viewport_diagonals: float = 1.0,
                     minimum_dash_pixels: float = 3.0, restitution: float = 0.0) -> np.ndarray:
        """updateTrajectory (GravityPipeline.kt:514-600) for every row of
        origins / velocities (px, px/s) on the field of the last force build:
        (count, steps * 6, 4) float32 vertices (x, y, dash px, distance
        fraction or -1)."""
        o = np.ascontiguousarray(origins_px, np.float32).reshape(-1, 2)
        v = np.ascontiguousarray(velocities_px, np.float32).reshape(-1, 2)
        if o.shape != v.shape:
            raise ValueError("origins and velocities must have the same shape")
        cfg = _abi.P3MTrajectoryConfig()
        self._check(self._lib.p3m_trajectory_config_default(ctypes.byref(cfg)))
        cfg.steps = steps
        cfg.maximum_time_step = maximum_time_step
        cfg.target_segment_pixels = target_segment_pixels
        cfg.maximum_path_viewport_diagonals = maximum_path_viewport_diagonals
        cfg.minimum_dash_pixels = minimum_dash_pixels
        cfg.restitution_coefficient = restitution
        out = np.empty((o.shape[0], steps * 6, 4), np.float32)
        self._check(self._lib.p3m_trajectories(self._ctx, n, ctypes.byref(cfg), o.shape[0],
                                               _ptr(o), _ptr(v), _ptr(out)))
        return out

    def nonfinite_count(self) -> int:
        c = ctypes.c_int64()
        self._check(self._lib.p3m_nonfinite_count(self._ctx, ctypes.byref(c)))
        return c.value

    def wait_timeouts(self) -> int:
        """Bounded device waits (sort look-back) that gave up; expected 0."""
        c = ctypes.c_int64()
        self._check(self._lib.p3m_wait_timeouts(self._ctx, ctypes.byref(c)))
        return c.value

    def set_lookback_fault(self, poll_limit: int = 200_000, withheld_tile: int = -1) -> None:
        """Test hook of the timeout path: a poll limit for the sort's look-back
        waits and a tile whose counts are never published (-1: none)."""
        self._check(self._lib.p3m_set_lookback_fault(self._ctx, int(poll_limit), int(withheld_tile)))

    def validate_fft(self) -> dict:
        """validateFft (GravityPipeline.kt:378-419): the FP32 density spectrum
        of the last force build against an FP64 transform of the same mesh."""
        out = np.zeros(3, np.float64)
        self._check(self._lib.p3m_validate_fft(self._ctx, _ptr(out)))
        return {"maximum_absolute_error": float(out[0]), "maximum_relative_error": float(out[1]),
                "root_mean_square_error": float(out[2])}

    def density_spectrum(self) -> np.ndarray:
        """FP32 spectrum of density / massScale of the last force build:
        (MH, MW/2+1) complex64, numpy.fft.rfft2's layout."""
        mw, mh = self.mesh_shape
        out = np.empty((mh, mw // 2 + 1), np.complex64)
        self._check(self._lib.p3m_density_spectrum(self._ctx, _ptr(out), out.nbytes))
        return out

    def direct_accel_f64(self, n: int, targets) -> np.ndarray:
        """FP64 direct-sum accelerations (unit/s^2) of the target bodies."""
        t = np.ascontiguousarray(targets, np.int32)
        out = np.empty((len(t), 2), np.float64)
        self._check(self._lib.p3m_direct_accel_f64(self._ctx, n, _ptr(t), len(t), _ptr(out)))
        return out

    def diagnostics_f64(self, n: int) -> dict:
        out = np.zeros(6, np.float64)
        self._check(self._lib.p3m_diagnostics_f64(self._ctx, n, _ptr(out)))
        return {"momentum": (out[0], out[1]), "kinetic_energy": out[2],
                "center_of_mass": (out[3], out[4]), "mass": out[5]}

    # ------------------------------------------------------ intermediates
    @property
    def mesh_shape(self) -> tuple[int, int]:
        g = self.config.gravity
        k = 2 if self._bounded else 1
        return g.grid_width * k, g.grid_height * k

    def cell_lists(self, n: int):
        """(keys[n], bodies[n], start[P], count[P], mass[P]) of the last cell sort."""
        g = self.config.gravity
        P = g.grid_width * g.grid_height
        keys = self.debug_get(_abi.BUF_CELL_KEYS, np.uint32, n)
        ids = self.debug_get(_abi.BUF_CELL_BODIES, np.int32, n)
        start = self.debug_get(_abi.BUF_CELL_START, np.int32, P)
        count = self.debug_get(_abi.BUF_CELL_COUNT, np.int32, P)
        mass = self.debug_get(_abi.BUF_CELL_MASS, np.uint32, P)
        return keys, ids, start, count, mass

    def density(self) -> np.ndarray:
        mw, mh = self.mesh_shape
        dt = np.int64 if self.config.deposit_mode == _abi.P3M_DEPOSIT_I64 else np.uint32
        return self.debug_get(_abi.BUF_DENSITY, dt, mw * mh).reshape(mh, mw)

    def force(self) -> np.ndarray:
        """Long-range mesh force, (MH, MW, 2) float32 (fx, fy)."""
        mw, mh = self.mesh_shape
        return self.debug_get(_abi.BUF_FORCE, np.float32, mw * mh * 2).reshape(mh, mw, 2)

    def destinations(self, n: int) -> np.ndarray:
        return self.debug_get(_abi.BUF_DESTINATIONS, np.uint32, n)

    def green(self) -> np.ndarray:
        mw, mh = self.mesh_shape
        return self.debug_get(_abi.BUF_GREEN, np.float32, (mw // 2 + 1) * mh * 2).reshape(mh, mw // 2 + 1, 2)


class PinnedArray:
    """A float32 numpy array over page-locked host memory (p3m_host_alloc)."""

    def __init__(self, shape):
        self._lib = _abi.load()
        count = int(np.prod(shape))
        self._ptr = ctypes.c_void_p()
        rc = self._lib.p3m_host_alloc(count * 4, ctypes.byref(self._ptr))
        if rc != _abi.P3M_OK:
            raise _abi.P3MError(rc, self._lib.p3m_last_error(None).decode())
        buf = (ctypes.c_float * count).from_address(self._ptr.value)
        self.array = np.ctypeslib.as_array(buf).reshape(shape)

    def free(self) -> None:
        if self._ptr:
            self.array = None
            self._lib.p3m_host_free(self._ptr)
            self._ptr = ctypes.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def kernel_launches() -> int:
    """Kernels the library has launched in this process."""
    return int(_abi.load().p3m_kernel_launches())
