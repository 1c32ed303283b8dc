"""CPU oracle of Gravity's P3M gravity step — TEST INFRASTRUCTURE ONLY.

A C++ restatement of the reference's GLSL shaders (p3m_oracle.cpp), built by
oracle/Makefile into oracle/_build/liboracle.so and loaded with ctypes. Only
the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` use it, always as the checker or the timed CPU baseline; the
product package ``gravity_b200`` never imports it.

Parity pins (what ties this restatement to the reference's own tests):
  * Morton keys and reorder invariants: SpatialSortIntegrationTest.kt:18-54,
    177-186 (fixtures in tests/golden/).
  * FFT layout and tolerances: Radix2FftLayoutTest.kt:17-188, with numpy's
    FP64 FFT in place of JTransforms 3.2 (not available here).
  * Config defaults: GravityConfigTest.kt:9-13 and GravityConfig.kt:641-654.
  * Deposit, cell lists, forces and positions: parity unpinned — the
    reference has no test that pins them and its GLSL cannot run here (no
    OpenGL); this restatement is their only oracle.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
import threading
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"
_lock = threading.Lock()
_lib = None


def build() -> Path:
    """Compile the oracle with its Makefile (g++, -ffp-contract=off, OpenMP)."""
    res = subprocess.run(["make", "-s", "-C", str(HERE)], capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{res.stdout}\n{res.stderr}")
    return LIB


def load() -> ctypes.CDLL:
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        newest = max((HERE / f).stat().st_mtime for f in ("p3m_oracle.cpp", "p3m_adjoint_f64.cpp"))
        if not LIB.exists() or LIB.stat().st_mtime < newest:
            build()
        lib = ctypes.CDLL(str(LIB))
        vp, i, f = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
        sigs = {
            "oracle_set_threads": (None, [i]),
            "oracle_max_threads": (i, []),
            "oracle_morton_key": (ctypes.c_uint32, [f, f, i, i]),
            "oracle_sort_axis_bits": (i, [i]),
            "oracle_mass_scale": (i, [f]),
            "oracle_neighbor_radii": (None, [vp, vp, vp]),
            "oracle_fft2d_f32": (None, [vp, i, i, i]),
            "oracle_fft2d_f64": (None, [vp, i, i, i]),
            "oracle_validate": (i, [vp]),
            "oracle_create": (vp, [vp]),
            "oracle_destroy": (None, [vp]),
            "oracle_set_bounded": (None, [vp, i]),
            "oracle_set_field": (None, [vp, f, f]),
            "oracle_set_mutual_gravity": (None, [vp, i]),
            "oracle_set_mass_excess": (None, [vp, f]),
            "oracle_upload": (None, [vp, vp, vp, vp, i]),
            "oracle_download": (None, [vp, vp, vp, vp, i]),
            "oracle_drift": (None, [vp, i, f, f]),
            "oracle_drift_raw": (None, [vp, vp, i, f, f, i]),
            "oracle_sort_bodies": (None, [vp, i]),
            "oracle_build_force": (None, [vp, i]),
            "oracle_build_grid": (None, [vp, i]),
            "oracle_apply_kick": (None, [vp, i, i]),
            "oracle_initialize_acceleration": (None, [vp, i]),
            "oracle_step": (None, [vp, i, i]),
            "oracle_normalization": (i, [vp, vp, vp]),
            "oracle_radii": (None, [vp, vp, vp]),
            "oracle_cell_lists": (None, [vp, i, vp, vp, vp, vp, vp]),
            "oracle_density_u32": (None, [vp, vp]),
            "oracle_density_i64": (None, [vp, vp]),
            "oracle_force": (None, [vp, vp]),
            "oracle_density_spectrum": (None, [vp, vp]),
            "oracle_kernel_spectra": (None, [vp, vp, vp]),
            "oracle_destinations": (None, [vp, vp, i]),
            "oracle_direct_sum_f64": (None, [vp, vp, i, vp, i, vp, f, i, vp]),
            "oracle_trajectory": (None, [vp, i, vp, f, f, f, f, vp]),
            "oracle_adj_create": (vp, [vp, vp, i, ctypes.c_double, ctypes.c_double]),
            "oracle_adj_destroy": (None, [vp]),
            "oracle_adj_force": (None, [vp, vp, vp]),
            "oracle_adj_mesh_force": (None, [vp, vp, vp, vp]),
            "oracle_adj_set_positions": (None, [vp, i, vp]),
            "oracle_adj_forward": (None, [vp, vp, vp, i, i, vp, vp]),
            "oracle_adj_backward": (None, [vp, vp, vp, vp, vp]),
        }
        for name, (res, args) in sigs.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def set_threads(n: int) -> None:
    load().oracle_set_threads(int(n))


def max_threads() -> int:
    return load().oracle_max_threads()


def morton_key(x: float, y: float, wbits: int, hbits: int) -> int:
    return load().oracle_morton_key(float(x), float(y), wbits, hbits)


def sort_axis_bits(extent: int) -> int:
    return load().oracle_sort_axis_bits(extent)


def mass_scale(total_mass: float) -> int:
    return load().oracle_mass_scale(float(total_mass))


def fft2d_f32(values: np.ndarray, inverse: bool) -> np.ndarray:
    """Mirror of fft_shared.comp on an (H, W) complex64 array."""
    a = np.ascontiguousarray(values, dtype=np.complex64).copy()
    h, w = a.shape
    load().oracle_fft2d_f32(_p(a), w, h, 1 if inverse else 0)
    return a


def fft2d_f64(values: np.ndarray, inverse: bool) -> np.ndarray:
    """FP64 radix-2 transform in the same layout (cpuFft2d)."""
    a = np.ascontiguousarray(values, dtype=np.complex128).copy()
    h, w = a.shape
    load().oracle_fft2d_f64(_p(a), w, h, 1 if inverse else 0)
    return a


def direct_sum_f64(bodies: np.ndarray, materials: np.ndarray, targets: np.ndarray, cfg_abi,
                   total_mass: float, bounded: bool) -> np.ndarray:
    """FP64 direct-sum accelerations (unit/s^2) of the target bodies."""
    b = np.ascontiguousarray(bodies, np.float32)
    m = np.ascontiguousarray(materials, np.float32)
    t = np.ascontiguousarray(targets, np.int32)
    out = np.empty((len(t), 2), np.float64)
    load().oracle_direct_sum_f64(_p(b), _p(m), b.shape[0], _p(t), len(t), ctypes.byref(cfg_abi),
                                 float(total_mass), 1 if bounded else 0, _p(out))
    return out


class OracleSim:
    """CPU restatement of the P3M path with GravityPipeline's method names."""

    def __init__(self, config):
        self.config = config
        self._abi_cfg = config.to_abi()
        self._lib = load()
        self._s = self._lib.oracle_create(ctypes.byref(self._abi_cfg))
        if not self._s:
            raise ValueError("oracle rejected the configuration")
        self._bounded = bool(config.bounded)

    def close(self):
        if self._s:
            self._lib.oracle_destroy(self._s)
            self._s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def bounded(self):
        return self._bounded

    @bounded.setter
    def bounded(self, v):
        self._lib.oracle_set_bounded(self._s, 1 if v else 0)
        self._bounded = bool(v)

    def set_field_acceleration(self, ax_px, ay_px):
        self._lib.oracle_set_field(self._s, float(ax_px), float(ay_px))

    def set_mutual_gravity(self, on):
        self._lib.oracle_set_mutual_gravity(self._s, 1 if on else 0)

    def set_mass_excess(self, e):
        self._lib.oracle_set_mass_excess(self._s, float(e))

    def upload(self, bodies, materials=None, acceleration=None):
        b = np.ascontiguousarray(bodies, np.float32).reshape(-1, 4)
        n = b.shape[0]
        m = None if materials is None else np.ascontiguousarray(materials, np.float32).reshape(n, 4)
        a = None if acceleration is None else np.ascontiguousarray(acceleration, np.float32).reshape(n, 2)
        self._lib.oracle_upload(self._s, _p(b), _p(m), _p(a), n)

    def download(self, n):
        b = np.empty((n, 4), np.float32)
        m = np.empty((n, 4), np.float32)
        a = np.empty((n, 2), np.float32)
        self._lib.oracle_download(self._s, _p(b), _p(m), _p(a), n)
        return b, m, a

    def initialize_acceleration(self, n):
        self._lib.oracle_initialize_acceleration(self._s, n)

    def step(self, n, steps=1):
        self._lib.oracle_step(self._s, n, steps)

    def build_force(self, n):
        self._lib.oracle_build_force(self._s, n)

    def build_grid(self, n):
        self._lib.oracle_build_grid(self._s, n)

    def apply_kick(self, n, initial):
        self._lib.oracle_apply_kick(self._s, n, 1 if initial else 0)

    def sort_bodies(self, n):
        self._lib.oracle_sort_bodies(self._s, n)

    def drift(self, n, kick_dt, drift_dt):
        self._lib.oracle_drift(self._s, n, float(kick_dt), float(drift_dt))

    def normalization(self):
        m = ctypes.c_float()
        s = ctypes.c_int()
        self._lib.oracle_normalization(self._s, ctypes.byref(m), ctypes.byref(s))
        return m.value, s.value

    def radii(self):
        rx, ry = ctypes.c_int(), ctypes.c_int()
        self._lib.oracle_radii(self._s, ctypes.byref(rx), ctypes.byref(ry))
        return rx.value, ry.value

    @property
    def mesh_shape(self):
        g = self.config.gravity
        k = 2 if self._bounded else 1
        return g.grid_width * k, g.grid_height * k

    def cell_lists(self, n):
        g = self.config.gravity
        P = g.grid_width * g.grid_height
        keys = np.empty(n, np.uint32)
        ids = np.empty(n, np.int32)
        start = np.empty(P, np.int32)
        count = np.empty(P, np.int32)
        mass = np.empty(P, np.uint32)
        self._lib.oracle_cell_lists(self._s, n, _p(keys), _p(ids), _p(start), _p(count), _p(mass))
        return keys, ids, start, count, mass

    def density(self):
        mw, mh = self.mesh_shape
        if self.config.deposit_mode == 1:
            out = np.empty(mw * mh, np.int64)
            self._lib.oracle_density_i64(self._s, _p(out))
        else:
            out = np.empty(mw * mh, np.uint32)
            self._lib.oracle_density_u32(self._s, _p(out))
        return out.reshape(mh, mw)

    def force(self):
        mw, mh = self.mesh_shape
        out = np.empty((mh, mw, 2), np.float32)
        self._lib.oracle_force(self._s, _p(out))
        return out

    def density_spectrum(self):
        mw, mh = self.mesh_shape
        out = np.empty((mh, mw), np.complex64)
        self._lib.oracle_density_spectrum(self._s, _p(out))
        return out

    def kernel_spectra(self):
        mw, mh = self.mesh_shape
        kx = np.empty((mh, mw), np.complex64)
        ky = np.empty((mh, mw), np.complex64)
        self._lib.oracle_kernel_spectra(self._s, _p(kx), _p(ky))
        return kx, ky

    def trajectory(self, n, origin_px, velocity_px, steps=1024, max_dt=1.0, segment_px=6.0,
                   path_diagonals=1.0, min_dash_px=3.0, restitution=0.0):
        """S/trajectory.comp for one preview: (steps * 6, 4) vertices."""
        prm = np.array([steps, max_dt, segment_px, path_diagonals, min_dash_px, restitution],
                       np.float32)
        out = np.empty((steps * 6, 4), np.float32)
        self._lib.oracle_trajectory(self._s, n, _p(prm), float(origin_px[0]), float(origin_px[1]),
                                    float(velocity_px[0]), float(velocity_px[1]), _p(out))
        return out

    def destinations(self, n):
        out = np.empty(n, np.uint32)
        self._lib.oracle_destinations(self._s, _p(out), n)
        return out


class Adjoint64:
    """FP64 reference of the differentiated gravity-only rollout on the torus
    (p3m_adjoint_f64.cpp): forward, then the hand-written reverse pass.

    field_px: uniform field in px/s^2, converted to unit/s^2 like the library.
    """

    def __init__(self, config, materials, field_px=(0.0, 0.0)):
        self._lib = load()
        self._abi_cfg = config.to_abi()
        m = np.ascontiguousarray(materials, np.float64).reshape(-1, 4)
        self.n = m.shape[0]
        fx = field_px[0] / config.viewport_width
        fy = field_px[1] / config.viewport_height
        self._s = self._lib.oracle_adj_create(ctypes.byref(self._abi_cfg), _p(m), self.n, fx, fy)
        if not self._s:
            raise ValueError("the FP64 adjoint covers the torus only, with n > 0")

    def close(self):
        if self._s:
            self._lib.oracle_adj_destroy(self._s)
            self._s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def force(self, positions):
        x = np.ascontiguousarray(positions, np.float64).reshape(-1, 2)
        out = np.empty_like(x)
        self._lib.oracle_adj_force(self._s, _p(x), _p(out))
        return out

    def mesh_force(self, positions):
        """The FP64 mesh force (H, W, 2) at `positions` (n, 2)."""
        x = np.ascontiguousarray(positions, np.float64).reshape(-1, 2)
        w, h = self._abi_cfg.grid_width, self._abi_cfg.grid_height
        ex = np.empty((h, w), np.float64)
        ey = np.empty((h, w), np.float64)
        self._lib.oracle_adj_mesh_force(self._s, _p(x), _p(ex), _p(ey))
        return np.stack([ex, ey], axis=-1)

    def forward(self, bodies, steps, acceleration=None):
        """Final (bodies (n,4), acceleration (n,2)) in float64. Without
        `acceleration`, a0 is the force at the initial positions."""
        b = np.ascontiguousarray(bodies, np.float64).reshape(-1, 4)
        a = None if acceleration is None else np.ascontiguousarray(acceleration, np.float64).reshape(-1, 2)
        out = np.empty_like(b)
        acc = np.empty((self.n, 2), np.float64)
        self._lib.oracle_adj_forward(self._s, _p(b), _p(a), 1 if a is None else 0, steps,
                                     _p(out), _p(acc))
        return out, acc

    def set_positions(self, k, positions):
        """Replace the recorded positions of step k (0 = initial)."""
        x = np.ascontiguousarray(positions, np.float64).reshape(self.n, 2)
        self._lib.oracle_adj_set_positions(self._s, int(k), _p(x))

    def backward(self, seed, seed_accel=None):
        """dL/d(initial bodies) (n,4) and dL/d(initial acceleration) (n,2)."""
        s4 = np.ascontiguousarray(seed, np.float64).reshape(-1, 4)
        sa = None if seed_accel is None else np.ascontiguousarray(seed_accel, np.float64).reshape(-1, 2)
        g = np.empty_like(s4)
        ga = np.empty((self.n, 2), np.float64)
        self._lib.oracle_adj_backward(self._s, _p(s4), _p(sa), _p(g), _p(ga))
        return g, ga
