"""ctypes binding of the C-ABI in include/p3m.h.

Loads the in-tree ``gravity_b200/lib/libgravity_p3m.so`` (building it with
nvcc first when it is missing or older than its sources). There is no other
implementation: if the library cannot be built or loaded, every call raises.
"""

from __future__ import annotations

import ctypes
import os
import threading
from pathlib import Path

from . import build as _build

P3M_OK = 0
P3M_ERR_INVALID_ARGUMENT = -1
P3M_ERR_OUT_OF_MEMORY = -2
P3M_ERR_CUDA = -3
P3M_ERR_TIMEOUT = -4
P3M_ERR_NON_FINITE = -5
P3M_ERR_CAPACITY = -6
P3M_ERR_UNSUPPORTED = -7
P3M_ERR_STATE = -8

P3M_ADJOINT_INITIAL_ACCELERATION = 1

P3M_DEPOSIT_U32 = 0
P3M_DEPOSIT_I64 = 1

BUF_BODIES = 0
BUF_ACCELERATION = 1
BUF_MATERIALS = 2
BUF_CELL_KEYS = 3
BUF_CELL_BODIES = 4
BUF_CELL_START = 5
BUF_CELL_COUNT = 6
BUF_CELL_MASS = 7
BUF_DENSITY = 8
BUF_FORCE = 9
BUF_DESTINATIONS = 10
BUF_GREEN = 11


class P3MConfig(ctypes.Structure):
    """Mirror of ``p3m_config`` (include/p3m.h)."""

    _fields_ = [
        ("struct_size", ctypes.c_int32),
        ("viewport_width", ctypes.c_int32),
        ("viewport_height", ctypes.c_int32),
        ("grid_width", ctypes.c_int32),
        ("grid_height", ctypes.c_int32),
        ("gravitational_constant", ctypes.c_float),
        ("softening_cells", ctypes.c_float),
        ("local_search_sigma_multiplier", ctypes.c_float),
        ("minimum_neighbor_radius_cells", ctypes.c_int32),
        ("maximum_neighbor_radius_cells", ctypes.c_int32),
        ("exact_neighbor_body_limit", ctypes.c_int32),
        ("maximum_home_body_interactions", ctypes.c_int32),
        ("minimum_distance_cell_fraction", ctypes.c_float),
        ("minimum_assignment_window_power", ctypes.c_float),
        ("time_step", ctypes.c_float),
        ("drift_substeps", ctypes.c_int32),
        ("spatial_sort_interval", ctypes.c_int32),
        ("capacity", ctypes.c_int32),
        ("bounded", ctypes.c_int32),
        ("deposit_mode", ctypes.c_int32),
        ("mutual_gravity", ctypes.c_int32),
    ]


class P3MTrajectoryConfig(ctypes.Structure):
    """Mirror of ``p3m_trajectory_config`` (include/p3m.h)."""

    _fields_ = [
        ("struct_size", ctypes.c_int32),
        ("steps", ctypes.c_int32),
        ("maximum_time_step", ctypes.c_float),
        ("target_segment_pixels", ctypes.c_float),
        ("maximum_path_viewport_diagonals", ctypes.c_float),
        ("minimum_dash_pixels", ctypes.c_float),
        ("restitution_coefficient", ctypes.c_float),
    ]


# Every symbol include/p3m.h declares, with (restype, argtypes).
_vp = ctypes.c_void_p
_i32 = ctypes.c_int32
_f = ctypes.c_float
SIGNATURES = {
    "p3m_config_default": (ctypes.c_int, [ctypes.POINTER(P3MConfig)]),
    "p3m_create": (ctypes.c_int, [ctypes.POINTER(P3MConfig), ctypes.POINTER(_vp)]),
    "p3m_destroy": (ctypes.c_int, [_vp]),
    "p3m_last_error": (ctypes.c_char_p, [_vp]),
    "p3m_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "p3m_upload_state": (ctypes.c_int, [_vp, _vp, _vp, _vp, _i32]),
    "p3m_upload_range": (ctypes.c_int, [_vp, _i32, _i32, _vp, _vp, _vp]),
    "p3m_download_state": (ctypes.c_int, [_vp, _vp, _vp, _vp, _i32]),
    "p3m_debug_get": (ctypes.c_int, [_vp, _i32, _vp, ctypes.c_size_t]),
    "p3m_device_pointer": (ctypes.c_int, [_vp, _i32, ctypes.POINTER(_vp),
                                          ctypes.POINTER(ctypes.c_size_t)]),
    "p3m_set_bounded": (ctypes.c_int, [_vp, _i32]),
    "p3m_set_field_acceleration": (ctypes.c_int, [_vp, _f, _f]),
    "p3m_set_mutual_gravity": (ctypes.c_int, [_vp, _i32]),
    "p3m_set_mass_excess": (ctypes.c_int, [_vp, _f]),
    "p3m_initialize_acceleration": (ctypes.c_int, [_vp, _i32]),
    "p3m_step": (ctypes.c_int, [_vp, _i32, _i32]),
    "p3m_sort_bodies": (ctypes.c_int, [_vp, _i32]),
    "p3m_drift": (ctypes.c_int, [_vp, _i32, _f, _f]),
    "p3m_build_force": (ctypes.c_int, [_vp, _i32]),
    "p3m_apply_kick": (ctypes.c_int, [_vp, _i32, _i32]),
    "p3m_build_cell_lists": (ctypes.c_int, [_vp, _i32]),
    "p3m_synchronize": (ctypes.c_int, [_vp]),
    "p3m_set_graphs": (ctypes.c_int, [_vp, _i32]),
    "p3m_profile_enable": (ctypes.c_int, [_vp, _i32]),
    "p3m_profile_read": (ctypes.c_int, [_vp, _vp, _vp]),
    "p3m_kernel_launches": (ctypes.c_int64, []),
    "p3m_get_stream": (ctypes.c_int, [_vp, ctypes.POINTER(_vp)]),
    "p3m_host_alloc": (ctypes.c_int, [ctypes.c_size_t, ctypes.POINTER(_vp)]),
    "p3m_host_free": (ctypes.c_int, [_vp]),
    "p3m_nonfinite_count": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int64)]),
    "p3m_wait_timeouts": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int64)]),
    "p3m_set_lookback_fault": (ctypes.c_int, [_vp, _i32, _i32]),
    "p3m_validate_fft": (ctypes.c_int, [_vp, _vp]),
    "p3m_density_spectrum": (ctypes.c_int, [_vp, _vp, ctypes.c_size_t]),
    "p3m_direct_accel_f64": (ctypes.c_int, [_vp, _i32, _vp, _i32, _vp]),
    "p3m_diagnostics_f64": (ctypes.c_int, [_vp, _i32, _vp]),
    "p3m_batch_create": (ctypes.c_int, [ctypes.POINTER(P3MConfig), _i32, ctypes.POINTER(_vp)]),
    "p3m_batch_destroy": (ctypes.c_int, [_vp]),
    "p3m_batch_last_error": (ctypes.c_char_p, [_vp]),
    "p3m_batch_size": (ctypes.c_int, [_vp, ctypes.POINTER(_i32)]),
    "p3m_batch_context": (ctypes.c_int, [_vp, _i32, ctypes.POINTER(_vp)]),
    "p3m_batch_upload": (ctypes.c_int, [_vp, _i32, _vp, _vp, _i32]),
    "p3m_batch_initialize_acceleration": (ctypes.c_int, [_vp]),
    "p3m_batch_step": (ctypes.c_int, [_vp, _i32]),
    "p3m_batch_autotune": (ctypes.c_int, [_vp, _i32, _vp]),
    "p3m_batch_set_fused": (ctypes.c_int, [_vp, _i32]),
    "p3m_batch_set_persistent": (ctypes.c_int, [_vp, _i32, _i32]),
    "p3m_set_launch_shape": (ctypes.c_int, [_vp, _i32, _i32]),
    "p3m_step_io": (ctypes.c_int, [_vp, _i32, _vp, _vp]),
    "p3m_batch_step_io": (ctypes.c_int, [_vp, _vp, _vp]),
    "p3m_autotune": (ctypes.c_int, [_vp, _i32, _i32, _vp]),
    "p3m_batch_set_barrier_fault": (ctypes.c_int, [_vp, _i32, _i32, _i32]),
    "p3m_batch_plan_info": (ctypes.c_int, [_vp, _vp]),
    "p3m_batch_phase_times": (ctypes.c_int, [_vp, _vp, _i32, ctypes.POINTER(_i32)]),
    "p3m_batch_synchronize": (ctypes.c_int, [_vp]),
    "p3m_batch_get_stream": (ctypes.c_int, [_vp, ctypes.POINTER(_vp)]),
    "p3m_adjoint_forward": (ctypes.c_int, [_vp, _i32, _i32, _i32, _i32]),
    "p3m_adjoint_backward": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "p3m_adjoint_release": (ctypes.c_int, [_vp]),
    "p3m_trajectory_config_default": (ctypes.c_int, [ctypes.POINTER(P3MTrajectoryConfig)]),
    "p3m_trajectories": (ctypes.c_int, [_vp, _i32, ctypes.POINTER(P3MTrajectoryConfig), _i32, _vp,
                                        _vp, _vp]),
    "p3m_cell_lists_static": (ctypes.c_int, [_vp, _vp, _i32, _i32, _i32, _vp, _vp, _vp, _vp,
                                             _vp, _vp, _vp]),
}

CELL_LISTS_STATIC_MAX_BODIES = 1 << 20

STAGES = ("spatial_sort", "drift", "cell_lists", "deposit", "forward_fft", "spectral",
          "inverse_fft", "kick", "short_range")

_lock = threading.Lock()
_lib = None


def library_path() -> Path:
    return _build.LIB_PATH


def load(rebuild_if_stale: bool = True) -> ctypes.CDLL:
    """Load (building when needed) the CUDA library; raises if impossible."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        path = library_path()
        if rebuild_if_stale and os.environ.get("GRAVITY_B200_NO_BUILD") != "1":
            if _build.needs_build():
                _build.build()
        if not path.exists():
            raise RuntimeError(f"{path} is missing; build it with `python -m gravity_b200.build`")
        lib = ctypes.CDLL(str(path))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


class P3MError(RuntimeError):
    """A non-zero p3m_status, with the library's message."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{message} (status {status})")
        self.status = status


def status_name(status: int) -> str:
    return load().p3m_status_string(status).decode()


def default_config() -> P3MConfig:
    c = P3MConfig()
    rc = load().p3m_config_default(ctypes.byref(c))
    if rc != P3M_OK:
        raise P3MError(rc, "p3m_config_default failed")
    return c
