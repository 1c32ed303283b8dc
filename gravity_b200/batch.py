"""``GravityBatch``: many independent P3M simulations stepped together.

The batched form of the C-ABI (include/p3m.h, p3m_batch_*): simulations of
uneven body counts and grid sizes — the application's trajectory previews and
ensembles — each keep a full context; one batch step is one CUDA graph launch
that runs every simulation's step on its own stream. ``autotune`` picks launch
shapes per grid by timing them.
"""

from __future__ import annotations

import ctypes
from typing import Sequence

import numpy as np

from . import _abi
from .config import P3MConfig
from .pipeline import GravityPipeline, P3MArgumentError, _ARG_STATUSES, _ptr


class GravityBatch:
    def __init__(self, configs: Sequence[P3MConfig]):
        self._lib = _abi.load()
        self.configs = list(configs)
        arr = (_abi.P3MConfig * len(self.configs))(*[c.to_abi() for c in self.configs])
        self._b = ctypes.c_void_p()
        rc = self._lib.p3m_batch_create(arr, len(self.configs), ctypes.byref(self._b))
        if rc != _abi.P3M_OK:
            self._raise(rc, self._lib.p3m_batch_last_error(None).decode())
        self.n = [0] * len(self.configs)

    @staticmethod
    def _raise(rc: int, msg: str):
        raise (P3MArgumentError if rc in _ARG_STATUSES else _abi.P3MError)(rc, msg)

    def _check(self, rc: int) -> None:
        if rc != _abi.P3M_OK:
            self._raise(rc, self._lib.p3m_batch_last_error(self._b).decode())

    def __len__(self) -> int:
        return len(self.configs)

    def close(self) -> None:
        if self._b:
            self._lib.p3m_batch_destroy(self._b)
            self._b = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, sim: int, bodies: np.ndarray, materials: np.ndarray | None = None) -> None:
        b = np.ascontiguousarray(bodies, np.float32).reshape(-1, 4)
        m = None if materials is None else np.ascontiguousarray(materials, np.float32).reshape(-1, 4)
        self._check(self._lib.p3m_batch_upload(self._b, sim, _ptr(b), _ptr(m), b.shape[0]))
        self.n[sim] = b.shape[0]

    def initialize_acceleration(self) -> None:
        self._check(self._lib.p3m_batch_initialize_acceleration(self._b))

    def step(self, steps: int = 1) -> None:
        self._check(self._lib.p3m_batch_step(self._b, steps))

    def set_fused(self, enabled: bool) -> None:
        """One launch per stage for all simulations (default) or one step
        per simulation inside one graph; the results are the same bits."""
        self._check(self._lib.p3m_batch_set_fused(self._b, 1 if enabled else 0))

    def synchronize(self) -> None:
        self._check(self._lib.p3m_batch_synchronize(self._b))

    def autotune(self, trial_steps: int = 3) -> list[tuple[int, int, int, int]]:
        """Per distinct grid: (width, height, FFT lines per CTA, short-range threads)."""
        out = np.zeros(64 * 4, np.int32)
        self._check(self._lib.p3m_batch_autotune(self._b, trial_steps, _ptr(out)))
        rows = [tuple(int(v) for v in out[4 * i:4 * i + 4]) for i in range(64)]
        return [r for r in rows if r[0] > 0]

    def download(self, sim: int):
        """(bodies, materials, acceleration) of simulation `sim` after the
        batch's queued steps."""
        return self.simulation(sim).download(self.n[sim])

    def simulation(self, sim: int) -> GravityPipeline:
        """A view of simulation `sim` (downloads, diagnostics, debug reads),
        taken after the batch's queued steps have finished."""
        self.synchronize()
        h = ctypes.c_void_p()
        self._check(self._lib.p3m_batch_context(self._b, sim, ctypes.byref(h)))
        return GravityPipeline.borrow(h, self.configs[sim])

    def stream_handle(self) -> int:
        s = ctypes.c_void_p()
        self._check(self._lib.p3m_batch_get_stream(self._b, ctypes.byref(s)))
        return s.value or 0
