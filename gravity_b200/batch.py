"""``GravityBatch``: many independent P3M simulations stepped together.

The batched form of the C-ABI (include/p3m.h, p3m_batch_*): simulations of
uneven body counts and grid sizes — the application's trajectory previews and
ensembles — each keep a full context. One batch step is, by default, one
launch per stage over all simulations (captured in a CUDA graph);
``set_persistent(True)`` makes it ONE persistent cooperative kernel launch
that runs every stage phase by phase, ``set_fused(False)`` one step per
simulation on its own stream. All forms give the same bits. ``autotune``
picks the form and launch shapes by timing whole batch steps.
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

    def step_io(self, bodies_in: np.ndarray | None = None,
                bodies_out: np.ndarray | None = None) -> None:
        """One batch step with its host copies pipelined (p3m_batch_step_io):
        bodies_in holds every simulation's bodies back to back (simulation
        order, n rows each) and becomes their bodies before the step; the
        stepped bodies go to bodies_out in the same layout. Asynchronous: keep
        both arrays (page-locked for overlap) alive and bodies_in unchanged
        until synchronize()."""
        rows = sum(self.n)
        for a, what in ((bodies_in, "input"), (bodies_out, "output")):
            if a is not None and (a.dtype != np.float32 or a.size < rows * 4 or not a.flags.c_contiguous):
                raise ValueError(f"{what} array must be contiguous float32 with sum(n) rows of 4")
        self._check(self._lib.p3m_batch_step_io(self._b, _ptr(bodies_in), _ptr(bodies_out)))

    def set_persistent(self, enabled: bool, ctas_per_sm: int = 0) -> None:
        """One persistent launch per batch step, or one launch per stage (the
        default); ``ctas_per_sm`` 0 keeps as many CTAs per SM as stay
        resident."""
        self._check(self._lib.p3m_batch_set_persistent(self._b, 1 if enabled else 0, ctas_per_sm))

    def set_barrier_fault(self, poll_limit: int = 1 << 20, withheld_cta: int = -1,
                          phase: int = -1) -> None:
        """Test hook of the persistent step's grid barrier: the poll limit of
        each wait, and a CTA that never arrives after ``phase``. The defaults
        clear it."""
        self._check(self._lib.p3m_batch_set_barrier_fault(self._b, poll_limit, withheld_cta, phase))

    def plan_info(self) -> dict:
        """The last fused step's plan: persistent or not, kernel launches per
        step, phases and CTAs of the persistent launch."""
        out = np.zeros(4, np.int32)
        self._check(self._lib.p3m_batch_plan_info(self._b, _ptr(out)))
        return {"persistent": bool(out[0]), "launches": int(out[1]), "phases": int(out[2]),
                "ctas": int(out[3])}

    def phase_times(self) -> list[float]:
        """Device milliseconds of each phase of the last persistent step."""
        out = np.zeros(64, np.float64)
        n = ctypes.c_int32(0)
        self._check(self._lib.p3m_batch_phase_times(self._b, _ptr(out), 64, ctypes.byref(n)))
        return [float(v) for v in out[:n.value]]

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
