"""Batching form: many solver states stepped by one persistent launch.

Members are Solver objects (ADR, same precision form). Each keeps its own
state, step number and damping coefficient, and computes exactly what a solo
launch computes; the batch shares the SMs among them (one work counter over
all members' node slices) and replays its launch from a captured CUDA graph
while the membership and launch length stay the same. Members may join and
leave between launches (continuous batching).
"""
from __future__ import annotations

import ctypes as C

from . import _native as N
from .solver import Solver


class Batch:
    def __init__(self, precision: str = "fp64", device: int = 0):
        self.precision = precision
        self.device = device
        h = C.c_void_p()
        prec = {"fp64": N.PREC_FP64, "fp32": N.PREC_FP32}[precision]
        N.check(N.lib().bbpd_batch_create(device, prec, C.byref(h)))
        self._h = h
        self.members: list[Solver] = []

    def add(self, s: Solver) -> None:
        N.check(N.lib().bbpd_batch_add(self._h, s.handle))
        self.members.append(s)

    def remove(self, s: Solver) -> None:
        N.check(N.lib().bbpd_batch_remove(self._h, s.handle))
        self.members.remove(s)

    def step(self, nsteps: int) -> None:
        N.check(N.lib().bbpd_batch_step(self._h, nsteps))

    def tune(self, nsteps_per_trial: int = 4) -> tuple[int, int]:
        """Autotune the schedule on real steps; returns (blocks per SM, slices per grab)."""
        b, g = C.c_int(), C.c_int()
        N.check(N.lib().bbpd_batch_tune(self._h, nsteps_per_trial, C.byref(b), C.byref(g)))
        return int(b.value), int(g.value)

    def set_schedule(self, blocks_per_sm: int, grab: int = 1, use_graph: bool = True) -> None:
        N.check(N.lib().bbpd_batch_set_schedule(self._h, blocks_per_sm, grab, int(use_graph)))

    def set_mixing(self, mixed: bool) -> None:
        """True: all laws in one launch per kernel variant; False (the default
        until tune() or this call chooses): one specialised launch per law and
        critical-stretch form."""
        N.check(N.lib().bbpd_batch_set_mixing(self._h, int(mixed)))

    def info(self) -> dict:
        i = N.BatchInfo()
        N.check(N.lib().bbpd_batch_get_info(self._h, C.byref(i)))
        return {f: getattr(i, f) for f, _ in N.BatchInfo._fields_}

    def last_kernel_ms(self) -> float:
        ms = C.c_float()
        N.check(N.lib().bbpd_batch_last_kernel_ms(self._h, C.byref(ms)))
        return float(ms.value)

    def close(self) -> None:
        if getattr(self, "_h", None):
            N.lib().bbpd_batch_destroy(self._h)
            self._h = None
            self.members = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
