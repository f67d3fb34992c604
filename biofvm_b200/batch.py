"""Many independent microenvironments advanced together, over the C ABI
(``bfvm_batch_*`` in include/bfvm.h).

``Batch.step(dt, n, flags)`` has the effect of ``Solver.step(dt, n, flags)``
on every member; the members are packed into L2-sized groups and the whole
run is one CUDA-graph replay: one launch per phase over a group
(``BATCH_FUSED``), every member's own kernels on concurrent graph branches
(``BATCH_BRANCHES``), or all steps of a group's members in one persistent
cooperative launch (``BATCH_PERSISTENT``: x, y, z phases of chunked line
tiles; ``BATCH_PLANES``: xy planes and xz strips staged in shared memory, two
phases per step).  The reference has no such object: its drivers loop over
Microenvironment instances one by one.
"""
from __future__ import annotations

import ctypes

from . import _abi
from ._abi import call
from .solver import Solver


class Batch:
    def __init__(self, device: int = 0):
        _abi.load_library()
        h = ctypes.c_void_p()
        call("bfvm_batch_create", ctypes.byref(h), device)
        self._h = h
        self.members: list[Solver] = []

    def close(self) -> None:
        if self._h is not None:
            call("bfvm_batch_destroy", self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, sv: Solver) -> None:
        call("bfvm_batch_add", self._h, sv.handle)
        self.members.append(sv)  # keeps the member alive while it is in the batch

    def clear(self) -> None:
        call("bfvm_batch_clear", self._h)
        self.members.clear()

    def __len__(self) -> int:
        n = ctypes.c_int()
        call("bfvm_batch_size", self._h, ctypes.byref(n))
        return n.value

    def step(self, dt: float, nsteps: int = 1, flags: int = _abi.STEP_ALL) -> None:
        call("bfvm_batch_step", self._h, dt, nsteps, flags)

    def tune(self, dt: float, flags: int = _abi.STEP_ALL, trial_steps: int = 5) -> None:
        call("bfvm_batch_tune", self._h, dt, flags, trial_steps)

    def set_config(self, chunk=(0, 0, 0), threads=(0, 0, 0), group_bytes: int = -1) -> None:
        ch = (ctypes.c_int * 3)(*chunk)
        th = (ctypes.c_int * 3)(*threads)
        call("bfvm_batch_set_config", self._h, ch, th, group_bytes)

    def get_config(self):
        ch = (ctypes.c_int * 3)()
        th = (ctypes.c_int * 3)()
        gb = ctypes.c_int64()
        call("bfvm_batch_get_config", self._h, ch, th, ctypes.byref(gb))
        return tuple(ch), tuple(th), gb.value

    def set_mode(self, mode: int) -> None:
        """BATCH_FUSED (one launch per phase over a group's members),
        BATCH_BRANCHES (every member's own kernels on concurrent graph
        branches), BATCH_PERSISTENT (all steps of a group's members in one
        persistent cooperative launch, x, y and z phases) or BATCH_PLANES
        (the same launch with two phases per step: xy planes solved along x
        and y in shared memory, then xz strips along z)."""
        call("bfvm_batch_set_mode", self._h, mode)

    def set_persistent_chunk(self, chunk: int) -> None:
        """Work split of the persistent kernel: 8 or 16 points per chunk
        (chunks folded across a block), 32 (tiles of 32 columns with the
        sweep kernels' chunk tables), or 0 (one thread per (line, density)
        column solving the whole line)."""
        call("bfvm_batch_set_persistent_chunk", self._h, chunk)

    def get_persistent_chunk(self) -> int:
        c = ctypes.c_int()
        call("bfvm_batch_get_persistent_chunk", self._h, ctypes.byref(c))
        return c.value

    def get_mode(self) -> int:
        m = ctypes.c_int()
        call("bfvm_batch_get_mode", self._h, ctypes.byref(m))
        return m.value

    def plan(self):
        """(groups of the last plan, kernel launches per step() call)."""
        g = ctypes.c_int()
        k = ctypes.c_int64()
        call("bfvm_batch_get_plan", self._h, ctypes.byref(g), ctypes.byref(k))
        return g.value, k.value

    def synchronize(self) -> None:
        call("bfvm_batch_synchronize", self._h)
