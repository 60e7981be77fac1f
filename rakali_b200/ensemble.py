"""Batches of independent simulations advanced together on one GPU.

An ``Ensemble`` groups finalised ``Rakali`` simulations (any sizes, each with
its own boundary parameters, dt and clock) and advances all of them with one
kernel launch per phase, chunks of steps captured in CUDA graphs.  Members
keep working as ordinary simulations: their host views, setters and
properties reflect the batch's steps.
"""
from __future__ import annotations

import ctypes

from . import _lib


class Ensemble:
    """``Ensemble(sims, precision=64)``; ``step``, ``advance``, ``autotune``."""

    def __init__(self, sims, precision: int = 64):
        if precision not in (32, 64):
            raise ValueError(f"precision must be 32 or 64, got {precision!r}")
        self._lib = _lib.load()
        self.members = list(sims)
        if not self.members:
            raise ValueError("an ensemble needs at least one simulation")
        arr = (ctypes.c_void_p * len(self.members))(*[s._handle.value for s in self.members])
        self._b = ctypes.c_void_p()
        rc = self._lib.rkb_batch_create(arr, len(self.members), int(precision),
                                        ctypes.byref(self._b))
        if rc != 0:
            raise RuntimeError(f"ensemble creation failed (rc={rc}): {_lib.last_error(self._lib)}")
        self.precision = precision

    def _rc(self, rc, what):
        if rc != 0:
            raise RuntimeError(f"{what} failed (rc={rc}): {_lib.last_error(self._lib)}")

    def _check(self):
        if not self._b:
            raise RuntimeError("ensemble is closed")

    def step(self, n: int = 1):
        self._check()
        self._rc(self._lib.rkb_batch_step(self._b, int(n)), "step")

    def advance(self, target_time: float):
        """Every member to ``target_time`` (each with its own CFL steps)."""
        self._check()
        self._rc(self._lib.rkb_batch_advance(self._b, float(target_time)), "advance")

    def time_steps(self, n: int) -> float:
        """Device milliseconds of ``n`` steps of every member (CUDA events)."""
        self._check()
        ms = ctypes.c_double()
        self._rc(self._lib.rkb_batch_time_steps(self._b, int(n), ctypes.byref(ms)), "time_steps")
        return ms.value

    def profile_steps(self, n: int) -> dict:
        """Mean device ms per step of each launch phase over ``n`` steps issued
        launch by launch (boundary fills and stages of every member), and of
        the whole sequence."""
        self._check()
        out = (ctypes.c_double * 5)()
        self._rc(self._lib.rkb_batch_profile_steps(self._b, int(n), out), "profile_steps")
        return {"bc_stage1": out[0], "stage1": out[1], "bc_stage2": out[2], "stage2": out[3],
                "launch_by_launch": out[4]}

    def autotune(self, trial_steps: int = 3) -> float:
        """Pick the fastest kernel shape on the live state (restored); ms per step."""
        self._check()
        ms = ctypes.c_double()
        self._rc(self._lib.rkb_batch_autotune(self._b, int(trial_steps), ctypes.byref(ms)),
                 "autotune")
        return ms.value

    def set_variant(self, a: int, b: int = 0):
        """Set the kernel shape without trials: FP64 (tile, 0), tiles 0-3 and
        6-10 (10: TMA-staged 16x15); FP32 (2 or 4 columns per lane, rows)."""
        self._check()
        self._rc(self._lib.rkb_batch_set_variant(self._b, int(a), int(b)), "set_variant")

    @property
    def variant(self):
        """FP64: (tile, 0); FP32: (columns per lane, rows per warp sweep)."""
        self._check()
        a, b = ctypes.c_int(), ctypes.c_int()
        self._rc(self._lib.rkb_batch_variant(self._b, ctypes.byref(a), ctypes.byref(b)), "variant")
        return a.value, b.value

    @property
    def cells(self) -> int:
        return sum(s.nx * s.ny for s in self.members)

    def close(self):
        if getattr(self, "_b", None):
            self._lib.rkb_batch_destroy(ctypes.byref(self._b))
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


__all__ = ["Ensemble"]
