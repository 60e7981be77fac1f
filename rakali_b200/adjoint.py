"""Gradients of a gauge misfit with respect to the bed and the Manning-n field.

``GaugeMisfit`` wraps the hand-written adjoint of the FP64 step in
librakali.so (rkb_adjoint_*): J = sum over steps 1..N and gauge cells of
(eta - eta_obs)^2, eta = h + b, for the SSP-RK2 step with wall boundaries,
HLL or HLLC fluxes and Manning friction with a per-cell n field, on a fixed dt
sequence (``record_dt`` takes CFL steps once and stores them; every later run
replays them, so J is a piecewise-smooth function of b and n).  The adjoint
uses sqrt(N)-step checkpointing with recompute.

``GaugeMisfitBatch`` advances many equally sized problems in the same
launches, in FP64 or FP32 (FP32 arithmetic, FP64 misfit and mass sums).

``misfit(problem, b, n)`` is the ``torch.autograd.Function`` front end: it
returns J as a 0-d float64 tensor and back-propagates dJ/db, dJ/dn.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

_DP = ctypes.POINTER(ctypes.c_double)
_IP = ctypes.POINTER(ctypes.c_int)


def _f(a, shape):
    a = np.asfortranarray(np.asarray(a, dtype=np.float64))
    if a.shape != shape:
        raise ValueError(f"expected shape {shape}, got {a.shape}")
    return a


class GaugeMisfit:
    """The misfit problem: initial state, gauges, observations, dt sequence."""

    def __init__(self, nx, ny, dx, dy, h0, gauges, n_steps, hu0=None, hv0=None, nghost=2,
                 cfl=0.45, use_hllc=False):
        self._lib = _lib.load()
        self.nx, self.ny, self.n_steps = int(nx), int(ny), int(n_steps)
        shape = (self.nx, self.ny)
        h0 = _f(h0, shape)
        hu0 = _f(np.zeros(shape) if hu0 is None else hu0, shape)
        hv0 = _f(np.zeros(shape) if hv0 is None else hv0, shape)
        gi = np.ascontiguousarray([int(g[0]) for g in gauges], dtype=np.int32)
        gj = np.ascontiguousarray([int(g[1]) for g in gauges], dtype=np.int32)
        self.n_gauges = len(gi)
        self._a = ctypes.c_void_p()
        rc = self._lib.rkb_adjoint_create(self.nx, self.ny, int(nghost), float(dx), float(dy),
                                          float(cfl), int(bool(use_hllc)), self.n_steps,
                                          h0.ctypes.data_as(_DP), hu0.ctypes.data_as(_DP),
                                          hv0.ctypes.data_as(_DP), gi.ctypes.data_as(_IP),
                                          gj.ctypes.data_as(_IP), self.n_gauges,
                                          ctypes.byref(self._a))
        if rc != 0:
            raise RuntimeError(f"adjoint setup failed (rc={rc}): {_lib.last_error(self._lib)}")
        self.set_observations(np.zeros((self.n_steps, self.n_gauges)))

    def _rc(self, rc, what):
        if rc != 0:
            raise RuntimeError(f"{what} failed (rc={rc}): {_lib.last_error(self._lib)}")

    def _fields(self, b, n):
        shape = (self.nx, self.ny)
        b = _f(b, shape)
        if n is None or np.ndim(n) == 0:
            return b, None, float(0.0 if n is None else n)
        return b, _f(n, shape), 0.0

    def set_observations(self, obs):
        obs = np.ascontiguousarray(obs, dtype=np.float64)
        if obs.shape != (self.n_steps, self.n_gauges):
            raise ValueError(f"observations must be ({self.n_steps}, {self.n_gauges})")
        self._rc(self._lib.rkb_adjoint_set_obs(self._a, obs.ctypes.data_as(_DP)), "set_observations")

    @property
    def dt(self):
        out = np.zeros(self.n_steps)
        self._rc(self._lib.rkb_adjoint_get_dt(self._a, out.ctypes.data_as(_DP)), "dt")
        return out

    def set_dt(self, dts):
        dts = np.ascontiguousarray(dts, dtype=np.float64)
        if dts.shape != (self.n_steps,):
            raise ValueError(f"dt must have {self.n_steps} entries")
        self._rc(self._lib.rkb_adjoint_set_dt(self._a, dts.ctypes.data_as(_DP)), "set_dt")

    def _forward(self, b, n, record):
        b, nf, ns = self._fields(b, n)
        J = ctypes.c_double()
        eta = np.zeros((self.n_steps, self.n_gauges))
        self._rc(self._lib.rkb_adjoint_forward(
            self._a, b.ctypes.data_as(_DP), nf.ctypes.data_as(_DP) if nf is not None else None, ns,
            int(record), ctypes.byref(J), eta.ctypes.data_as(_DP)), "forward")
        return J.value, eta

    def record_dt(self, b, n=None):
        """Forward run with CFL steps; stores the dt sequence; returns (J, eta_gauges)."""
        return self._forward(b, n, True)

    def forward(self, b, n=None):
        """(J, eta_gauges (n_steps, n_gauges)) on the stored dt sequence."""
        return self._forward(b, n, False)

    def gradient(self, b, n=None):
        """(J, dJ/db, dJ/dn), the gradients as (nx, ny) arrays."""
        b, nf, ns = self._fields(b, n)
        J = ctypes.c_double()
        gb = np.zeros((self.nx, self.ny), order="F")
        gn = np.zeros((self.nx, self.ny), order="F")
        self._rc(self._lib.rkb_adjoint_gradient(
            self._a, b.ctypes.data_as(_DP), nf.ctypes.data_as(_DP) if nf is not None else None, ns,
            ctypes.byref(J), gb.ctypes.data_as(_DP), gn.ctypes.data_as(_DP)), "gradient")
        return J.value, gb, gn

    def set_frozen_slopes(self, on=True):
        """Hold the limited slopes fixed in later gradients (bounded over long
        windows; not the exact derivative of the limiter)."""
        self._rc(self._lib.rkb_adjoint_set_frozen_slopes(self._a, int(bool(on))), "set_frozen_slopes")

    @property
    def checkpoint_interval(self):
        """1 once a gradient run kept every state in device memory, else the
        sqrt(n_steps) checkpoint interval."""
        return int(self._lib.rkb_adjoint_checkpoint_interval(self._a))

    def set_state_budget(self, nbytes):
        """Device bytes a gradient run may allocate to keep every state instead
        of recomputing them from sqrt(n_steps) checkpoints: 0 (the default)
        never, None half the free device memory.  The gradients are the same
        bits either way."""
        self._rc(self._lib.rkb_adjoint_set_state_budget(self._a, -1 if nbytes is None else int(nbytes)),
                 "set_state_budget")

    @property
    def last_ms(self) -> float:
        """Device milliseconds of the last forward / gradient call."""
        return float(self._lib.rkb_adjoint_last_ms(self._a))

    def close(self):
        if getattr(self, "_a", None):
            self._lib.rkb_adjoint_destroy(ctypes.byref(self._a))
            self._a = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _stack(a, nm, nx, ny):
    """(n_members, nx, ny) -> contiguous float64 buffer, each member Fortran-ordered."""
    a = np.asarray(a, dtype=np.float64)
    if a.shape != (nm, nx, ny):
        raise ValueError(f"expected shape {(nm, nx, ny)}, got {a.shape}")
    return np.ascontiguousarray(np.stack([a[m].ravel(order="F") for m in range(nm)]))


def _unstack(buf, nm, nx, ny):
    return np.stack([buf[m].reshape((nx, ny), order="F") for m in range(nm)])


class GaugeMisfitBatch:
    """n_members equally sized misfit problems advanced together, FP64 or FP32.

    Every kernel launch covers all members; each member has its own initial
    state, gauges, observations, dt sequence, bed and n field.  precision=32
    runs the forward and the adjoint in FP32 arithmetic with the misfit and
    the domain mass summed in FP64.  Arrays: h0, b, n and the gradients are
    (n_members, nx, ny); gauges is a list (one per member) of n_gauges (i, j)
    interior cells; observations and gauge surfaces are
    (n_steps, n_members, n_gauges); dt is (n_members, n_steps).
    """

    def __init__(self, n_members, nx, ny, dx, dy, h0, gauges, n_steps, precision=32, hu0=None,
                 hv0=None, nghost=2, cfl=0.45, use_hllc=False):
        self._lib = _lib.load()
        self.nm, self.nx, self.ny, self.n_steps = int(n_members), int(nx), int(ny), int(n_steps)
        dims = (self.nm, self.nx, self.ny)
        h0 = _stack(h0, *dims)
        hu0 = None if hu0 is None else _stack(hu0, *dims)
        hv0 = None if hv0 is None else _stack(hv0, *dims)
        if len(gauges) != self.nm:
            raise ValueError("one gauge list per member")
        self.n_gauges = len(gauges[0])
        if any(len(gl) != self.n_gauges for gl in gauges):
            raise ValueError("every member needs the same number of gauges")
        gi = np.ascontiguousarray([int(g[0]) for gl in gauges for g in gl], dtype=np.int32)
        gj = np.ascontiguousarray([int(g[1]) for gl in gauges for g in gl], dtype=np.int32)
        self._a = ctypes.c_void_p()
        nul = ctypes.POINTER(ctypes.c_double)()
        rc = self._lib.rkb_adjoint_batch_create(
            int(precision), self.nm, self.nx, self.ny, int(nghost), float(dx), float(dy),
            float(cfl), int(bool(use_hllc)), self.n_steps, h0.ctypes.data_as(_DP),
            hu0.ctypes.data_as(_DP) if hu0 is not None else nul,
            hv0.ctypes.data_as(_DP) if hv0 is not None else nul,
            gi.ctypes.data_as(_IP), gj.ctypes.data_as(_IP), self.n_gauges, ctypes.byref(self._a))
        if rc != 0:
            raise RuntimeError(f"adjoint setup failed (rc={rc}): {_lib.last_error(self._lib)}")
        self.precision = int(self._lib.rkb_adjoint_precision(self._a))
        self.set_observations(np.zeros((self.n_steps, self.nm, self.n_gauges)))

    def _rc(self, rc, what):
        if rc != 0:
            raise RuntimeError(f"{what} failed (rc={rc}): {_lib.last_error(self._lib)}")

    def _fields(self, b, n):
        dims = (self.nm, self.nx, self.ny)
        b = _stack(b, *dims)
        if n is None or np.ndim(n) == 0:
            return b, None, float(0.0 if n is None else n)
        return b, _stack(n, *dims), 0.0

    def set_observations(self, obs):
        obs = np.ascontiguousarray(obs, dtype=np.float64)
        if obs.shape != (self.n_steps, self.nm, self.n_gauges):
            raise ValueError(f"observations must be {(self.n_steps, self.nm, self.n_gauges)}")
        self._rc(self._lib.rkb_adjoint_set_obs(self._a, obs.ctypes.data_as(_DP)), "set_observations")

    @property
    def dt(self):
        out = np.zeros((self.nm, self.n_steps))
        self._rc(self._lib.rkb_adjoint_get_dt(self._a, out.ctypes.data_as(_DP)), "dt")
        return out

    def set_dt(self, dts):
        dts = np.ascontiguousarray(dts, dtype=np.float64)
        if dts.shape != (self.nm, self.n_steps):
            raise ValueError(f"dt must be {(self.nm, self.n_steps)}")
        self._rc(self._lib.rkb_adjoint_set_dt(self._a, dts.ctypes.data_as(_DP)), "set_dt")

    def _forward(self, b, n, record):
        b, nf, ns = self._fields(b, n)
        J = np.zeros(self.nm)
        eta = np.zeros((self.n_steps, self.nm, self.n_gauges))
        self._rc(self._lib.rkb_adjoint_forward(
            self._a, b.ctypes.data_as(_DP), nf.ctypes.data_as(_DP) if nf is not None else None, ns,
            int(record), J.ctypes.data_as(_DP), eta.ctypes.data_as(_DP)), "forward")
        return J, eta

    def record_dt(self, b, n=None):
        """Forward run with CFL steps; stores the dt sequences; returns (J, eta_gauges)."""
        return self._forward(b, n, True)

    def forward(self, b, n=None):
        """(J (n_members,), eta_gauges) on the stored dt sequences."""
        return self._forward(b, n, False)

    def gradient(self, b, n=None):
        """(J, dJ/db, dJ/dn), the gradients as (n_members, nx, ny) arrays."""
        b, nf, ns = self._fields(b, n)
        J = np.zeros(self.nm)
        gb = np.zeros((self.nm, self.nx * self.ny))
        gn = np.zeros((self.nm, self.nx * self.ny))
        self._rc(self._lib.rkb_adjoint_gradient(
            self._a, b.ctypes.data_as(_DP), nf.ctypes.data_as(_DP) if nf is not None else None, ns,
            J.ctypes.data_as(_DP), gb.ctypes.data_as(_DP), gn.ctypes.data_as(_DP)), "gradient")
        dims = (self.nm, self.nx, self.ny)
        return J, _unstack(gb, *dims), _unstack(gn, *dims)

    @property
    def mass(self):
        """FP64 interior sum(h) per member: row 0 before, row 1 after the last forward run."""
        out = np.zeros((2, self.nm))
        self._rc(self._lib.rkb_adjoint_mass(self._a, out.ctypes.data_as(_DP)), "mass")
        return out

    def set_frozen_slopes(self, on=True):
        """Hold the limited slopes fixed in later gradients (bounded over long
        windows; not the exact derivative of the limiter)."""
        self._rc(self._lib.rkb_adjoint_set_frozen_slopes(self._a, int(bool(on))), "set_frozen_slopes")

    @property
    def checkpoint_interval(self):
        """1 once a gradient run kept every state in device memory, else the
        sqrt(n_steps) checkpoint interval."""
        return int(self._lib.rkb_adjoint_checkpoint_interval(self._a))

    def set_state_budget(self, nbytes):
        """Device bytes a gradient run may allocate to keep every state instead
        of recomputing them from sqrt(n_steps) checkpoints: 0 (the default)
        never, None half the free device memory.  The gradients are the same
        bits either way."""
        self._rc(self._lib.rkb_adjoint_set_state_budget(self._a, -1 if nbytes is None else int(nbytes)),
                 "set_state_budget")

    @property
    def last_ms(self) -> float:
        """Device milliseconds of the last forward / gradient call."""
        return float(self._lib.rkb_adjoint_last_ms(self._a))

    def close(self):
        if getattr(self, "_a", None):
            self._lib.rkb_adjoint_destroy(ctypes.byref(self._a))
            self._a = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _function():
    import torch

    class _Misfit(torch.autograd.Function):
        @staticmethod
        def forward(ctx, b, n, problem):
            bn = b.detach().to("cpu", torch.float64).numpy()
            nn = n.detach().to("cpu", torch.float64).numpy()
            if ctx.needs_input_grad[0] or ctx.needs_input_grad[1]:
                J, gb, gn = problem.gradient(bn, nn)
                ctx.save_for_backward(torch.from_numpy(np.ascontiguousarray(gb)).to(b.device),
                                      torch.from_numpy(np.ascontiguousarray(gn)).to(n.device))
            else:
                J, _ = problem.forward(bn, nn)
            return torch.tensor(J, dtype=torch.float64, device=b.device)

        @staticmethod
        def backward(ctx, gJ):
            gb, gn = ctx.saved_tensors
            return gJ * gb, gJ * gn, None

    return _Misfit


_MISFIT = None


def misfit(problem: GaugeMisfit, b, n):
    """J(b, n) as a differentiable float64 tensor (b, n: (nx, ny) tensors)."""
    global _MISFIT
    if _MISFIT is None:
        _MISFIT = _function()
    return _MISFIT.apply(b, n, problem)


__all__ = ["GaugeMisfit", "GaugeMisfitBatch", "misfit"]
