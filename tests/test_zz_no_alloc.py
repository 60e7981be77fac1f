"""The allocation-free dt entry point against the allocating one (GPU).

rkb_compute_timestep_noalloc exists for callers that cannot allocate device
memory when they need dt - a host application whose memory pool already owns
the GPU, or a loop that must not block on the device-wide synchronisation of
cudaMalloc/cudaFree.  Its scratch is a fixed array compiled into the
library.  This file is collected last so a failure here leaves every other
test already run; it passes alone in a fresh process and after the others.

Checked through the C ABI on two calls in a row with different states (the
shared scratch keeps the previous call's contents), each against
rkb_compute_timestep with the tolerance the other dt tests use (exact), plus
the size limit.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(np.asfortranarray(a).T)).cuda()


def _state(shape, seed, dry_frac):
    rng = np.random.default_rng(seed)
    h = rng.random(shape) * 3.0
    h[rng.random(shape) < dry_frac] = 0.0
    hu = rng.normal(0.0, 1.5, shape)
    hv = rng.normal(0.0, 0.5, shape)
    return [np.asfortranarray(a) for a in (h, hu, hv)]


def _dt(fn, arrays, ng, dx, dy, cfl):
    dev = [_dev(a) for a in arrays]
    out = ctypes.c_double(-1.0)
    nx, ny = arrays[0].shape
    rc = fn(*(t.data_ptr() for t in dev), nx, ny, ng, nx, dx, dy, cfl, ctypes.byref(out))
    return rc, out.value


def test_noalloc_matches_allocating_dt_twice():
    from rakali_b200 import _lib
    lib = _lib.load()
    cases = [((300, 517), 1, 0.2, 3, 5.0, 5.0, 0.45),
             ((64, 40), 2, 0.0, 2, 2.0, 7.0, 0.9)]
    for shape, seed, dry, ng, dx, dy, cfl in cases:
        arrays = _state(shape, seed, dry)
        rc_a, dt_a = _dt(lib.rkb_compute_timestep, arrays, ng, dx, dy, cfl)
        rc_b, dt_b = _dt(lib.rkb_compute_timestep_noalloc, arrays, ng, dx, dy, cfl)
        assert rc_a == 0 and rc_b == 0
        assert dt_b == dt_a  # same reduction, exact


def test_noalloc_rejects_too_many_rows():
    from rakali_b200 import _lib
    lib = _lib.load()
    arrays = [np.zeros((8, 32768 + 2 * 2 + 1), order="F") for _ in range(3)]
    rc, _ = _dt(lib.rkb_compute_timestep_noalloc, arrays, 2, 1.0, 1.0, 0.45)
    assert rc == -2
    assert "exceed" in _lib.last_error(lib)
