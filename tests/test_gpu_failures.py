"""Failure detection on the device, made to happen without faulting the GPU.

* A bulk-copy wait that runs out (FP32 sweep; FP64 TMA-staged tiles, single
  and batched): the limit of the device-side waits is set to one cycle, so
  the first wait of every warp (block) gives up; the kernel flags the step,
  still waits (with the default limit) for the copies it issued, and
  returns.  The step fails with a message naming the wait (a batch: naming a
  member's device error); with the default limit restored the same handle
  steps normally.
* A non-finite state: a NaN put into the momentum through the setter is
  caught by the stage-2 epilogue; the step that produced it completes, the
  rest of the requested steps do not run, and the call fails with a message
  naming the step.  Restoring a finite state makes the handle usable again.
"""
import numpy as np
import pytest

from helpers import gaussian_bed, hump_depth

pytestmark = pytest.mark.gpu

NX, NY, DX = 200, 150, 5.0


def _sim(precision):
    from rakali_b200 import Rakali
    b = gaussian_bed(NX, NY, DX, DX, 8, seed=2, width=(30.0, 150.0))
    h = hump_depth(b, DX, DX, width=80.0)
    s = Rakali(defer_init=True, nx=NX, ny=NY, dx=DX, dy=DX, t_end=1e6, cfl=0.45,
               manning_n=0.025)
    s.set_bathymetry(b)
    s.set_initial_h(h)
    s.finalize()
    s.set_precision(precision)
    return s


@pytest.mark.parametrize("precision,tile", [(32, None), (64, 10)])
def test_expired_bulk_copy_wait_fails_the_step_and_the_handle_recovers(precision, tile):
    with _sim(precision) as s:
        if tile is not None:
            s.set_tile(tile)
            assert s._lib.rkb_tma_tile_status(s._handle) == 0  # the TMA-staged kernel runs
        s.step(2)
        state = [a.copy() for a in (s.h_phys, s.hu_phys, s.hv_phys)]
        lib = s._lib
        assert lib.rkb_set_wait_limit(s._handle, 1) == 0
        with pytest.raises(RuntimeError, match="wait for a bulk copy expired"):
            s.step(3)
        assert lib.rkb_set_wait_limit(s._handle, 0) == 0
        s.set_h(state[0])
        s.set_hu(state[1])
        s.set_hv(state[2])
        n0 = s.step_count
        s.step(3)
        assert s.step_count == n0 + 3
        assert np.all(np.isfinite(s.h_phys))


def test_expired_tma_wait_in_a_batch_fails_the_step_and_the_batch_recovers():
    """The batched TMA-staged kernel: one member's wait limit set to one cycle
    makes its blocks give up; the batch step fails naming a member's device
    error, the other members step normally, and with the limit restored the
    whole batch steps again."""
    from rakali_b200 import workloads as wl
    from rakali_b200.ensemble import Ensemble
    sims = [wl.build_member(m) for m in wl.ensemble_members(n_inst=3, seed=6, size=(40, 120))]
    lib = sims[0]._lib
    with Ensemble(sims) as ens:
        ens.set_variant(10, 0)
        assert all(lib.rkb_tma_tile_status(s._handle) == 0 for s in sims)
        ens.step(2)
        state = [(s.h_phys.copy(), s.hu_phys.copy(), s.hv_phys.copy()) for s in sims]
        n_ok = sims[0].step_count
        assert lib.rkb_set_wait_limit(sims[1]._handle, 1) == 0
        with pytest.raises(RuntimeError, match="device error"):
            ens.step(3)
        assert sims[0].step_count == n_ok + 3  # the others stepped
        assert lib.rkb_set_wait_limit(sims[1]._handle, 0) == 0
        for s, (h, hu, hv) in zip(sims, state):
            s.set_h(h)
            s.set_hu(hu)
            s.set_hv(hv)
        counts = [s.step_count for s in sims]
        ens.step(3)
        assert [s.step_count for s in sims] == [c + 3 for c in counts]
        assert all(np.all(np.isfinite(s.h_phys)) for s in sims)
    for s in sims:
        s.close()


@pytest.mark.parametrize("precision", [64, 32])
def test_nan_in_the_state_is_reported_not_propagated_silently(precision):
    with _sim(precision) as s:
        s.step(2)
        good = [a.copy() for a in (s.h_phys, s.hu_phys, s.hv_phys)]
        wet = np.argwhere(good[0] > 0.5)
        i, j = wet[len(wet) // 2]
        bad_hu = good[1].copy()
        bad_hu[i, j] = np.nan
        s.set_hu(bad_hu)
        n0 = s.step_count
        with pytest.raises(RuntimeError, match="non-finite"):
            s.step(5)
        assert s.step_count == n0 + 1  # the step that met the NaN, none after it
        s.set_h(good[0])
        s.set_hu(good[1])
        s.set_hv(good[2])
        s.step(3)
        assert s.step_count == n0 + 4
        assert np.all(np.isfinite(s.h_phys)) and np.all(np.isfinite(s.hu_phys))
