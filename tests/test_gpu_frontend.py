"""The B200 front end's chunked advance with a callback (python/rakali/_core.py
:945-1035 is the reference's: advance to each interval boundary, refresh the
host state, call back).

The callback fires once per interval with the host views refreshed, and the
run equals the oracle advancing to the same interval boundaries: the state
seen inside every callback and the final state are bit-identical to the
oracle's at those times.
"""
import numpy as np
import pytest

from helpers import gaussian_bed, hump_depth, pair

pytestmark = pytest.mark.gpu


def test_callback_fires_at_interval_with_the_state_of_that_time():
    nx, ny, dx = 80, 64, 5.0
    b = gaussian_bed(nx, ny, dx, dx, 6, seed=5, width=(30.0, 100.0))
    h = hump_depth(b, dx, dx, width=60.0)
    cfg = dict(nx=nx, ny=ny, dx=dx, dy=dx, t_end=1e6, cfl=0.45, manning_n=0.025, use_hllc=True)
    sim, orc = pair(cfg, bathymetry=b, initial_h=h)
    seen = []

    def cb(s):
        seen.append((s.time, s.step_count, s.h_phys.copy(), s.hu_phys.copy()))

    with sim:
        sim.advance(20.0, callback=cb, callback_interval=5.0)
        assert [round(t, 9) for t, *_ in seen] == [5.0, 10.0, 15.0, 20.0]
        assert all(b_[1] > a_[1] for a_, b_ in zip(seen, seen[1:]))
        for t, n, hh, hu in seen:
            orc.advance(t)
            assert orc.step_count == n
            assert np.array_equal(hh, orc.interior("h")) and np.array_equal(hu, orc.interior("hu"))
        assert sim.time == orc.time
        assert np.array_equal(sim.h, orc.arrays["h"])


def test_default_interval_is_a_tenth_of_the_span():
    cfg = dict(nx=32, ny=16, dx=10.0, dy=10.0, t_end=1e6, cfl=0.45, init_condition="dam_break")
    from rakali_b200 import Rakali
    times = []
    with Rakali(**cfg) as sim:
        sim.advance(10.0, callback=lambda s: times.append(s.time))
        assert len(times) == 10 and abs(times[-1] - 10.0) < 1e-9
        with pytest.raises(ValueError):
            sim.advance(20.0, callback=lambda s: None, callback_interval=-1.0)
