"""The headline single-instance workload at its full size (4096 x 4096).

The wet/dry benchmark configuration itself - dx = dy = 5 m, a bed of 32 seeded
Gaussians (amplitudes U[-4, 12] m, widths U[50, 500] m) with emergent
islands, a 0.5 m / 200 m hump at the centre, Manning n = 0.025, walls - is
checked here at 4096^2, not only the smaller grids of the other parity tests:

* the FP64 step against the oracle for 20 steps, bit-identical, ghosts
  included (the oracle runs on every host core: ~15 s);
* the lake-at-rest variant (the same bed, no hump) for 1000 steps: |eta| <=
  1e-13 m in FP64, and |hu|, |hv| within round-off of the natural momentum
  scale, 1e-12 H sqrt(g H) with H the deepest water (the bound of the
  reference's tests/test_c_property.F90:97-104); exactly stationary in the
  FP32 surface form;
* the domain volume over 1000 steps with the hump: closed walls, so it is
  conserved to round-off (1e-12 relative in FP64; FP32 state with FP64 sums:
  1e-6 relative, the FP32 surface's own rounding).
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 4096


def _sim(b, h, precision=64):
    from rakali_b200 import Rakali
    from rakali_b200 import workloads as wl
    s = Rakali(defer_init=True, nx=N, ny=N, **wl.CONFIG2_KW)
    s.set_bathymetry(b)
    s.set_initial_h(h)
    s.finalize()
    s.set_precision(precision)
    return s


@pytest.fixture(scope="module")
def config2():
    from rakali_b200 import workloads as wl
    return wl.config2(n=N, seed=2024)


def test_fp64_step_matches_oracle_at_4096(config2):
    from oracle import oracle as orc
    from rakali_b200 import workloads as wl
    b, h = config2
    orc.set_threads(os.cpu_count() or 1)
    o = orc.OracleSim.from_config(dict(nx=N, ny=N, **wl.CONFIG2_KW), bathymetry=b, initial_h=h)
    o.step(20)
    with _sim(b, h) as s:
        s.step(20)
        assert s.step_count == o.step_count == 20
        assert s.time == o.time and s.dt == o.dt
        for name in ("h", "hu", "hv", "b"):
            got = getattr(s, name)
            want = o.arrays[name]
            assert np.array_equal(got, want), \
                (name, float(np.max(np.abs(got - want))), int(np.sum(got != want)))


@pytest.mark.parametrize("precision", [64, 32])
def test_lake_at_rest_4096_1000_steps(precision):
    from rakali_b200 import workloads as wl
    b, h = wl.config2(n=N, seed=2024, hump=False)
    assert (h == 0).any() and (h > 0).any()  # emergent islands: dry cells inside the domain
    with _sim(b, h, precision) as s:
        s.step(1000)
        eta = s.h_phys + b
        wet = s.h_phys > 0
        eta_max = float(np.abs(eta[wet]).max())
        mom = max(float(np.abs(s.hu_phys).max()), float(np.abs(s.hv_phys).max()))
        if precision == 64:
            assert eta_max <= 1e-13, eta_max
            H = float(h.max())
            assert mom <= 1e-12 * H * np.sqrt(9.80665 * H), mom
        else:
            # the surface form is exactly stationary: depths read back as
            # eta - b with eta = 0 on every wet cell
            assert np.array_equal(s.h_phys, h)
            assert mom == 0.0


@pytest.mark.parametrize("precision,tol", [(64, 1e-12), (32, 1e-6)])
def test_domain_volume_4096_1000_steps(config2, precision, tol):
    b, h = config2
    with _sim(b, h, precision) as s:
        v0 = float(np.sum(s.h_phys))
        s.step(1000)
        v1 = float(np.sum(s.h_phys))
        out, src = s.mass_budget()
        assert out == 0.0 or abs(out) <= 1e-9 * v0 * 25.0  # walls: nothing leaves
        assert abs(v1 - v0) / v0 <= tol, (v0, v1, (v1 - v0) / v0)
        assert float(np.abs(s.h_phys - h).max()) > 1e-3  # the hump moved
