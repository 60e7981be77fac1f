"""Batched ensembles (GPU): members of uneven sizes advanced by one launch per phase.

A batch runs the same stage code as a single simulation, so each member's
state after batched steps must be bit-identical to the same member stepped
alone (FP64 and FP32 forms), and the FP64 batch bit-identical to the oracle.
Autotuning runs trial steps on the live state and must leave it exactly as
it found it.
"""
import numpy as np
import pytest

from rakali_b200 import workloads as wl
from rakali_b200.ensemble import Ensemble

pytestmark = pytest.mark.gpu


def _members(n, seed, size=(40, 200)):
    return wl.ensemble_members(n_inst=n, seed=seed, size=size)


def _state(s):
    return (s.h_phys.copy(), s.hu_phys.copy(), s.hv_phys.copy(), s.time, s.step_count, s.dt)


def _assert_same(a, b):
    for x, y in zip(a, b):
        if isinstance(x, np.ndarray):
            assert np.array_equal(x, y)
        else:
            assert x == y


@pytest.mark.parametrize("precision", [64, 32])
def test_batch_matches_members_stepped_alone(precision):
    ms = _members(6, seed=3)
    alone = [wl.build_member(m, precision) for m in ms]
    for s in alone:
        s.step(30)
    ref = [_state(s) for s in alone]
    for s in alone:
        s.close()
    sims = [wl.build_member(m, precision) for m in ms]
    with Ensemble(sims, precision=precision) as ens:
        ens.step(30)
        for s, r in zip(sims, ref):
            _assert_same(_state(s), r)
    for s in sims:
        s.close()


def test_fp32_batch_mixes_plain_and_forced_members():
    """One member with wind and rain, the others without: the batch runs the
    sweep with forcing terms for all, and every member still matches its own
    single run bit for bit (the single runs use the plain build where they can)."""
    ms = _members(4, seed=5)
    rng = np.random.default_rng(8)
    nx, ny = ms[1]["b"].shape
    wx = rng.uniform(0.0, 0.2, (nx, ny))
    wy = rng.uniform(-0.1, 0.1, (nx, ny))
    rain = np.full((nx, ny), 1.0e-5)

    def build():
        sims = [wl.build_member(mm, 32) for mm in ms]
        sims[1].set_wind(wx, wy)
        sims[1].set_precipitation(rain)
        return sims

    alone = build()
    for s in alone:
        s.step(25)
    ref = [_state(s) for s in alone]
    for s in alone:
        s.close()
    sims = build()
    with Ensemble(sims, precision=32) as ens:
        ens.step(25)
        for k, (s, r) in enumerate(zip(sims, ref)):
            got = _state(s)
            diff = [float(np.abs(x - y).max()) for x, y in zip(got[:3], r[:3])]
            assert got[3:] == r[3:], (k, got[3:], r[3:])
            assert max(diff) == 0.0, (k, diff)
    for s in sims:
        s.close()


@pytest.mark.parametrize("tile", [1, 10])
def test_fp64_batch_matches_oracle(tile):
    """Tile 1 (32x16) and tile 10 (16x15, TMA-loaded through each member's own
    tensor maps)."""
    from oracle.oracle import OracleSim
    ms = _members(3, seed=11)
    sims = [wl.build_member(m) for m in ms]
    with Ensemble(sims) as ens:
        ens.set_variant(tile, 0)
        assert ens.variant == (tile, 0)
        ens.step(25)
        for m, s in zip(ms, sims):
            o = OracleSim.from_config(m["kw"], bathymetry=m["b"], initial_h=m["h"])
            o.set_tidal_constituents(*m["tide"])
            o.step(25)
            assert np.array_equal(s.h_phys, o.interior("h"))
            assert np.array_equal(s.hu_phys, o.interior("hu"))
            assert s.time == o.time
    for s in sims:
        s.close()


def test_batch_advance_each_member_own_dt():
    ms = _members(5, seed=5)
    sims = [wl.build_member(m) for m in ms]
    with Ensemble(sims) as ens:
        ens.advance(120.0)
        counts = [s.step_count for s in sims]
        for s in sims:
            assert abs(s.time - 120.0) < 1e-9
    assert len(set(counts)) > 1  # members took different numbers of steps
    alone = wl.build_member(ms[0])
    alone.advance(120.0)
    _assert_same(_state(alone), _state(sims[0]))
    alone.close()
    for s in sims:
        s.close()


@pytest.mark.parametrize("precision", [64, 32])
def test_autotune_leaves_state_unchanged(precision):
    ms = _members(4, seed=9)
    ref_sims = [wl.build_member(m, precision) for m in ms]
    with Ensemble(ref_sims, precision=precision) as ens:
        ens.step(10)
        ref = [_state(s) for s in ref_sims]
    sims = [wl.build_member(m, precision) for m in ms]
    with Ensemble(sims, precision=precision) as ens:
        ens.step(4)
        best = ens.autotune(trial_steps=2)
        assert best > 0.0
        ens.step(6)
        for s, r in zip(sims, ref):
            _assert_same(_state(s), r)
        a, b = ens.variant
        assert (a in (0, 1, 2, 3, 6, 7, 8, 9, 10)) if precision == 64 else (a in (2, 4))
    for s in ref_sims + sims:
        s.close()


def test_set_variant_checks_the_shape():
    sims = [wl.build_member(m) for m in _members(2, seed=4)]
    with Ensemble(sims) as ens:
        for a, b in ((4, 0), (11, 0), (1, 3), (-1, 0)):
            with pytest.raises(RuntimeError, match="variant"):
                ens.set_variant(a, b)
        ens.set_variant(8, 0)
        ens.step(2)
    sims32 = [wl.build_member(m, 32) for m in _members(2, seed=4)]
    with Ensemble(sims32, precision=32) as ens:
        with pytest.raises(RuntimeError, match="variant"):
            ens.set_variant(3, 0)
        ens.set_variant(4, 16)
        assert ens.variant == (4, 16)
        ens.step(2)
    for s in sims + sims32:
        s.close()


def test_batch_rejects_bad_members():
    ms = _members(2, seed=1)
    a = wl.build_member(ms[0])
    b = wl.build_member(dict(ms[1], kw=dict(ms[1]["kw"], use_hllc=True)))
    with pytest.raises(RuntimeError, match="Riemann"):
        Ensemble([a, b])
    c = wl.build_member(ms[1])
    ens = Ensemble([a, c])
    with pytest.raises(RuntimeError, match="one batch"):
        Ensemble([a])
    c.close()  # destroying a member disables the batch
    with pytest.raises(RuntimeError, match="destroyed"):
        ens.step(1)
    ens.close()
    a.close()
    b.close()


@pytest.mark.parametrize("precision", [64, 32])
def test_batch_records_member_gauges(precision):
    """A member's gauge stations record inside the batch's step graphs exactly as
    when that member steps alone; autotuning trial steps leave no records."""
    ms = _members(3, seed=4)
    sims = [wl.build_member(m, precision) for m in ms]
    alone = wl.build_member(ms[1], precision)
    nx, ny, dx = ms[1]["kw"]["nx"], ms[1]["kw"]["ny"], ms[1]["kw"]["dx"]
    xs, ys = [0.3 * nx * dx, 0.7 * nx * dx], [0.5 * ny * dx, 0.25 * ny * dx]
    for s in (sims[1], alone):
        s.set_gauges(xs, ys, names=["a", "b"])
    with Ensemble(sims, precision=precision) as ens:
        ens.autotune(trial_steps=2)
        ens.step(7)
    alone.step(7)
    got, ref = sims[1].gauge_records(), alone.gauge_records()
    assert got["time"].size == ref["time"].size == 7
    assert np.array_equal(got["time"], ref["time"])
    for key in ("eta", "u", "v"):
        assert np.array_equal(got[key], ref[key])
    for s in sims + [alone]:
        s.close()
