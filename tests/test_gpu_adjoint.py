"""Adjoint of the FP64 step (GPU): gauge-misfit gradients w.r.t. bed and Manning n.

* the adjoint's forward is the production step: with a uniform n field and
  the recorded CFL dt sequence its gauge surfaces are bit-identical to
  Rakali's FP64 step;
* dJ/db and dJ/dn equal torch.autograd through the plain FP64 torch
  transcription (tests/torch_step.py, itself pinned to the oracle) to 1e-8
  relative;
* directional derivatives match central finite differences on random smooth
  directions to 1e-6 relative.  J is piecewise smooth, and at a lake at rest
  it is not differentiable with respect to b at all: the minmod limiter sits
  at (0, 0), where a bed perturbation e d gives slopes e minmod(d_a, d_b),
  not linear in d, so no gradient (this adjoint's or autograd's) matches
  finite differences there.  The finite-difference case therefore starts
  from a surface with nonzero gradients everywhere;
* the torch.autograd.Function front end back-propagates the same gradient.
"""
import numpy as np
import pytest

from rakali_b200.adjoint import GaugeMisfit, misfit
from tests.helpers import gaussian_bed, hump_depth

pytestmark = pytest.mark.gpu


def _problem(nx, ny, steps, n_gauges, seed, hllc=False, dx=10.0, generic=False):
    rng = np.random.default_rng(seed)
    b = gaussian_bed(nx, ny, dx, dx, 8, seed=seed, base=-6.0, amp=(-2.0, 3.0), width=(30.0, 90.0))
    h = hump_depth(b, dx, dx, amp=0.3, width=60.0)
    if generic:  # a surface with nonzero gradients everywhere (no resting water)
        x = (np.arange(nx) + 0.5) * dx
        y = (np.arange(ny) + 0.5) * dx
        X, Y = np.meshgrid(x, y, indexing="ij")
        surf = 0.02 * np.sin(X / 37.0 + 0.3) * np.cos(Y / 23.0 + 0.7) + 0.01 * np.sin((X + 2 * Y) / 51.0)
        h = np.asfortranarray(np.where(h > 0, np.maximum(h + surf, 0.0), 0.0))
    cells = rng.choice(nx * ny, size=n_gauges, replace=False)
    gauges = [(int(c % nx), int(c // nx)) for c in cells]
    p = GaugeMisfit(nx, ny, dx, dx, h, gauges, steps, use_hllc=hllc)
    n = np.full((nx, ny), 0.025)
    p.record_dt(b, n)
    # observations: the forward run of a perturbed bed
    noise = 0.2 * np.asfortranarray(gaussian_bed(nx, ny, dx, dx, 5, seed=seed + 1, base=0.0,
                                                 amp=(-1.0, 1.0), width=(40.0, 120.0)))
    _, obs = p.forward(b + noise, n)
    p.set_observations(obs)
    return p, b, h, n, gauges, obs


def test_forward_matches_production_step():
    from rakali_b200 import Rakali
    nx, ny, dx, steps = 40, 32, 10.0, 25
    b = gaussian_bed(nx, ny, dx, dx, 8, seed=2, base=-6.0, amp=(-2.0, 3.0), width=(30.0, 90.0))
    h = hump_depth(b, dx, dx, amp=0.3, width=60.0)
    gauges = [(3, 4), (20, 16), (39, 31), (10, 25)]
    p = GaugeMisfit(nx, ny, dx, dx, h, gauges, steps)
    _, eta = p.record_dt(b, np.full((nx, ny), 0.025))
    sim = Rakali(defer_init=True, nx=nx, ny=ny, dx=dx, dy=dx, nghost=2, t_end=1e6, cfl=0.45,
                 manning_n=0.025)
    sim.set_bathymetry(b)
    sim.set_initial_h(h)
    sim.finalize()
    with sim:
        for k in range(steps):
            sim.step(1)
            assert sim.dt == p.dt[k]
            e = sim.h_phys + sim.b_phys
            for m, (i, j) in enumerate(gauges):
                assert e[i, j] == eta[k, m]
    p.close()


def test_uniform_field_equals_scalar():
    p, b, h, n, _, _ = _problem(24, 20, 10, 5, seed=3)
    J1, _ = p.forward(b, n)
    J2, _ = p.forward(b, 0.025)
    assert J1 == J2
    p.close()


@pytest.mark.parametrize("hllc", [False, True])
def test_gradient_matches_torch_autograd(hllc):
    import torch

    from tests import torch_step as ts
    nx, ny, steps = 28, 22, 14
    p, b, h, n, gauges, obs = _problem(nx, ny, steps, 6, seed=5, hllc=hllc)
    J, gb, gn = p.gradient(b, n)
    obs = torch.from_numpy(obs)
    bt = torch.tensor(b, dtype=torch.float64, requires_grad=True)
    nt = torch.tensor(n, dtype=torch.float64, requires_grad=True)
    z = torch.zeros((nx, ny), dtype=torch.float64)
    Jt = ts.misfit(bt, nt, torch.from_numpy(h), z, z, gauges, obs, list(p.dt), 2, 10.0, 10.0,
                   hllc=hllc)
    Jt.backward()
    assert abs(float(Jt) - J) <= 1e-10 * abs(J)
    for got, ref in ((gb, bt.grad.numpy()), (gn, nt.grad.numpy())):
        scale = float(np.abs(ref).max())
        assert scale > 0.0
        assert float(np.abs(got - ref).max()) <= 1e-8 * scale
    p.close()


def test_gradient_matches_central_differences():
    nx, ny, steps = 40, 32, 29  # 29 steps: checkpoint segments of 6, the last one short
    p, b, h, n, _, _ = _problem(nx, ny, steps, 10, seed=7, generic=True)
    assert p.checkpoint_interval == 6  # the default: segments recomputed
    J, gb, gn = p.gradient(b, n)
    assert p.checkpoint_interval == 6
    rng = np.random.default_rng(11)
    for k in range(5):
        db = np.asfortranarray(gaussian_bed(nx, ny, 10.0, 10.0, 3, seed=100 + k, base=0.0,
                                            amp=(-1.0, 1.0), width=(50.0, 150.0)))
        dn = np.asfortranarray(0.005 * rng.standard_normal((nx, ny)))
        eps = 1e-6
        Jp, _ = p.forward(b + eps * db, n + eps * dn)
        Jm, _ = p.forward(b - eps * db, n - eps * dn)
        fd = (Jp - Jm) / (2 * eps)
        ad = float(np.sum(gb * db) + np.sum(gn * dn))
        assert abs(fd - ad) <= 1e-6 * max(abs(fd), 1e-12), (k, fd, ad)
    p.close()


def test_kept_states_and_checkpoints_give_the_same_bits():
    """A gradient run that keeps every state (given a state budget) and one
    that checkpoints every ~sqrt(N) steps and recomputes the segments (the
    default) return identical J and gradients."""
    nx, ny, steps = 40, 32, 29
    p, b, h, n, _, _ = _problem(nx, ny, steps, 10, seed=7, generic=True)
    p.set_state_budget(None)
    J1, gb1, gn1 = p.gradient(b, n)
    assert p.checkpoint_interval == 1  # every state kept
    p.set_state_budget(0)
    J0, gb0, gn0 = p.gradient(b, n)
    assert p.checkpoint_interval == 6
    assert J0 == J1 and np.array_equal(gb0, gb1) and np.array_equal(gn0, gn1)
    p.set_state_budget(None)
    J2, gb2, gn2 = p.gradient(b, n)
    assert p.checkpoint_interval == 1
    assert J2 == J1 and np.array_equal(gb2, gb1) and np.array_equal(gn2, gn1)
    p.close()


def test_autograd_function_backward():
    import torch
    p, b, h, n, _, _ = _problem(24, 20, 12, 5, seed=9)
    J, gb, gn = p.gradient(b, n)
    bt = torch.tensor(b, dtype=torch.float64, requires_grad=True)
    nt = torch.tensor(n, dtype=torch.float64, requires_grad=True)
    Jt = misfit(p, bt, nt)
    assert float(Jt) == J
    (3.0 * Jt).backward()
    assert np.array_equal(bt.grad.numpy(), 3.0 * gb)
    assert np.array_equal(nt.grad.numpy(), 3.0 * gn)
    p.close()


def test_gradient_matches_torch_autograd_128():
    """The autograd comparison at 128 x 128, 30 steps, 16 gauges.

    The transcription agrees with the CUDA forward to ~1e-12, not bit for bit;
    on resting water the limiter and wave-speed branches are decided by
    rounding-level differences, so the two would differentiate different
    pieces there.  The case starts from a moving surface."""
    import torch

    from tests import torch_step as ts
    nx = ny = 128
    p, b, h, n, gauges, obs = _problem(nx, ny, 30, 16, seed=13, generic=True)
    J, gb, gn = p.gradient(b, n)
    bt = torch.tensor(b, dtype=torch.float64, requires_grad=True)
    nt = torch.tensor(n, dtype=torch.float64, requires_grad=True)
    z = torch.zeros((nx, ny), dtype=torch.float64)
    Jt = ts.misfit(bt, nt, torch.from_numpy(h), z, z, gauges, torch.from_numpy(obs), list(p.dt),
                   2, 10.0, 10.0)
    Jt.backward()
    assert abs(float(Jt) - J) <= 1e-10 * abs(J)
    for got, ref in ((gb, bt.grad.numpy()), (gn, nt.grad.numpy())):
        assert float(np.abs(got - ref).max()) <= 1e-8 * float(np.abs(ref).max())
    p.close()


# ---------------------------------------------------------------------------
# batches: many problems in the same launches, FP64 and FP32
# ---------------------------------------------------------------------------

def _batch_inputs(nm, nx, ny, steps, n_gauges, seed, dx=10.0):
    """Per-member beds, moving initial surfaces, gauges and observation beds."""
    from tests.helpers import gaussian_bed
    x = (np.arange(nx) + 0.5) * dx
    y = (np.arange(ny) + 0.5) * dx
    X, Y = np.meshgrid(x, y, indexing="ij")
    bs, hs, gs, obs_b = [], [], [], []
    rng = np.random.default_rng(seed)
    for m in range(nm):
        b = gaussian_bed(nx, ny, dx, dx, 8, seed=seed + 10 * m, base=-6.0, amp=(-2.0, 3.0),
                         width=(30.0, 90.0))
        h = hump_depth(b, dx, dx, amp=0.3, width=60.0)
        surf = 0.02 * np.sin(X / (37.0 + m) + 0.3) * np.cos(Y / 23.0 + 0.7)
        h = np.where(h > 0, np.maximum(h + surf, 0.0), 0.0)
        cells = rng.choice(nx * ny, size=n_gauges, replace=False)
        bs.append(b)
        hs.append(h)
        gs.append([(int(c % nx), int(c // nx)) for c in cells])
        obs_b.append(b + 0.2 * gaussian_bed(nx, ny, dx, dx, 5, seed=seed + 10 * m + 1, base=0.0,
                                            amp=(-1.0, 1.0), width=(40.0, 120.0)))
    return np.array(bs), np.array(hs), gs, np.array(obs_b)


def test_batch_fp64_equals_single_problems():
    """Members of an FP64 batch reproduce their single-problem runs bit for bit."""
    from rakali_b200.adjoint import GaugeMisfitBatch
    nm, nx, ny, steps = 3, 28, 22, 14
    b, h, gauges, ob = _batch_inputs(nm, nx, ny, steps, 5, seed=31)
    n = np.full((nm, nx, ny), 0.025)
    with GaugeMisfitBatch(nm, nx, ny, 10.0, 10.0, h, gauges, steps, precision=64) as pb:
        assert pb.precision == 64
        pb.set_state_budget(None)  # every state kept: the singles checkpoint
        pb.record_dt(b, n)
        _, obs = pb.forward(ob, n)
        pb.set_observations(obs)
        J, gb, gn = pb.gradient(b, n)
        dts = pb.dt
        assert pb.checkpoint_interval == 1  # every state kept
    for m in range(nm):
        with GaugeMisfit(nx, ny, 10.0, 10.0, h[m], gauges[m], steps) as p:
            p.record_dt(b[m], n[m])
            assert np.array_equal(p.dt, dts[m])
            p.set_observations(obs[:, m, :])
            Jm, gbm, gnm = p.gradient(b[m], n[m])
        assert Jm == J[m]
        assert np.array_equal(gbm, gb[m]) and np.array_equal(gnm, gn[m])


def test_batch_fp32_kept_states_and_checkpoints_give_the_same_bits():
    from rakali_b200.adjoint import GaugeMisfitBatch
    nm, nx, ny, steps = 2, 30, 24, 17
    b, h, gauges, ob = _batch_inputs(nm, nx, ny, steps, 4, seed=37)
    n = np.full((nm, nx, ny), 0.025)
    with GaugeMisfitBatch(nm, nx, ny, 10.0, 10.0, h, gauges, steps, precision=32) as pb:
        pb.set_state_budget(None)
        pb.record_dt(b, n)
        _, obs = pb.forward(ob, n)
        pb.set_observations(obs)
        J1, gb1, gn1 = pb.gradient(b, n)
        assert pb.checkpoint_interval == 1
        pb.set_state_budget(0)
        J0, gb0, gn0 = pb.gradient(b, n)
        assert pb.checkpoint_interval == 5
    assert np.array_equal(J0, J1) and np.array_equal(gb0, gb1) and np.array_equal(gn0, gn1)


def test_batch_fp32_against_fp64():
    """FP32 forward and adjoint against the FP64 batch on the same dt sequence.

    Forward: gauge surfaces within 2e-4 m, J within 1e-3 relative, the FP64
    mass sum of the FP32 state drifts by < 1e-6 relative in a closed basin.

    Gradients: J is piecewise smooth and its gradient jumps across the kinks
    of the limiter and wave-speed branches, so the FP64 gradient itself moves
    when the bed moves by FP32 rounding (its "floor": the FP64 gradient at
    b + 1e-7 |b|max noise against the FP64 gradient at b; the worst member).
    The FP32 gradient's relative L2 error (worst member) must stay within 4x
    that floor plus 1e-3, and its directional derivatives along smooth
    directions, where isolated branch flips average out, within 1e-2 relative
    of the FP64 ones."""
    from rakali_b200.adjoint import GaugeMisfitBatch
    from tests.helpers import gaussian_bed
    nm, nx, ny, steps = 4, 64, 48, 40
    b, h, gauges, ob = _batch_inputs(nm, nx, ny, steps, 8, seed=41)
    n = np.full((nm, nx, ny), 0.025)
    rng = np.random.default_rng(7)
    noise = 1e-7 * float(np.abs(b).max()) * rng.standard_normal(b.shape)
    with GaugeMisfitBatch(nm, nx, ny, 10.0, 10.0, h, gauges, steps, precision=64) as p64:
        p64.record_dt(b, n)
        dts = p64.dt
        _, obs = p64.forward(ob, n)
        p64.set_observations(obs)
        J64, eta64 = p64.forward(b, n)
        _, gb64, gn64 = p64.gradient(b, n)
        _, gbf, gnf = p64.gradient(b + noise, n)
    with GaugeMisfitBatch(nm, nx, ny, 10.0, 10.0, h, gauges, steps, precision=32) as p32:
        assert p32.precision == 32
        p32.set_dt(dts)
        p32.set_observations(obs)
        J32, eta32 = p32.forward(b, n)
        mass = p32.mass
        _, gb32, gn32 = p32.gradient(b, n)

    def rel(a, r):
        return np.array([np.linalg.norm(a[m] - r[m]) / np.linalg.norm(r[m]) for m in range(nm)])

    eta_err = float(np.abs(eta32 - eta64).max())
    J_err = float(np.abs(J32 - J64).max() / np.abs(J64).max())
    drift = float(np.abs(mass[1] - mass[0]).max() / mass[0].min())
    gb_err, gn_err = rel(gb32, gb64), rel(gn32, gn64)
    gb_floor, gn_floor = rel(gbf, gb64), rel(gnf, gn64)
    dd = []
    for k in range(6):
        db = np.array([gaussian_bed(nx, ny, 10.0, 10.0, 3, seed=200 + 10 * k + m, base=0.0,
                                    amp=(-1.0, 1.0), width=(60.0, 200.0)) for m in range(nm)])
        dn = np.array([gaussian_bed(nx, ny, 10.0, 10.0, 3, seed=300 + 10 * k + m, base=0.0,
                                    amp=(-0.01, 0.01), width=(60.0, 200.0)) for m in range(nm)])
        d64 = np.sum(gb64 * db, axis=(1, 2)) + np.sum(gn64 * dn, axis=(1, 2))
        d32 = np.sum(gb32 * db, axis=(1, 2)) + np.sum(gn32 * dn, axis=(1, 2))
        dd.extend(np.abs(d32 - d64) / np.abs(d64))
    print(f"fp32 vs fp64: eta {eta_err:.2e} m, J {J_err:.2e}, mass drift {drift:.2e}, "
          f"grad b {gb_err.max():.2e} (floor {gb_floor.max():.2e}), "
          f"grad n {gn_err.max():.2e} (floor {gn_floor.max():.2e}), "
          f"directional max {max(dd):.2e} median {np.median(dd):.2e}")
    assert eta_err <= 2e-4
    assert J_err <= 1e-3
    assert drift <= 1e-6
    assert gb_err.max() <= 4.0 * gb_floor.max() + 1e-3
    assert gn_err.max() <= 4.0 * gn_floor.max() + 1e-3
    assert max(dd) <= 1e-2



@pytest.mark.parametrize("hllc", [False, True])
def test_frozen_slope_gradient_matches_autograd_with_detached_slopes(hllc):
    """set_frozen_slopes(True): the gradient with the limited slopes held constant
    equals torch.autograd through the transcription with its slopes detached; J
    is unchanged, and set_frozen_slopes(False) gives the exact gradient back bit
    for bit."""
    import torch

    from tests import torch_step as ts
    nx, ny, steps = 28, 22, 14
    p, b, h, n, gauges, obs = _problem(nx, ny, steps, 6, seed=5, hllc=hllc, generic=True)
    J0, gb0, gn0 = p.gradient(b, n)
    p.set_frozen_slopes(True)
    J, gb, gn = p.gradient(b, n)
    assert J == J0
    bt = torch.tensor(b, dtype=torch.float64, requires_grad=True)
    nt = torch.tensor(n, dtype=torch.float64, requires_grad=True)
    z = torch.zeros((nx, ny), dtype=torch.float64)
    Jt = ts.misfit(bt, nt, torch.from_numpy(h), z, z, gauges, torch.from_numpy(obs), list(p.dt),
                   2, 10.0, 10.0, hllc=hllc, frozen=True)
    Jt.backward()
    assert abs(float(Jt.detach()) - J) <= 1e-10 * abs(J)
    for got, ref in ((gb, bt.grad.numpy()), (gn, nt.grad.numpy())):
        scale = float(np.abs(ref).max())
        assert scale > 0.0
        assert float(np.abs(got - ref).max()) <= 1e-8 * scale
    assert float(np.abs(gb - gb0).max()) > 0.0  # the slopes do carry sensitivity
    p.set_frozen_slopes(False)
    J1, gb1, gn1 = p.gradient(b, n)
    assert J1 == J0 and np.array_equal(gb1, gb0) and np.array_equal(gn1, gn0)
    p.close()


def test_frozen_slope_gradient_fp32_against_fp64():
    """Frozen-slope gradients of an FP32 batch against the FP64 batch on the same
    dt sequence: relative L2 error (worst member) within 1e-2 and directional
    derivatives along smooth directions within 2e-3 relative."""
    from rakali_b200.adjoint import GaugeMisfitBatch
    nm, nx, ny, steps = 3, 64, 48, 40
    b, h, gauges, ob = _batch_inputs(nm, nx, ny, steps, 8, seed=43)
    n = np.full((nm, nx, ny), 0.025)
    with GaugeMisfitBatch(nm, nx, ny, 10.0, 10.0, h, gauges, steps, precision=64) as p64:
        p64.record_dt(b, n)
        dts = p64.dt
        _, obs = p64.forward(ob, n)
        p64.set_observations(obs)
        p64.set_frozen_slopes(True)
        _, gb64, gn64 = p64.gradient(b, n)
    with GaugeMisfitBatch(nm, nx, ny, 10.0, 10.0, h, gauges, steps, precision=32) as p32:
        p32.set_dt(dts)
        p32.set_observations(obs)
        p32.set_frozen_slopes(True)
        _, gb32, gn32 = p32.gradient(b, n)
    rel = max(float(np.linalg.norm(gb32[m] - gb64[m]) / np.linalg.norm(gb64[m])) for m in range(nm))
    dd = []
    for k in range(4):
        db = np.array([gaussian_bed(nx, ny, 10.0, 10.0, 3, seed=500 + 10 * k + m, base=0.0,
                                    amp=(-1.0, 1.0), width=(60.0, 200.0)) for m in range(nm)])
        d64 = np.sum(gb64 * db, axis=(1, 2))
        d32 = np.sum(gb32 * db, axis=(1, 2))
        dd.extend(np.abs(d32 - d64) / np.abs(d64))
    print(f"frozen fp32 vs fp64: grad b rel L2 {rel:.2e}, directional max {max(dd):.2e}")
    assert rel <= 1e-2
    assert max(dd) <= 2e-3
