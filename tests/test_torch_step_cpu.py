"""The torch FP64 transcription used as the autograd reference, against the oracle (CPU).

Same configuration (walls, islands, Manning friction, fixed dt) through the C
oracle and through tests/torch_step.py: the states agree to 1e-12 relative
(the transcription evaluates h**(1/3) with torch's pow, the oracle correctly
rounded, so the last bits may differ).
"""
import numpy as np
import pytest
import torch

from tests import torch_step as ts
from tests.helpers import gaussian_bed, hump_depth


@pytest.mark.parametrize("hllc", [False, True])
def test_torch_transcription_matches_oracle(oracle, hllc):
    nx, ny, dx, ng = 24, 20, 10.0, 2
    b = gaussian_bed(nx, ny, dx, dx, 6, seed=4, base=-3.0, amp=(-1.0, 4.0), width=(15.0, 60.0))
    h = hump_depth(b, dx, dx, amp=0.4, width=50.0)
    assert (h == 0).any()
    dt, steps = 0.4, 12
    cfg = dict(nx=nx, ny=ny, dx=dx, dy=dx, nghost=ng, t_end=1e6, cfl=0.45, manning_n=0.03,
               use_hllc=hllc, dt_fixed=dt)
    o = oracle.OracleSim.from_config(cfg, bathymetry=b, initial_h=h)
    o.step(steps)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a))
    bf = ts.embed(t(b), ng)
    H, HU, HV = ts.embed(t(h), ng), torch.zeros_like(bf), torch.zeros_like(bf)
    n = torch.full((nx, ny), 0.03, dtype=torch.float64)
    for _ in range(steps):
        H, HU, HV, bf = ts.walls(H, HU, HV, bf, ng)
        base = (H[ng:-ng, ng:-ng], HU[ng:-ng, ng:-ng], HV[ng:-ng, ng:-ng])
        a, u, v = ts.stage(H, HU, HV, bf, n, dt, ng, dx, dx, hllc)
        hs, hus, hvs, bf = ts.walls(ts.embed(a, ng), ts.embed(u, ng), ts.embed(v, ng), bf, ng)
        a, u, v = ts.stage(hs, hus, hvs, bf, n, dt, ng, dx, dx, hllc, base=base)
        H, HU, HV = ts.embed(a, ng), ts.embed(u, ng), ts.embed(v, ng)
    for got, ref in ((a, o.interior("h")), (u, o.interior("hu")), (v, o.interior("hv"))):
        scale = max(1e-6, float(np.abs(ref).max()))
        assert float(np.abs(got.numpy() - ref).max()) / scale <= 1e-12
