"""Configurations run for their stated lengths.

Configuration 0 as defined: TG channel 64 x 64 x 64 on Lx = 4 pi, Ly = 2
(tanh stretching beta = 2), Lz = 4 pi / 3, Re_b = 2800, dt = 1e-3, seed 0,
amplitude 0.1, NS = 0 projection, then 100 full RK3 steps.  The FP64 form
stays within 1e-10 relative (max |a - b| / max |b|) of the FP64 oracle on u,
v, w and p at every 25th step, and a second run repeats the first bitwise.

The mixed form (FP64 state, FP32 temporaries and spectra, FP64 Poisson lines,
one FP64-residual refinement sweep) over 50 steps against the FP64 oracle,
with its errors on u, p and max |div u| printed per checkpoint; stated
tolerances over 50 steps: u, v, w <= 1e-5, p <= 1e-4, max |div u| <= 1e-8.
"""
import math

import numpy as np
import pytest

from tests.conftest import relerr

pytestmark = pytest.mark.gpu


def _need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


C0 = dict(nx=64, ny=64, nz=64, lx=4 * math.pi, lz=4 * math.pi / 3, ren=2800.0, dt=1e-3)


def test_config0_100_steps_fp64_parity_and_bitwise_repeat():
    _need_gpu()
    from chapsim1ww_b200 import TGChannel
    from oracle.pyoracle import OracleTG
    dims = (C0["nx"], C0["ny"], C0["nz"])
    kw = dict(lx=C0["lx"], lz=C0["lz"], ren=C0["ren"], dt=C0["dt"])
    g = TGChannel(*dims, **kw)
    o = OracleTG(*dims, **kw)
    g.random_fl_fld_tg(0, 0.1, project=True)
    o.init_random(0, 0.1)
    o.substep(0)
    worst = {}
    for chunk in range(4):
        g.step(25)
        o.step(25)
        for n in ("u", "v", "w", "p"):
            e = relerr(g.get_field(n), o.get(n))
            worst[n] = max(worst.get(n, 0.0), e)
            assert e <= 1e-10, (25 * (chunk + 1), n, e)
    print(f"config 0, 100 steps, FP64 vs oracle: worst relative errors {worst}, "
          f"max|div u| = {g.divgck_tg():.3e} (oracle {o.divmax():.3e})")
    assert g.divgck_tg() <= 1e-11
    # a second FP64 run from the same seed repeats the first bit for bit
    h = TGChannel(*dims, **kw)
    h.random_fl_fld_tg(0, 0.1, project=True)
    h.step(100)
    for n in ("u", "v", "w", "p"):
        assert np.array_equal(h.get_field(n), g.get_field(n)), n


def test_mixed_form_50_steps_against_fp64_oracle():
    _need_gpu()
    from chapsim1ww_b200 import MIXED, TGChannel
    from oracle.pyoracle import OracleTG
    dims = (96, 64, 64)
    g = TGChannel(*dims, precision=MIXED)
    o = OracleTG(*dims)
    g.random_fl_fld_tg(1, 0.1, project=True)
    o.init_random(1, 0.1)
    o.substep(0)
    rows = []
    for chunk in range(5):
        g.step(10)
        o.step(10)
        errs = {n: relerr(g.get_field(n), o.get(n)) for n in ("u", "v", "w", "p")}
        rows.append((10 * (chunk + 1), errs, g.divgck_tg()))
    for step, errs, div in rows:
        print(f"mixed 96x64x64 step {step}: u {errs['u']:.2e} v {errs['v']:.2e} w {errs['w']:.2e} "
              f"p {errs['p']:.2e} max|div u| {div:.2e}")
    for step, errs, div in rows:
        assert max(errs["u"], errs["v"], errs["w"]) <= 1e-5, (step, errs)
        assert errs["p"] <= 1e-4, (step, errs)
        assert div <= 1e-8, (step, div)
