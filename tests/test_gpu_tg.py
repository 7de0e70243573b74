"""GPU parity of the TG RK3 substep (libchapsim, sm_100a) against the FP64
CPU oracle and the golden fixtures.  Tolerance: FP64 form within 1e-10
relative (max |a-b| / max |b|) on u, v, w, p after every checked stage."""
import math
import os

import numpy as np
import pytest

from tests.conftest import relerr

pytestmark = pytest.mark.gpu

TOL = 1e-10
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def pair(nx, ny, nz, lx=4 * math.pi, lz=4 * math.pi / 3, ren=2800.0, dt=1e-3, seed=0, amp=0.1, **kw):
    _need_gpu()
    from chapsim1ww_b200 import TGChannel
    from oracle.pyoracle import OracleTG
    g = TGChannel(nx, ny, nz, lx=lx, lz=lz, ren=ren, dt=dt, **kw)
    o = OracleTG(nx, ny, nz, lx=lx, lz=lz, ren=ren, dt=dt, **kw)
    g.random_fl_fld_tg(seed, amp, project=False)
    o.init_random(seed, amp)
    return g, o


def compare(g, o, names=("u", "v", "w", "p"), tol=TOL, tag=""):
    errs = {n: relerr(g.get_field(n), o.get(n)) for n in names}
    bad = {n: e for n, e in errs.items() if not e <= tol}
    assert not bad, f"{tag}: relative errors above {tol}: {errs}"
    return errs


@pytest.mark.parametrize("dims", [(16, 12, 8), (24, 16, 12), (64, 64, 64), (48, 20, 40), (60, 18, 36)])
def test_substep_parity(dims):
    g, o = pair(*dims)
    compare(g, o, ("u", "v", "w"), tol=1e-14, tag="init")
    g.solverrk3_mom_tg(0)
    o.substep(0)
    compare(g, o, tag="ns0")
    for step in range(2):
        for ns in (1, 2, 3):
            g.solverrk3_mom_tg(ns)
            o.substep(ns)
            compare(g, o, tag=f"step{step} ns{ns}")
    compare(g, o, ("h0u", "h0v", "h0w"), tag="h0")
    assert g.divgck_tg() < 1e-11
    assert abs(g.bulk_velocity_tg() - o.bulk()) < 1e-12


@pytest.mark.parametrize("dims", [(112, 16, 176), (80, 12, 96)])
def test_radix_7_11_lengths(dims):
    # lengths outside FFT99's 2/3/5 support (112 = 7*16, 176 = 11*16)
    g, o = pair(*dims, seed=3)
    g.solverrk3_mom_tg(0)
    o.substep(0)
    for ns in (1, 2, 3):
        g.solverrk3_mom_tg(ns)
        o.substep(ns)
    compare(g, o, tag="radix")


def test_graph_step_matches_eager_bitwise():
    _need_gpu()
    from chapsim1ww_b200 import TGChannel
    a = TGChannel(32, 24, 16)
    b = TGChannel(32, 24, 16)
    for s in (a, b):
        s.random_fl_fld_tg(7, 0.1, project=True)
    a.step(3)
    for _ in range(3):
        for ns in (1, 2, 3):
            b.solverrk3_mom_tg(ns)
    for n in ("u", "v", "w", "p"):
        assert np.array_equal(a.get_field(n), b.get_field(n)), n


def test_async_transfers_match_blocking_copies():
    """Stream-ordered uploads, a step and downloads queued on one context's
    stream give the same bits as blocking copies around the same step, with
    pinned and with pageable host buffers."""
    _need_gpu()
    import torch
    from chapsim1ww_b200 import TGChannel
    a = TGChannel(32, 24, 16)
    b = TGChannel(32, 24, 16)
    a.random_fl_fld_tg(5, 0.1, project=True)
    names = ("u", "v", "w", "p")
    start = {n: a.get_field(n) for n in names}
    for pinned in (True, False):
        host = {}
        for n in names:
            h = (torch.empty(a.shape, dtype=torch.float64, pin_memory=True).numpy() if pinned
                 else np.empty(a.shape))
            h[...] = start[n]
            host[n] = h
            b.set_field_async(n, h)
        b.step(2)
        for n in names:
            b.get_field_async(n, out=host[n])
        b.sync()
        for n in names:
            a.set_field(n, start[n])
        a.step(2)
        for n in names:
            assert np.array_equal(host[n], a.get_field(n)), (pinned, n)
    with pytest.raises(ValueError):
        b.set_field_async("u", np.zeros(3))
    a.close()
    b.close()


def test_fp64_bit_reproducible():
    _need_gpu()
    from chapsim1ww_b200 import TGChannel
    outs = []
    for _ in range(2):
        s = TGChannel(64, 48, 32, ren=3000.0)
        s.random_fl_fld_tg(11, 0.1, project=True)
        s.step(5)
        outs.append([s.get_field(n) for n in ("u", "v", "w", "p")])
        s.close()
    for x, y in zip(*outs):
        assert np.array_equal(x, y)


def test_poisson_piece_parity():
    g, o = pair(32, 24, 16, seed=4)
    rng = np.random.default_rng(5)
    rhs = np.zeros(g.shape)
    rhs[:, 1:-1, :] = rng.standard_normal((16, 24, 32))
    g.set_field("rhsphi", rhs)
    o.set("rhsphi", rhs)
    g.fft99_pois3d()
    o.pois3d()
    e = relerr(g.get_field("phi")[:, 1:-1, :], o.get("phi")[:, 1:-1, :])
    assert e < 1e-12, e


def test_analytic_poisson():
    """TEST_POISSON (src/SOLVERRK3_MOM_IO.f90:171-202): rhs = -4 sin x cos x."""
    _need_gpu()
    from chapsim1ww_b200 import TGChannel
    nx, ny, nz, lx = 64, 16, 8, 4 * math.pi
    g = TGChannel(nx, ny, nz, lx=lx)
    x = (np.arange(nx) + 0.5) * lx / nx
    rhs = np.zeros(g.shape)
    rhs[:, 1:-1, :] = (-4.0 * np.sin(x) * np.cos(x))[None, None, :]
    g.set_field("rhsphi", rhs)
    g.fft99_pois3d()
    phi = g.get_field("phi")[:, 1:-1, :]
    m = round(lx / math.pi)  # sin(2x) is wavenumber index lx/pi
    ak1 = 2.0 * (1.0 - math.cos(2.0 * math.pi * m / nx)) * (nx / lx) ** 2
    exact = 2.0 * np.sin(2.0 * x) / ak1
    assert np.abs(phi - exact[None, None, :]).max() < 1e-12


def test_divg_and_correction_pieces():
    g, o = pair(24, 16, 12, seed=9)
    for s in (g,):
        s.divg_tg(1)
    o.divg(1)
    assert relerr(g.get_field("rhsphi")[:, 1:-1, :], o.get("rhsphi")[:, 1:-1, :]) < 1e-13
    rng = np.random.default_rng(1)
    phi = rng.standard_normal(g.shape)
    g.set_field("phi", phi)
    o.set("phi", phi)
    g.veloupdt_tg(2)
    o.velo_correction(2)
    compare(g, o, tag="correction")


@pytest.mark.parametrize("name", ["tg_16x12x8_seed0", "tg_24x16x12_seed5"])
def test_golden_fixture(name):
    _need_gpu()
    from chapsim1ww_b200 import TGChannel
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    nx, ny, nz, lx, lz, ren, dt, seed, amp, steps = z["meta"]
    g = TGChannel(int(nx), int(ny), int(nz), lx=lx, lz=lz, ren=ren, dt=dt)
    g.random_fl_fld_tg(int(seed), amp, project=True)
    for n in ("u", "v", "w", "p"):
        assert relerr(g.get_field(n), z["ns0_" + n]) < 1e-10, n
    g.step(int(steps))
    for n in ("u", "v", "w", "p"):
        assert relerr(g.get_field(n), z["end_" + n]) < 1e-10, n


def test_flowdrvtp2_constant_pressure_gradient():
    g, o = pair(24, 16, 12, flowdrvtp=2, cfgv=8.18e-3)
    g.solverrk3_mom_tg(0)
    o.substep(0)
    for ns in (1, 2, 3):
        g.solverrk3_mom_tg(ns)
        o.substep(ns)
    compare(g, o, tag="flowdrvtp2")


def test_uniform_grid_istr2_0():
    g, o = pair(16, 16, 16, istr2=0)
    for ns in (0, 1, 2, 3):
        g.solverrk3_mom_tg(ns)
        o.substep(ns)
    compare(g, o, tag="uniform")


def test_nan_scan_and_divmax():
    _need_gpu()
    from chapsim1ww_b200 import TGChannel
    s = TGChannel(32, 16, 16)
    s.random_fl_fld_tg(2, 0.1, project=True)
    s.step(2)
    assert s.nan_count() == 0
    u = s.get_field("u")
    u[3, 5, 7] = float("nan")
    s.set_field("u", u)
    assert s.nan_count() == 1
    assert math.isinf(s.divgck_tg())


def test_adi_fallback_wide_inverse():
    # Re = 1, dt = 0.05: the x/z inverses are too wide for the banded kernel,
    # so the shared-memory cyclic Thomas kernels run instead
    g, o = pair(32, 24, 16, ren=1.0, dt=0.05)
    for ns in (0, 1):
        g.solverrk3_mom_tg(ns)
        o.substep(ns)
    compare(g, o, tag="fallback")


def test_short_lines_wrap():
    # nx, nz shorter than a 32 x 8 tile plus its halo
    g, o = pair(8, 8, 8, lx=1.0, lz=0.5)
    for ns in (0, 1, 2, 3):
        g.solverrk3_mom_tg(ns)
        o.substep(ns)
    compare(g, o, tag="short")


def test_line_tuning_does_not_change_results():
    """The y-line block width of the Poisson solve (64, 128, 256: one of the
    autotuner's launch shapes) leaves every field bitwise unchanged, TG and
    IO."""
    _need_gpu()
    from chapsim1ww_b200 import IOChannel, TGChannel
    from oracle.pyoracle import synth_table
    out = []
    for bx in (64, 128, 256):
        g = TGChannel(48, 20, 40)
        g.set_line_tuning(bx)
        assert g.get_line_tuning() == bx
        g.random_fl_fld_tg(3, 0.1, project=True)
        g.step(2)
        out.append([g.get_field(n) for n in ("u", "v", "w", "p")])
        g.close()
    for a in out[1:]:
        assert all(np.array_equal(x, y) for x, y in zip(out[0], a))
    table = synth_table(4096)
    res = []
    for bx in (64, 256):
        g = IOChannel(40, 18, 24, table=table)
        g.set_line_tuning(bx)
        g.random_fl_theml_fld_io(2, 0.1)
        g.step(1)
        res.append([g.get_field(n) for n in ("gx", "p", "h")])
        g.close()
    assert all(np.array_equal(x, y) for x, y in zip(*res))
