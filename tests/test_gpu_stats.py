"""On-device statistics of the TG channel: PP_MEAN_ZX_FLOW_TG against the
oracle's restatement (1e-12 relative per statistic group), the running time
average of PP_MEAN_T_TG, and the PP_MONITOR_TG numbers derived from them."""
import numpy as np
import pytest

from tests.conftest import relerr

pytestmark = pytest.mark.gpu

GROUPS = {"U1": (0, 4), "UP": (4, 7), "U2": (7, 13), "U3": (13, 23), "DVDL1": (23, 32), "DVDLP": (32, 41),
          "DVDL2": (41, 122)}


def _need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _pair():
    _need_gpu()
    from chapsim1ww_b200 import TGChannel
    from oracle.pyoracle import OracleTG
    g, o = TGChannel(48, 20, 40), OracleTG(48, 20, 40)
    g.random_fl_fld_tg(4, 0.1, project=True)
    o.init_random(4, 0.1)
    o.substep(0)
    return g, o


def test_xz_statistics_parity():
    g, o = _pair()
    g.step(1)
    o.step(1)
    g.pp_mean_zx()
    a, n = g.stats(0)
    assert n == 0
    # the statistics kernel on its own: the oracle's restatement applied to
    # the GPU's own fields, 1e-12 per group
    for f in ("u", "v", "w", "p"):
        o.set(f, g.get_field(f))
    b = o.stats()
    for name, (lo, hi) in GROUPS.items():
        assert relerr(a[:, lo:hi], b[:, lo:hi]) <= 1e-12, name
    # end to end (each side's own step): the fields agree to round-off
    # (1e-10 is the field parity bound), and the velocity-pressure
    # correlations, a few percent of max|u| max|p|, show that round-off
    # magnified; every group within the field bound
    from oracle.pyoracle import OracleTG
    o2 = OracleTG(48, 20, 40)
    o2.init_random(4, 0.1)
    o2.substep(0)
    o2.step(1)
    c = o2.stats()
    for name, (lo, hi) in GROUPS.items():
        assert relerr(a[:, lo:hi], c[:, lo:hi]) <= 1e-10, name
    # DVDL2 is symmetric in (m,h) <-> (n,p)
    d2 = a[:, 41:].reshape(-1, 9, 9)
    assert np.array_equal(d2, np.transpose(d2, (0, 2, 1)))


def test_time_average_and_monitor():
    g, o = _pair()
    g.stats_reset()
    g.pp_mean_zx(accumulate=True)
    s1 = o.stats()
    g.step(1)
    o.step(1)
    g.pp_mean_zx(accumulate=True)
    s2 = o.stats()
    t, n = g.stats(1)
    assert n == 2
    assert relerr(t, 0.5 * (s1 + s2)) <= 1e-12
    mon = g.monitor()
    assert all(np.isfinite(v) for v in mon.values())
    assert abs(mon["u1mean"] - g.bulk_velocity_tg()) < 1e-12
    assert mon["cf_bottom_xz"] > 0 and mon["cf_top_xz"] > 0


def test_statistics_bit_reproducible():
    g, _ = _pair()
    g.pp_mean_zx()
    a, _ = g.stats(0)
    g.pp_mean_zx()
    b, _ = g.stats(0)
    assert np.array_equal(a, b)
