"""On-device statistics of the x-periodic IO section:
PP_MEAN_ZX_FLOW_Xperiodic_IO (src/processing/PP_MEAN_ZX.f90:299-872) against
the oracle's restatement applied to the GPU's own fields (1e-12 per statistic
group, relative to the group's largest value), the running time average of
PP_MEAN_T_Xperiodic_IO (src/processing/PP_MEAN_T.f90:436-520), the bulk
numbers that close the reference routine, and bit-reproducibility."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FLOW = ("u", "v", "w", "p", "gx", "gy", "gz")
THERMAL = ("h", "t", "rho", "mu", "k")


def _need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _pair(thermal, dims=(40, 18, 24)):
    _need_gpu()
    from chapsim1ww_b200 import IOChannel
    from oracle.pyoracle import OracleIO, synth_table
    table = synth_table(4096) if thermal else None
    g = IOChannel(*dims, thermal=thermal, table=table)
    o = OracleIO(*dims, thermal=thermal, table=table)
    g.random_fl_theml_fld_io(5, 0.1)
    g.step(1)
    return g, o


def _oracle_on(g, o, thermal):
    for f in FLOW + (THERMAL if thermal else ()):
        o.set(f, g.get_field(f))
    return o.stats()


def _check_groups(g, a, b, thermal):
    lo = 0
    for name, width in g.STATS_LAYOUT:
        x, y = a[:, lo:lo + width], b[:, lo:lo + width]
        lo += width
        if not thermal and lo > 141:
            assert not np.any(x), name
            continue
        assert np.abs(x - y).max() <= 1e-12 * max(np.abs(y).max(), 1e-300), name
    assert lo == 360


@pytest.mark.parametrize("thermal", [1, 0])
def test_io_xz_statistics_parity(thermal):
    g, o = _pair(thermal)
    g.pp_mean_zx()
    a, n = g.stats(0)
    assert n == 0 and a.shape == (18, 360)
    _check_groups(g, a, _oracle_on(g, o, thermal), thermal)
    # DVDL2 is symmetric in (m,h) <-> (n,p)
    d2 = a[:, 60:141].reshape(-1, 9, 9)
    assert np.allclose(d2, np.transpose(d2, (0, 2, 1)), rtol=0, atol=1e-14 * np.abs(d2).max())


def test_io_time_average_and_monitor():
    g, o = _pair(1)
    g.stats_reset()
    g.pp_mean_zx(accumulate=True)
    s1 = _oracle_on(g, o, 1)
    g.step(1)
    g.pp_mean_zx(accumulate=True)
    s2 = _oracle_on(g, o, 1)
    t, n = g.stats(1)
    assert n == 2
    assert np.abs(t - 0.5 * (s1 + s2)).max() <= 1e-12 * np.abs(s1).max()
    mon = g.monitor()
    assert all(np.isfinite(v) for v in mon.values())
    # G1BULK of the statistics is BULK_MASSFLUX_IO (the x-mean of the
    # cell-centred flux is the x-mean of the face flux)
    assert abs(mon["g1bulk"] - g.bulk_massflux_io()) <= 1e-12
    assert mon["t1maxx"] > 0


def test_io_statistics_bit_reproducible():
    g, _ = _pair(1)
    g.pp_mean_zx()
    a, _ = g.stats(0)
    g.pp_mean_zx()
    b, _ = g.stats(0)
    assert np.array_equal(a, b)


def test_io_driven_force():
    """PP_DRIVEN_FORCE (src/processing/PP_MEAN_ZX.f90:969-1056) from the device
    statistics against the reference's sums over the fields themselves: the
    wall frictions from u in the first and last rows (wall viscosity 1, or
    M_WAL_GV of iso-thermal walls), no buoyancy; FUxzL_IO = FcDrv (U1, 1).
    A heated channel with two iso-flux walls, where the reference reads an
    array it never allocated, is refused."""
    _need_gpu()
    from chapsim1ww_b200 import IOChannel
    from oracle.pyoracle import synth_table
    table = synth_table(4096)
    for thermal, iso in ((0, 0), (1, 3), (1, 1)):
        g = IOChannel(40, 18, 24, thermal=thermal, table=table if thermal else None,
                      qw=(0.95, 0.80) if iso else (1.0, 1.0), isothermal=iso)
        g.random_fl_theml_fld_io(5, 0.1)
        g.step(1)
        g.pp_mean_zx()
        fc, fu = g.driven_force()
        u = g.get_field("u")
        mu_w = g.wall_values()[:, 3] if thermal else np.ones(2)
        ynd, ycc = g.mesh(0), g.mesh(1)
        nxz = u.shape[0] * u.shape[2]
        f1 = mu_w[0] * u[:, 1, :].sum() / (ycc[0] - ynd[0]) / g.cfg.ren / nxz
        f2 = mu_w[1] * u[:, -2, :].sum() / (ycc[-1] - ynd[-1]) / g.cfg.ren / nxz
        ref = (abs(f1) + abs(f2)) / 2.0
        assert abs(fc - ref) <= 1e-12 * abs(ref), (thermal, iso, fc, ref)
        assert fu.shape == (18, 4) and np.all(fu[:, 3] == fc)
        g.close()
    g = IOChannel(16, 12, 8, table=table)
    g.random_fl_theml_fld_io(5, 0.1)
    g.pp_mean_zx()
    with pytest.raises(ValueError):
        g.driven_force()
