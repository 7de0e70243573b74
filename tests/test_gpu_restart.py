"""Restart from instantaneous-field files written by the library (TG and IO
sections): the restarted state equals the written one, a TG run continues
bit for bit (CONVH0 is not needed at NS = 1), and an IO run from the restarted
state stays in parity with the oracle given the same state."""
import numpy as np
import pytest

from tests.conftest import relerr

pytestmark = pytest.mark.gpu


def _need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def test_tg_restart_continues_bitwise(tmp_path):
    _need_gpu()
    from chapsim1ww_b200 import TGChannel
    d = str(tmp_path) + "/"
    a = TGChannel(48, 20, 40)
    a.random_fl_fld_tg(6, 0.1)
    a.step(2)
    a.write_instant(d, 2, 0.002)
    b = TGChannel(48, 20, 40)
    it, tm = b.read_instant(d, 0.002)
    assert (it, tm) == (2, 0.002)
    for n in ("u", "v", "w", "p"):
        assert np.array_equal(a.get_field(n), b.get_field(n)), n
    a.step(2)
    b.step(2)
    for n in ("u", "v", "w", "p"):
        assert np.array_equal(a.get_field(n), b.get_field(n)), n


def test_io_restart_state_and_oracle_parity(tmp_path):
    _need_gpu()
    from chapsim1ww_b200 import IOChannel
    from oracle.pyoracle import OracleIO, synth_table
    d = str(tmp_path) + "/"
    table = synth_table(4096)
    a = IOChannel(40, 18, 24, table=table)
    a.random_fl_theml_fld_io(3, 0.1)
    a.step(2)
    a.write_instant(d, 6, 0.002)
    b = IOChannel(40, 18, 24, table=table)
    assert b.read_instant(d, 0.002) == (6, 0.002)
    for n in ("gx", "gy", "gz", "p", "t", "rho", "h", "mu", "k"):
        assert relerr(b.get_field(n)[:, 1:-1, :], a.get_field(n)[:, 1:-1, :]) <= 1e-14, n
    assert np.all(b.get_field("g0x") == 0.0)
    o = OracleIO(40, 18, 24, table=table)
    for n in ("u", "v", "w", "p", "gx", "gy", "gz", "g0x", "g0y", "g0z", "h", "t", "rho", "mu", "k", "rhoh", "rho0",
              "mu0", "ex0x", "ex0y", "ex0z", "rhse0", "drho"):
        o.set(n, b.get_field(n))
    b.step(1)
    o.step(1)
    for n in ("u", "v", "w", "p", "gx", "h", "rho"):
        assert relerr(b.get_field(n), o.get(n)) <= 1e-10, n


def test_tg_and_io_sections_share_a_directory(tmp_path):
    """TG and coupled IO sections written into one directory keep separate
    files (DNS_perixz / DNS_perioz) and each restarts from its own."""
    _need_gpu()
    import os

    from chapsim1ww_b200 import IOChannel, TGChannel
    from oracle.pyoracle import synth_table
    d = str(tmp_path) + "/"
    table = synth_table(4096)
    tg = TGChannel(40, 18, 24)
    tg.random_fl_fld_tg(1, 0.1)
    io = IOChannel(40, 18, 24, table=table, coupled=1)
    io.random_fl_theml_fld_io(2, 0.1)
    tg.write_instant(d, 3, 0.003)
    io.write_instant(d, 3, 0.003)
    names = sorted(os.listdir(d))
    assert sum(n.startswith("DNS_perixz") for n in names) == 4
    assert sum(n.startswith("DNS_perioz") for n in names) == 7
    tg2 = TGChannel(40, 18, 24)
    tg2.read_instant(d, 0.003)
    io2 = IOChannel(40, 18, 24, table=table, coupled=1)
    io2.read_instant(d, 0.003)
    for n in ("u", "v", "w", "p"):
        assert np.array_equal(tg2.get_field(n), tg.get_field(n)), n
    for n in ("gx", "gy", "gz", "p", "t", "rho", "h"):
        assert relerr(io2.get_field(n)[:, 1:-1, :], io.get_field(n)[:, 1:-1, :]) <= 1e-14, n
