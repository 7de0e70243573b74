"""CFL reductions (CFL_tg, CFL_io + CFL_VISCOUS, src/CFL.f90) against the
oracle, and a time-step change (the adaptive-DT variable of SOLVE.f90)
followed by steps that stay in parity with the oracle at the new DT
(FP64, 1e-10 relative)."""
import numpy as np
import pytest

from tests.conftest import relerr

pytestmark = pytest.mark.gpu


def _need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def test_tg_cfl_and_set_dt():
    _need_gpu()
    from chapsim1ww_b200 import TGChannel
    from oracle.pyoracle import OracleTG
    g, o = TGChannel(48, 20, 40), OracleTG(48, 20, 40)
    g.random_fl_fld_tg(3, 0.1, project=True)
    o.init_random(3, 0.1)
    o.substep(0)
    assert abs(g.cfl() - o.cfl()) <= 1e-13 * o.cfl()
    g.step(1)  # captures the step graph at the first dt
    o.step(1)
    g.set_dt(5e-4)
    o.set_dt(5e-4)
    g.step(2)
    o.step(2)
    for n in ("u", "v", "w", "p"):
        assert relerr(g.get_field(n), o.get(n)) <= 1e-10, n
    assert abs(g.cfl() - o.cfl()) <= 1e-12 * o.cfl()


def test_io_cfl_and_set_dt():
    _need_gpu()
    from chapsim1ww_b200 import IOChannel
    from oracle.pyoracle import OracleIO, synth_table
    table = synth_table(4096)
    g, o = IOChannel(40, 18, 24, table=table), OracleIO(40, 18, 24, table=table)
    g.random_fl_theml_fld_io(2, 0.1)
    o.init_random(2, 0.1)
    assert abs(g.cfl() - o.cfl()) <= 1e-13 * o.cfl()
    g.step(1)
    o.step(1)
    g.set_dt(2e-3)
    o.set_dt(2e-3)
    g.step(2)
    o.step(2)
    for n in ("u", "v", "w", "p", "gx", "h", "rho"):
        assert relerr(g.get_field(n), o.get(n)) <= 1e-10, n
    assert g.divgck_io() < 1e-10
