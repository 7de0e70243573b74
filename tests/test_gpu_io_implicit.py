"""GPU parity of the IO section's semi-implicit viscous scheme (visthemflg = 1:
VISCOUS_PAR_EXPLT_*_io, RHS_MOM_EXPLICIT_io's implicit branch, the MOMFA_io
factored solves, DENSITY_implicit_add and the implicit PRCALC_io) against the
FP64 CPU oracle.  Tolerance: FP64 within 1e-10 relative (max |a-b| / max |b|)
on every state field after every substep."""
import numpy as np
import pytest

from tests.conftest import relerr

pytestmark = pytest.mark.gpu

TOL = 1e-10
FLOW = ("u", "v", "w", "p", "gx", "gy", "gz")
THERMAL = ("h", "t", "rho", "mu", "k", "rhoh")


def _need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def pair(nx, ny, nz, thermal, seed=2, amp=0.1, **kw):
    _need_gpu()
    from chapsim1ww_b200 import IOChannel
    from oracle.pyoracle import OracleIO, synth_table
    table = synth_table(4096)
    g = IOChannel(nx, ny, nz, thermal=thermal, table=table if thermal else None, visc_scheme=1, **kw)
    o = OracleIO(nx, ny, nz, thermal=thermal, table=table, visc_scheme=1, **kw)
    g.random_fl_theml_fld_io(seed, amp)
    o.init_random(seed, amp)
    return g, o


def compare(g, o, names, tol=TOL, tag=""):
    errs = {n: relerr(g.get_field(n), o.get(n)) for n in names}
    bad = {n: e for n, e in errs.items() if not e <= tol}
    assert not bad, f"{tag}: relative errors above {tol}: {errs}"
    return errs


@pytest.mark.parametrize("dims", [(16, 12, 8), (40, 18, 24)])
def test_io_implicit_isothermal_parity(dims):
    g, o = pair(*dims, thermal=0)
    compare(g, o, FLOW + ("ex0x", "ex0y", "ex0z"), tag="init+projection")
    for step in range(2):
        for ns in (1, 2, 3):
            g.solverrk3_mom_io(ns)
            o.mom(ns)
            compare(g, o, FLOW + ("ex0x", "ex0y", "ex0z"), tag=f"step{step} ns{ns}")
    assert g.divgck_io() < 1e-11 and o.divmax() < 1e-11


@pytest.mark.parametrize("dims", [(16, 12, 8), (48, 20, 40)])
def test_io_implicit_thermal_parity(dims):
    g, o = pair(*dims, thermal=1)
    compare(g, o, FLOW + THERMAL, tag="init+projection")
    for step in range(2):
        for ns in (1, 2, 3):
            g.solverrk3_eng_io(ns)
            o.eng(ns)
            compare(g, o, THERMAL + ("rho0", "mu0", "rhse0"), tag=f"step{step} eng{ns}")
            g.solverrk3_mom_io(ns)
            o.mom(ns)
            compare(g, o, FLOW + ("ex0x", "ex0y", "ex0z"), tag=f"step{step} mom{ns}")
    assert g.bad_cells() == 0 and o.bad_cells() == 0
    assert g.divgck_io() < 1e-10


def test_io_implicit_graph_step_and_cfl():
    """Graph-replayed steps match the oracle; the CFL has no viscous limit
    (CFL_VISCOUS is zero for the semi-implicit scheme)."""
    g, o = pair(32, 16, 16, thermal=1, seed=5)
    g.step(2)
    o.step(2)
    compare(g, o, FLOW + THERMAL, tag="graph steps")
    assert abs(g.cfl() - o.cfl()) <= 1e-12 * o.cfl()


def test_io_implicit_density_correction_active():
    """Plant a non-uniform density history so DRHOI_STG and the density part
    of the split viscous terms are far from zero, then compare one substep."""
    g, o = pair(24, 16, 12, thermal=1, seed=7)
    rng = np.random.default_rng(11)
    for name in ("rho", "rho0", "mu", "mu0"):
        a = g.get_field(name) * (1.0 + 0.2 * rng.random(g.shape))
        g.set_field(name, a)
        o.set(name, a)
    g.solverrk3_mom_io(1)
    o.mom(1)
    compare(g, o, FLOW + ("ex0x", "ex0y", "ex0z"), tag="planted density")
